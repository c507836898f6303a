// Skinny GETT: contractions with one small free extent, FP32 on the CUDA cores.
//
// When one GETT extent -- M or N, the narrow side S -- is small, the
// contraction has few FMAs per byte: the wide operand P (W rows x K) and C
// (W x S) dominate, and each should cross HBM once. The tile kernels pad S
// to their tile width and, for most layouts, pay a packing pass that
// transposes P first. This kernel keeps a chunk of the narrow operand Q
// (S x K) in shared memory (every CTA reads it, from L2), streams P straight
// from the caller's tensor and writes every element of C once, in C's own
// layout -- the GETT property of TCCG's micro-kernel (C written in its
// original layout, tccg/gett.py:192-223), with TCCG's packing step
// (tccg/gett.py:440-470) replaced by loads that follow P's layout.
//
// W blocking. The W modes split into X -- the W mode C stores contiguously
// (its smallest C stride) -- and the Y space: all other W modes, linearised
// in order of increasing P stride. A block is a box of tx x ty positions
// (x, y), tx * ty <= SK_BW (256):
//   P(x, y, k) = P[x px + p_y_off[y] + p_k_off[k]]
//   Q(s, k)    = Q[q_s_off[s] + q_k_off[k]]
//   C(x, y, s) = C[x cx + c_y_off[y] + c_s_off[s]]
// When P's stride-one W mode is not X (P and C order the W modes
// differently: a transposition), the box spans X and the first Y mode, so
// the P loads run along y and the C stores along x, each over runs of the
// box's extent.
//
// Jobs. A job is one block x one pass over S (4 RS rows: RS = 4, 8 or 12
// rows per thread) x one k slice; an S above 48 runs passes of 32 rows,
// neighbouring jobs whose P chunks the later passes read from L2. The CTAs are persistent
// (two 256-thread CTAs per SM) and walk their jobs' k chunks (32 k each) as one sequence,
// double buffered through element-wise cp.async: the copies of the next
// chunk -- of the same job, or the first of the next job, whose box offsets
// are computed then -- are in flight while the CTA multiplies the current
// chunk and, after a job's last chunk, stores its C block. That keeps loads
// in flight through the FMA and store phases of every block.
//
// Per chunk thread (wg, sg) accumulates 4 positions x RS rows in FP32 FMAs, k
// in increasing order. The epilogue stages 32 rows at a time in the P stage
// just consumed and stores them in C's address order (SK_C_*): alpha * acc,
// then fma with beta * C (not read when beta = 0).
//
// Offsets are 32-bit: the plan takes this kernel only for tensors whose
// element offsets stay below 2^31 (8 GiB of FP32 each), which halves the
// integer work of every load and store address and of the offset tables.
//
// With a k-split (few jobs, long K: a matrix-vector shape) the job of slice
// z writes its raw sums densely to partial[z][block][pass][row][position]
// and skinny_reduce_kernel (one CTA per block and pass) adds the slices in
// split order before the same store walk. Results are deterministic: a fixed k order within a slice,
// slices in order.
#pragma once
#include <cuda.h>
#include "common.cuh"

namespace tccg {

// 256 threads (two CTAs per SM); 128-thread CTAs (four per SM, boxes of
// 128 positions) measured 24 % slower on the largest transposing item and
// faster only on multi-pass ones
#ifndef TCCG_SK_THREADS
#define TCCG_SK_THREADS 256
#endif
constexpr int SK_THREADS = TCCG_SK_THREADS;
constexpr int SK_BW = SK_THREADS;      // box positions per block (one per thread)
constexpr int SK_WG = SK_BW / 4;       // position groups of 4: a thread owns one ...
constexpr int SK_SG = SK_THREADS / SK_WG;  // ... in one of 4 row groups
static_assert(SK_SG == 4 && SK_WG % 32 == 0, "a warp's threads share one row group");
constexpr int SK_KC = 32;              // k per chunk
constexpr int SK_LDP = SK_BW + 4;      // P stage row stride (floats): [k][position]
constexpr int SK_SMAX = 256;           // largest narrow extent
constexpr int SK_SPMAX = 48;           // rows of one pass
constexpr int SK_QLD = SK_SPMAX + 4;   // Q stage row stride (floats): [k][row]
constexpr int SK_SUB = 32;             // rows of S staged per epilogue step
// shared memory: P stages [2][KC][LDP], Q stages [2][KC][QLD], then per job
// slot (two) the box positions' P and C offsets and the pass rows' C offsets
constexpr size_t SK_P_STAGE = (size_t)SK_KC * SK_LDP * 4;
constexpr size_t SK_Q_STAGE = (size_t)SK_KC * SK_QLD * 4;
constexpr size_t SK_OFF_TAB = 2 * (SK_P_STAGE + SK_Q_STAGE);
constexpr size_t SK_SMEM_BYTES = SK_OFF_TAB + (size_t)(4 * SK_BW + 2 * SK_SPMAX) * 4;
constexpr int SK_CTAS_PER_SM = SK_THREADS == 128 ? 4 : 2;
static_assert(SK_SUB == SK_KC, "the epilogue staging reuses one P stage");
static_assert(SK_CTAS_PER_SM * (SK_SMEM_BYTES + 1024) <= 228 * 1024, "CTAs per SM");

// P load order: lanes along x (X is P's stride-one W mode), along y (the
// first Y mode is), or along k (a K mode is). Box positions are numbered
// x-fastest (SK_P_X, SK_P_K) or y-fastest (SK_P_Y).
enum SkinnyPWalk : int { SK_P_X = 0, SK_P_Y = 1, SK_P_K = 2 };
// C store order of a staged step: (x, s) planes per y (C's next stride after
// X is S's); (x, y) planes per s (it is a Y mode's); runs of C's stride-one
// S mode, then x, per y (C's stride-one index is on the narrow side).
enum SkinnyCWalk : int { SK_C_XS = 0, SK_C_XY = 1, SK_C_SX = 2 };
// Contiguous C rows of a box (each y of the box): C(x, y, s) = C(0, y, s0) +
// x + ex (s - s0) with the box covering all of X (SK_CLIN_XS), or C(x0 + x,
// y, s) = C(x0, y, 0) + s + S x with all of S in one staged step
// (SK_CLIN_SX).
// C's stride-one S mode of extent e0 (s_run) directly followed in C by X:
// C(x, y, u e0 + o) = C(0, y, u e0) + x e0 + o, passes of whole runs, each
// (run, box row) one range of e0 x floats (SK_CLIN_RUNS; staged like the
// general case, copied range by range).
enum SkinnyCLin : int { SK_CLIN_NONE = 0, SK_CLIN_XS = 1, SK_CLIN_SX = 2, SK_CLIN_RUNS = 3 };

struct SkinnyArgs {
  const float* P;
  const float* Q;
  float* C;
  const int32_t* p_y_off;  // [ey]
  const int32_t* c_y_off;  // [ey]
  const int32_t* p_k_off;  // [K]
  const int32_t* q_s_off;  // [S]
  const int32_t* q_k_off;  // [K]
  const int32_t* c_s_off;  // [S]
  int32_t px, cx;          // P and C strides of X
  int32_t ex, ey;          // extents of X and of the Y space
  int32_t nblk;            // boxes: bxn along x, ceil(ey / ty) along y
  int32_t njobs;           // nblk x npass x ksplit
  int32_t tx, ty, bxn;
  int32_t S, K;
  int32_t rs;              // rows of S per thread; a pass covers 4 * rs rows
  int32_t npass;           // passes over S (> 1 only with one chunk and no k-split)
  int32_t spr;             // rows per pass: pass p covers S rows [p spr, p spr + spr), spr <= 4 rs
  int32_t ksplit;
  int32_t nchunks, chunks_per_split;
  int32_t kr_log2;         // SK_P_K: log2 of the lanes along k per position
  int32_t p_walk, c_walk;
  int32_t q_kfast;         // Q loads along k (its stride-one index is a K mode)
  int32_t s_run;           // SK_C_SX: extent of C's stride-one S mode
  // SK_P_X with unit x stride, every k offset and P itself 16-byte aligned:
  // four positions that are consecutive in P move as one 16-byte copy
  int32_t p_vec;
  // C of a box row is one contiguous range (SkinnyCLin): staged in that
  // order and stored as a straight copy
  int32_t c_lin;
  // SK_CLIN_XS with beta = 0 and C 16-byte aligned: each box row's
  // 16-byte-aligned range leaves as one bulk copy (cp.async.bulk) instead of
  // per-element stores; alpha is applied when staging
  int32_t c_bulk;
  float alpha, beta;
  float* partial;          // k-split slices (null: store to C)
};

constexpr int32_t SK_NONE = INT32_MIN;  // position outside the tensor (offsets may be negative)

// Job J of an item: block b, pass p, k slice z over chunks [c0, c1).
struct SkJob {
  int b, p, z, c0, c1;
};

__device__ __forceinline__ SkJob skinny_job(const SkinnyArgs& a, int J) {
  SkJob j;
  if (a.ksplit == 1 && a.npass == 1) {  // the common case: a job is a block
    j.b = J;
    j.p = j.z = 0;
  } else {
    j.z = J % a.ksplit;
    const int r = J / a.ksplit;
    j.p = r % a.npass;
    j.b = r / a.npass;
  }
  j.c0 = j.z * a.chunks_per_split;
  j.c1 = j.c0 + a.chunks_per_split < a.nchunks ? j.c0 + a.chunks_per_split : a.nchunks;
  return j;
}

// The fields the P copies of a chunk read (skinny_kc, skinny_p_ko,
// skinny_issue_p): a caller that issues many chunks of one item keeps them in
// registers (a grouped launch's item is in global memory, and every cp.async
// clobbers memory: read through the item, each chunk would load them again).
struct SkPFields {
  const float* P;
  const int32_t* p_k_off;
  int32_t K, p_walk, p_vec, kr_log2;
};

__device__ __forceinline__ SkPFields skinny_p_fields(const SkinnyArgs& a) {
  return SkPFields{a.P, a.p_k_off, a.K, a.p_walk, a.p_vec, a.kr_log2};
}

template <typename A>
__device__ __forceinline__ int skinny_kc(const A& a, int c) {
  const int64_t k0 = (int64_t)c * SK_KC;
  return a.K - k0 < SK_KC ? (int)(a.K - k0) : SK_KC;
}

// Offsets of block b's box positions (one per thread) into pw / cw, and the
// C offsets of pass p's rows into cs (when the job stores to C).
__device__ __forceinline__ void skinny_begin(const SkinnyArgs& a, int b, int p, int sp,
                                             int32_t* pw, int32_t* cw, int32_t* cs) {
  const int w = threadIdx.x;
  const int ix = a.bxn == 1 ? 0 : b % a.bxn, iy = a.bxn == 1 ? b : b / a.bxn;
  int xl, yl;
  if (a.p_walk == SK_P_Y) {
    yl = w % a.ty;
    xl = w / a.ty;
  } else {
    xl = w % a.tx;
    yl = w / a.tx;
  }
  const int x = ix * a.tx + xl, y = iy * a.ty + yl;
  const bool ok = w < a.tx * a.ty && x < a.ex && y < a.ey;
  pw[w] = ok ? x * a.px + __ldg(a.p_y_off + y) : SK_NONE;
  cw[w] = ok ? x * a.cx + __ldg(a.c_y_off + y) : SK_NONE;
  if (!a.partial && w < a.spr) {
    const int s = p * a.spr + w;
    cs[w] = s < a.S ? __ldg(a.c_s_off + s) : 0;
  }
}

// The P k offset thread tid's copies of chunk c start from: k = tid % kr
// of the chunk for the walk along k, else k = lane (passed around the warp
// by shuffles); 0 past the chunk's extent. A table load whose result the
// copies wait for: callers load it a chunk ahead.
template <typename A>
__device__ __forceinline__ int32_t skinny_p_ko(const A& a, int c) {
  const int tid = threadIdx.x;
  const int kl = a.p_walk == SK_P_K ? tid & ((1 << a.kr_log2) - 1) : tid & 31;
  return kl < skinny_kc(a, c) ? __ldg(a.p_k_off + c * SK_KC + kl) : 0;
}

// Issues the P copies of chunk c ([k][position], k < the chunk's extent) of
// the box whose offsets pw holds (visible to all threads; positions outside
// the tensor are zeros); ko = skinny_p_ko(a, c). Threads 0 .. SK_THREADS - 1
// take part; no commit. SKIP: positions outside the tensor are left
// unwritten (the consumer substitutes zeros for them).
template <bool SKIP = false, typename A = SkinnyArgs>
__device__ __forceinline__ void skinny_issue_p(const A& a, int c, float* ps,
                                               const int32_t* pw, int32_t ko) {
  auto zero = [&](float* d) {
    if (!SKIP) *d = 0.0f;
  };
  const int tid = threadIdx.x;
  const int kc = skinny_kc(a, c);
  // read once: each cp.async clobbers memory, and a grouped launch's item is
  // in global memory, which the compiler would otherwise read again
  const float* const P = a.P;
  if (a.p_walk == SK_P_K) {
    // lanes along k: thread tid takes k = tid % kr of positions tid / kr + i * 256 / kr
    const int lg = a.kr_log2, kl = tid & ((1 << lg) - 1);
    if (kl < kc) {
      float* d = ps + kl * SK_LDP;
#pragma unroll 4
      for (int w = tid >> lg; w < SK_BW; w += SK_THREADS >> lg) {
        const int32_t po = pw[w];
        if (po != SK_NONE)
          cp_async_elem<4>(d + w, P + po + ko);
        else
          zero(d + w);
      }
    }
  } else if (a.p_vec) {
    // four consecutive positions per 16-byte copy where they are consecutive
    // and aligned in P (else four element copies): thread tid takes
    // positions 4 (tid % WG) .. + 3 at k = tid / WG, tid / WG + 4, ...
    const int g = 4 * (tid % SK_WG);
    const int32_t o0 = pw[g], o1 = pw[g + 1], o2 = pw[g + 2], o3 = pw[g + 3];
    const bool vec = o0 != SK_NONE && (o0 & 3) == 0 && o1 == o0 + 1 && o2 == o0 + 2 && o3 == o0 + 3;
    for (int k = tid / SK_WG; k < kc; k += SK_SG) {  // warp-uniform k
      const int32_t kok = __shfl_sync(0xffffffffu, ko, k);
      float* d = ps + k * SK_LDP + g;
      if (vec) {
        cp_async_16(d, P + o0 + kok);
      } else {
        const int32_t o[4] = {o0, o1, o2, o3};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          if (o[e] != SK_NONE)
            cp_async_elem<4>(d + e, P + o[e] + kok);
          else
            zero(d + e);
        }
      }
    }
  } else {
    // lanes along the positions: thread tid takes position tid at every k;
    // the chunk's k offsets are loaded once per warp (lane k) and passed
    // around by shuffles, so no copy waits on a table load
    const int32_t po = pw[tid];
    float* d = ps + tid;
    const float* src = P + (po != SK_NONE ? po : 0);
#pragma unroll 4
    for (int k = 0; k < kc; ++k) {
      const int32_t kok = __shfl_sync(0xffffffffu, ko, k);
      if (po != SK_NONE)
        cp_async_elem<4>(d + k * SK_LDP, src + kok);
      else
        zero(d + k * SK_LDP);
    }
  }
}

// Issues the copies of chunk c of job j (P: [k][position], Q: the pass's
// rows, [k][row]) as one cp.async group; elements outside the tensors are
// zeros. pw must hold the job's box offsets (visible to all threads); ko =
// skinny_p_ko(a, c).
__device__ __forceinline__ void skinny_issue(const SkinnyArgs& a, const SkJob& j, int c, int sp,
                                             float* ps, float* qs, const int32_t* pw, int32_t ko) {
  skinny_issue_p(a, c, ps, pw, ko);
  const int tid = threadIdx.x, lane = tid & 31;
  const int k0 = c * SK_KC;
  const int kc = skinny_kc(a, c);
  // Q rows p spr .. p spr + spr - 1 of k [0, kc) in the pass's sp slots;
  // slots >= spr and rows >= S are zeros
  const int s0 = j.p * a.spr;
  // fields read once (see skinny_issue_p); rows valid below nr
  const float* const Q = a.Q;
  const int32_t* const qso = a.q_s_off + s0;
  const int32_t* const qko = a.q_k_off + k0;
  const int nr = a.S - s0 < a.spr ? a.S - s0 : a.spr;
  if (a.q_kfast) {
    if (lane < kc) {
      const int32_t ko = __ldg(qko + lane);
      for (int r = tid >> 5; r < sp; r += SK_THREADS / 32) {
        float* d = qs + lane * SK_QLD + r;
        if (r < nr)
          cp_async_elem<4>(d, Q + __ldg(qso + r) + ko);
        else
          *d = 0.0f;
      }
    }
  } else {
    for (int r = tid % sp, k = tid / sp; k < kc;) {
      float* d = qs + k * SK_QLD + r;
      if (r < nr)
        cp_async_elem<4>(d, Q + __ldg(qso + r) + __ldg(qko + k));
      else
        *d = 0.0f;
      r += SK_THREADS % sp;
      k += SK_THREADS / sp;
      if (r >= sp) {
        r -= sp;
        ++k;
      }
    }
  }
  cp_async_commit();
}

// One warp's share of a staged plane of L0 x L1 elements (i0 fastest, 32
// consecutive elements per step): element (i, j) is box position w0 + wi i
// + wj j of staged row r0 + ri i + rj j, stored at C + cw[w] + cs[r].
// Positions and rows advance by fixed steps (one carry at most per step).
__device__ __forceinline__ void skinny_plane(const SkinnyArgs& a, const float* os,
                                             const int32_t* cw, const int32_t* cs, int L0, int L1,
                                             int w0, int wi, int wj, int r0, int ri, int rj) {
  const int lane = threadIdx.x & 31;
  const int total = L0 * L1, di = 32 % L0, dj = 32 / L0;
  int i = lane % L0;
  const int j = lane / L0;
  int w = w0 + wi * i + wj * j, r = r0 + ri * i + rj * j;
  const int dw = wi * di + wj * dj, dr = ri * di + rj * dj;
  const int cw_carry = wj - wi * L0, cr_carry = rj - ri * L0;
  const float alpha = a.alpha, beta = a.beta;
  float* const Cb = a.C;  // read once (a grouped launch's item is in global memory)
  for (int f = lane; f < total; f += 32) {
    const int32_t o = cw[w];
    if (o != SK_NONE) {
      float* d = Cb + o + cs[r];
      const float v = alpha * os[r * SK_LDP + w];
      *d = beta != 0.0f ? fmaf(beta, *d, v) : v;
    }
    i += di;
    w += dw;
    r += dr;
    if (i >= L0) {
      i -= L0;
      w += cw_carry;
      r += cr_carry;
    }
  }
}

// Stores staged rows [0, ns) (C rows s0 .. s0 + ns - 1; cs[r] = C offset of
// row s0 + r) in the walk's address order; the NT / 32 warps share the planes.
// Parts of the x range per plane so that a walk of n planes gives every warp
// work: at least 2 NW pieces where the box is flat (few y), at least 32
// positions a piece.
__device__ __forceinline__ int skinny_xparts(int n, int tx, int nw) {
  if (n >= 2 * nw) return 1;
  const int want = (2 * nw + n - 1) / n, most = (tx + 31) / 32;
  return want < most ? want : most;
}

template <int NT = SK_THREADS>
__device__ __forceinline__ void skinny_store(const SkinnyArgs& a, const float* os,
                                             const int32_t* cw, const int32_t* cs, int s0, int ns,
                                             int tid) {
  constexpr int NW = NT / 32;
  const int warp = tid >> 5;
  const bool py = a.p_walk == SK_P_Y;
  const int tx = a.tx, ty = a.ty;
  const int xs = py ? ty : 1;  // position step along x
  if (a.c_walk == SK_C_XS) {
    // (x, s) planes per y, split along x when there are few y (a flat box
    // would leave most warps without a plane)
    const int parts = skinny_xparts(ty, tx, NW), xp = (tx + parts - 1) / parts;
    for (int job = warp; job < ty * parts; job += NW) {
      const int yl = job / parts, x0 = (job % parts) * xp;
      const int xn = tx - x0 < xp ? tx - x0 : xp;
      if (xn > 0)
        skinny_plane(a, os, cw, cs, xn, ns, (py ? yl : tx * yl) + x0 * xs, xs, 0, 0, 0, 1);
    }
  } else if (a.c_walk == SK_C_XY) {
    for (int r = warp; r < ns; r += NW)
      skinny_plane(a, os, cw, cs, tx, ty, 0, xs, py ? 1 : tx, r, 0, 0);
  } else {
    // runs of e0 consecutive rows (C stride one), clipped to [s0, s0 + ns),
    // then x, per y; split along x like the (x, s) planes
    const int e0 = a.s_run;
    const int first = (s0 / e0) * e0;
    const int nruns = (s0 + ns - first + e0 - 1) / e0;
    const int parts = skinny_xparts(nruns * ty, tx, NW), xp = (tx + parts - 1) / parts;
    for (int job = warp; job < nruns * ty * parts; job += NW) {
      const int part = job % parts, rj = job / parts;
      const int run = rj % nruns, yl = rj / nruns;
      const int rs = first + run * e0;
      const int ra = rs > s0 ? rs : s0;
      const int rb = rs + e0 < s0 + ns ? rs + e0 : s0 + ns;
      const int x0 = part * xp, xn = tx - x0 < xp ? tx - x0 : xp;
      if (rb <= ra || xn <= 0) continue;
      skinny_plane(a, os, cw, cs, rb - ra, xn, (py ? yl : tx * yl) + x0 * xs, 0, xs, ra - s0, 1, 0);
    }
  }
}

template <int RS>
struct SkAcc {
  float v[RS][4];
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int i = 0; i < RS; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) v[i][j] = 0.0f;
  }
};

// acc += P chunk (positions 4 wg .. 4 wg + 3) x Q chunk (rows sg RS ..), k < kc
template <int RS>
__device__ __forceinline__ void skinny_fma(SkAcc<RS>& acc, const float* ps, const float* qs, int kc) {
  const int tid = threadIdx.x;
  const float* pp = ps + 4 * (tid % SK_WG);
  const float* qq = qs + (tid / SK_WG) * RS;
#pragma unroll 4
  for (int k = 0; k < kc; ++k) {
    const float4 pv = *reinterpret_cast<const float4*>(pp + k * SK_LDP);
    float q[RS];
#pragma unroll
    for (int i = 0; i < RS; i += 4) {
      const float4 t = *reinterpret_cast<const float4*>(qq + k * SK_QLD + i);
      q[i] = t.x; q[i + 1] = t.y; q[i + 2] = t.z; q[i + 3] = t.w;
    }
#pragma unroll
    for (int i = 0; i < RS; ++i) {
      acc.v[i][0] = fmaf(q[i], pv.x, acc.v[i][0]);
      acc.v[i][1] = fmaf(q[i], pv.y, acc.v[i][1]);
      acc.v[i][2] = fmaf(q[i], pv.z, acc.v[i][2]);
      acc.v[i][3] = fmaf(q[i], pv.w, acc.v[i][3]);
    }
  }
}

// x extent of block b's box inside the tensor.
__device__ __forceinline__ int skinny_box_xn(const SkinnyArgs& a, int b) {
  const int ix = a.bxn == 1 ? 0 : b % a.bxn;
  return a.ex - ix * a.tx < a.tx ? a.ex - ix * a.tx : a.tx;
}

// SK_CLIN_RUNS: stores staged rows [0, ns) (whole runs u = 0 .. ns / e0 - 1
// of C's stride-one S mode, row u e0 + o of position w at os[(u e0 + o)
// SK_LDP + w]) as ranges: run u of box row yl is the xn e0 consecutive floats
// from C + cw(0, yl) + cs[u e0], element f = x e0 + o. A warp per range when
// there are at least NT / 32 ranges, else the whole CTA per range; (x, o)
// and the staging index advance by fixed steps (one carry at most per step).
template <int NT = SK_THREADS>
__device__ __forceinline__ void skinny_copy_runs(const SkinnyArgs& a, const float* os,
                                                 const int32_t* cw, const int32_t* cs, int ns,
                                                 int xn, int tid) {
  constexpr int NW = NT / 32;
  const int e0 = a.s_run, ty = a.ty;
  const bool py = a.p_walk == SK_P_Y;
  const int wx = py ? ty : 1;  // position step along x
  const int n = xn * e0, nr = (ns / e0) * ty;
  const bool per_warp = nr >= NW;
  const int g0 = per_warp ? tid >> 5 : 0, gs = per_warp ? NW : 1;
  const int f0 = per_warp ? tid & 31 : tid, fs = per_warp ? 32 : NT;
  const int dx = fs / e0, dox = fs - dx * e0;
  const int x0 = f0 / e0, o0 = f0 - x0 * e0;
  const int dsi = dox * SK_LDP + dx * wx, csi = wx - e0 * SK_LDP;
  const float alpha = a.alpha, beta = a.beta;
  for (int g = g0; g < nr; g += gs) {
    const int u = g / ty, yl = g - u * ty;
    const int wy = py ? yl : a.tx * yl;  // position (0, yl)
    const int32_t cy = cw[wy];
    if (cy == SK_NONE) continue;  // y past the tensor (uniform per range)
    float* c = a.C + cy + cs[u * e0];
    int o = o0, si = (u * e0 + o0) * SK_LDP + wy + x0 * wx;
    for (int f = f0; f < n; f += fs) {
      const float v = alpha * os[si];
      c[f] = beta != 0.0f ? fmaf(beta, c[f], v) : v;
      o += dox;
      si += dsi;
      if (o >= e0) {
        o -= e0;
        si += csi;
      }
    }
  }
}

// Stores the staged range [0, n) of box row yl (os[f]) at C + base + f; one
// warp per row when there are at least 8 rows, else the whole CTA per row.
// With c_bulk (staged values already scaled by alpha, beta = 0) a row whose
// C start is 16-byte aligned leaves as one bulk copy of its first 4 [n / 4]
// elements (issued by the row's first thread; every address and size a
// multiple of 16 bytes: C, the staging rows and n / 4 quads), the rest by the
// threads.
template <int NT = SK_THREADS>
__device__ __forceinline__ void skinny_copy_rows(const SkinnyArgs& a, const float* os, int plane,
                                                 const int32_t* cw, int32_t cs0, int n, int tid) {
  const int lane = tid & 31, warp = tid >> 5;
  const bool py = a.p_walk == SK_P_Y;
  const bool per_warp = a.ty >= NT / 32;
  const int y0 = per_warp ? warp : 0, ys = per_warp ? NT / 32 : 1;
  const int f0 = per_warp ? lane : tid, fs = per_warp ? 32 : NT;
  const float alpha = a.alpha, beta = a.beta;
  bool issued = false;
  for (int yl = y0; yl < a.ty; yl += ys) {
    const int32_t o = cw[py ? yl : a.tx * yl];  // position (0, yl)
    if (o == SK_NONE) continue;                 // y past the tensor (uniform per row)
    float* c = a.C + o + cs0;
    const float* src = os + yl * plane;
    if (a.c_bulk) {
      const int body = ((o + cs0) & 3) == 0 ? (n & ~3) : 0;
      if (body > 0 && f0 == 0) {
        bulk_store_1d(c, src, (uint32_t)body * 4);
        bulk_commit();
        issued = true;
      }
      for (int f = body + f0; f < n; f += fs) c[f] = src[f];
    } else {
      for (int f = f0; f < n; f += fs) {
        const float v = alpha * src[f];
        c[f] = beta != 0.0f ? fmaf(beta, c[f], v) : v;
      }
    }
  }
  if (issued) bulk_wait_read_all();  // the staging is reused by the next copies
}

// Linear C (SkinnyCLin): the pass's rows are staged per box row yl in C's own
// order -- [s][x] (SK_CLIN_XS, one 32-row step at a time) or [x][s]
// (SK_CLIN_SX, all of S at once) -- and leave as straight copies.
template <int RS>
__device__ __forceinline__ void skinny_finish_lin(const SkinnyArgs& a, const SkJob& j,
                                                  const SkAcc<RS>& acc, float* os,
                                                  const int32_t* cw, const int32_t* cs) {
  constexpr int SP = 4 * RS;
  const int tid = threadIdx.x, wg = tid % SK_WG, sg = tid / SK_WG;
  const bool py = a.p_walk == SK_P_Y;
  const int tx = a.tx, ty = a.ty;
  const bool xs = a.c_lin == SK_CLIN_XS;
  const int plane = xs ? tx * SK_SUB : tx * a.S;
  // staging index of row 0 of the thread's four positions 4 wg .. 4 wg + 3
  // (-1: past the box): y plane + x (XS, rows tx apart) or + x S (SX, rows 1 apart)
  int ob[4];
  {
    const int w = 4 * wg, npos = tx * ty;
    int u = py ? w % ty : w % tx, v = py ? w / ty : w / tx;  // fast / slow index
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int x = py ? v : u, y = py ? u : v;
      ob[e] = w + e < npos ? y * plane + (xs ? x : x * a.S) : -1;
      if (++u == (py ? ty : tx)) {
        u = 0;
        ++v;
      }
    }
  }
  if (xs) {
#pragma unroll 1
    for (int h = 0; h < SP; h += SK_SUB) {
      const int s0 = j.p * SP + h;
      if (s0 >= a.S) break;
      int ns = SP - h < SK_SUB ? SP - h : SK_SUB;
      if (ns > a.S - s0) ns = a.S - s0;
      __syncthreads();  // the stage's last reader is done
      const float sc = a.c_bulk ? a.alpha : 1.0f;
#pragma unroll
      for (int i = 0; i < RS; ++i) {
        const int r = sg * RS + i - h;
        if (r >= 0 && r < SK_SUB) {
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (ob[e] >= 0) os[ob[e] + r * tx] = sc * acc.v[i][e];
        }
      }
      if (a.c_bulk) fence_proxy_async_smem();  // the bulk copies read the staging
      __syncthreads();
      skinny_copy_rows(a, os, plane, cw, cs[h], tx * ns, threadIdx.x);
    }
  } else {  // SK_CLIN_SX: all of S (<= 32 rows) in one step
    const int S = a.S;
    const int ix = a.bxn == 1 ? 0 : j.b % a.bxn;
    const int xn = a.ex - ix * tx < tx ? a.ex - ix * tx : tx;  // x of the box inside the tensor
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RS; ++i) {
      const int r = sg * RS + i;
      if (r < S) {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (ob[e] >= 0) os[ob[e] + r] = acc.v[i][e];
      }
    }
    __syncthreads();
    skinny_copy_rows(a, os, plane, cw, cs[0], xn * S, threadIdx.x);
  }
}

// The end of job j: raw sums to its k slice, or its pass's rows to C staged
// 32 at a time through os (the P stage just consumed).
template <int RS>
__device__ __forceinline__ void skinny_finish(const SkinnyArgs& a, const SkJob& j, const SkAcc<RS>& acc,
                                              float* os, const int32_t* cw, const int32_t* cs) {
  constexpr int SP = 4 * RS;
  const int tid = threadIdx.x, wg = tid % SK_WG, sg = tid / SK_WG;
  if (a.partial) {
    float* dst = a.partial + (((size_t)j.z * a.nblk + j.b) * a.npass + j.p) * SP * SK_BW + 4 * wg;
#pragma unroll
    for (int i = 0; i < RS; ++i)
      *reinterpret_cast<float4*>(dst + (size_t)(sg * RS + i) * SK_BW) =
          make_float4(acc.v[i][0], acc.v[i][1], acc.v[i][2], acc.v[i][3]);
    return;
  }
  if (a.c_lin == SK_CLIN_XS || a.c_lin == SK_CLIN_SX) {
    skinny_finish_lin<RS>(a, j, acc, os, cw, cs);
    return;
  }
#pragma unroll 1
  for (int h = 0; h < a.spr; h += SK_SUB) {
    const int s0 = j.p * a.spr + h;
    if (s0 >= a.S) break;
    int ns = a.spr - h < SK_SUB ? a.spr - h : SK_SUB;
    if (ns > a.S - s0) ns = a.S - s0;
    __syncthreads();  // the stage's last reader (the FMAs, or the previous step's stores) is done
#pragma unroll
    for (int i = 0; i < RS; ++i) {
      const int r = sg * RS + i - h;
      if (r >= 0 && r < SK_SUB)
        *reinterpret_cast<float4*>(os + r * SK_LDP + 4 * wg) =
            make_float4(acc.v[i][0], acc.v[i][1], acc.v[i][2], acc.v[i][3]);
    }
    __syncthreads();
    if (a.c_lin == SK_CLIN_RUNS)
      skinny_copy_runs(a, os, cw, cs, ns, skinny_box_xn(a, j.b), threadIdx.x);
    else
      skinny_store(a, os, cw, cs + h, s0, ns, threadIdx.x);
  }
}

// A CTA's sequence of jobs: global job indices j0, j0 + jstep, ... < njobs;
// resolve(J) gives the job's item (its SkinnyArgs) and its index in the item.
struct SkRef {
  const SkinnyArgs* a;
  int J;
};

template <int RS, typename Resolve>
__device__ __forceinline__ void skinny_loop(int j0, int jstep, int njobs, Resolve&& resolve,
                                            uint8_t* smem) {
  constexpr int SP = 4 * RS;
  float* Ps = reinterpret_cast<float*>(smem);
  float* Qs = reinterpret_cast<float*>(smem + 2 * SK_P_STAGE);
  int32_t* pw = reinterpret_cast<int32_t*>(smem + SK_OFF_TAB);  // [2][BW]
  int32_t* cw = pw + 2 * SK_BW;                                  // [2][BW]
  int32_t* cs = cw + 2 * SK_BW;                                  // [2][SPMAX]
  if (j0 >= njobs) return;
  // loop state: the current step (job jg of this CTA's sequence, chunk c of
  // its [.., c1)), its P / Q stage st and its job's offset slot; the job's
  // fields are recomputed where needed (fewer registers across the FMAs)
  int jg = j0;
  SkRef cur = resolve(jg);
  int c, c1;
  {
    const SkJob job = skinny_job(*cur.a, cur.J);
    c = job.c0;
    c1 = job.c1;
    skinny_begin(*cur.a, job.b, job.p, SP, pw, cw, cs);
    __syncthreads();
    skinny_issue(*cur.a, job, c, SP, Ps, Qs, pw, skinny_p_ko(*cur.a, c));
  }
  int st = 0, slot = 0;
  SkAcc<RS> acc;
  acc.clear();
#pragma unroll 1
  while (true) {
    // the step after: the job's next chunk, or the next job's first
    const bool last = c + 1 >= c1;
    const int jn = last ? jg + jstep : jg;
    const bool has_next = jn < njobs;
    SkRef nref = cur;
    int nc = c + 1, nc1 = c1;
    __syncthreads();  // stage st ^ 1 and job slot slot ^ 1 are free
    if (has_next) {
      const int ns = last ? slot ^ 1 : slot;
      if (last) nref = resolve(jn);
      const SkJob njob = skinny_job(*nref.a, nref.J);
      if (last) {
        nc = njob.c0;
        nc1 = njob.c1;
        skinny_begin(*nref.a, njob.b, njob.p, SP, pw + ns * SK_BW, cw + ns * SK_BW,
                     cs + ns * SK_SPMAX);
        // the copies below read other threads' box offsets only along k or
        // in 16-byte groups; otherwise each thread reads its own
        if (nref.a->p_walk == SK_P_K || nref.a->p_vec) __syncthreads();
      }
      skinny_issue(*nref.a, njob, nc, SP, Ps + (st ^ 1) * (SK_P_STAGE / 4),
                   Qs + (st ^ 1) * (SK_Q_STAGE / 4), pw + ns * SK_BW, skinny_p_ko(*nref.a, nc));
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();  // chunk c is in stage st
    float* ps = Ps + st * (SK_P_STAGE / 4);
    skinny_fma<RS>(acc, ps, Qs + st * (SK_Q_STAGE / 4), skinny_kc(*cur.a, c));
    if (last) {
      skinny_finish<RS>(*cur.a, skinny_job(*cur.a, cur.J), acc, ps, cw + slot * SK_BW,
                        cs + slot * SK_SPMAX);
      acc.clear();
    }
    if (!has_next) break;
    if (last) {
      slot ^= 1;
      jg = jn;
    }
    cur = nref;
    c = nc;
    c1 = nc1;
    st ^= 1;
  }
}

// C of pass p of block b = alpha * (slice 0 + slice 1 + ...) + beta * C,
// slices in order; r = b npass + p.
template <int RS>
__device__ __forceinline__ void skinny_reduce_block(const SkinnyArgs& a, int r, uint8_t* smem) {
  constexpr int SP = 4 * RS;
  static_assert(SP <= 2 * SK_SPMAX, "the rows' C offsets fit the two offset slots");
  float* os = reinterpret_cast<float*>(smem);
  int32_t* pw = reinterpret_cast<int32_t*>(smem + SK_OFF_TAB);
  int32_t* cw = pw + 2 * SK_BW;
  int32_t* cs = cw + 2 * SK_BW;
  const int tid = threadIdx.x;
  const int b = r / a.npass, p = r % a.npass;
  SkinnyArgs ac = a;
  ac.partial = nullptr;  // stage the rows' C offsets
  skinny_begin(ac, b, p, SP, pw, cw, cs);
  const size_t slice = (size_t)a.nblk * a.npass * SP * SK_BW;
  const float* src = a.partial + (size_t)r * SP * SK_BW + tid;
#pragma unroll 1
  for (int h = 0; h < a.spr; h += SK_SUB) {
    const int s0 = p * a.spr + h;
    if (s0 >= a.S) break;
    int ns = a.spr - h < SK_SUB ? a.spr - h : SK_SUB;
    if (ns > a.S - s0) ns = a.S - s0;
    __syncthreads();
    for (int rr = 0; rr < ns; ++rr) {
      const float* q = src + (size_t)(h + rr) * SK_BW;
      float v = q[0];
      for (int z = 1; z < a.ksplit; ++z) v = __fadd_rn(v, q[z * slice]);
      os[rr * SK_LDP + tid] = v;
    }
    __syncthreads();
    if (a.c_lin == SK_CLIN_RUNS)
      skinny_copy_runs(a, os, cw, cs, ns, skinny_box_xn(a, b), threadIdx.x);
    else
      skinny_store(a, os, cw, cs + h, s0, ns, threadIdx.x);
  }
}

template <typename F>
__device__ __forceinline__ void skinny_dispatch(int rs, F&& f) {
  switch (rs) {
    case 4: f(std::integral_constant<int, 4>()); break;
    case 8: f(std::integral_constant<int, 8>()); break;
    default: f(std::integral_constant<int, 12>()); break;
  }
}

// The reductions also serve the tensor-core kernel's slices (skinny_tc.cuh:
// one pass of up to 64 rows, RS = 16).
template <typename F>
__device__ __forceinline__ void skinny_reduce_dispatch(int rs, F&& f) {
  switch (rs) {
    case 4: f(std::integral_constant<int, 4>()); break;
    case 8: f(std::integral_constant<int, 8>()); break;
    case 12: f(std::integral_constant<int, 12>()); break;
    default: f(std::integral_constant<int, 16>()); break;
  }
}

// A grouped launch's item (see the grouped kernels below).
struct SkinnyItem {
  SkinnyArgs args;
  int64_t begin;
};

// ---- register path: a narrow side of at most 16 rows ------------------------
// With 4 rows per thread the tile path reads each staged P value four times
// from shared memory (once per row group): 5 shared-memory wavefronts per 16
// FMAs of a warp, more than the FMA pipe's time for them, and its copies land
// through the same L1 data path, so copies and FMAs queue behind each other.
// Here P goes from global memory straight to registers: 128 threads, thread t
// owns positions t and t + 128 of the block and all 16 rows (32 sums); each
// step of 16 k loads the next step's 2 x 16 P values while it multiplies the
// current ones with the step's Q values, broadcast from shared memory (4
// wavefronts per 32 FMAs of a warp). Same boxes, jobs, k slices and C stores
// as the tile path (rows staged in shared memory, then the store walks or the
// linear / bulk copies); four CTAs per SM.
constexpr int SKR_THREADS = 128;
constexpr int SKR_ROWS = 16;
constexpr int SKR_KR = 16;  // k per step
constexpr size_t SKR_OFF_OS = (size_t)2 * SKR_KR * SKR_ROWS * 4;  // after Qs[2][KR][ROWS]
constexpr size_t SKR_OFF_TAB = SKR_OFF_OS + (size_t)SKR_ROWS * SK_LDP * 4;
constexpr size_t SKR_SMEM_BYTES = SKR_OFF_TAB + (size_t)(4 * SK_BW + 2 * SKR_ROWS) * 4;
constexpr int SKR_CTAS_PER_SM = 4;
static_assert(SK_BW == 2 * SKR_THREADS, "two positions per thread");
static_assert(SKR_CTAS_PER_SM * (SKR_SMEM_BYTES + 1024) <= 228 * 1024, "CTAs per SM");

// Box offsets of positions w = tid, tid + 128 and the C offsets of the 16 rows.
__device__ __forceinline__ void skinny_reg_begin(const SkinnyArgs& a, int b, int32_t* pw,
                                                 int32_t* cw, int32_t* cs) {
  const int ix = a.bxn == 1 ? 0 : b % a.bxn, iy = a.bxn == 1 ? b : b / a.bxn;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int w = threadIdx.x + h * SKR_THREADS;
    int xl, yl;
    if (a.p_walk == SK_P_Y) {
      yl = w % a.ty;
      xl = w / a.ty;
    } else {
      xl = w % a.tx;
      yl = w / a.tx;
    }
    const int x = ix * a.tx + xl, y = iy * a.ty + yl;
    const bool ok = w < a.tx * a.ty && x < a.ex && y < a.ey;
    pw[w] = ok ? x * a.px + __ldg(a.p_y_off + y) : SK_NONE;
    cw[w] = ok ? x * a.cx + __ldg(a.c_y_off + y) : SK_NONE;
  }
  if (!a.partial && threadIdx.x < SKR_ROWS) {
    const int s = threadIdx.x;
    cs[s] = s < a.S ? __ldg(a.c_s_off + s) : 0;
  }
}

// Q rows 0..ROWS-1 of k [kb, kb + 16) into qs[k][row] (zeros past S or ke).
template <int ROWS>
__device__ __forceinline__ void skinny_reg_q(const SkinnyArgs& a, int kb, int ke, float* qs) {
  // fields read once (each cp.async clobbers memory; a grouped item is in
  // global memory)
  const float* const Q = a.Q;
  const int32_t* const qso = a.q_s_off;
  const int32_t* const qko = a.q_k_off + kb;
  const int S = a.S;
#pragma unroll
  for (int i = 0; i < SKR_KR * ROWS / SKR_THREADS; ++i) {
    const int e = threadIdx.x + i * SKR_THREADS;
    const int kk = e / ROWS, r = e % ROWS;
    float* d = qs + e;
    if (r < S && kb + kk < ke)
      cp_async_elem<4>(d, Q + __ldg(qso + r) + __ldg(qko + kk));
    else
      *d = 0.0f;
  }
  cp_async_commit();
}

// The P k offset of k = kb + lane (lanes < 16, k < ke; else 0): loaded a
// step ahead of the copies that use it.
__device__ __forceinline__ int32_t skinny_reg_ko(const SkinnyArgs& a, int kb, int ke) {
  const int lane = threadIdx.x & 31;
  return lane < SKR_KR && kb + lane < ke ? __ldg(a.p_k_off + kb + lane) : 0;
}

// P of the thread's two positions at k [kb, kb + 16) (zeros past ke or the
// box); ko_lane = skinny_reg_ko(a, kb, ke).
__device__ __forceinline__ void skinny_reg_p(const SkinnyArgs& a, int kb, int ke, int32_t po0,
                                             int32_t po1, float (&p0)[SKR_KR], float (&p1)[SKR_KR],
                                             int32_t ko_lane) {
#pragma unroll
  for (int kk = 0; kk < SKR_KR; ++kk) {
    const int32_t ko = __shfl_sync(0xffffffffu, ko_lane, kk);
    const bool kok = kb + kk < ke;
    p0[kk] = kok && po0 != SK_NONE ? __ldg(a.P + po0 + ko) : 0.0f;
    p1[kk] = kok && po1 != SK_NONE ? __ldg(a.P + po1 + ko) : 0.0f;
  }
}

// The end of a job: raw sums to its k slice, or the rows to C (staged in os).
template <int ROWS>
__device__ __forceinline__ void skinny_reg_finish(const SkinnyArgs& a, const SkJob& j,
                                                  const float (&acc)[2][ROWS], float* os,
                                                  const int32_t* cw, const int32_t* cs) {
  const int tid = threadIdx.x;
  if (a.partial) {  // layout of the 16-row (RS = 4) tile path; rows >= ROWS not written
    float* dst = a.partial + (((size_t)j.z * a.nblk + j.b) * a.npass + j.p) * SKR_ROWS * SK_BW + tid;
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
      dst[(size_t)r * SK_BW] = acc[0][r];
      dst[(size_t)r * SK_BW + SKR_THREADS] = acc[1][r];
    }
    return;
  }
  const int S = a.S;
  if (a.c_lin != SK_CLIN_NONE) {
    // staged per box row in C's order: [s][x] (XS, rows tx apart) or [x][s] (SX)
    const bool py = a.p_walk == SK_P_Y, xs = a.c_lin == SK_CLIN_XS;
    const int tx = a.tx, ty = a.ty, plane = tx * (xs ? SKR_ROWS : S);
    const float sc = a.c_bulk ? a.alpha : 1.0f;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int w = tid + h * SKR_THREADS;
      if (w >= tx * ty) continue;
      const int xl = py ? w / ty : w % tx, yl = py ? w % ty : w / tx;
      float* o = os + yl * plane + (xs ? xl : xl * S);
#pragma unroll
      for (int r = 0; r < ROWS; ++r)
        if (r < S) o[xs ? r * tx : r] = sc * acc[h][r];
    }
    if (a.c_bulk) fence_proxy_async_smem();
    __syncthreads();
    if (xs) {
      skinny_copy_rows<SKR_THREADS>(a, os, plane, cw, cs[0], tx * S, tid);
    } else {
      const int ix = a.bxn == 1 ? 0 : j.b % a.bxn;
      const int xn = a.ex - ix * tx < tx ? a.ex - ix * tx : tx;
      skinny_copy_rows<SKR_THREADS>(a, os, plane, cw, cs[0], xn * S, tid);
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < ROWS; ++r) {
    os[r * SK_LDP + tid] = acc[0][r];
    os[r * SK_LDP + tid + SKR_THREADS] = acc[1][r];
  }
  __syncthreads();
  skinny_store<SKR_THREADS>(a, os, cw, cs, 0, S, tid);
}

// One job of the register path with ROWS computed rows (16, or 8 for a
// narrow side of at most 8: half the FMAs and Q copies).
template <int ROWS>
__device__ __forceinline__ void skinny_reg_job(const SkinnyArgs& a, const SkJob& job, float* Qs,
                                               float* os, const int32_t* pw, const int32_t* cw,
                                               const int32_t* cs) {
  const int tid = threadIdx.x;
  const int32_t po0 = pw[tid], po1 = pw[tid + SKR_THREADS];
  const int kbeg = job.c0 * SK_KC;
  const int kend = job.c1 * SK_KC < a.K ? job.c1 * SK_KC : a.K;
  float acc[2][ROWS];
#pragma unroll
  for (int r = 0; r < ROWS; ++r) acc[0][r] = acc[1][r] = 0.0f;
  float pc0[SKR_KR], pc1[SKR_KR];
  skinny_reg_q<ROWS>(a, kbeg, kend, Qs);
  skinny_reg_p(a, kbeg, kend, po0, po1, pc0, pc1, skinny_reg_ko(a, kbeg, kend));
  int32_t ko_next = skinny_reg_ko(a, kbeg + SKR_KR, kend);  // the next step's
  int st = 0;
#pragma unroll 1
  for (int kb = kbeg; kb < kend; kb += SKR_KR) {
    const int nb = kb + SKR_KR;
    float pn0[SKR_KR], pn1[SKR_KR];
    if (nb < kend) {
      __syncthreads();  // stage st ^ 1 was read by the previous step
      skinny_reg_q<ROWS>(a, nb, kend, Qs + (st ^ 1) * SKR_KR * SKR_ROWS);
      skinny_reg_p(a, nb, kend, po0, po1, pn0, pn1, ko_next);
      ko_next = skinny_reg_ko(a, nb + SKR_KR, kend);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();  // Q of this step landed
    const float* q = Qs + st * SKR_KR * SKR_ROWS;
#pragma unroll
    for (int kk = 0; kk < SKR_KR; ++kk) {
      float qv[ROWS];
#pragma unroll
      for (int r = 0; r < ROWS; r += 4) {
        const float4 t = *reinterpret_cast<const float4*>(q + kk * ROWS + r);
        qv[r] = t.x; qv[r + 1] = t.y; qv[r + 2] = t.z; qv[r + 3] = t.w;
      }
#pragma unroll
      for (int r = 0; r < ROWS; ++r) {
        acc[0][r] = fmaf(qv[r], pc0[kk], acc[0][r]);
        acc[1][r] = fmaf(qv[r], pc1[kk], acc[1][r]);
      }
    }
    if (nb < kend) {
#pragma unroll
      for (int kk = 0; kk < SKR_KR; ++kk) {
        pc0[kk] = pn0[kk];
        pc1[kk] = pn1[kk];
      }
    }
    st ^= 1;
  }
  skinny_reg_finish<ROWS>(a, job, acc, os, cw, cs);
}

template <int ROWS, typename Resolve>
__device__ __forceinline__ void skinny_reg_loop(int j0, int jstep, int njobs, Resolve&& resolve,
                                                uint8_t* smem) {
  float* Qs = reinterpret_cast<float*>(smem);  // [2][KR][ROWS], stages SKR_ROWS rows apart
  float* os = reinterpret_cast<float*>(smem + SKR_OFF_OS);
  int32_t* pw = reinterpret_cast<int32_t*>(smem + SKR_OFF_TAB);
  int32_t* cw = pw + SK_BW;
  int32_t* cs = cw + SK_BW;
#pragma unroll 1
  for (int jg = j0; jg < njobs; jg += jstep) {
    const SkRef ref = resolve(jg);
    const SkinnyArgs& a = *ref.a;
    const SkJob job = skinny_job(a, ref.J);
    __syncthreads();  // the previous job's stores are done with os, pw, cw, cs
    skinny_reg_begin(a, job.b, pw, cw, cs);
    __syncthreads();
    skinny_reg_job<ROWS>(a, job, Qs, os, pw, cw, cs);
  }
}

// ROWS = 16, or 8 for a narrow side of at most 8 (one kernel per row count:
// both in one kernel would need more registers than four CTAs per SM leave)
template <int ROWS>
__global__ void __launch_bounds__(SKR_THREADS, SKR_CTAS_PER_SM)
    skinny_reg_kernel(const __grid_constant__ SkinnyArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  grid_dep_wait();
  auto resolve = [&](int J) { return SkRef{&a, J}; };
  skinny_reg_loop<ROWS>(blockIdx.x, gridDim.x, a.njobs, resolve, smem);
  bulk_wait_all();  // bulk C copies complete before the CTA exits
}

template <int ROWS>
__global__ void __launch_bounds__(SKR_THREADS, SKR_CTAS_PER_SM)
    skinny_reg_group_kernel(const SkinnyItem* items, const int64_t* begin, int n, int njobs) {
  extern __shared__ __align__(16) uint8_t smem[];
  auto resolve = [&](int J) {
    const SkinnyItem& it = items[find_segment(begin, n, J)];
    return SkRef{&it.args, (int)(J - it.begin)};
  };
  skinny_reg_loop<ROWS>(blockIdx.x, gridDim.x, njobs, resolve, smem);
  bulk_wait_all();
}

// persistent grid (SK_CTAS_PER_SM CTAs per SM) over the plan's jobs; one
// instantiation per rows-per-thread class (RS = a.rs)
template <int RS>
__global__ void __launch_bounds__(SK_THREADS, SK_CTAS_PER_SM)
    skinny_gett_kernel(const __grid_constant__ SkinnyArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  grid_dep_wait();
  auto resolve = [&](int J) { return SkRef{&a, J}; };
  skinny_loop<RS>(blockIdx.x, gridDim.x, a.njobs, resolve, smem);
  bulk_wait_all();  // bulk C copies complete before the CTA exits
}

// grid (blocks x passes)
__global__ void __launch_bounds__(SK_THREADS, SK_CTAS_PER_SM)
    skinny_reduce_kernel(const __grid_constant__ SkinnyArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  grid_dep_wait();  // slices written by the kernel before
  skinny_reduce_dispatch(a.rs, [&](auto r) { skinny_reduce_block<decltype(r)::value>(a, blockIdx.x, smem); });
}

// Grouped launches. Contraction items: item i owns the global job indices
// [begin[i], begin[i + 1]); one persistent launch per rows-per-thread class
// (RS = the items' rs) walks all of them. Reduction items:
// CTAs [begin[i], begin[i + 1]) are the (block, pass) pairs of a k-split item.

template <int RS>
__global__ void __launch_bounds__(SK_THREADS, SK_CTAS_PER_SM)
    skinny_group_kernel(const SkinnyItem* items, const int64_t* begin, int n, int njobs) {
  extern __shared__ __align__(16) uint8_t smem[];
  auto resolve = [&](int J) {
    const SkinnyItem& it = items[find_segment(begin, n, J)];
    return SkRef{&it.args, (int)(J - it.begin)};
  };
  skinny_loop<RS>(blockIdx.x, gridDim.x, njobs, resolve, smem);
  bulk_wait_all();  // bulk C copies complete before the CTA exits
}

__global__ void __launch_bounds__(SK_THREADS, SK_CTAS_PER_SM)
    skinny_reduce_group_kernel(const SkinnyItem* items, const int64_t* begin, int n) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int64_t t = blockIdx.x;
  const SkinnyItem& it = items[find_segment(begin, n, t)];
  skinny_reduce_dispatch(it.args.rs, [&](auto r) {
    skinny_reduce_block<decltype(r)::value>(it.args, (int)(t - it.begin), smem);
  });
}

}  // namespace tccg
