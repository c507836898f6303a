// Skinny GETT: contractions with one small free extent, FP32 on the CUDA cores.
//
// When one GETT extent -- M or N, the narrow side S -- is small, the
// contraction has few FMAs per byte: the wide operand P (W rows x K) and C
// (W x S) dominate, and each should cross HBM once. The tile kernels pad S
// to their tile width and, for most layouts, pay a packing pass that
// transposes P first. This kernel keeps the narrow operand Q (S x K) in
// shared memory chunk by chunk (every CTA reads it, from L2), streams P
// straight from the caller's tensor and writes every element of C once, in
// C's own layout -- the GETT property of TCCG's micro-kernel (C written in
// its original layout, tccg/gett.py:192-223), with TCCG's packing step
// (tccg/gett.py:440-470) replaced by loads that follow P's layout.
//
// W blocking. The W modes split into X -- the W mode C stores contiguously
// (its smallest C stride) -- and the Y space: all other W modes, linearised
// in order of increasing P stride. A block is a box of tx x ty positions
// (x, y), tx * ty <= 256:
//   P(x, y, k) = P[x px + p_y_off[y] + p_k_off[k]]
//   Q(s, k)    = Q[q_s_off[s] + q_k_off[k]]
//   C(x, y, s) = C[x cx + c_y_off[y] + c_s_off[s]]
// When P's stride-one W mode is not X (P and C order the W modes
// differently: a transposition), the box spans X and the first Y mode, so
// the P loads run along y and the C stores along x, each over runs of the
// box's extent.
//
// Per block (256 threads, two CTAs per SM): K in chunks of 32, double
// buffered through element-wise cp.async (no packing pass, no alignment
// requirement); thread (wg, sg) accumulates 4 positions x RS rows of S
// (RS = 4, 8, 12 or 16; a pass covers 4 RS rows) in FP32 FMAs, k in
// increasing order. S up to 64 takes one pass; up to 256 several passes over
// one chunk when K <= 32. The epilogue stages 32 rows at a time in shared
// memory and stores them in C's address order (SK_C_*), alpha * acc, then
// fma with beta * C (not read when beta = 0).
//
// With a k-split (few blocks, long K: a matrix-vector shape) split z writes
// its raw sums densely to partial[z][block][row][position] and
// skinny_reduce_kernel adds the slices in split order before the same store
// walk. Results are deterministic: a fixed k order within a slice, slices in
// order.
#pragma once
#include <cuda.h>
#include "common.cuh"

namespace tccg {

constexpr int SK_THREADS = 256;
constexpr int SK_BW = 256;             // box positions per block (one per thread)
constexpr int SK_KC = 32;              // k per chunk
constexpr int SK_LDP = SK_BW + 4;      // P stage row stride (floats): [k][position]
constexpr int SK_SMAX = 256;           // largest narrow extent
constexpr int SK_SUB = 32;             // rows of S staged per epilogue step
constexpr int SK_QCAP = SK_KC * (SK_SMAX + 4);  // floats of the Q region
// shared memory: P stages [2][KC][LDP], Q region, then position / row offsets
constexpr size_t SK_P_BYTES = (size_t)2 * SK_KC * SK_LDP * 4;
constexpr size_t SK_Q_BYTES = (size_t)SK_QCAP * 4;
constexpr size_t SK_SMEM_BYTES = SK_P_BYTES + SK_Q_BYTES + (size_t)(2 * SK_BW + SK_SMAX) * 8;
static_assert(SK_SUB == SK_KC, "the epilogue staging reuses one P stage");
static_assert(2 * (SK_SMEM_BYTES + 1024) <= 228 * 1024, "two CTAs per SM");

// P load order: lanes along x (X is P's stride-one W mode), along y (the
// first Y mode is), or along k (a K mode is). Box positions are numbered
// x-fastest (SK_P_X, SK_P_K) or y-fastest (SK_P_Y).
enum SkinnyPWalk : int { SK_P_X = 0, SK_P_Y = 1, SK_P_K = 2 };
// C store order of a staged step: (x, s) planes per y (C's next stride after
// X is S's); (x, y) planes per s (it is a Y mode's); runs of C's stride-one
// S mode, then x, per y (C's stride-one index is on the narrow side).
enum SkinnyCWalk : int { SK_C_XS = 0, SK_C_XY = 1, SK_C_SX = 2 };

struct SkinnyArgs {
  const float* P;
  const float* Q;
  float* C;
  const int64_t* p_y_off;  // [ey]
  const int64_t* c_y_off;  // [ey]
  const int64_t* p_k_off;  // [K]
  const int64_t* q_s_off;  // [S]
  const int64_t* q_k_off;  // [K]
  const int64_t* c_s_off;  // [S]
  int64_t px, cx;          // P and C strides of X
  int64_t ex, ey;          // extents of X and of the Y space
  int64_t nblk;            // boxes: bxn along x, ceil(ey / ty) along y
  int32_t tx, ty, bxn;
  int32_t S, K;
  int32_t rs;              // rows of S per thread; a pass covers 4 * rs rows
  int32_t npass;           // passes over S (> 1 only with one chunk, no k-split)
  int32_t nchunks, chunks_per_split;
  int32_t kr_log2;         // SK_P_K: log2 of the lanes along k per position
  int32_t p_walk, c_walk;
  int32_t q_kfast;         // Q loads along k (its stride-one index is a K mode)
  int32_t s_run;           // SK_C_SX: extent of C's stride-one S mode
  float alpha, beta;
  float* partial;          // k-split slices (null: store to C)
};

constexpr int64_t SK_NONE = INT64_MIN;  // position outside the tensor (offsets may be negative)

// Offsets of this block's box positions (one per thread) into pw / cw.
__device__ __forceinline__ void skinny_box(const SkinnyArgs& a, int64_t b, int64_t* pw,
                                           int64_t* cw) {
  const int w = threadIdx.x;
  const int64_t ix = b % a.bxn, iy = b / a.bxn;
  int xl, yl;
  if (a.p_walk == SK_P_Y) {
    yl = w % a.ty;
    xl = w / a.ty;
  } else {
    xl = w % a.tx;
    yl = w / a.tx;
  }
  const int64_t x = ix * a.tx + xl, y = iy * a.ty + yl;
  const bool ok = w < a.tx * a.ty && x < a.ex && y < a.ey;
  pw[w] = ok ? x * a.px + __ldg(a.p_y_off + y) : SK_NONE;
  cw[w] = ok ? x * a.cx + __ldg(a.c_y_off + y) : SK_NONE;
}

// Box position of (xl, yl) in the block's numbering.
__device__ __forceinline__ int skinny_pos(const SkinnyArgs& a, int xl, int yl) {
  return a.p_walk == SK_P_Y ? yl + a.ty * xl : xl + a.tx * yl;
}

// Issues the copies of chunk c (P: [k][position], Q: [k][row], qld floats
// per k) as one cp.async group; elements outside the tensors are zeros.
__device__ __forceinline__ void skinny_load(const SkinnyArgs& a, int c, float* ps, float* qs,
                                            int sq, int qld, const int64_t* pw) {
  const int tid = threadIdx.x;
  const int64_t k0 = (int64_t)c * SK_KC;
  const int kc = a.K - k0 < SK_KC ? (int)(a.K - k0) : SK_KC;
  if (a.p_walk == SK_P_K) {
    // lanes along k: thread tid takes k = tid % kr of positions tid / kr + j * 256 / kr
    const int lg = a.kr_log2, kl = tid & ((1 << lg) - 1);
    if (kl < kc) {
      const int64_t ko = __ldg(a.p_k_off + k0 + kl);
      float* d = ps + kl * SK_LDP;
#pragma unroll 4
      for (int w = tid >> lg; w < SK_BW; w += SK_THREADS >> lg) {
        const int64_t po = pw[w];
        if (po != SK_NONE)
          cp_async_elem<4>(d + w, a.P + po + ko);
        else
          d[w] = 0.0f;
      }
    }
  } else {
    // lanes along the positions: thread tid takes position tid at every k
    const int64_t po = pw[tid];
    float* d = ps + tid;
    if (po != SK_NONE) {
      const float* src = a.P + po;
#pragma unroll 4
      for (int k = 0; k < kc; ++k) cp_async_elem<4>(d + k * SK_LDP, src + __ldg(a.p_k_off + k0 + k));
    } else {
      for (int k = 0; k < kc; ++k) d[k * SK_LDP] = 0.0f;
    }
  }
  // Q rows [0, sq) of k [0, kc); rows >= S are zeros
  if (a.q_kfast) {
    const int kl = tid & 31;
    if (kl < kc) {
      const int64_t ko = __ldg(a.q_k_off + k0 + kl);
      for (int s = tid >> 5; s < sq; s += SK_THREADS / 32) {
        float* d = qs + kl * qld + s;
        if (s < a.S)
          cp_async_elem<4>(d, a.Q + __ldg(a.q_s_off + s) + ko);
        else
          *d = 0.0f;
      }
    }
  } else {
    for (int s = tid % sq, k = tid / sq; k < kc;) {
      float* d = qs + k * qld + s;
      if (s < a.S)
        cp_async_elem<4>(d, a.Q + __ldg(a.q_s_off + s) + __ldg(a.q_k_off + k0 + k));
      else
        *d = 0.0f;
      s += SK_THREADS % sq;
      k += SK_THREADS / sq;
      if (s >= sq) {
        s -= sq;
        ++k;
      }
    }
  }
  cp_async_commit();
}

// Stores staged rows [s0, s0 + ns) of S (os[row - s0][position]) to C in
// the walk's address order; 8 warps share the planes.
__device__ __forceinline__ void skinny_store(const SkinnyArgs& a, const float* os,
                                             const int64_t* cw, const int64_t* cs, int s0, int ns) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const float alpha = a.alpha, beta = a.beta;
  auto put = [&](int w, int r) {
    const int64_t o = cw[w];
    if (o == SK_NONE) return;
    float* d = a.C + o + cs[s0 + r];
    const float v = alpha * os[r * SK_LDP + w];
    *d = beta != 0.0f ? fmaf(beta, *d, v) : v;
  };
  // plane of L0 x L1 elements (i0 fastest), 32 consecutive per step
  auto plane = [&](int L0, int L1, auto&& elem) {
    const int total = L0 * L1, di = 32 % L0, dj = 32 / L0;
    int i = lane % L0, j = lane / L0;
    for (int f = lane; f < total; f += 32) {
      elem(i, j);
      i += di;
      j += dj;
      if (i >= L0) {
        i -= L0;
        ++j;
      }
    }
  };
  if (a.c_walk == SK_C_XS) {
    for (int yl = warp; yl < a.ty; yl += SK_THREADS / 32)
      plane(a.tx, ns, [&](int xl, int r) { put(skinny_pos(a, xl, yl), r); });
  } else if (a.c_walk == SK_C_XY) {
    for (int r = warp; r < ns; r += SK_THREADS / 32)
      plane(a.tx, a.ty, [&](int xl, int yl) { put(skinny_pos(a, xl, yl), r); });
  } else {
    // runs of e0 consecutive rows (C stride one), clipped to [s0, s0 + ns)
    const int e0 = a.s_run;
    const int first = (s0 / e0) * e0;
    const int nruns = (s0 + ns - first + e0 - 1) / e0;
    for (int job = warp; job < nruns * a.ty; job += SK_THREADS / 32) {
      const int run = job % nruns, yl = job / nruns;
      const int rs = first + run * e0;
      const int ra = rs > s0 ? rs : s0;
      const int rb = rs + e0 < s0 + ns ? rs + e0 : s0 + ns;
      if (rb <= ra) continue;
      plane(rb - ra, a.tx, [&](int i, int xl) { put(skinny_pos(a, xl, yl), ra - s0 + i); });
    }
  }
}

// One block of split z (partial != null) or of the whole K.
template <int RS>
__device__ __forceinline__ void skinny_block(const SkinnyArgs& a, int64_t b, int z, uint8_t* smem) {
  constexpr int SP = 4 * RS;
  float* Ps = reinterpret_cast<float*>(smem);
  float* Qs = reinterpret_cast<float*>(smem + SK_P_BYTES);
  int64_t* pw = reinterpret_cast<int64_t*>(smem + SK_P_BYTES + SK_Q_BYTES);
  int64_t* cw = pw + SK_BW;
  int64_t* cs = cw + SK_BW;
  const int tid = threadIdx.x;
  const int wg = tid & 63, sg = tid >> 6;  // positions 4 wg .. 4 wg + 3, rows sg RS .. sg RS + RS - 1
  skinny_box(a, b, pw, cw);
  if (!a.partial)
    for (int s = tid; s < a.S; s += SK_THREADS) cs[s] = __ldg(a.c_s_off + s);
  __syncthreads();

  const int sq = SP * a.npass;  // rows of Q in shared memory
  const int qld = sq + 4;
  const int c0 = z * a.chunks_per_split;
  const int c1 = c0 + a.chunks_per_split < a.nchunks ? c0 + a.chunks_per_split : a.nchunks;
  float acc[RS][4];
  auto clear = [&] {
#pragma unroll
    for (int i = 0; i < RS; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  };
  auto fma_chunk = [&](const float* ps, const float* qs, int kc) {
    const float* pp = ps + 4 * wg;
    const float* qq = qs + sg * RS;
#pragma unroll 2
    for (int k = 0; k < kc; ++k) {
      const float4 pv = *reinterpret_cast<const float4*>(pp + k * SK_LDP);
      float q[RS];
#pragma unroll
      for (int i = 0; i < RS; i += 4) {
        const float4 t = *reinterpret_cast<const float4*>(qq + k * qld + i);
        q[i] = t.x; q[i + 1] = t.y; q[i + 2] = t.z; q[i + 3] = t.w;
      }
#pragma unroll
      for (int i = 0; i < RS; ++i) {
        acc[i][0] = fmaf(q[i], pv.x, acc[i][0]);
        acc[i][1] = fmaf(q[i], pv.y, acc[i][1]);
        acc[i][2] = fmaf(q[i], pv.z, acc[i][2]);
        acc[i][3] = fmaf(q[i], pv.w, acc[i][3]);
      }
    }
  };
  auto kc_of = [&](int c) {
    const int64_t k0 = (int64_t)c * SK_KC;
    return a.K - k0 < SK_KC ? (int)(a.K - k0) : SK_KC;
  };
  // staged store of pass p's rows (32 at a time through P stage 1)
  float* os = Ps + SK_KC * SK_LDP;
  auto store_pass = [&](int p) {
#pragma unroll 1
    for (int h = 0; h < SP; h += SK_SUB) {
      const int s0 = p * SP + h;
      if (s0 >= a.S) break;
      int ns = SP - h < SK_SUB ? SP - h : SK_SUB;
      if (ns > a.S - s0) ns = a.S - s0;
      __syncthreads();  // the stage (and earlier staged rows) are no longer read
#pragma unroll
      for (int i = 0; i < RS; ++i) {
        const int r = sg * RS + i - h;
        if (r >= 0 && r < SK_SUB)
          *reinterpret_cast<float4*>(os + r * SK_LDP + 4 * wg) =
              make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
      }
      __syncthreads();
      skinny_store(a, os, cw, cs, s0, ns);
    }
  };

  if (a.npass > 1) {
    // one chunk (K <= 32), every row of Q at once, passes over S
    skinny_load(a, 0, Ps, Qs, sq, qld, pw);
    cp_async_wait<0>();
    __syncthreads();
    const int kc = kc_of(0);
#pragma unroll 1
    for (int p = 0; p < a.npass; ++p) {
      clear();
      fma_chunk(Ps, Qs + p * SP, kc);
      store_pass(p);
    }
    return;
  }

  clear();
  if (c0 < c1) skinny_load(a, c0, Ps, Qs, sq, qld, pw);
#pragma unroll 1
  for (int c = c0; c < c1; ++c) {
    const int st = (c - c0) & 1;
    if (c + 1 < c1) {
      // the other stage was last read by chunk c - 1: all threads are past it
      __syncthreads();
      skinny_load(a, c + 1, Ps + (st ^ 1) * SK_KC * SK_LDP, Qs + (st ^ 1) * SK_KC * qld, sq, qld, pw);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    fma_chunk(Ps + st * SK_KC * SK_LDP, Qs + st * SK_KC * qld, kc_of(c));
  }
  if (a.partial) {
    float* dst = a.partial + ((size_t)z * a.nblk + b) * SP * SK_BW + 4 * wg;
#pragma unroll
    for (int i = 0; i < RS; ++i)
      *reinterpret_cast<float4*>(dst + (size_t)(sg * RS + i) * SK_BW) =
          make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
    return;
  }
  store_pass(0);
}

// C of block b = alpha * (slice 0 + slice 1 + ...) + beta * C, slices in order.
template <int RS>
__device__ __forceinline__ void skinny_reduce_block(const SkinnyArgs& a, int64_t b, int splits,
                                                    uint8_t* smem) {
  constexpr int SP = 4 * RS;
  float* os = reinterpret_cast<float*>(smem);
  int64_t* pw = reinterpret_cast<int64_t*>(smem + SK_P_BYTES + SK_Q_BYTES);
  int64_t* cw = pw + SK_BW;
  int64_t* cs = cw + SK_BW;
  const int tid = threadIdx.x;
  skinny_box(a, b, pw, cw);
  for (int s = tid; s < a.S; s += SK_THREADS) cs[s] = __ldg(a.c_s_off + s);
  const size_t slice = (size_t)a.nblk * SP * SK_BW;
  const float* src = a.partial + (size_t)b * SP * SK_BW + tid;
#pragma unroll 1
  for (int h = 0; h < SP; h += SK_SUB) {
    if (h >= a.S) break;
    int ns = SP - h < SK_SUB ? SP - h : SK_SUB;
    if (ns > a.S - h) ns = a.S - h;
    __syncthreads();
    for (int r = 0; r < ns; ++r) {
      const float* p = src + (size_t)(h + r) * SK_BW;
      float v = p[0];
      for (int zz = 1; zz < splits; ++zz) v = __fadd_rn(v, p[zz * slice]);
      os[r * SK_LDP + tid] = v;
    }
    __syncthreads();
    skinny_store(a, os, cw, cs, h, ns);
  }
}

template <typename F>
__device__ __forceinline__ void skinny_dispatch(int rs, F&& f) {
  switch (rs) {
    case 4: f(std::integral_constant<int, 4>()); break;
    case 8: f(std::integral_constant<int, 8>()); break;
    case 12: f(std::integral_constant<int, 12>()); break;
    default: f(std::integral_constant<int, 16>()); break;
  }
}

// grid (blocks, k slices)
__global__ void __launch_bounds__(SK_THREADS, 2) skinny_gett_kernel(const SkinnyArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  grid_dep_wait();
  skinny_dispatch(a.rs, [&](auto r) { skinny_block<decltype(r)::value>(a, blockIdx.x, blockIdx.y, smem); });
}

// grid (blocks)
__global__ void __launch_bounds__(SK_THREADS, 2) skinny_reduce_kernel(const SkinnyArgs a, int splits) {
  extern __shared__ __align__(16) uint8_t smem[];
  grid_dep_wait();  // slices written by the kernel before
  skinny_dispatch(a.rs, [&](auto r) { skinny_reduce_block<decltype(r)::value>(a, blockIdx.x, splits, smem); });
}

// Grouped launches: item i owns CTAs [begin[i], begin[i + 1]) -- (block,
// slice) pairs of its contraction, or its blocks in the reduction.
struct SkinnyItem {
  SkinnyArgs args;
  int64_t begin;
  int32_t ksplit;
};

__global__ void __launch_bounds__(SK_THREADS, 2) skinny_group_kernel(const SkinnyItem* items,
                                                                      const int64_t* begin, int n) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int64_t t = blockIdx.x;
  const SkinnyItem& it = items[find_segment(begin, n, t)];
  const int64_t local = t - it.begin;
  const int64_t b = local % it.args.nblk;
  const int z = (int)(local / it.args.nblk);
  skinny_dispatch(it.args.rs, [&](auto r) { skinny_block<decltype(r)::value>(it.args, b, z, smem); });
}

__global__ void __launch_bounds__(SK_THREADS, 2) skinny_reduce_group_kernel(const SkinnyItem* items,
                                                                             const int64_t* begin,
                                                                             int n) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int64_t t = blockIdx.x;
  const SkinnyItem& it = items[find_segment(begin, n, t)];
  skinny_dispatch(it.args.rs, [&](auto r) {
    skinny_reduce_block<decltype(r)::value>(it.args, t - it.begin, it.ksplit, smem);
  });
}

}  // namespace tccg
