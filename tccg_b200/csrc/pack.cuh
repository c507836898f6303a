// Operand packing: GETT's "pack the sub-tensor, keep the stride-one index"
// step (TCCG packs A-hat -> A-tilde per cache block with HPTT,
// tccg/gett.py:346-391, 700-753). Here each operand is packed once per call
// into a layout the GEMM kernels read with 16-byte (SIMT) or TMA (tcgen05)
// loads; the packing pass is bandwidth-bound and fused with the element-type
// conversion (FP32 -> BF16, or FP32 -> BF16 hi/lo pair for split-BF16x3).
//
// Source addressing is separable: element (r, k) of the operand lives at
// src[row_off[r] + col_off[k]], where r is the linear M (or N) index and k the
// linear K index; the host builds both tables from the tensor's strides, so
// any permutation of the modes (and any strides) is handled.
#pragma once
#include "common.cuh"

namespace tccg {

enum PackLayout : int {
  PACK_MN = 0,        // dst[k * ld + r], rows padded to Rcover, k padded to Kcover (zeros)
  PACK_K_BF16 = 1,    // dst[r * ld + k], bf16, k < Kcover (zeros beyond K)
  PACK_K_BF16X3 = 2,  // dst[r * ld + (k/32)*64 + k%32] = hi, +32 = lo (bf16)
  PACK_MN_BF16 = 3,   // as PACK_MN, each value rounded to bf16 (BF16 semantics on CUDA cores)
};

struct PackOperand {
  const void* src;
  const int64_t* row_off;
  const int64_t* col_off;
  int64_t R, Kk;          // logical extents
  int64_t Rcover, Kcover; // extents written (padding is written as zeros)
  void* dst;
  int64_t ld;             // dst leading dimension in elements
  int32_t read_k_fast;    // 1: consecutive threads read consecutive k
  int32_t active;
  // K-major layouts only: null, or the destination row of tile row r (then
  // row_off is indexed by the same visit order). Lets the pass walk the rows
  // along the operand's unit-stride mode when that is not the first mode of
  // the destination order; each destination row is written whole either way.
  const int64_t* row_dst;
  // K-major layouts only: k-block tiles (kb_lo > 0) for an operand whose
  // unit-stride mode is a K mode u other than the first. A tile covers kb_rows
  // rows x (kb_lo * kb_run) consecutive k -- kb_lo = the product of the extents
  // of the K modes before u, kb_run consecutive values of u -- and is read with
  // u fastest (coalesced), reordered in shared memory and written K-major.
  // kb_ext = u's extent, kb_step = u's stride (+1 or -1). kb_quad = 1: every
  // 4 consecutive u (u % 4 == 0) are 4 consecutive, 16-byte aligned source
  // elements, and kb_lo, kb_run and kb_ext are multiples of 4: the tile
  // moves them as one 16-byte copy.
  int32_t kb_lo, kb_run, kb_rows, kb_ext, kb_step, kb_quad;
  // K-major layouts only: 1 = every quad of k (k % 4 == 0) is 4 consecutive,
  // 16-byte aligned source elements (the first K mode has unit stride): the
  // pass streams 16-byte loads straight into K-major stores.
  int32_t kstream;
  // tile grid of this operand: tiles along k and in total (set by the host)
  int64_t ktiles, tiles;
};

struct PackArgs {
  PackOperand op[2];
};

template <typename T>
struct AccOf {
  using type = float;
};
template <>
struct AccOf<double> {
  using type = double;
};

template <typename T>
__device__ __forceinline__ typename AccOf<T>::type load_as_acc(const T* p) {
  return static_cast<typename AccOf<T>::type>(*p);
}
template <>
__device__ __forceinline__ float load_as_acc<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __bfloat162float(*p);
}

// Writes 4 consecutive k (k .. k+3, k % 4 == 0) of destination row `base`
// in a K-major layout: bf16, or [hi x32 | lo x32] per 32-wide k block.
template <int LAYOUT>
__device__ __forceinline__ void store_k4(__nv_bfloat16* base, int64_t k, int64_t kcover,
                                         int64_t ld, const float (&x)[4]) {
  if constexpr (LAYOUT == PACK_K_BF16) {
    if (k + 3 < kcover && (ld & 3) == 0) {
      __nv_bfloat162 p0 = __floats2bfloat162_rn(x[0], x[1]);
      __nv_bfloat162 p1 = __floats2bfloat162_rn(x[2], x[3]);
      uint2 u;
      u.x = *reinterpret_cast<uint32_t*>(&p0);
      u.y = *reinterpret_cast<uint32_t*>(&p1);
      *reinterpret_cast<uint2*>(base + k) = u;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (k + j < kcover) base[k + j] = __float2bfloat16_rn(x[j]);
    }
  } else {  // PACK_K_BF16X3 (kcover is a multiple of 32)
    __nv_bfloat16* row = base + (k / 32) * 64;  // 16-byte aligned: ld % 64 == 0
    uint2 uh, ul;
    split_bf16x2(x[0], x[1], uh.x, ul.x);
    split_bf16x2(x[2], x[3], uh.y, ul.y);
    *reinterpret_cast<uint2*>(row + k % 32) = uh;
    *reinterpret_cast<uint2*>(row + 32 + k % 32) = ul;
  }
}

// One CTA (32 x 8 threads) packs 32 rows x 128 k of an operand. All 16 loads
// of a thread are issued before the first shared-memory store, so each thread
// keeps 16 global loads in flight (32 x 32 tiles left the pass
// latency-bound). Reads run along the operand's fast direction (k or rows);
// writes along the destination's: rows for the MN layouts, k for K-major.
constexpr int PACK_KT_WIDE = 128;
constexpr int PACK_KB_ELEMS = 4096;  // k-block tiles: rows x k elements per CTA (at most)

template <int LAYOUT>
__host__ __device__ constexpr int pack_k_tile() {
  return PACK_KT_WIDE;
}

template <typename Tin, typename Tout, int LAYOUT>
__device__ __forceinline__ void pack_tile_wide(const PackOperand& o, int64_t kt, int64_t rt,
                                               typename AccOf<Tin>::type (&tile)[PACK_KT_WIDE][33]) {
  using Acc = typename AccOf<Tin>::type;
  constexpr int KT = PACK_KT_WIDE, SB = KT / 32;
  const int64_t k0 = kt * KT, r0 = rt * 32;
  if (k0 >= o.Kcover || r0 >= o.Rcover) return;
  // tile: [k_local][r_local]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const Tin* src = static_cast<const Tin*>(o.src);
  Acc v[SB][4];
  if (o.read_k_fast) {
    int64_t roff[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t r = r0 + ty + 8 * i;
      roff[i] = (r < o.R) ? o.row_off[r] : -1;
    }
#pragma unroll
    for (int sb = 0; sb < SB; ++sb) {
      const int64_t k = k0 + sb * 32 + tx;
      const int64_t coff = (k < o.Kk) ? o.col_off[k] : -1;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        v[sb][i] = (roff[i] >= 0 && coff >= 0) ? load_as_acc<Tin>(src + roff[i] + coff) : Acc(0);
    }
#pragma unroll
    for (int sb = 0; sb < SB; ++sb)
#pragma unroll
      for (int i = 0; i < 4; ++i) tile[sb * 32 + tx][ty + 8 * i] = v[sb][i];
  } else {
    const int64_t r = r0 + tx;
    const int64_t roff = (r < o.R) ? o.row_off[r] : -1;
#pragma unroll
    for (int sb = 0; sb < SB; ++sb)
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int64_t k = k0 + sb * 32 + ty + 8 * i;
        v[sb][i] = (roff >= 0 && k < o.Kk) ? load_as_acc<Tin>(src + roff + o.col_off[k]) : Acc(0);
      }
#pragma unroll
    for (int sb = 0; sb < SB; ++sb)
#pragma unroll
      for (int i = 0; i < 4; ++i) tile[sb * 32 + ty + 8 * i][tx] = v[sb][i];
  }
  __syncthreads();
  if constexpr (LAYOUT == PACK_MN || LAYOUT == PACK_MN_BF16) {
    // MN layouts: dst[k * ld + r], lanes along r (32 consecutive rows)
    const int64_t r = r0 + tx;
    if (r >= o.Rcover) return;
    Tout* dst = static_cast<Tout*>(o.dst);
#pragma unroll
    for (int i = 0; i < KT / 8; ++i) {
      const int kl = ty + 8 * i;
      const int64_t k = k0 + kl;
      if (k < o.Kcover) {
        if constexpr (LAYOUT == PACK_MN_BF16)
          dst[k * o.ld + r] = static_cast<Tout>(__bfloat162float(__float2bfloat16_rn((float)tile[kl][tx])));
        else
          dst[k * o.ld + r] = static_cast<Tout>(tile[kl][tx]);
      }
    }
    return;
  }
  // K-major: thread t packs 4 consecutive k of row t/8 per 32-wide k block
  const int t = ty * 32 + tx;
  const int rl = t >> 3, kq = (t & 7) * 4;
  const int64_t r = r0 + rl;
  if (r >= o.Rcover) return;
  const int64_t rd = o.row_dst ? o.row_dst[r] : r;
  __nv_bfloat16* base = static_cast<__nv_bfloat16*>(o.dst) + rd * o.ld;
#pragma unroll
  for (int sb = 0; sb < SB; ++sb) {
    const int kl = sb * 32 + kq;
    const int64_t k = k0 + kl;
    if (k >= o.Kcover) break;
    const float x[4] = {(float)tile[kl][rl], (float)tile[kl + 1][rl], (float)tile[kl + 2][rl],
                        (float)tile[kl + 3][rl]};
    store_k4<LAYOUT>(base, k, o.Kcover, o.ld, x);
  }
}

// Position (r, l, u) of element f = r * T + l * run + u of a k-block tile,
// stepped by `step` elements without divisions (one carry per level: the
// step is below T and run).
struct KbWalk {
  int r, l, u, dr, dl, du;
  __device__ __forceinline__ KbWalk(int f, int step, int lo, int run) {
    const int T = lo * run;
    r = f / T;
    l = (f - r * T) / run;
    u = f - r * T - l * run;
    dr = step / T;
    dl = (step - dr * T) / run;
    du = step - dr * T - dl * run;
  }
  __device__ __forceinline__ void next(int lo, int run) {
    u += du;
    l += dl;
    if (u >= run) { u -= run; ++l; }
    if (l >= lo) { l -= lo; ++r; }
    r += dr;
  }
};

// k-block tile (K-major layouts): rows [rt R, rt R + R) x k [kt T, kt T + T),
// T = kb_lo * kb_run. Element e = l * kb_run + u of a row's run is k_local =
// l + kb_lo * u: consecutive threads read consecutive u (unit stride) of one
// l, at col_off[k0 + l] + u * kb_step (the table only where the run wraps
// into the next value of the higher modes). Values land in shared memory at
// k_local's padded position k + k / 32 (threads reading along u write kb_lo
// apart: the padding spreads them over the banks) by cp.async; every thread
// issues all its copies (R T / 256 <= 16) before it waits. FP32 sources only.
template <typename Tin, int LAYOUT>
__device__ __forceinline__ void pack_kblock(const PackOperand& o, int64_t kt, int64_t rt,
                                            float* tile) {
  constexpr int NV = PACK_KB_ELEMS / 256;
  const int lo = o.kb_lo, run = o.kb_run, T = lo * run, R = o.kb_rows, TP = T + T / 32;
  const int64_t k0 = kt * T, r0 = rt * R;
  if (k0 >= o.Kcover || r0 >= o.Rcover) return;
  const int tid = threadIdx.x + 32 * threadIdx.y;
  const Tin* src = static_cast<const Tin*>(o.src);
  const int u0 = (int)((kt * run) % o.kb_ext);  // u of the tile's first run
  // source element of (r, l, u), or null (zero) past K or the last row
  auto source = [&](const KbWalk& w) -> const Tin* {
    const int64_t row = r0 + w.r, k = k0 + w.l + (int64_t)lo * w.u;
    if (k >= o.Kk || row >= o.R) return nullptr;
    const int64_t coff =
        u0 + w.u < o.kb_ext ? o.col_off[k0 + w.l] + (int64_t)o.kb_step * w.u : o.col_off[k];
    return src + o.row_off[row] + coff;
  };
  auto slot = [&](const KbWalk& w) {
    const int kl = w.l + lo * w.u;
    return w.r * TP + kl + kl / 32;
  };
  static_assert(sizeof(Tin) == 4, "k-block tiles take FP32 sources");
  KbWalk w(tid, 256, lo, run);
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    if (w.r < R) {
      const Tin* p = source(w);
      float* d = tile + slot(w);
      if (p)
        cp_async_elem<4>(d, p);
      else
        *d = 0.f;
    }
    w.next(lo, run);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  const int Q = T / 4;  // quads of k per row
  for (int f = tid; f < R * Q; f += 256) {
    const int r = f / Q, kq = (f - r * Q) * 4;
    const int64_t k = k0 + kq, row = r0 + r;
    if (row >= o.Rcover || k >= o.Kcover) continue;
    const float* t = tile + r * TP + kq + kq / 32;  // kq % 4 == 0: the quad shares one 32-group
    const float x[4] = {t[0], t[1], t[2], t[3]};
    store_k4<LAYOUT>(static_cast<__nv_bfloat16*>(o.dst) + row * o.ld, k, o.Kcover, o.ld, x);
  }
}

// k-block tile with 16-byte copies (kb_quad): the tile is kept as the source
// lays it out, raw[r][l][u] (u contiguous), 4 consecutive u per cp.async; the
// 16-byte chunks of row (r, l) are rotated by l / 4 so that the write-out,
// which reads 4 consecutive l of one u per quad of k, spreads over the banks.
// Quads past K or the last row are read element by element (or zero).
template <int LAYOUT>
__device__ __forceinline__ void pack_kblock_quad(const PackOperand& o, int64_t kt, int64_t rt,
                                                 float* tile) {
  constexpr int NQ = PACK_KB_ELEMS / 4 / 256;  // 16-byte copies per thread at most
  const int lo = o.kb_lo, run = o.kb_run, T = lo * run, R = o.kb_rows;
  const int nch = run / 4;  // 16-byte chunks per (r, l) row
  const int64_t k0 = kt * T, r0 = rt * R;
  if (k0 >= o.Kcover || r0 >= o.Rcover) return;
  const int tid = threadIdx.x + 32 * threadIdx.y;
  const float* src = static_cast<const float*>(o.src);
  const int u0 = (int)((kt * run) % o.kb_ext);  // u of the tile's first run (a multiple of 4)
  // chunk c of row (r, l) lives at raw position ((r lo + l) run + 4 ((c + l/4) % nch))
  auto chunk = [&](int r, int l, int c) {
    return tile + (r * lo + l) * run + 4 * ((c + (l >> 2)) % nch);
  };
#pragma unroll
  for (int i = 0; i < NQ; ++i) {
    const int f = tid + 256 * i;  // f = (r lo + l) nch + c
    if (f >= R * lo * nch) break;
    const int c = f % nch, rl = f / nch, l = rl % lo, r = rl / lo;
    const int u = 4 * c;
    const int64_t row = r0 + r, k = k0 + l + (int64_t)lo * u;
    float* d = chunk(r, l, c);
    if (row < o.R && k + 3 * (int64_t)lo < o.Kk) {
      const int64_t coff = u0 + u < o.kb_ext ? o.col_off[k0 + l] + u : o.col_off[k];
      cp_async_16(d, src + o.row_off[row] + coff);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t kj = k + (int64_t)lo * j;
        d[j] = (row < o.R && kj < o.Kk) ? src[o.row_off[row] + o.col_off[kj]] : 0.f;
      }
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  const int Q = T / 4;  // quads of k per row: 4 consecutive l (lo % 4 == 0) of one u
  for (int f = tid; f < R * Q; f += 256) {
    const int r = f / Q, kq = (f - r * Q) * 4;
    const int64_t k = k0 + kq, row = r0 + r;
    if (row >= o.Rcover || k >= o.Kcover) continue;
    const int l = kq % lo, u = kq / lo;
    float x[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) x[j] = chunk(r, l + j, u >> 2)[u & 3];
    store_k4<LAYOUT>(static_cast<__nv_bfloat16*>(o.dst) + row * o.ld, k, o.Kcover, o.ld, x);
  }
}

// Streaming K-major pack (kstream): quad q of the operand (quads numbered
// row-major over Rcover x Kcover / 4) is k .. k+3 of one row, 4 consecutive
// source elements (16 bytes, 8 for bf16 sources). A CTA moves 256 x
// PACK_KS_Q quads: every thread issues its quads as cp.async copies into
// shared memory (no registers held while they are in flight), then converts
// its quads and stores them at the same place of the K-major rows. Quads past
// K (or past the last row) are written as zeros; a quad that straddles K is
// read element by element.
constexpr int PACK_KS_Q = 4;

template <typename Tin, int LAYOUT>
__device__ __forceinline__ void pack_kstream(const PackOperand& o, int64_t blk, float* smem) {
  static_assert(sizeof(Tin) == 4 || sizeof(Tin) == 2, "float or bf16 sources");
  const int64_t qr = o.Kcover / 4;  // quads per row
  const int tid = threadIdx.x + 32 * threadIdx.y;
  const Tin* src = static_cast<const Tin*>(o.src);
  Tin* buf = reinterpret_cast<Tin*>(smem);  // [PACK_KS_Q][256][4]
  // quad q = (blk PACK_KS_Q + i) 256 + tid = row qr + kq, stepped by 256
  const int64_t q0 = blk * PACK_KS_Q * 256 + tid;
  const int64_t row0 = q0 / qr, drow = 256 / qr;
  const int64_t kq0 = q0 - row0 * qr, dkq = 256 - drow * qr;
  int64_t row = row0, kq = kq0;
#pragma unroll
  for (int i = 0; i < PACK_KS_Q; ++i) {
    const int64_t k = kq * 4;
    Tin* d = buf + (i * 256 + tid) * 4;
    if (row < o.R && k + 3 < o.Kk) {
      const Tin* p = src + o.row_off[row] + o.col_off[k];
      if constexpr (sizeof(Tin) == 4)
        cp_async_16(d, p);
      else
        cp_async_elem<8>(d, p);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        d[j] = (row < o.R && k + j < o.Kk) ? src[o.row_off[row] + o.col_off[k + j]] : Tin(0.0f);
    }
    kq += dkq;
    row += drow;
    if (kq >= qr) { kq -= qr; ++row; }
  }
  cp_async_commit();
  cp_async_wait<0>();  // each thread reads back only its own quads
  row = row0;
  kq = kq0;
#pragma unroll
  for (int i = 0; i < PACK_KS_Q; ++i) {
    if (row < o.Rcover) {
      const Tin* d = buf + (i * 256 + tid) * 4;
      float x[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) x[j] = load_as_acc<Tin>(d + j);
      store_k4<LAYOUT>(static_cast<__nv_bfloat16*>(o.dst) + row * o.ld, kq * 4, o.Kcover, o.ld, x);
    }
    kq += dkq;
    row += drow;
    if (kq >= qr) { kq -= qr; ++row; }
  }
}

// Read schedules compiled into one pack kernel: the 32-row tiles, the
// streaming pass or the k-block tiles only, or all three (chosen per operand
// at run time: the grouped kernel). The narrower kernels keep their register
// counts -- and so their occupancy -- free of the paths they do not run.
enum PackRead : int {
  PACK_READ_WIDE = 0,
  PACK_READ_STREAM = 1,
  PACK_READ_KBLOCK = 2,
  PACK_READ_ANY = 3
};

template <typename Tin, typename Tout, int LAYOUT, int READ>
__device__ __forceinline__ void pack_any(const PackOperand& o, int64_t kt, int64_t rt) {
  using Acc = typename AccOf<Tin>::type;
  __shared__ __align__(16) Acc tile[PACK_KT_WIDE][33];
  static_assert(PACK_KB_ELEMS + PACK_KB_ELEMS / 32 <= PACK_KT_WIDE * 33, "k-block tile fits");
  static_assert(PACK_KS_Q * 256 * 4 <= PACK_KT_WIDE * 33, "streaming buffer fits");
  constexpr bool KMAJOR = LAYOUT == PACK_K_BF16 || LAYOUT == PACK_K_BF16X3;
  if constexpr (KMAJOR && (READ == PACK_READ_STREAM || READ == PACK_READ_ANY)) {
    if (READ == PACK_READ_STREAM || o.kstream) {
      pack_kstream<Tin, LAYOUT>(o, rt, &tile[0][0]);  // one tile along k
      return;
    }
  }
  if constexpr (KMAJOR && sizeof(Tin) == 4 && (READ == PACK_READ_KBLOCK || READ == PACK_READ_ANY)) {
    if (READ == PACK_READ_KBLOCK || o.kb_lo > 0) {
      if (o.kb_quad)
        pack_kblock_quad<LAYOUT>(o, kt, rt, &tile[0][0]);
      else
        pack_kblock<Tin, LAYOUT>(o, kt, rt, &tile[0][0]);
      return;
    }
  }
  if constexpr (!KMAJOR || READ == PACK_READ_WIDE || READ == PACK_READ_ANY)
    pack_tile_wide<Tin, Tout, LAYOUT>(o, kt, rt, tile);
}

// grid = (max tiles of the two operands, 1, 2), block = (32, 8); CTA x covers
// k tile x % ktiles of row tile x / ktiles of operand z.
template <typename Tin, typename Tout, int LAYOUT, int READ>
__global__ void __launch_bounds__(256) pack_kernel(const PackArgs args) {
  grid_dep_launch();  // the GETT kernel may launch now; it waits for this grid's writes
  const PackOperand& o = args.op[blockIdx.z];
  if (!o.active || (int64_t)blockIdx.x >= o.tiles) return;
  pack_any<Tin, Tout, LAYOUT, READ>(o, (int64_t)blockIdx.x % o.ktiles, (int64_t)blockIdx.x / o.ktiles);
}

// Grouped packing: job j (an operand of one contraction) owns the CTAs
// [job_begin[j], job_begin[j+1]); its tiles are numbered k fastest.
struct PackJob {
  PackOperand op;
  int64_t begin;  // first CTA of this job
};

template <typename Tin, typename Tout, int LAYOUT>
__global__ void __launch_bounds__(256) pack_group_kernel(const PackJob* jobs, const int64_t* begin,
                                                         int n_jobs) {
  const int64_t t = blockIdx.x + (int64_t)gridDim.x * blockIdx.y;
  // the job's fields by value: loaded together up front instead of one
  // dependent global load at a time inside the tile code
  const PackJob j = jobs[find_segment(begin, n_jobs, t)];
  const int64_t local = t - j.begin;
  pack_any<Tin, Tout, LAYOUT, PACK_READ_ANY>(j.op, local % j.op.ktiles, local / j.op.ktiles);
}

}  // namespace tccg
