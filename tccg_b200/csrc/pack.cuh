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

// One CTA (32 x 8 threads) packs 32 rows x 128 k of an operand. All 16 loads
// of a thread are issued before the first shared-memory store, so each thread
// keeps 16 global loads in flight (32 x 32 tiles left the pass
// latency-bound). Reads run along the operand's fast direction (k or rows);
// writes along the destination's: rows for the MN layouts, k for K-major.
constexpr int PACK_KT_WIDE = 128;

template <int LAYOUT>
__host__ __device__ constexpr int pack_k_tile() {
  return PACK_KT_WIDE;
}

template <typename Tin, typename Tout, int LAYOUT>
__device__ __forceinline__ void pack_tile_wide(const PackOperand& o, int64_t kt, int64_t rt) {
  using Acc = typename AccOf<Tin>::type;
  constexpr int KT = PACK_KT_WIDE, SB = KT / 32;
  const int64_t k0 = kt * KT, r0 = rt * 32;
  if (k0 >= o.Kcover || r0 >= o.Rcover) return;
  __shared__ Acc tile[KT][33];  // [k_local][r_local]
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
    if constexpr (LAYOUT == PACK_K_BF16) {
      if (k + 3 < o.Kcover && (o.ld & 3) == 0) {
        __nv_bfloat162 p0 = __floats2bfloat162_rn(tile[kl][rl], tile[kl + 1][rl]);
        __nv_bfloat162 p1 = __floats2bfloat162_rn(tile[kl + 2][rl], tile[kl + 3][rl]);
        uint2 u;
        u.x = *reinterpret_cast<uint32_t*>(&p0);
        u.y = *reinterpret_cast<uint32_t*>(&p1);
        *reinterpret_cast<uint2*>(base + k) = u;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (k + j < o.Kcover) base[k + j] = __float2bfloat16_rn(tile[kl + j][rl]);
      }
    } else {  // PACK_K_BF16X3: each 32-wide k block becomes [hi x32 | lo x32]
      __nv_bfloat16 hi[4], lo[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float x = tile[kl + j][rl];
        hi[j] = __float2bfloat16_rn(x);
        lo[j] = __float2bfloat16_rn(x - __bfloat162float(hi[j]));
      }
      __nv_bfloat16* row = base + ((k0 + sb * 32) / 32) * 64;  // 16-byte aligned: ld % 64 == 0
      __nv_bfloat162 h0 = __halves2bfloat162(hi[0], hi[1]), h1 = __halves2bfloat162(hi[2], hi[3]);
      __nv_bfloat162 l0 = __halves2bfloat162(lo[0], lo[1]), l1 = __halves2bfloat162(lo[2], lo[3]);
      uint2 uh, ul;
      uh.x = *reinterpret_cast<uint32_t*>(&h0);
      uh.y = *reinterpret_cast<uint32_t*>(&h1);
      ul.x = *reinterpret_cast<uint32_t*>(&l0);
      ul.y = *reinterpret_cast<uint32_t*>(&l1);
      *reinterpret_cast<uint2*>(row + kq) = uh;
      *reinterpret_cast<uint2*>(row + 32 + kq) = ul;
    }
  }
}

template <typename Tin, typename Tout, int LAYOUT>
__device__ __forceinline__ void pack_any(const PackOperand& o, int64_t kt, int64_t rt) {
  pack_tile_wide<Tin, Tout, LAYOUT>(o, kt, rt);
}

// grid = (ktiles * rtiles, 1, 2) with ktiles = ceil(Kcover / pack_k_tile),
// block = (32, 8); CTA x covers k tile x % ktiles of row tile x / ktiles.
template <typename Tin, typename Tout, int LAYOUT>
__global__ void __launch_bounds__(256) pack_kernel(const PackArgs args, int64_t ktiles) {
  const PackOperand& o = args.op[blockIdx.z];
  if (!o.active) return;
  pack_any<Tin, Tout, LAYOUT>(o, (int64_t)blockIdx.x % ktiles, (int64_t)blockIdx.x / ktiles);
}

// Grouped packing: job j (an operand of one contraction) owns the CTAs
// [job_begin[j], job_begin[j+1]); its tiles are numbered k fastest.
struct PackJob {
  PackOperand op;
  int64_t begin;   // first CTA of this job
  int64_t ktiles;  // tiles along k (pack_k_tile<LAYOUT>() wide)
};

template <typename Tin, typename Tout, int LAYOUT>
__global__ void __launch_bounds__(256) pack_group_kernel(const PackJob* jobs, const int64_t* begin,
                                                         int n_jobs) {
  const int64_t t = blockIdx.x + (int64_t)gridDim.x * blockIdx.y;
  // the job's fields by value: loaded together up front instead of one
  // dependent global load at a time inside the tile code
  const PackJob j = jobs[find_segment(begin, n_jobs, t)];
  const int64_t local = t - j.begin;
  pack_any<Tin, Tout, LAYOUT>(j.op, local % j.ktiles, local / j.ktiles);
}

}  // namespace tccg
