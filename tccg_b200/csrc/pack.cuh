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

// One 32 (rows) x 32 (k) tile of operand o; block = (32, 8).
template <typename Tin, typename Tout, int LAYOUT>
__device__ __forceinline__ void pack_tile(const PackOperand& o, int64_t kt, int64_t rt) {
  using Acc = typename AccOf<Tin>::type;
  const int64_t k0 = kt * 32, r0 = rt * 32;
  if (k0 >= o.Kcover || r0 >= o.Rcover) return;
  __shared__ Acc tile[32][33];  // [k_local][r_local]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const Tin* src = static_cast<const Tin*>(o.src);
  if (o.read_k_fast) {
    const int64_t k = k0 + tx;
    const int64_t coff = (k < o.Kk) ? o.col_off[k] : 0;
#pragma unroll
    for (int i = ty; i < 32; i += 8) {
      const int64_t r = r0 + i;
      Acc v = 0;
      if (r < o.R && k < o.Kk) v = load_as_acc<Tin>(src + o.row_off[r] + coff);
      tile[tx][i] = v;
    }
  } else {
    const int64_t r = r0 + tx;
    const int64_t roff = (r < o.R) ? o.row_off[r] : 0;
#pragma unroll
    for (int i = ty; i < 32; i += 8) {
      const int64_t k = k0 + i;
      Acc v = 0;
      if (r < o.R && k < o.Kk) v = load_as_acc<Tin>(src + roff + o.col_off[k]);
      tile[i][tx] = v;
    }
  }
  __syncthreads();
  Tout* dst = static_cast<Tout*>(o.dst);
  if constexpr (LAYOUT == PACK_MN) {
    const int64_t r = r0 + tx;
#pragma unroll
    for (int i = ty; i < 32; i += 8) {
      const int64_t k = k0 + i;
      if (k < o.Kcover && r < o.Rcover) dst[k * o.ld + r] = static_cast<Tout>(tile[i][tx]);
    }
  } else if constexpr (LAYOUT == PACK_K_BF16) {
    const int64_t k = k0 + tx;
#pragma unroll
    for (int i = ty; i < 32; i += 8) {
      const int64_t r = r0 + i;
      if (r < o.Rcover && k < o.Kcover) dst[r * o.ld + k] = __float2bfloat16_rn((float)tile[tx][i]);
    }
  } else {  // PACK_K_BF16X3: each 32-wide k block becomes [hi x32 | lo x32]
#pragma unroll
    for (int i = ty; i < 32; i += 8) {
      const int64_t r = r0 + i;
      if (r < o.Rcover) {
        const float v = (float)tile[tx][i];
        const __nv_bfloat16 hi = __float2bfloat16_rn(v);
        const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
        __nv_bfloat16* row = reinterpret_cast<__nv_bfloat16*>(dst) + r * o.ld + (k0 / 32) * 64;
        row[tx] = hi;
        row[32 + tx] = lo;
      }
    }
  }
}

// grid = (ceil(Kcover/32), ceil(Rcover/32), 2), block = (32, 8)
template <typename Tin, typename Tout, int LAYOUT>
__global__ void __launch_bounds__(256) pack_kernel(const PackArgs args) {
  const PackOperand& o = args.op[blockIdx.z];
  if (!o.active) return;
  pack_tile<Tin, Tout, LAYOUT>(o, blockIdx.x, blockIdx.y);
}

// Grouped packing: job j (an operand of one contraction) owns the CTAs
// [job_begin[j], job_begin[j+1]); its tiles are numbered k fastest.
struct PackJob {
  PackOperand op;
  int64_t begin;   // first CTA of this job
  int64_t ktiles;  // tiles along k
};

template <typename Tin, typename Tout, int LAYOUT>
__global__ void __launch_bounds__(256) pack_group_kernel(const PackJob* jobs, int n_jobs) {
  const int64_t t = blockIdx.x + (int64_t)gridDim.x * blockIdx.y;
  int lo = 0, hi = n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].begin <= t) lo = mid; else hi = mid - 1;
  }
  const PackJob& j = jobs[lo];
  const int64_t local = t - j.begin;
  pack_tile<Tin, Tout, LAYOUT>(j.op, local % j.ktiles, local / j.ktiles);
}

}  // namespace tccg
