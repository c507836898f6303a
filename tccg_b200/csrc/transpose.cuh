// Out-of-place tensor transposition  B[perm(i)] = alpha * A[i] + beta * B[perm(i)]
// -- the operation TCCG's TTGT emits through HPTT (tccg/transpose.py:110-144).
// One 32x32 shared-memory tile per CTA over (output dim 0, the output dim that
// is A's stride-one dim), so that both the reads and the writes are coalesced;
// all other dimensions are decoded from the CTA index.
#pragma once
#include "common.cuh"

namespace tccg {

constexpr int PERM_MAX_DIMS = 16;

struct PermArgs {
  const void* A;
  void* B;
  int32_t dim;
  int32_t da;               // output dim whose A-stride is 1 (0 => both fast dims coincide)
  int64_t ext[PERM_MAX_DIMS];  // extents in OUTPUT order
  int64_t sa[PERM_MAX_DIMS];   // A stride of each output dim
  int64_t sb[PERM_MAX_DIMS];   // B stride of each output dim
  int64_t nt0, nta;         // tiles along dim 0 and dim da
  int64_t rest;             // product of the remaining extents
  double alpha, beta;
};

template <typename T>
__global__ void __launch_bounds__(256) permute_kernel(const PermArgs p) {
  __shared__ T tile[32][33];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const T alpha = (T)p.alpha, beta = (T)p.beta;
  const T* A = static_cast<const T*>(p.A);
  T* B = static_cast<T*>(p.B);
  for (int64_t r = (int64_t)blockIdx.y + (int64_t)gridDim.y * blockIdx.z; r < p.rest;
       r += (int64_t)gridDim.y * gridDim.z) {
    // decode the remaining dims (all except 0 and da) from r
    int64_t rr = r, offa = 0, offb = 0;
    for (int d = 1; d < p.dim; ++d) {
      if (d == p.da) continue;
      const int64_t i = rr % p.ext[d];
      rr /= p.ext[d];
      offa += i * p.sa[d];
      offb += i * p.sb[d];
    }
    if (p.da == 0) {  // dim 0 is stride one on both sides: straight streaming copy
      const int64_t i0 = (int64_t)blockIdx.x * 256 + ty * 32 + tx;
      if (i0 < p.ext[0]) {
        T v = alpha * A[offa + i0 * p.sa[0]];
        T* dst = B + offb + i0 * p.sb[0];
        if (beta != T(0)) v += beta * *dst;
        *dst = v;
      }
      continue;
    }
    const int64_t t0 = blockIdx.x % p.nt0, ta = blockIdx.x / p.nt0;
    {
      const int64_t ia = ta * 32 + tx;
#pragma unroll
      for (int i = ty; i < 32; i += 8) {
        const int64_t i0 = t0 * 32 + i;
        if (ia < p.ext[p.da] && i0 < p.ext[0])
          tile[i][tx] = A[offa + ia * p.sa[p.da] + i0 * p.sa[0]];
      }
    }
    __syncthreads();
    {
      const int64_t i0 = t0 * 32 + tx;
#pragma unroll
      for (int i = ty; i < 32; i += 8) {
        const int64_t ia = ta * 32 + i;
        if (ia < p.ext[p.da] && i0 < p.ext[0]) {
          T* dst = B + offb + i0 * p.sb[0] + ia * p.sb[p.da];
          T v = alpha * tile[tx][i];
          if (beta != T(0)) v += beta * *dst;
          *dst = v;
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace tccg
