// Out-of-place tensor transposition  B[perm(i)] = alpha * A[i] + beta * B[perm(i)]
// -- the operation TCCG's TTGT emits through HPTT (tccg/transpose.py:110-144).
//
// The host side (permute_launch) drops unit extents, fuses neighbouring
// output dimensions that are contiguous in both tensors, and orders the
// output dimensions so that dim 0 has B's smallest stride. Then:
//   * dim 0 is also A's smallest stride: a streaming copy along dim 0, 8
//     elements per thread with all loads issued before the stores (one
//     warp per row when dim 0 is short);
//   * otherwise shared-memory tiles over (dim 0, the dim `da` with A's
//     smallest stride): reads along da, writes along dim 0, 16 loads in
//     flight per thread (one 64 x 64 tile, or four 32 x 32 tiles of
//     consecutive rows when 64 would pad the extents by more than 5 %).
// The remaining dimensions are decoded once per CTA from its row index.
#pragma once
#include "common.cuh"

namespace tccg {

constexpr int PERM_MAX_DIMS = 16;
constexpr int PERM_STREAM = 8;   // elements per thread in the streaming copy

struct PermArgs {
  const void* A;
  void* B;
  int32_t dim;
  int32_t da;                  // output dim with A's smallest stride (0: same as B's)
  int64_t ext[PERM_MAX_DIMS];  // extents in OUTPUT order
  int64_t sa[PERM_MAX_DIMS];   // A stride of each output dim
  int64_t sb[PERM_MAX_DIMS];   // B stride of each output dim
  int64_t nt0, nta;            // tiles (or chunks) along dim 0 and dim da
  int64_t rest;                // product of the remaining extents
  double alpha, beta;
};

// offsets of row r over the dims other than 0 and da
__device__ __forceinline__ void perm_decode(const PermArgs& p, int64_t r, int64_t& offa,
                                            int64_t& offb) {
  offa = 0;
  offb = 0;
  for (int d = 1; d < p.dim; ++d) {
    if (d == p.da) continue;
    const int64_t i = r % p.ext[d];
    r /= p.ext[d];
    offa += i * p.sa[d];
    offb += i * p.sb[d];
  }
}

// dim 0 has the smallest stride in both tensors; grid.x = chunks of
// 256 * PERM_STREAM elements of dim 0, grid.y/z = rows
template <typename T>
__global__ void __launch_bounds__(256) permute_stream_kernel(const PermArgs p) {
  const T alpha = (T)p.alpha, beta = (T)p.beta;
  const T* A = static_cast<const T*>(p.A);
  T* B = static_cast<T*>(p.B);
  const int tid = threadIdx.x + 32 * threadIdx.y;
  const int64_t L = p.ext[0], sa0 = p.sa[0], sb0 = p.sb[0];
  for (int64_t r = (int64_t)blockIdx.y + (int64_t)gridDim.y * blockIdx.z; r < p.rest;
       r += (int64_t)gridDim.y * gridDim.z) {
    int64_t offa, offb;
    perm_decode(p, r, offa, offb);
    const int64_t base = (int64_t)blockIdx.x * (256 * PERM_STREAM);
    T v[PERM_STREAM];
#pragma unroll
    for (int u = 0; u < PERM_STREAM; ++u) {
      const int64_t i0 = base + u * 256 + tid;
      v[u] = i0 < L ? A[offa + i0 * sa0] : T(0);
    }
    if (beta != T(0)) {
      T old[PERM_STREAM];
#pragma unroll
      for (int u = 0; u < PERM_STREAM; ++u) {
        const int64_t i0 = base + u * 256 + tid;
        old[u] = i0 < L ? B[offb + i0 * sb0] : T(0);
      }
#pragma unroll
      for (int u = 0; u < PERM_STREAM; ++u) v[u] = alpha * v[u] + beta * old[u];
    } else {
#pragma unroll
      for (int u = 0; u < PERM_STREAM; ++u) v[u] = alpha * v[u];
    }
#pragma unroll
    for (int u = 0; u < PERM_STREAM; ++u) {
      const int64_t i0 = base + u * 256 + tid;
      if (i0 < L) B[offb + i0 * sb0] = v[u];
    }
  }
}

// dim 0 has the smallest stride in both tensors and is short (< PERM_ROWS_MAX
// elements): one warp per row of dim 0 (rows r = global warp index + k *
// warps in the grid), lanes along dim 0, 4 x 32 elements per pass with all
// loads issued before the stores. The chunked kernel above gives every row a
// CTA of 256 x PERM_STREAM slots, most of them empty on short rows.
constexpr int PERM_ROWS_MAX = 1024;

template <typename T>
__global__ void __launch_bounds__(256) permute_rows_kernel(const PermArgs p) {
  const T alpha = (T)p.alpha, beta = (T)p.beta;
  const T* A = static_cast<const T*>(p.A);
  T* B = static_cast<T*>(p.B);
  const int lane = threadIdx.x, w = threadIdx.y;  // block (32, 8)
  const int64_t L = p.ext[0], sa0 = p.sa[0], sb0 = p.sb[0];
  const int64_t warps = (int64_t)gridDim.x * 8;
  for (int64_t r = (int64_t)blockIdx.x * 8 + w; r < p.rest; r += warps) {
    int64_t offa, offb;
    perm_decode(p, r, offa, offb);
    for (int64_t c0 = 0; c0 < L; c0 += 128) {
      T v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t i0 = c0 + u * 32 + lane;
        v[u] = i0 < L ? A[offa + i0 * sa0] : T(0);
      }
      if (beta != T(0)) {
        T old[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int64_t i0 = c0 + u * 32 + lane;
          old[u] = i0 < L ? B[offb + i0 * sb0] : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = alpha * v[u] + beta * old[u];
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = alpha * v[u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t i0 = c0 + u * 32 + lane;
        if (i0 < L) B[offb + i0 * sb0] = v[u];
      }
    }
  }
}

// grid.x = nt0 * nta tile groups, grid.y/z = row groups; block (32, 8). A
// thread issues (TE / 8) * (TE / 32) * ROWS loads before its first
// shared-memory store: one 64 x 64 tile for large extents, or ROWS 32 x 32
// tiles where 64 would leave much of a tile empty -- of ROWS consecutive rows,
// or (ALONG0, for few rows) of ROWS consecutive tiles along dim 0.
template <typename T, int TE, int ROWS, bool ALONG0>
__global__ void __launch_bounds__(256) permute_kernel(const PermArgs p) {
  constexpr int H = TE / 32, I = TE / 8;
  __shared__ T tile[ROWS][TE][TE + 1];  // [row][dim-0 index][da index]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const T alpha = (T)p.alpha, beta = (T)p.beta;
  const T* A = static_cast<const T*>(p.A);
  T* B = static_cast<T*>(p.B);
  const int64_t e0 = p.ext[0], ea = p.ext[p.da];
  const int64_t sa0 = p.sa[0], saa = p.sa[p.da], sb0 = p.sb[0], sba = p.sb[p.da];
  // da tiles vary fastest: the CTAs that run together read the whole
  // stride-one span of A (and write neighbouring row groups of B)
  const int64_t ta = blockIdx.x % p.nta, t0 = blockIdx.x / p.nta;
  const int64_t groups = ALONG0 ? p.rest : (p.rest + ROWS - 1) / ROWS;
  for (int64_t gr = (int64_t)blockIdx.y + (int64_t)gridDim.y * blockIdx.z; gr < groups;
       gr += (int64_t)gridDim.y * gridDim.z) {
    int64_t offa[ROWS], offb[ROWS], t0q[ROWS];
    bool rok[ROWS];
#pragma unroll
    for (int q = 0; q < ROWS; ++q) {
      const int64_t r = ALONG0 ? gr : gr * ROWS + q;
      t0q[q] = ALONG0 ? t0 * ROWS + q : t0;
      rok[q] = r < p.rest;
      perm_decode(p, rok[q] ? r : 0, offa[q], offb[q]);
    }
    // read along da (A's fast dim)
    T v[ROWS][I][H];
#pragma unroll
    for (int q = 0; q < ROWS; ++q)
#pragma unroll
      for (int i = 0; i < I; ++i)
#pragma unroll
        for (int h = 0; h < H; ++h) {
          const int64_t i0 = t0q[q] * TE + ty + 8 * i, ia = ta * TE + tx + 32 * h;
          v[q][i][h] = (rok[q] && i0 < e0 && ia < ea) ? A[offa[q] + ia * saa + i0 * sa0] : T(0);
        }
#pragma unroll
    for (int q = 0; q < ROWS; ++q)
#pragma unroll
      for (int i = 0; i < I; ++i)
#pragma unroll
        for (int h = 0; h < H; ++h) tile[q][ty + 8 * i][tx + 32 * h] = v[q][i][h];
    __syncthreads();
    // write along dim 0 (B's fast dim); B is read first only when beta != 0
#pragma unroll
    for (int q = 0; q < ROWS; ++q) {
      T o[I][H];
      if (beta != T(0)) {
#pragma unroll
        for (int i = 0; i < I; ++i)
#pragma unroll
          for (int h = 0; h < H; ++h) {
            const int64_t i0 = t0q[q] * TE + tx + 32 * h, ia = ta * TE + ty + 8 * i;
            o[i][h] = (rok[q] && i0 < e0 && ia < ea) ? B[offb[q] + i0 * sb0 + ia * sba] : T(0);
          }
      }
#pragma unroll
      for (int i = 0; i < I; ++i)
#pragma unroll
        for (int h = 0; h < H; ++h) {
          const int64_t i0 = t0q[q] * TE + tx + 32 * h, ia = ta * TE + ty + 8 * i;
          if (rok[q] && i0 < e0 && ia < ea) {
            T x = alpha * tile[q][tx + 32 * h][ty + 8 * i];
            if (beta != T(0)) x += beta * o[i][h];
            B[offb[q] + i0 * sb0 + ia * sba] = x;
          }
        }
    }
    __syncthreads();
  }
}

}  // namespace tccg
