// SIMT GETT kernels: FP32 FFMA and FP64 DFMA on the CUDA cores.
//
// Operands come packed MN-major by pack_kernel (Ap[k][Mp], Bp[k][Np], zero
// padded), so the main loop is a dense 16-byte cp.async pipeline -- or, for
// bandwidth-bound contractions (short K), straight from the user's tensors
// through the offset tables with element-wise cp.async ("direct": one read of
// each operand instead of read + packed write + packed read). The
// epilogue writes C straight into its own (multi-index) layout through the
// offset tables: element (m, n) of the GETT view is C[c_m_off[m] + c_n_off[n]].
// That is GETT's defining property (TCCG's micro-kernel stores into C's
// original layout, tccg/gett.py:192-223) -- there is no C transposition.
//
// FP32 tiles come in three shapes (128x128, and 128x32 / 32x128 for a small
// N / M); simt_shortk_kernel is the K <= 32 variant that reads the tile's C
// block under the FMA phase (below).
//
// beta == 0 writes C without reading it (TCCG's update = 0 path,
// tccg/gett.py:516-525). With a k-split the CTAs of split z write raw partial
// sums to a workspace and simt_reduce_kernel adds them (in T: FP64 for the
// double path) and applies alpha/beta, like TCCG's k-split with one private C
// per k-group and a final sum (tccg/gett.py:755-781).
#pragma once
#include <cuda.h>
#include "common.cuh"

namespace tccg {

// Tile shapes S: 0 = the square tile; FP32 also 1 = 128 x 32 (small N) and
// 2 = 32 x 128 (small M), for contractions whose small extent would leave
// most of a 128 x 128 tile empty (4 x 4 per thread instead of 8 x 8).
enum SimtShape : int { SIMT_SQUARE = 0, SIMT_NARROW_N = 1, SIMT_NARROW_M = 2 };

template <typename T, int S = SIMT_SQUARE>
struct SimtCfg;

template <>
struct SimtCfg<float, SIMT_SQUARE> {
  static constexpr int BM = 128, BN = 128, BK = 16;
  static constexpr int WARPS_M = 2, WARPS_N = 4;
  static constexpr int TMG = 2, TNG = 2;  // 4-wide groups per thread along m / n
  static constexpr int STAGES = 4;
  static constexpr int EPN = 128;         // epilogue columns per pass (the whole tile)
  static constexpr int PAD = 4;
  static constexpr int MIN_BLOCKS = 2;    // CTAs per SM the register budget allows
  static constexpr int LDA = BM, LDB = BN;  // stage row strides (elements)
};

template <>
struct SimtCfg<float, SIMT_NARROW_N> {
  static constexpr int BM = 128, BN = 32, BK = 16;
  static constexpr int WARPS_M = 4, WARPS_N = 2;
  static constexpr int TMG = 1, TNG = 1;
  static constexpr int STAGES = 4;
  static constexpr int EPN = 32;
  static constexpr int PAD = 4;
  static constexpr int MIN_BLOCKS = 3;
  // padded stage rows: gathers along k (lanes 4 elements apart in k) spread
  // over the banks
  static constexpr int LDA = BM + 4, LDB = BN + 4;
};

template <>
struct SimtCfg<float, SIMT_NARROW_M> {
  static constexpr int BM = 32, BN = 128, BK = 16;
  static constexpr int WARPS_M = 1, WARPS_N = 8;
  static constexpr int TMG = 1, TNG = 1;
  static constexpr int STAGES = 4;
  static constexpr int EPN = 128;
  static constexpr int PAD = 4;
  static constexpr int MIN_BLOCKS = 3;
  static constexpr int LDA = BM + 4, LDB = BN + 4;
};

template <>
struct SimtCfg<double, SIMT_SQUARE> {
  static constexpr int BM = 128, BN = 64, BK = 8;
  static constexpr int WARPS_M = 2, WARPS_N = 4;
  static constexpr int TMG = 2, TNG = 1;
  static constexpr int STAGES = 4;
  static constexpr int EPN = 64;
  static constexpr int PAD = 2;
  static constexpr int MIN_BLOCKS = 2;
  static constexpr int LDA = BM, LDB = BN;
};

template <typename T>
struct SimtArgs {
  const T* Ap;  // [Kp][Mp]
  const T* Bp;  // [Kp][Np]
  int64_t Mp, Np, M, N;
  int32_t ktiles;          // Kp / BK
  int32_t ktiles_per_split;
  T* C;
  const int64_t* c_m_off;
  const int64_t* c_n_off;
  T alpha, beta;
  T* partial;  // non-null: write raw sums to partial[z][n][Mp]
  // direct != 0: no packing pass; the stage loader gathers A[k][m] =
  // Asrc[a_m_off[m] + a_k_off[k]] and B[k][n] = Bsrc[b_n_off[n] + b_k_off[k]]
  // element by element (zeros beyond M, N, K)
  int32_t direct;
  // narrow tiles, direct: 1 = the operand is gathered along k (its unit
  // stride is a K mode)
  int32_t a_kfast, b_kfast;
  int64_t K;
  const T* Asrc;
  const T* Bsrc;
  const int64_t* a_m_off;
  const int64_t* a_k_off;
  const int64_t* b_n_off;
  const int64_t* b_k_off;
  int32_t* status;  // device error word (bounded waits of the short-K kernel)
  // C layout (as TcArgs::crun): e0 in [2, 31] = C's stride-one index is the
  // first M mode, of extent e0, directly followed in C by the first N mode;
  // the epilogue then stores runs of e0 m by 32 / e0 columns per warp
  // instruction (consecutive addresses); 0 = quads along m
  int32_t crun;
};

template <typename T, int S = SIMT_SQUARE>
constexpr size_t simt_smem_bytes() {
  using Cfg = SimtCfg<T, S>;
  size_t pipe = (size_t)Cfg::STAGES * Cfg::BK * (Cfg::LDA + Cfg::LDB) * sizeof(T);
  // epilogue: the C tile (one pass of EPN columns), C offsets of the pass's
  // columns and of the tile's rows
  size_t epi = (size_t)Cfg::EPN * (Cfg::BM + Cfg::PAD) * sizeof(T) +
               (Cfg::EPN + Cfg::BM) * sizeof(int64_t);
  return pipe > epi ? pipe : epi;
}

template <typename T>
struct Vec4 {
  T v[4];
};

template <typename T>
__device__ __forceinline__ Vec4<T> lds4(const T* p) {
  Vec4<T> r;
  if constexpr (sizeof(T) == 4) {
    float4 x = *reinterpret_cast<const float4*>(p);
    r.v[0] = x.x; r.v[1] = x.y; r.v[2] = x.z; r.v[3] = x.w;
  } else {
    double2 x = *reinterpret_cast<const double2*>(p);
    double2 y = *reinterpret_cast<const double2*>(p + 2);
    r.v[0] = x.x; r.v[1] = x.y; r.v[2] = y.x; r.v[3] = y.y;
  }
  return r;
}

// Thread fragment geometry of the 256-thread CUDA-core tiles: warps WARPS_M x
// WARPS_N, lanes 8 (m) x 4 (n), each thread TMG groups of 4 m and TNG groups of
// 4 n. A fragment: per group g of 32 m, a thread owns 4 m. FP32: m = 4 lm + i,
// one 16-byte load. FP64: two 16-byte loads at m = 2 lm + {0,1} and
// 16 + 2 lm + {0,1}, so the 8 lane groups of each load read 128 contiguous
// bytes (4 consecutive doubles per lane would put lanes lm and lm + 4 on
// the same banks: a 2-way conflict on every A load).
template <typename T, int S = SIMT_SQUARE>
struct SimtFrag {
  using Cfg = SimtCfg<T, S>;
  static constexpr int TM = Cfg::TMG * 4, TN = Cfg::TNG * 4;
  static constexpr bool PAIRS = sizeof(T) == 8;
  int a_off, b_off;
  __device__ __forceinline__ explicit SimtFrag(int tid) {
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp % Cfg::WARPS_M, wn = warp / Cfg::WARPS_M;
    a_off = wm * (Cfg::TMG * 32) + (lane & 7) * (PAIRS ? 2 : 4);
    b_off = wn * (Cfg::TNG * 16) + (lane >> 3) * 4;
  }
  // tile-local m of accumulator row i and n of accumulator column j
  __device__ __forceinline__ int m(int i) const {
    return PAIRS ? a_off + (i / 4) * 32 + ((i % 4) / 2) * 16 + (i % 2) : a_off + (i / 4) * 32 + (i % 4);
  }
  __device__ __forceinline__ int n(int j) const { return b_off + (j / 4) * 16 + (j % 4); }
};

// One k-tile: acc += A[k][m] * B[k][n] over the BK rows of the stage's
// A [BK][LDA] and B [BK][LDB] panels, k in increasing order.
template <typename T, int S = SIMT_SQUARE>
__device__ __forceinline__ void simt_fma_ktile(const T* as, const T* bs, int a_off, int b_off,
                                               T (&acc)[SimtFrag<T, S>::TM][SimtFrag<T, S>::TN]) {
  using Cfg = SimtCfg<T, S>;
  constexpr int BK = Cfg::BK;
  constexpr int TM = SimtFrag<T, S>::TM, TN = SimtFrag<T, S>::TN;
#pragma unroll
  for (int k = 0; k < BK; ++k) {
    T av[TM], bv[TN];
#pragma unroll
    for (int g = 0; g < Cfg::TMG; ++g) {
      Vec4<T> x;
      if constexpr (SimtFrag<T, S>::PAIRS) {
        const double2 lo = *reinterpret_cast<const double2*>(as + k * Cfg::LDA + a_off + g * 32);
        const double2 hi = *reinterpret_cast<const double2*>(as + k * Cfg::LDA + a_off + g * 32 + 16);
        x.v[0] = lo.x; x.v[1] = lo.y; x.v[2] = hi.x; x.v[3] = hi.y;
      } else {
        x = lds4<T>(as + k * Cfg::LDA + a_off + g * 32);
      }
      av[g * 4 + 0] = x.v[0]; av[g * 4 + 1] = x.v[1]; av[g * 4 + 2] = x.v[2]; av[g * 4 + 3] = x.v[3];
    }
#pragma unroll
    for (int g = 0; g < Cfg::TNG; ++g) {
      Vec4<T> x = lds4<T>(bs + k * Cfg::LDB + b_off + g * 16);
      bv[g * 4 + 0] = x.v[0]; bv[g * 4 + 1] = x.v[1]; bv[g * 4 + 2] = x.v[2]; bv[g * 4 + 3] = x.v[3];
    }
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
  }
}

// One BM x BN tile (bx, by) of split bz; all 256 threads of the CTA take part.
// Operand loading of simt_gett_tile: packed operands only, direct gathers
// only, or either by a.direct at run time (the grouped kernel). The packed
// instantiation carries none of the gather code, so its register allocation
// and epilogue stay those of a pure packed kernel.
enum SimtLoad : int { SIMT_PACKED = 0, SIMT_DIRECT = 1, SIMT_EITHER = 2 };

template <typename T, int LOAD = SIMT_EITHER, int S = SIMT_SQUARE>
__device__ __forceinline__ void simt_gett_tile(const SimtArgs<T>& a, int bx, int by, int bz) {
  using Cfg = SimtCfg<T, S>;
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, STAGES = Cfg::STAGES;
  constexpr int LDA = Cfg::LDA, LDB = Cfg::LDB;
  constexpr int TM = Cfg::TMG * 4, TN = Cfg::TNG * 4;
  constexpr int VEC = 16 / sizeof(T);                 // elements per 16-byte chunk
  constexpr int A_CHUNKS = BK * BM / VEC, B_CHUNKS = BK * BN / VEC;
  constexpr int A_ROW_CHUNKS = BM / VEC, B_ROW_CHUNKS = BN / VEC;
  static_assert(Cfg::WARPS_M * Cfg::TMG * 32 == BM, "tile M");
  static_assert(Cfg::WARPS_N * Cfg::TNG * 16 == BN, "tile N");

  extern __shared__ __align__(16) uint8_t smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);              // [STAGES][BK][LDA]
  T* Bs = As + (size_t)STAGES * BK * LDA;              // [STAGES][BK][LDB]

  const int tid = threadIdx.x;
  const int64_t m0 = (int64_t)bx * BM, n0 = (int64_t)by * BN;
  const int kt_begin = bz * a.ktiles_per_split;
  int kt_end = kt_begin + a.ktiles_per_split;
  if (kt_end > a.ktiles) kt_end = a.ktiles;

  // direct loads: thread tid always fills column tid % BM of A's stage and
  // tid % BN of B's (256 is a multiple of both), rows tid / BM + j * 256 / BM
  static_assert(256 % BM == 0 && 256 % BN == 0, "direct loader layout");
  const int dcol_a = tid % BM, drow_a = tid / BM;
  const int dcol_b = tid % BN, drow_b = tid / BN;
  constexpr int64_t NONE = INT64_MIN;  // offsets may be negative (negative strides)
  int64_t dm_off = NONE, dn_off = NONE;
  const bool direct = LOAD == SIMT_DIRECT || (LOAD == SIMT_EITHER && a.direct);
  if (direct) {
    if (m0 + dcol_a < a.M) dm_off = a.a_m_off[m0 + dcol_a];
    if (n0 + dcol_b < a.N) dn_off = a.b_n_off[n0 + dcol_b];
  }
  // Narrow tiles: an operand whose unit stride is along k (a_kfast /
  // b_kfast) is gathered with lanes along k instead -- thread tid fills
  // k = tid % BK of rows tid / BK + j * (256 / BK) -- so each warp reads two
  // 64-byte runs; the rows' offsets are loaded once per tile.
  constexpr bool KFAST = S != SIMT_SQUARE;
  constexpr int KR = 256 / BK;  // rows per pass of the k-fast gather
  constexpr int JAK = KFAST ? BM / KR : 1, JBK = KFAST ? BN / KR : 1;
  const int kk = tid % BK, kr = tid / BK;
  int64_t kfa[JAK], kfb[JBK];
  const bool kfast_a = KFAST && direct && a.a_kfast, kfast_b = KFAST && direct && a.b_kfast;
  if constexpr (KFAST) {
    static_assert(BM % KR == 0 && BN % KR == 0, "k-fast gather layout");
#pragma unroll
    for (int j = 0; j < JAK; ++j) {
      const int64_t m = m0 + kr + j * KR;
      kfa[j] = kfast_a && m < a.M ? a.a_m_off[m] : NONE;
    }
#pragma unroll
    for (int j = 0; j < JBK; ++j) {
      const int64_t n = n0 + kr + j * KR;
      kfb[j] = kfast_b && n < a.N ? a.b_n_off[n] : NONE;
    }
  }

  auto load_stage = [&](int stage, int kt) {
    T* as = As + (size_t)stage * BK * LDA;
    T* bs = Bs + (size_t)stage * BK * LDB;
    const int64_t krow = (int64_t)kt * BK;
    if (KFAST && (kfast_a || kfast_b)) {
      // one operand (or both) along k; the other, if any, along its rows
      const int64_t k = krow + kk;
      const int64_t koa = k < a.K ? __ldg(a.a_k_off + k) : NONE;
      const int64_t kob = k < a.K ? __ldg(a.b_k_off + k) : NONE;
      constexpr int JA = BK * BM / 256, JB = BK * BN / 256;
      if (kfast_a) {
#pragma unroll
        for (int j = 0; j < JAK; ++j) {
          T* dst = as + kk * LDA + kr + j * KR;
          if (kfa[j] != NONE && koa != NONE)
            cp_async_elem<sizeof(T)>(dst, a.Asrc + kfa[j] + koa);
          else
            *dst = T(0);
        }
      } else {
#pragma unroll
        for (int j = 0; j < JA; ++j) {
          const int64_t kj = krow + drow_a + j * (256 / BM);
          T* dst = as + (drow_a + j * (256 / BM)) * LDA + dcol_a;
          if (dm_off != NONE && kj < a.K)
            cp_async_elem<sizeof(T)>(dst, a.Asrc + dm_off + __ldg(a.a_k_off + kj));
          else
            *dst = T(0);
        }
      }
      if (kfast_b) {
#pragma unroll
        for (int j = 0; j < JBK; ++j) {
          T* dst = bs + kk * LDB + kr + j * KR;
          if (kfb[j] != NONE && kob != NONE)
            cp_async_elem<sizeof(T)>(dst, a.Bsrc + kfb[j] + kob);
          else
            *dst = T(0);
        }
      } else {
#pragma unroll
        for (int j = 0; j < JB; ++j) {
          const int64_t kj = krow + drow_b + j * (256 / BN);
          T* dst = bs + (drow_b + j * (256 / BN)) * LDB + dcol_b;
          if (dn_off != NONE && kj < a.K)
            cp_async_elem<sizeof(T)>(dst, a.Bsrc + dn_off + __ldg(a.b_k_off + kj));
          else
            *dst = T(0);
        }
      }
    } else if (direct) {
      // all k offsets first (independent loads), then the copies: an offset
      // load between two asynchronous copies would serialise them
      constexpr int JA = BK * BM / 256, JB = BK * BN / 256;
      int64_t koa[JA], kob[JB];
#pragma unroll
      for (int j = 0; j < JA; ++j) {
        const int64_t k = krow + drow_a + j * (256 / BM);
        koa[j] = k < a.K ? __ldg(a.a_k_off + k) : NONE;
      }
#pragma unroll
      for (int j = 0; j < JB; ++j) {
        const int64_t k = krow + drow_b + j * (256 / BN);
        kob[j] = k < a.K ? __ldg(a.b_k_off + k) : NONE;
      }
#pragma unroll
      for (int j = 0; j < JA; ++j) {
        T* dst = as + (drow_a + j * (256 / BM)) * LDA + dcol_a;
        if (dm_off != NONE && koa[j] != NONE)
          cp_async_elem<sizeof(T)>(dst, a.Asrc + dm_off + koa[j]);
        else
          *dst = T(0);
      }
#pragma unroll
      for (int j = 0; j < JB; ++j) {
        T* dst = bs + (drow_b + j * (256 / BN)) * LDB + dcol_b;
        if (dn_off != NONE && kob[j] != NONE)
          cp_async_elem<sizeof(T)>(dst, a.Bsrc + dn_off + kob[j]);
        else
          *dst = T(0);
      }
    } else if constexpr (LOAD != SIMT_DIRECT) {
#pragma unroll
      for (int c = tid; c < A_CHUNKS; c += 256) {
        const int row = c / A_ROW_CHUNKS, col = (c % A_ROW_CHUNKS) * VEC;
        cp_async_16(as + row * LDA + col, a.Ap + (krow + row) * a.Mp + m0 + col);
      }
#pragma unroll
      for (int c = tid; c < B_CHUNKS; c += 256) {
        const int row = c / B_ROW_CHUNKS, col = (c % B_ROW_CHUNKS) * VEC;
        cp_async_16(bs + row * LDB + col, a.Bp + (krow + row) * a.Np + n0 + col);
      }
    }
  };

  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = T(0);

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (kt_begin + s < kt_end) load_stage(s, kt_begin + s);
    cp_async_commit();
  }

  const SimtFrag<T, S> frag(tid);
  const int a_off = frag.a_off, b_off = frag.b_off;
  for (int kt = kt_begin; kt < kt_end; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + STAGES - 1;
      if (nk < kt_end) load_stage((nk - kt_begin) % STAGES, nk);
      cp_async_commit();
    }
    const int stage = (kt - kt_begin) % STAGES;
    const T* as = As + (size_t)stage * BK * LDA;
    const T* bs = Bs + (size_t)stage * BK * LDB;
    simt_fma_ktile<T, S>(as, bs, a_off, b_off, acc);
  }
  cp_async_wait<0>();
  __syncthreads();

  auto mloc = [&](int i) { return frag.m(i); };
  auto nloc = [&](int j) { return frag.n(j); };

  if (a.partial != nullptr) {
    T* P = a.partial + (size_t)bz * a.Np * a.Mp;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int64_t n = n0 + nloc(j);
#pragma unroll
      for (int i = 0; i < TM; ++i) P[n * a.Mp + m0 + mloc(i)] = acc[i][j];
    }
    return;
  }

  // Epilogue through shared memory. Each thread owns 4 consecutive m of one
  // column at a time; where those 4 elements of C are contiguous and 16-byte
  // aligned (C's stride-one index is the first M mode) they move as one
  // vector, otherwise element by element. All C loads of a pass are issued
  // before its stores, so a thread keeps several loads in flight.
  constexpr int EPN = Cfg::EPN, LDC = BM + Cfg::PAD;
  constexpr int QPC = BM / 4;              // m quads per column
  constexpr int CPI = 256 / QPC;           // columns per iteration
  constexpr int ITER = EPN / CPI;
  T* Cs = reinterpret_cast<T*>(smem_raw);  // [EPN][LDC]
  // C offsets of the pass's columns, staged once: the C loads of a chunk then
  // depend on shared memory only, not on a table load from L2
  int64_t* Cn = reinterpret_cast<int64_t*>(smem_raw + (size_t)EPN * LDC * sizeof(T));
  int64_t* Cm = Cn + EPN;  // C offsets of the tile's rows (staged C stores)
  static_assert((EPN * LDC * sizeof(T)) % 8 == 0 && EPN <= 256, "column offset staging");
  if (a.crun > 0)
    for (int r = tid; r < BM; r += 256) Cm[r] = m0 + r < a.M ? a.c_m_off[m0 + r] : 0;
  const int q = tid % QPC, cl = tid / QPC;
  const int64_t mq = m0 + 4 * q;
  int64_t cmo[4];
  bool mok[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    mok[i] = mq + i < a.M;
    cmo[i] = mok[i] ? a.c_m_off[mq + i] : 0;
  }
  const bool vec_m = mok[3] && cmo[1] == cmo[0] + 1 && cmo[2] == cmo[0] + 2 && cmo[3] == cmo[0] + 3;
  const T alpha = a.alpha, beta = a.beta;
  for (int p = 0; p < BN / EPN; ++p) {
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int nl = nloc(j) - p * EPN;
      if (nl >= 0 && nl < EPN) {
#pragma unroll
        for (int i = 0; i < TM; ++i) Cs[nl * LDC + mloc(i)] = acc[i][j];
      }
    }
    if (tid < EPN) {
      const int64_t n = n0 + p * EPN + tid;
      Cn[tid] = n < a.N ? a.c_n_off[n] : 0;
    }
    __syncthreads();
    if (a.crun > 0) {
      // runs of e0 consecutive m (clipped to the tile and M, length L), one
      // per warp at a time: the run's L x ncols block is stored in C's
      // address order, element f = i + L * j (row ma + i, column j) by lane
      // f % 32, so a store instruction covers 32 consecutive positions of
      // one contiguous stretch of C; the C offsets of rows and columns come
      // from shared memory. Same arithmetic as the quad path (alpha * acc,
      // then fma with beta).
      const int e0 = a.crun;
      const int lane = tid & 31, w = tid >> 5;
      const int64_t rfirst = (m0 / e0) * e0;
      const int nruns = (int)((m0 + BM - rfirst + e0 - 1) / e0);
      const int64_t nleft = a.N - (n0 + p * EPN);
      const int ncols = nleft < EPN ? (int)nleft : EPN;
#pragma unroll 1
      for (int ri = w; ri < nruns; ri += 8) {
        const int64_t rs = rfirst + (int64_t)ri * e0;
        const int64_t ma = rs > m0 ? rs : m0;
        int64_t mb = rs + e0 < m0 + BM ? rs + e0 : m0 + BM;
        if (mb > a.M) mb = a.M;
        const int L = (int)(mb - ma);
        if (L <= 0 || ncols <= 0) continue;
        const int total = L * ncols;
        int i = lane % L, j = lane / L;
        const int di = 32 % L, dj = 32 / L;
        const int moff = (int)(ma - m0);
#pragma unroll 2
        for (int f = lane; f < total; f += 32) {
          T* d = a.C + Cm[moff + i] + Cn[j];
          T v = alpha * Cs[j * LDC + moff + i];
          if (beta != T(0)) v = fma(beta, *d, v);
          *d = v;
          i += di;
          j += dj;
          if (i >= L) {
            i -= L;
            ++j;
          }
        }
      }
    } else if (mok[0]) {
      constexpr int CH = sizeof(T) == 8 ? 4 : 8;  // columns whose C loads are in flight together
#pragma unroll 1
      for (int it0 = 0; it0 < ITER; it0 += CH) {
        int64_t coff[CH];
        bool nok[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) {
          const int64_t n = n0 + p * EPN + (it0 + u) * CPI + cl;
          nok[u] = (it0 + u < ITER) && n < a.N;
          coff[u] = nok[u] ? Cn[(it0 + u) * CPI + cl] : 0;
        }
        T old[CH][4];
        if (beta != T(0)) {
#pragma unroll
          for (int u = 0; u < CH; ++u) {
            if (!nok[u]) continue;
            const T* d = a.C + cmo[0] + coff[u];
            if (vec_m && (reinterpret_cast<uintptr_t>(d) % (4 * sizeof(T))) == 0) {
              const Vec4<T> v = lds4<T>(d);  // 16/32-byte vector load
              old[u][0] = v.v[0]; old[u][1] = v.v[1]; old[u][2] = v.v[2]; old[u][3] = v.v[3];
            } else {
#pragma unroll
              for (int i = 0; i < 4; ++i) old[u][i] = mok[i] ? a.C[cmo[i] + coff[u]] : T(0);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) {
          if (!nok[u]) continue;
          const int nl = (it0 + u) * CPI + cl;
          T v[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            v[i] = alpha * Cs[nl * LDC + 4 * q + i];
            if (beta != T(0)) v[i] = fma(beta, old[u][i], v[i]);
          }
          T* d = a.C + cmo[0] + coff[u];
          if (vec_m && (reinterpret_cast<uintptr_t>(d) % (4 * sizeof(T))) == 0) {
            if constexpr (sizeof(T) == 4) {
              *reinterpret_cast<float4*>(d) = make_float4(v[0], v[1], v[2], v[3]);
            } else {
              reinterpret_cast<double2*>(d)[0] = make_double2(v[0], v[1]);
              reinterpret_cast<double2*>(d)[1] = make_double2(v[2], v[3]);
            }
          } else {
#pragma unroll
            for (int i = 0; i < 4; ++i)
              if (mok[i]) a.C[cmo[i] + coff[u]] = v[i];
          }
        }
      }
    }
    __syncthreads();
  }
}

template <typename T, int LOAD, int S = SIMT_SQUARE>
__global__ void __launch_bounds__(256, SimtCfg<T, S>::MIN_BLOCKS) simt_gett_kernel(const SimtArgs<T> a) {
  grid_dep_wait();  // packed operands written by the kernel before
  simt_gett_tile<T, LOAD, S>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// Short-K kernel (packed operands, K <= KP, no k-split). For K = 16 a tile's
// FMA work (16 FMAs per C element) is short next to its C traffic, and
// simt_gett_tile reads C only in its epilogue, where the loads' latency
// stalls the CTA, then spends its own issue slots on the stores. Here the CTA
// brings its C block into shared memory right after the operand panels, so
// the read runs under the FMA phase; the epilogue combines in shared memory
// (alpha * acc + beta * C, 16-byte accesses at the fragment positions) and
// the block leaves as one bulk store.
//   TMA = true  (C is a 2-D matrix in the GETT view: unit M stride, one N
//               stride): the C block comes in and goes out by TMA -- one
//               instruction each, the store draining while the next CTA on
//               the SM computes.
//   TMA = false (any layout): cp.async per thread through the offset tables,
//               stores from the threads (16-byte vectors where 4 consecutive
//               m are contiguous and aligned in C).
// Two CTAs per SM. Same k order and epilogue arithmetic as simt_gett_tile:
// the results are bitwise equal.
template <typename T>
struct SimtShortKCfg {
  using Cfg = SimtCfg<T>;
  static constexpr int KP = sizeof(T) == 4 ? 32 : 16;  // longest padded K it takes
  static constexpr size_t C_BYTES = (size_t)Cfg::BN * Cfg::BM * sizeof(T);  // [BN][BM], dense
  static constexpr size_t N_BYTES = (size_t)Cfg::BN * sizeof(int64_t);
  static constexpr size_t A_BYTES = (size_t)KP * Cfg::BM * sizeof(T);
  static constexpr size_t B_BYTES = (size_t)KP * Cfg::BN * sizeof(T);
  static constexpr size_t USED = C_BYTES + N_BYTES + A_BYTES + B_BYTES + 16;  // + mbarrier
  static constexpr size_t SMEM_BYTES = USED + 128;  // slack to align the C block to 128 bytes
  static_assert(C_BYTES % 128 == 0 && N_BYTES % 16 == 0 && A_BYTES % 16 == 0, "aligned panels");
  static_assert(2 * (SMEM_BYTES + 1024) <= 228 * 1024, "two CTAs per SM");
};

template <typename T, bool TMA>
__global__ void __launch_bounds__(256, 2)
    simt_shortk_kernel(const SimtArgs<T> a, const __grid_constant__ CUtensorMap tmC) {
  using Cfg = SimtCfg<T>;
  using SC = SimtShortKCfg<T>;
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK;
  constexpr int VEC = 16 / sizeof(T);  // elements per 16-byte access
  constexpr int QPC = BM / 4, CPI = 256 / QPC, ITER = BN / CPI;
  constexpr int TM = SimtFrag<T>::TM, TN = SimtFrag<T>::TN;
  constexpr int64_t NONE = INT64_MIN;  // offsets may be negative (negative strides)
  static_assert(BN <= 256, "one column offset per thread");
  extern __shared__ __align__(16) uint8_t smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + (((raw_addr + 127u) & ~127u) - raw_addr);  // TMA: 128-byte aligned
  T* Cs = reinterpret_cast<T*>(smem);                                  // [BN][BM]
  int64_t* Cn = reinterpret_cast<int64_t*>(smem + SC::C_BYTES);        // [BN]
  T* As = reinterpret_cast<T*>(smem + SC::C_BYTES + SC::N_BYTES);      // [KP][BM]
  T* Bs = As + (size_t)SC::KP * BM;                                    // [KP][BN]
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + SC::USED - 16);
  const int tid = threadIdx.x;
  const SimtFrag<T> frag(tid);
  const int64_t m0 = (int64_t)blockIdx.x * BM, n0 = (int64_t)blockIdx.y * BN;
  const int kp = a.ktiles * BK;
  const T alpha = a.alpha, beta = a.beta;
  const bool read_c = beta != T(0);

  if constexpr (TMA) {
    if (tid == 0) {
      mbar_init(bar, 1);
      fence_mbar_init();
    }
    __syncthreads();
    // the packing kernel before this one does not write C: the block comes
    // in while that kernel may still run
    if (read_c && tid == 0) {
      mbar_arrive_expect_tx(bar, (uint32_t)SC::C_BYTES);
      tma_load_2d(Cs, &tmC, (int32_t)m0, (int32_t)n0, bar);
    }
  }
  grid_dep_wait();  // packed operands written by the kernel before
  // operand panels first: their latency runs under the offset loads
  for (int c = tid; c < kp * (BM / VEC); c += 256) {
    const int row = c / (BM / VEC), col = (c % (BM / VEC)) * VEC;
    cp_async_16(As + row * BM + col, a.Ap + (int64_t)row * a.Mp + m0 + col);
  }
  for (int c = tid; c < kp * (BN / VEC); c += 256) {
    const int row = c / (BN / VEC), col = (c % (BN / VEC)) * VEC;
    cp_async_16(Bs + row * BN + col, a.Bp + (int64_t)row * a.Np + n0 + col);
  }
  cp_async_commit();
  // element path: the thread's 4 m (quad q) of columns cl + u * CPI
  const int q = tid % QPC, cl = tid / QPC;
  int64_t cmo[4] = {NONE, NONE, NONE, NONE};
  bool vq = false;
  if constexpr (!TMA) {
    if (tid < BN) Cn[tid] = n0 + tid < a.N ? __ldg(a.c_n_off + n0 + tid) : NONE;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t m = m0 + 4 * q + i;
      cmo[i] = m < a.M ? __ldg(a.c_m_off + m) : NONE;
    }
    vq = cmo[3] != NONE && cmo[1] == cmo[0] + 1 && cmo[2] == cmo[0] + 2 && cmo[3] == cmo[0] + 3;
  }
  auto aligned16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  if constexpr (!TMA) {
    __syncthreads();  // Cn staged
    if (read_c && cmo[0] != NONE) {
#pragma unroll
      for (int u = 0; u < ITER; ++u) {
        const int col = u * CPI + cl;
        const int64_t no = Cn[col];
        if (no == NONE) continue;
        T* dst = Cs + col * BM + 4 * q;
        const T* src = a.C + cmo[0] + no;
        if (vq && aligned16(src)) {
          cp_async_16(dst, src);
          if constexpr (sizeof(T) == 8) cp_async_16(dst + 2, src + 2);
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if (cmo[i] != NONE) cp_async_elem<sizeof(T)>(dst + i, a.C + cmo[i] + no);
        }
      }
    }
  }
  cp_async_commit();
  cp_async_wait<1>();  // operand panels in place; the C block may still be in flight
  __syncthreads();
  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
  for (int kt = 0; kt < a.ktiles; ++kt)
    simt_fma_ktile<T>(As + kt * BK * BM, Bs + kt * BK * BN, frag.a_off, frag.b_off, acc);
  if constexpr (TMA) {
    if (read_c && !mbar_wait(bar, 0)) {
      record_error(a.status, 4);
      return;  // nothing stored; the block's load never completed
    }
  } else {
    cp_async_wait<0>();
    __syncthreads();
  }
  // combine at the fragment positions: runs of VEC consecutive m (16 bytes)
#pragma unroll
  for (int j = 0; j < TN; ++j)
#pragma unroll
    for (int i0 = 0; i0 < TM; i0 += VEC) {
      T* c = Cs + frag.n(j) * BM + frag.m(i0);
      T v[VEC];
#pragma unroll
      for (int e = 0; e < VEC; ++e) v[e] = alpha * acc[i0 + e][j];
      if (read_c) {
        if constexpr (sizeof(T) == 4) {
          const float4 o = *reinterpret_cast<const float4*>(c);
          v[0] = fma(beta, o.x, v[0]); v[1] = fma(beta, o.y, v[1]);
          v[2] = fma(beta, o.z, v[2]); v[3] = fma(beta, o.w, v[3]);
        } else {
          const double2 o = *reinterpret_cast<const double2*>(c);
          v[0] = fma(beta, o.x, v[0]); v[1] = fma(beta, o.y, v[1]);
        }
      }
      if constexpr (sizeof(T) == 4)
        *reinterpret_cast<float4*>(c) = make_float4(v[0], v[1], v[2], v[3]);
      else
        *reinterpret_cast<double2*>(c) = make_double2(v[0], v[1]);
    }
  if constexpr (TMA) {
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tma_store_2d(&tmC, Cs, (int32_t)m0, (int32_t)n0);
      bulk_commit();
      bulk_wait_read_all();  // shared memory stays valid until the store has read it
    }
    return;
  }
  __syncthreads();
  if (cmo[0] == NONE) return;
#pragma unroll
  for (int u = 0; u < ITER; ++u) {
    const int col = u * CPI + cl;
    const int64_t no = Cn[col];
    if (no == NONE) continue;
    const T* src = Cs + col * BM + 4 * q;
    T* d = a.C + cmo[0] + no;
    if (vq && aligned16(d)) {
      if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(d) = *reinterpret_cast<const float4*>(src);
      } else {
        reinterpret_cast<double2*>(d)[0] = reinterpret_cast<const double2*>(src)[0];
        reinterpret_cast<double2*>(d)[1] = reinterpret_cast<const double2*>(src)[1];
      }
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (cmo[i] != NONE) a.C[cmo[i] + no] = src[i];
    }
  }
}

// Grouped launch: item i owns CTAs [tile_begin[i], tile_begin[i+1]); the CTA
// finds its item by binary search and runs the same tile code.
template <typename T>
struct SimtGroupItem {
  SimtArgs<T> args;
  int64_t tile_begin;
  int32_t tiles_m, tiles_n;  // tiles of one k-split slice
  int32_t shape;             // SimtShape (FP32 items)
};

// Shared memory of the grouped kernel: the largest of its tile shapes.
template <typename T>
constexpr size_t simt_group_smem_bytes() {
  if constexpr (sizeof(T) == 4) {
    constexpr size_t a = simt_smem_bytes<T, SIMT_SQUARE>(), b = simt_smem_bytes<T, SIMT_NARROW_N>(),
                     c = simt_smem_bytes<T, SIMT_NARROW_M>();
    return a > b ? (a > c ? a : c) : (b > c ? b : c);
  } else {
    return simt_smem_bytes<T, SIMT_SQUARE>();
  }
}

template <typename T>
__global__ void __launch_bounds__(256, 2) simt_gett_group_kernel(const SimtGroupItem<T>* items,
                                                                  const int64_t* begin,
                                                                  int n_items) {
  const int64_t t = blockIdx.x;
  const SimtGroupItem<T>& it = items[find_segment(begin, n_items, t)];
  const int64_t local = t - it.tile_begin;
  const int64_t mn = (int64_t)it.tiles_m * it.tiles_n;
  const int64_t rem = local % mn;
  const int bx = (int)(rem % it.tiles_m), by = (int)(rem / it.tiles_m), bz = (int)(local / mn);
  if constexpr (sizeof(T) == 4) {  // the item's tile shape (uniform over the CTA)
    if (it.shape == SIMT_NARROW_N) {
      simt_gett_tile<T, SIMT_EITHER, SIMT_NARROW_N>(it.args, bx, by, bz);
      return;
    }
    if (it.shape == SIMT_NARROW_M) {
      simt_gett_tile<T, SIMT_EITHER, SIMT_NARROW_M>(it.args, bx, by, bz);
      return;
    }
  }
  simt_gett_tile<T>(it.args, bx, by, bz);
}

// C = alpha * sum_z partial[z] + beta * C.
// grid = (ceil(M/256), min(N, 65535)), block 256; n strides by gridDim.y.
template <typename T>
__global__ void __launch_bounds__(256) simt_reduce_kernel(const T* __restrict__ partial,
                                                          int splits, int64_t Mp, int64_t Np,
                                                          int64_t M, int64_t N, T* C,
                                                          const int64_t* c_m_off,
                                                          const int64_t* c_n_off, T alpha,
                                                          T beta) {
  grid_dep_wait();  // partial sums written by the GETT kernel before
  const int64_t m = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (m >= M) return;
  const int64_t cmo = c_m_off[m];
  for (int64_t n = blockIdx.y; n < N; n += gridDim.y) {
    T s = T(0);
#pragma unroll 4
    for (int z = 0; z < splits; ++z) s += partial[(size_t)z * Np * Mp + n * Mp + m];
    T* dst = C + cmo + c_n_off[n];
    T v = alpha * s;
    if (beta != T(0)) v = fma(beta, *dst, v);
    *dst = v;
  }
}

// Grouped k-split reduction: job j (one contraction with a k-split) owns the
// CTAs [begin, begin + mblocks * nblocks); CTA (mb, nb) sums the slices of
// 256 rows over columns [ncols nb, ncols nb + ncols) in split order.
template <typename T>
struct ReduceJob {
  const T* partial;
  int64_t Mp, Np, M, N;
  T* C;
  const int64_t* c_m_off;
  const int64_t* c_n_off;
  T alpha, beta;
  int64_t begin;
  int32_t splits, mblocks;
  int32_t ncols;  // columns per CTA: fewer when there are many slices
};

template <typename T>
__global__ void __launch_bounds__(256) reduce_group_kernel(const ReduceJob<T>* jobs,
                                                           const int64_t* begin, int n_jobs) {
  const int64_t t = blockIdx.x;
  const ReduceJob<T> j = jobs[find_segment(begin, n_jobs, t)];  // fields loaded up front
  const int64_t local = t - j.begin;
  const int64_t m = (local % j.mblocks) * 256 + threadIdx.x;
  if (m >= j.M) return;
  const int64_t n0 = (local / j.mblocks) * j.ncols;
  const int64_t n1 = n0 + j.ncols < j.N ? n0 + j.ncols : j.N;
  const int64_t cmo = j.c_m_off[m];
  for (int64_t n = n0; n < n1; ++n) {
    T s = T(0);
#pragma unroll 4
    for (int z = 0; z < j.splits; ++z) s += j.partial[(size_t)z * j.Np * j.Mp + n * j.Mp + m];
    T* dst = j.C + cmo + j.c_n_off[n];
    T v = j.alpha * s;
    if (j.beta != T(0)) v = fma(j.beta, *dst, v);
    *dst = v;
  }
}

}  // namespace tccg
