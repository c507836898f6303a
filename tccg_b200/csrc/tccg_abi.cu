// C ABI of tccg_b200 (declared in include/tccg_b200.h): plan objects, kernel
// dispatch, tensor-map encoding, transposition and grouped launches.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/tccg_b200.h"
#include "common.cuh"
#include "pack.cuh"
#include "simt_gemm.cuh"
#include "skinny_gett.cuh"
#include "skinny_tc.cuh"
#include "tc2_gemm.cuh"
#include "tc_gemm.cuh"
#include "transpose.cuh"

using namespace tccg;

// --------------------------------------------------------------------------
// errors
// --------------------------------------------------------------------------
static thread_local char g_err[1024] = "";

static int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

#define CUDA_TRY(expr)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (expr);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(TCCG_ERR_CUDA, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                     \
  } while (0)

extern "C" const char* tccg_last_error(void) { return g_err; }
extern "C" const char* tccg_version(void) { return "tccg_b200 0.1 (sm_100a)"; }

// --------------------------------------------------------------------------
// plan
// --------------------------------------------------------------------------
struct tccg_plan {
  tccg_desc d;
  int32_t dtype = 0, prec = 0;
  tccg_tuning tune{};
  int device = 0;
  int num_sms = 148;
  int64_t M = 1, N = 1, K = 1;
  // device offset tables (elements)
  int64_t* t_a_m = nullptr;
  int64_t* t_a_k = nullptr;
  int64_t* t_b_n = nullptr;
  int64_t* t_b_k = nullptr;
  int64_t* t_c_m = nullptr;
  int64_t* t_c_n = nullptr;
  int64_t* t_id_m = nullptr;  // TTGT: identity tables of the contiguous C' = [M][N]
  int64_t* t_id_n = nullptr;
  // tensor-core packs: rows visited along the operand's unit-stride mode
  // (source offsets and destination rows in that order), or null
  int64_t* t_a_vsrc = nullptr;
  int64_t* t_a_vdst = nullptr;
  int64_t* t_b_vsrc = nullptr;
  int64_t* t_b_vdst = nullptr;
  // tensor-core packs: k-block tiles {kb_lo, kb_run, kb_rows} (PackOperand), or zeros
  int32_t kb_a[5] = {0, 0, 0, 0, 0}, kb_b[5] = {0, 0, 0, 0, 0};  // {lo, run, rows, ext, step}
  // offset tables allow the streaming K-major pack (every quad of k is 4
  // consecutive elements, every quad start and row offset a multiple of 4)
  bool ks_a = false, ks_b = false;
  // the k-block tiles of A / B may move 16-byte quads along u (kb_quad)
  bool kbq_a = false, kbq_b = false;
  int32_t* d_status = nullptr;
  int32_t read_k_fast_a = 0, read_k_fast_b = 0;
  bool c_is_mn_dense = false;  // C is already the column-major [M-modes][N-modes] matrix
  int64_t c_ldc = 0;  // > 0: C(m, n) = C[m + c_ldc * n] (a 2-D matrix in the GETT view)
  // SIMT geometry
  int64_t Mp = 0, Np = 0, Kp = 0;
  int32_t ktiles = 0, ksplit = 1, ktiles_per_split = 0;
  // tcgen05 geometry
  int64_t Kc = 0;
  int32_t num_kb = 0, tiles_m = 0, tiles_n = 0, raster = 8, grid = 0, chunk_kb = 1, bn = 256;
  int32_t kb_per_split = 0;
  // tail split of the tcgen05 tile order (TcArgs): tiles [0, full_tiles) over
  // all of K, the rest as tail_split slices of tail_kb k-blocks; 1 = none
  int32_t full_tiles = 0, tail_split = 1, tail_kb = 0;
  bool direct = false;  // CUDA-core kernel gathers operands without a packing pass
  bool gather_k_a = false, gather_k_b = false;  // direct, narrow tiles: gathers along k
  bool shortk = false;  // short-K CUDA-core kernel prefetching C (simt_shortk_kernel)
  int32_t simt_shape = 0;             // SimtShape of the CUDA-core tiles
  int32_t simt_bm = 0, simt_bn = 0;   // its tile extents
  bool simt = false;    // CUDA-core kernels (else tcgen05)
  // tcgen05 BF16X3: gather loader (operands read straight from the caller's
  // tensors, no packing pass) and its read schedule per operand (GatherRead)
  bool gather = false;
  int32_t gread_a = 0, gread_b = 0;
  // tcgen05 epilogue: C's stride-one index is the first M mode of extent
  // crun < 32, directly followed in C by the first N mode (staged C stores,
  // TcArgs::crun), or 0
  int32_t crun = 0;
  int32_t tcv = 0;  // TcVariant of a tensor-core plan
  // skinny kernel (skinny_gett.cuh): geometry and tables in sk (operand, C
  // and slice pointers are filled in per run); s_is_n: the narrow side is N
  bool skinny = false, sk_s_is_n = false, sk_p_vec = false;
  bool sk_reg = false;  // the register path (narrow side <= 16 rows)
  // the tensor-core skinny kernel (skinny_tc.cuh, split-BF16x3): MMA N = S
  // rounded up to 16; Q packed K-major [hi | lo] per 32 k at off_q
  bool sk_tc = false;
  int32_t sk_spad = 0;
  size_t off_q = 0;
  int32_t sk_ksplit = 1;
  SkinnyArgs sk{};
  // its 32-bit offset tables in one allocation: P and C offsets of the Y
  // space, P's k, Q's rows and k, C's rows (start of each in sk_tab[])
  int32_t* t_sk = nullptr;
  size_t sk_tab[6] = {};
  // workspace layout
  size_t off_a = 0, off_b = 0, off_part = 0, off_cprime = 0, off_tail = 0, ws_bytes = 0;
  char describe[512] = "";
};

// tcgen05 kernel variants: precision x operand loader x tile width (the
// autotuner's tile-shape choices). A plan runs one; a grouped run launches
// one grouped kernel per variant its items use.
enum TcVariant : int {
  TCV_X3 = 0,         // split-BF16x3, packing pass + TMA, 128 x 192
  TCV_X3_N128,        // split-BF16x3, packing pass + TMA, 128 x 128
  TCV_X3_GATHER,      // split-BF16x3, gather loader, 128 x 128
  TCV_BF16,           // BF16, packing pass + TMA, 128 x 256
  TCV_BF16_N192,      // BF16, packing pass + TMA, 128 x 192
  TCV_BF16_N128,      // BF16, packing pass + TMA, 128 x 128
  TCV_COUNT
};

template <int MODE, int LOAD, int BNV>
struct TcKernels {
  using Cfg = TcCfgT<MODE, LOAD, BNV>;
  static constexpr bool GATHER = LOAD == TC_LOAD_GATHER;
  static constexpr auto single = &gett_tc_kernel<MODE, LOAD, BNV>;
  static constexpr auto group = &gett_tc_group_kernel<MODE, LOAD, BNV>;
  static constexpr auto tail = &tc_tail_reduce_kernel<MODE, LOAD, BNV>;
};

// Calls f(TcKernels<...>{}) for variant v.
template <typename F>
static void with_tc_variant(int v, F&& f) {
  switch (v) {
    case TCV_X3: f(TcKernels<TC_BF16X3, TC_LOAD_TMA, 0>{}); break;
    case TCV_X3_N128: f(TcKernels<TC_BF16X3, TC_LOAD_TMA, 128>{}); break;
    case TCV_X3_GATHER: f(TcKernels<TC_BF16X3, TC_LOAD_GATHER, 0>{}); break;
    case TCV_BF16: f(TcKernels<TC_BF16, TC_LOAD_TMA, 0>{}); break;
    case TCV_BF16_N192: f(TcKernels<TC_BF16, TC_LOAD_TMA, 192>{}); break;
    default: f(TcKernels<TC_BF16, TC_LOAD_TMA, 128>{}); break;
  }
}

// The variant of a tensor-core plan: its precision, loader and the tuning's
// tile width (0 = the loader's default); -1 when the width is not built.
static int tc_variant(bool x3, bool gather, int32_t tile_n) {
  if (gather) return (tile_n == 0 || tile_n == 128) ? TCV_X3_GATHER : -1;
  if (x3) return tile_n == 0 || tile_n == 192 ? TCV_X3 : tile_n == 128 ? TCV_X3_N128 : -1;
  return tile_n == 0 || tile_n == 256 ? TCV_BF16
         : tile_n == 192              ? TCV_BF16_N192
         : tile_n == 128              ? TCV_BF16_N128
                                      : -1;
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
static int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }
static int64_t cdiv(int64_t x, int64_t a) { return (x + a - 1) / a; }

// The CUDA-core (SIMT) kernels run FP32 and FP64, and the BF16 precisions too
// when that is faster (operands rounded to bf16 by the pack for
// TCCG_PREC_BF16; FP32 FFMA accumulation, more accurate than split-BF16x3):
// tuning.variant < 0 asks for them, > 0 for the tensor cores, 0 lets a
// bandwidth/compute model decide.
static bool simt_path(const tccg_plan* p) { return p->simt; }

// CUDA-core tile extents of a shape (FP64: the square tile only).
static void simt_dims(bool dbl, int shape, int* bm, int* bn, int* bk) {
  if (dbl) {
    *bm = SimtCfg<double>::BM, *bn = SimtCfg<double>::BN, *bk = SimtCfg<double>::BK;
  } else if (shape == SIMT_NARROW_N) {
    *bm = SimtCfg<float, SIMT_NARROW_N>::BM, *bn = SimtCfg<float, SIMT_NARROW_N>::BN;
    *bk = SimtCfg<float, SIMT_NARROW_N>::BK;
  } else if (shape == SIMT_NARROW_M) {
    *bm = SimtCfg<float, SIMT_NARROW_M>::BM, *bn = SimtCfg<float, SIMT_NARROW_M>::BN;
    *bk = SimtCfg<float, SIMT_NARROW_M>::BK;
  } else {
    *bm = SimtCfg<float>::BM, *bn = SimtCfg<float>::BN, *bk = SimtCfg<float>::BK;
  }
}

// CUDA-core tile shape: the tuning's, or the one with the least padded work,
// the narrow tiles' work counted at NARROW_COST per element (their 4 x 4
// fragments do fewer FMAs per shared-memory load). FP64: square only.
static constexpr double NARROW_COST = 1.6;
static int choose_simt_shape(const tccg_plan* p, double* padded_work) {
  const bool dbl = p->prec == TCCG_PREC_FP64;
  int best = SIMT_SQUARE;
  double best_w = 0;
  for (int sh = SIMT_SQUARE; sh <= (dbl ? SIMT_SQUARE : SIMT_NARROW_M); ++sh) {
    int bm, bn, bk;
    simt_dims(dbl, sh, &bm, &bn, &bk);
    const double w = (double)round_up(p->M, bm) * (double)round_up(p->N, bn) *
                     (sh == SIMT_SQUARE ? 1.0 : NARROW_COST);
    const bool forced = !dbl && p->tune.simt_tile == sh + 1;
    if (forced || (p->tune.simt_tile == 0 && (sh == SIMT_SQUARE || w < best_w))) {
      best = sh;
      best_w = w;
      if (forced) break;
    }
  }
  if (padded_work) *padded_work = best_w;
  return best;
}

static bool direct_eligible(const tccg_plan* p, int shape);
static bool unit_first(int n, const int64_t* ext, const int64_t* str);

// The gather loader of the tcgen05 BF16X3 kernel (TC_LOAD_GATHER) can serve
// the plan: FP32 operands, GETT, one-SM tiles, and each operand read
// coalesced along its gather direction (k quads, a unit-stride first K mode
// read along k, a unit-stride first row mode read along rows) or small
// enough (<= 4 MiB) to stay in L2 across its re-reads.
static bool gather_eligible(const tccg_plan* p) {
  if (p->prec != TCCG_PREC_BF16X3 || p->dtype != TCCG_F32 || p->tune.method != TCCG_METHOD_GETT ||
      p->tune.pair || p->tune.load == 1 || (p->tune.tile_n != 0 && p->tune.tile_n != 128))
    return false;
  if (p->tune.load == 2) return true;
  const tccg_desc& d = p->d;
  const int64_t small = 4 << 20;
  const bool a_ok = p->ks_a || unit_first(d.nk, d.k_ext, d.a_k_stride) ||
                    unit_first(d.nm, d.m_ext, d.a_m_stride) || p->M * p->K * 4 <= small;
  const bool b_ok = p->ks_b || unit_first(d.nk, d.k_ext, d.b_k_stride) ||
                    unit_first(d.nn, d.n_ext, d.b_n_stride) || p->N * p->K * 4 <= small;
  return a_ok && b_ok;
}

// Tensor-core time model (seconds), fitted on B200 timings of the 256-item
// batched workload: tensor cores at 0.6 PFLOP/s effective (x3 for
// split-BF16x3) on 128 x 192 tiles, the C epilogue at 3 TB/s, operands
// streamed at 4.5 TB/s three times with the packing pass (pack read, packed
// write, GEMM read); the gather loader's 128 x 128 tiles at 0.5 PFLOP/s with
// one operand pass. Tile padding counts as work.
static double tc_time(const tccg_plan* p, bool gather) {
  const double M = (double)p->M, N = (double)p->N, K = (double)p->K;
  const double Mt = (double)round_up(p->M, 128), Nt = (double)round_up(p->N, gather ? 128 : 192);
  const double op = (M + N) * K * (p->dtype == TCCG_BF16 ? 2.0 : 4.0), cb = M * N * 4.0;
  const double x3 = p->prec == TCCG_PREC_BF16X3 ? 3.0 : 1.0;
  return std::max(2.0 * Mt * Nt * K * x3 / (gather ? 0.5e15 : 0.6e15),
                  cb / 3e12 + (gather ? 1.0 : 3.0) * op / 4.5e12);
}

// The gather loader runs only when asked for (tuning.load = 2, which the
// autotuner tries): measured on the 256-item batched workload, its producer
// warps bring in 0.3-0.7 TB/s per kernel where the packing pass plus TMA
// loads move operands at 3-5 TB/s, so the model never picks it.
static bool choose_gather(const tccg_plan* p) {
  return p->tune.load == 2 && gather_eligible(p);
}

// CUDA-core tile kernel model (seconds): 35 TFLOP/s on the tile shape
// choose_simt_shape picks (its padding counted as work), operands streamed
// at 4.5 TB/s three times with a packing pass, once where the kernel reads
// them in place.
static double simt_time(const tccg_plan* p) {
  const double M = (double)p->M, N = (double)p->N, K = (double)p->K;
  double simt_work = 0;  // padded M x N of the CUDA-core tile shape it would use
  const int shape = choose_simt_shape(p, &simt_work);
  const double simt_passes = direct_eligible(p, shape) ? 1.0 : 3.0;  // operand reads
  const double op = (M + N) * K * (p->dtype == TCCG_BF16 ? 2.0 : 4.0), cb = M * N * 4.0;
  return std::max(2.0 * simt_work * K / 35e12, (cb + simt_passes * op) / 4.5e12);
}

static bool choose_simt(const tccg_plan* p) {
  if (p->prec == TCCG_PREC_FP32 || p->prec == TCCG_PREC_FP64) return true;
  if (p->tune.pair || p->tune.variant > 0 || p->tune.load > 0) return false;
  if (p->tune.variant < 0) return true;
  // against the tensor-core model (tc_time, with the loader the tuning asks for)
  return simt_time(p) < tc_time(p, p->tune.load == 2 && gather_eligible(p));
}

// First mode of extent > 1 has unit stride (or no such mode).
static bool unit_first(int n, const int64_t* ext, const int64_t* str) {
  for (int i = 0; i < n; ++i)
    if (ext[i] > 1) return str[i] == 1;
  return true;
}

// Whether the CUDA-core kernel with tile shape `shape` reads the operands in
// place (no packing pass): asked for by the tuning, or -- automatically --
// when the pack's extra traffic matters and each operand's gather runs along
// a unit-stride mode (narrow tiles: a row mode or a K mode) or the operand is
// small enough to stay cached; short K only for the square tile. Not for
// TTGT (whose point is the transposition) and not where the pack converts
// (bf16 operands, BF16 rounding).
static bool direct_eligible(const tccg_plan* p, int shape) {
  if (p->tune.method != TCCG_METHOD_GETT || p->tune.direct < 0) return false;
  if (p->dtype == TCCG_BF16 || p->prec == TCCG_PREC_BF16) return false;
  if (p->tune.direct > 0) return true;
  if (p->tune.shortk > 0) return false;  // the short-K kernel reads packed operands
  const bool narrow = shape != SIMT_SQUARE;
  if (p->K > 256 && !narrow) return false;
  // the pack's extra traffic (2 x the operands) must matter next to C's;
  // otherwise the 16-byte loads of packed operands win
  if (4 * (p->M + p->N) * p->K < p->M * p->N) return false;
  const int64_t es = p->prec == TCCG_PREC_FP64 ? 8 : 4, small = 4 << 20;
  const tccg_desc& d = p->d;
  const bool a_ok = unit_first(d.nm, d.m_ext, d.a_m_stride) || p->M * p->K * es <= small ||
                    (narrow && unit_first(d.nk, d.k_ext, d.a_k_stride));
  const bool b_ok = unit_first(d.nn, d.n_ext, d.b_n_stride) || p->N * p->K * es <= small ||
                    (narrow && unit_first(d.nk, d.k_ext, d.b_k_stride));
  return a_ok && b_ok;
}

static bool choose_direct(const tccg_plan* p) {
  return simt_path(p) && direct_eligible(p, p->simt_shape);
}

// Narrow tiles, direct loads: gather an operand along k when its unit
// stride is a K mode and not a row mode.
static void choose_gather_k(tccg_plan* p) {
  const tccg_desc& d = p->d;
  const bool narrow = p->simt_shape != SIMT_SQUARE;
  p->gather_k_a = p->direct && narrow && !unit_first(d.nm, d.m_ext, d.a_m_stride) &&
                  unit_first(d.nk, d.k_ext, d.a_k_stride);
  p->gather_k_b = p->direct && narrow && !unit_first(d.nn, d.n_ext, d.b_n_stride) &&
                  unit_first(d.nk, d.k_ext, d.b_k_stride);
}

// The short-K kernel moves its C block by TMA when C is a 2-D matrix
// C[m + ldc n] with a 16-byte column stride and at least one full tile in
// each direction (else by cp.async through the offset tables).
static bool shortk_tma(const tccg_plan* p, int64_t ldc) {
  const bool dbl = p->prec == TCCG_PREC_FP64;
  const int64_t es = dbl ? 8 : 4;
  const int BM = dbl ? SimtCfg<double>::BM : SimtCfg<float>::BM;
  const int BN = dbl ? SimtCfg<double>::BN : SimtCfg<float>::BN;
  return ldc > 0 && (ldc * es) % 16 == 0 && p->M >= BM && p->N >= BN &&
         p->M < (int64_t(1) << 31) && p->N < (int64_t(1) << 31);
}

// The short-K kernel that prefetches its C block under the FMA phase:
// packed operands, the whole K in one panel, no k-split. Automatically only
// with the TMA C block (the cp.async one measured no faster than the tile
// kernel) and at least two tiles per SM. TTGT writes the contiguous C'
// (ldc = M).
static bool choose_shortk(const tccg_plan* p, int64_t tiles) {
  if (p->direct || p->ksplit > 1 || p->tune.shortk < 0 || p->simt_shape != SIMT_SQUARE) return false;
  const int kp = p->prec == TCCG_PREC_FP64 ? SimtShortKCfg<double>::KP : SimtShortKCfg<float>::KP;
  if (p->Kp > kp) return false;
  if (p->tune.shortk > 0) return true;
  const int64_t ldc = p->tune.method == TCCG_METHOD_TTGT ? p->M : p->c_ldc;
  return shortk_tma(p, ldc) && tiles >= 2 * (int64_t)p->num_sms;
}

// K slices for `tiles` C tiles over `kblocks` k-blocks when `slots` CTAs run
// at once: the requested count, or (requested == 0) as many slices as fill
// the idle slots, each at least `min_kb` k-blocks long. Returns the k-blocks
// per slice; *splits gets the slice count (no empty slices).
static int64_t choose_ksplit(int32_t requested, int64_t tiles, int64_t kblocks, int64_t slots,
                             int64_t min_kb, int32_t* splits) {
  int64_t ks = 1;
  if (requested > 1)
    ks = requested;
  else if (requested == 0 && 2 * tiles <= slots)
    ks = std::min<int64_t>(slots / tiles, kblocks / min_kb);
  ks = std::max<int64_t>(1, std::min<int64_t>(ks, kblocks));
  const int64_t per = cdiv(kblocks, ks);
  *splits = (int32_t)cdiv(kblocks, per);
  return per;
}

// offsets[l] = sum_i idx_i(l) * stride_i, l the linear index over the modes
// (first mode fastest).
static void build_offsets(int n, const int64_t* ext, const int64_t* stride,
                          std::vector<int64_t>& out) {
  int64_t total = 1;
  for (int i = 0; i < n; ++i) total *= ext[i];
  out.resize((size_t)total);
  int64_t idx[TCCG_MAX_MODES] = {0};
  int64_t off = 0;
  for (int64_t l = 0; l < total; ++l) {
    out[(size_t)l] = off;
    for (int i = 0; i < n; ++i) {
      idx[i]++;
      off += stride[i];
      if (idx[i] < ext[i]) break;
      off -= idx[i] * stride[i];
      idx[i] = 0;
    }
  }
}

static int upload(const std::vector<int64_t>& h, int64_t** dptr) {
  size_t bytes = std::max<size_t>(h.size(), 1) * sizeof(int64_t);
  CUDA_TRY(cudaMalloc((void**)dptr, bytes));
  if (!h.empty()) CUDA_TRY(cudaMemcpy(*dptr, h.data(), h.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  return TCCG_OK;
}

// Fast read direction of an operand: 1 when its first K mode (extent > 1) has
// a smaller stride than its first row mode, i.e. consecutive k are closer in
// memory than consecutive m (or n).
static int32_t pick_read_k_fast(int nr, const int64_t* rext, const int64_t* rstr, int nk,
                                const int64_t* kext, const int64_t* kstr) {
  int64_t rs = INT64_MAX, ks = INT64_MAX;
  for (int i = 0; i < nr; ++i)
    if (rext[i] > 1) { rs = rstr[i] < 0 ? -rstr[i] : rstr[i]; break; }
  for (int i = 0; i < nk; ++i)
    if (kext[i] > 1) { ks = kstr[i] < 0 ? -kstr[i] : kstr[i]; break; }
  return ks < rs ? 1 : 0;
}

// ---- skinny kernel: eligibility, geometry and model ----------------------
// FP32 operands (FP32 accumulation serves BF16X3 as well: more accurate
// than its three-product split), GETT, a narrow side of at most 256 rows (one
// pass of up to 64 rows, or passes of 32 / 64 rows).
static bool skinny_eligible(const tccg_plan* p) {
  if (p->dtype != TCCG_F32 || (p->prec != TCCG_PREC_FP32 && p->prec != TCCG_PREC_BF16X3)) return false;
  if (p->tune.method != TCCG_METHOD_GETT || p->tune.pair) return false;
  return std::min(p->M, p->N) <= SK_SMAX && p->K <= INT32_MAX;
}

// The tensor-core skinny kernel: split-BF16x3, the skinny kernel's narrow
// sides (<= 256: passes of 64 rows above 64), K whose packed Q columns (2 x
// K rounded up to 32) stay TMA coordinates.
static bool skinny_tc_eligible(const tccg_plan* p) {
  return skinny_eligible(p) && p->prec == TCCG_PREC_BF16X3 && p->K <= (int64_t(1) << 29);
}

static long long abs_ll(int64_t v) { return v < 0 ? -(long long)v : (long long)v; }

// Smallest |stride| over modes of extent > 1 (LLONG_MAX when there is none).
static long long min_abs_stride(int n, const int64_t* ext, const int64_t* str) {
  long long m = LLONG_MAX;
  for (int i = 0; i < n; ++i)
    if (ext[i] > 1) m = std::min(m, abs_ll(str[i]));
  return m;
}

// Geometry of the skinny kernel (SkinnyArgs without pointers) and the Y-space
// mode list (W modes other than X, by increasing P stride). False when the
// blocks would not fit one launch. tc: the tensor-core kernel's rows (one
// pass of S rounded up to 16) and k slices (one CTA per SM).
static bool skinny_geometry(tccg_plan* p, std::vector<int>& ym, int* xmode, bool tc = false) {
  const tccg_desc& d = p->d;
  const bool sn = p->N <= p->M;  // narrow side: N (W = M, P = GA) or M (W = N, P = GB)
  p->sk_s_is_n = sn;
  const int nw = sn ? d.nm : d.nn, nsm = sn ? d.nn : d.nm;
  const int64_t* wext = sn ? d.m_ext : d.n_ext;
  const int64_t* wp = sn ? d.a_m_stride : d.b_n_stride;
  const int64_t* wc = sn ? d.c_m_stride : d.c_n_stride;
  const int64_t* kp = sn ? d.a_k_stride : d.b_k_stride;
  const int64_t* kq = sn ? d.b_k_stride : d.a_k_stride;
  const int64_t* sext = sn ? d.n_ext : d.m_ext;
  const int64_t* sq = sn ? d.b_n_stride : d.a_m_stride;
  const int64_t* sc = sn ? d.c_n_stride : d.c_m_stride;
  SkinnyArgs& a = p->sk;
  a = SkinnyArgs{};
  int X = -1;  // the W mode C stores contiguously
  for (int i = 0; i < nw; ++i)
    if (wext[i] > 1 && (X < 0 || abs_ll(wc[i]) < abs_ll(wc[X]))) X = i;
  ym.clear();
  for (int i = 0; i < nw; ++i)
    if (i != X && wext[i] > 1) ym.push_back(i);
  std::stable_sort(ym.begin(), ym.end(), [&](int u, int v) { return abs_ll(wp[u]) < abs_ll(wp[v]); });
  *xmode = X;
  // 32-bit offsets: every element offset of P, Q and C below 2^31
  auto span = [](int n, const int64_t* ext, const int64_t* str) {
    long long t = 0;
    for (int i = 0; i < n; ++i) t += (long long)(ext[i] - 1) * abs_ll(str[i]);
    return t;
  };
  const long long lim = INT32_MAX;
  if (span(nw, wext, wp) + span(d.nk, d.k_ext, kp) >= lim ||
      span(nsm, sext, sq) + span(d.nk, d.k_ext, kq) >= lim ||
      span(nw, wext, wc) + span(nsm, sext, sc) >= lim || p->K >= lim)
    return false;
  a.ex = (int32_t)(X >= 0 ? wext[X] : 1);
  a.px = (int32_t)(X >= 0 ? wp[X] : 0);
  a.cx = (int32_t)(X >= 0 ? wc[X] : 0);
  int64_t ey = 1;
  for (int i : ym) ey *= wext[i];
  a.ey = (int32_t)ey;
  // P loads along its stride-one direction
  const long long px = X >= 0 ? abs_ll(wp[X]) : LLONG_MAX;
  const long long py = ym.empty() ? LLONG_MAX : abs_ll(wp[ym[0]]);
  const long long pk = min_abs_stride(d.nk, d.k_ext, kp);
  a.p_walk = pk < std::min(px, py) ? SK_P_K : py < px ? SK_P_Y : SK_P_X;
  // box: along X (and the first Y modes) when P and C agree on X; a
  // transposition needs runs both ways -- all of X up to 32, else 16 x 16
  int64_t tx, ty;
  if (a.p_walk == SK_P_Y) {
    tx = a.ex <= 32 ? a.ex : a.ey <= 16 ? std::min<int64_t>(a.ex, SK_BW / a.ey) : 16;
    ty = std::min<int64_t>(a.ey, SK_BW / tx);
    tx = std::min<int64_t>(a.ex, SK_BW / ty);
  } else {
    tx = std::min<int64_t>(a.ex, SK_BW);
    ty = std::min<int64_t>(a.ey, SK_BW / tx);
  }
  a.tx = (int32_t)tx;
  a.ty = (int32_t)ty;
  a.bxn = (int32_t)cdiv(a.ex, tx);
  const int64_t nblk = (int64_t)a.bxn * cdiv(a.ey, ty);
  if (nblk > INT32_MAX / 4) return false;
  a.nblk = (int32_t)nblk;
  // C walk: C's stride-one index on the narrow side (runs of that S mode,
  // when it is the first one), else X then the next C stride's side
  const long long cs = min_abs_stride(nsm, sext, sc), cx = X >= 0 ? abs_ll(wc[X]) : LLONG_MAX;
  long long cymin = LLONG_MAX;
  for (int i : ym) cymin = std::min(cymin, abs_ll(wc[i]));
  a.c_walk = cymin < cs ? SK_C_XY : SK_C_XS;
  a.s_run = 0;
  if (cs < cx) {
    int s0 = -1;  // first S mode of extent > 1
    for (int i = 0; i < nsm && s0 < 0; ++i)
      if (sext[i] > 1) s0 = i;
    if (s0 >= 0 && abs_ll(sc[s0]) == 1) {
      a.c_walk = SK_C_SX;
      a.s_run = (int32_t)sext[s0];
    }
  }
  a.q_kfast = min_abs_stride(d.nk, d.k_ext, kq) < min_abs_stride(nsm, sext, sq) ? 1 : 0;
  // rows per thread: one pass of the smallest of 16 / 32 / 48 rows; a longer
  // S runs passes of 32 rows (the passes of a block are neighbouring jobs:
  // their P chunks come from L2). 64-row passes (16 rows per thread) need
  // more than the 128 registers two CTAs per SM leave a thread.
  const int64_t S = sn ? p->N : p->M;
  p->sk_tc = tc;
  p->sk_spad = (int32_t)std::min<int64_t>(round_up(S, 16), SKT_SMAX);
  if (tc) {  // passes of spad rows (MMA N)
    a.rs = p->sk_spad / 4;
    a.npass = (int32_t)cdiv(S, p->sk_spad);
  } else if (S <= 48) {
    a.rs = (int32_t)std::max<int64_t>(4, round_up(cdiv(S, 4), 4));
    a.npass = 1;
  } else {
    a.rs = 8;
    a.npass = (int32_t)cdiv(S, 32);
  }
  a.S = (int32_t)S;
  a.K = (int32_t)p->K;
  a.nchunks = (int32_t)cdiv(p->K, SK_KC);
  int lg = 0;
  while ((1 << lg) < std::min<int64_t>(p->K, SK_KC)) ++lg;
  a.kr_log2 = lg;
  // a narrow side of at most 16 rows: P straight to registers (skinny_reg_kernel);
  // TCCG_B200_SKINNY_REG=0 keeps the shared-memory path
  const char* reg_env = std::getenv("TCCG_B200_SKINNY_REG");
  p->sk_reg = !tc && a.rs == 4 && a.npass == 1 && !(reg_env && std::strcmp(reg_env, "0") == 0);
  a.spr = 4 * a.rs;
  // C's stride-one S mode (extent e0 < S, unit stride) directly followed in C
  // by X: passes of whole runs (spr = the most runs in one 32-row staging
  // step), each (run, box row) stored as one range of e0 x floats
  // (SK_CLIN_RUNS), when that takes no more passes
  bool runs = false;
  if (!tc && !p->sk_reg && a.c_walk == SK_C_SX && a.s_run < S && a.cx == a.s_run) {
    const int32_t spr = (std::min<int32_t>(a.spr, SK_SUB) / a.s_run) * a.s_run;
    int sfirst = -1;
    for (int i = 0; i < nsm && sfirst < 0; ++i)
      if (sext[i] > 1) sfirst = i;
    if (spr > 0 && cdiv(S, spr) == a.npass && sc[sfirst] == 1) {
      runs = true;
      a.spr = spr;
    }
  }
  // k-split: (block, pass) jobs that cannot fill the persistent CTAs,
  // slices of >= 4 chunks
  const int64_t per_sm = tc ? 1 : p->sk_reg ? SKR_CTAS_PER_SM : SK_CTAS_PER_SM;
  a.chunks_per_split = (int32_t)choose_ksplit(p->tune.ksplit, (int64_t)a.nblk * a.npass, a.nchunks,
                                              per_sm * p->num_sms, 4, &p->sk_ksplit);
  if (tc && p->tune.ksplit == 0) {
    // one CTA per SM runs whole jobs: the split whose busiest CTA has the
    // fewest chunks, each slice counted two chunks more (its partial sums
    // written and read again), slices of >= 4 chunks
    double best = 1e300;
    for (int64_t s = 1; s <= std::max<int64_t>(1, std::min<int64_t>(2 * p->num_sms, a.nchunks / 4)); ++s) {
      const int64_t per = cdiv(a.nchunks, s), ns = cdiv(a.nchunks, per);
      const double cost =
          (double)cdiv((int64_t)a.nblk * a.npass * ns, p->num_sms) * (double)(per + (ns > 1 ? 2 : 0));
      if (cost < best) {
        best = cost;
        a.chunks_per_split = (int32_t)per;
        p->sk_ksplit = (int32_t)ns;
      }
    }
  }
  a.ksplit = p->sk_ksplit;
  const int64_t njobs = (int64_t)a.nblk * a.npass * a.ksplit;
  if (njobs > INT32_MAX) return false;
  a.njobs = (int32_t)njobs;
  // 16-byte P copies: x at unit stride, every k offset a multiple of 4 (the
  // run checks P's alignment); linear C rows of a box (SkinnyCLin)
  std::vector<int64_t> t;
  build_offsets(d.nk, d.k_ext, kp, t);
  bool k4 = true;
  for (int64_t v : t) k4 &= v % 4 == 0;
  p->sk_p_vec = a.p_walk == SK_P_X && a.px == 1 && k4;
  build_offsets(nsm, sext, sc, t);
  auto affine = [&](int64_t st) {
    for (size_t i = 0; i < t.size(); ++i)
      if (t[i] != t[0] + (int64_t)i * st) return false;
    return true;
  };
  a.c_lin = runs ? SK_CLIN_RUNS : SK_CLIN_NONE;
  if (runs)
    ;
  else if (a.c_walk == SK_C_XS && a.cx == 1 && a.tx == a.ex && a.bxn == 1 && affine(a.ex))
    a.c_lin = SK_CLIN_XS;
  else if (a.c_walk == SK_C_SX && a.npass == 1 && S <= SK_SUB && a.cx == S && affine(1))
    a.c_lin = SK_CLIN_SX;
  a.alpha = 1.0f;
  a.beta = 0.0f;
  return true;
}

// Skinny kernel model (seconds), fitted on B200 timings of eleven items of
// the 256-item batched workload (0.08-1.4 ms; within 25 % of each): FP32
// FMAs over the blocks' positions and padded rows at 18 TFLOP/s, C written at
// 2.0 TB/s and P read at 6 TB/s (its copies overlap the FMAs and stores), as
// a sum -- a job's phases follow one another in its CTA -- plus 4 us; a
// k-split adds its slices' traffic and the reduction's launch.
static double skinny_time(const tccg_plan* p) {
  const SkinnyArgs& a = p->sk;
  const double W = (double)a.ex * (double)a.ey, K = (double)p->K, S = (double)a.S;
  const double rows = 4.0 * a.rs * a.npass;
  const double fma = 2.0 * (double)a.nblk * SK_BW * rows * K;
  double t = fma / 18e12 + 4.0 * W * S / 2.0e12 + 4.0 * W * K / 6e12;
  // the rates need every persistent CTA busy
  const double slots = (double)(p->sk_reg ? SKR_CTAS_PER_SM : SK_CTAS_PER_SM) * p->num_sms;
  if ((double)a.njobs < slots) t *= slots / (double)a.njobs;
  t += 4e-6;
  if (p->sk_ksplit > 1) t += 8.0 * p->sk_ksplit * (double)a.nblk * rows * SK_BW / 3e12 + 5e-6;
  return t;
}

// The persistent skinny kernel of a rows-per-thread class (4, 8 or 12).
template <typename F>
static void with_skinny_rs(int rs, F&& f) {
  switch (rs) {
    case 4: f(std::integral_constant<int, 4>()); break;
    case 8: f(std::integral_constant<int, 8>()); break;
    default: f(std::integral_constant<int, 12>()); break;
  }
}

// Whether the plan runs the skinny kernel: asked for, or -- unless the
// tuning asks for another kernel family -- where it was measured to win or
// its model beats the others'. Measured on the 233 items of the 256-item
// batched workload it can take (standalone runs, L2 flushed): with K <= 32,
// a narrow side of at most 48 and at least 65536 positions on the wide side
// it was the fastest kernel on 10 of 13 items (0.38-0.9x the time of the best
// other one; 1.1-1.4x on the three others), and with K <= 32 and over 2^20
// positions on all three such items (any narrow side up to 256). There the
// tile kernels' models undercount the packing pass, which must transpose the
// wide operand (0.9 TB/s measured where they assume 4.5), and the tcgen05
// epilogue's short C runs (0.4-0.5 TB/s measured where it assumes 3).
// Whether a plan runs the tensor-core skinny kernel (skinny_tc.cuh): asked
// for with tuning.skinny = 2, or -- unless the tuning asks for something
// else -- K > 32 (two chunks or more), at least 48 blocks of positions
// (enough CTAs without a deep k-split) and 17-64 rows. Measured on the 169
// items of the 256-item batched workload it can take (standalone, L2
// flushed): on the 20 such items 0.52 ms less in sum than the kernels chosen
// before; it loses where K <= 32 (C stores dominate) and on a few blocks
// with a very long K (few CTAs, deep k-splits).
static bool choose_skinny_tc(const tccg_plan* p) {
  if (p->tune.skinny == 2) return true;
  if (p->tune.skinny != 0) return false;
  const tccg_tuning& t = p->tune;
  if (t.variant != 0 || t.load != 0 || t.direct != 0 || t.shortk != 0 || t.simt_tile != 0 ||
      t.tile_n != 0 || t.ksplit != 0)
    return false;
  // a narrow side of at most 16 takes the CUDA-core register path instead
  // (choose_skinny): on the 8 such items 1.36 ms in sum against 1.50 ms here
  // -- except where P's stride-one index is contracted and K spans at least
  // 8 chunks: the register path's loads (16 consecutive k per lane) then
  // touch 32 rows per warp load (items 40 / 48 of the 256-item batched
  // workload: 0.21 / 0.31 ms there, 0.20 / 0.25 ms here)
  if (p->K > SK_KC && p->sk.nblk >= 48 && p->sk.S <= 16 && p->sk.p_walk == SK_P_K &&
      p->sk.nchunks >= 8)
    return true;
  return p->K > SK_KC && p->sk.nblk >= 48 && p->sk.S > 16 && p->sk.S <= SKT_SMAX;
}

static bool choose_skinny(const tccg_plan* p) {
  if (p->tune.skinny > 0) return true;
  if (p->tune.skinny < 0) return false;
  const tccg_tuning& t = p->tune;
  if (t.variant != 0 || t.load != 0 || t.direct != 0 || t.shortk != 0 || t.simt_tile != 0 ||
      t.tile_n != 0)
    return false;
  const SkinnyArgs& a = p->sk;
  const int64_t W = (int64_t)a.ex * a.ey;
  if (p->K <= SK_KC && ((a.S <= 48 && W >= 65536) || W >= (int64_t(1) << 20))) return true;
  // FP32 precision (the CUDA-core tiles its only other choice): a narrow side
  // of at most 48 and at least 4096 positions, any K -- on the 59 such items
  // 2.6 ms less in sum than the CUDA-core tiles (21 % of their time)
  if (p->prec == TCCG_PREC_FP32 && a.S <= 48 && W >= 4096) return true;
  // split-BF16x3, a narrow side of at most 16 (the register path), K > 32
  // and at least 48 blocks: on the 8 such items 1.36 ms in sum where the
  // kernels chosen before took 2.13 ms (the tensor-core skinny kernel 1.50 ms)
  if (p->sk_reg && p->K > SK_KC && a.nblk >= 48) return true;
  double other = simt_time(p);
  if (p->prec == TCCG_PREC_BF16X3) other = std::min(other, tc_time(p, false));
  return skinny_time(p) < other;
}

static void plan_free(tccg_plan* p) {
  if (!p) return;
  int64_t* ts[] = {p->t_a_m, p->t_a_k, p->t_b_n, p->t_b_k, p->t_c_m, p->t_c_n, p->t_id_m, p->t_id_n,
                   p->t_a_vsrc, p->t_a_vdst, p->t_b_vsrc, p->t_b_vdst};
  for (auto t : ts)
    if (t) cudaFree(t);
  if (p->d_status) cudaFree(p->d_status);
  if (p->t_sk) cudaFree(p->t_sk);
  delete p;
}

static int plan_layout(tccg_plan* p);
static int pair_clusters(bool x3, int* clusters);

// Smallest |stride| of the modes of extent > 1 (INT64_MAX if none).
static long long min_stride(int n, const int64_t* ext, const int64_t* str) {
  long long best = INT64_MAX;
  for (int i = 0; i < n; ++i)
    if (ext[i] > 1) best = std::min(best, std::llabs(str[i]));
  return best;
}

// Streaming K-major pack: every row offset is a multiple of 4 elements, and
// every quad of k (k % 4 == 0, k + 3 < K) starts at a multiple of 4 and runs
// over 4 consecutive elements -- 16-byte loads once the base is aligned.
static bool rows_by_4(const std::vector<int64_t>& roff) {
  for (int64_t o : roff)
    if (o % 4 != 0) return false;
  return true;
}
static bool k_quads(const std::vector<int64_t>& coff) {
  if (coff.size() < 4) return false;
  for (size_t k = 0; k + 3 < coff.size(); k += 4) {
    if (coff[k] % 4 != 0) return false;
    for (size_t j = 1; j < 4; ++j)
      if (coff[k + j] != coff[k] + (int64_t)j) return false;
  }
  return true;
}

// k-block tiles of a K-major pack (PackOperand::kb_*) when the operand's
// unit-stride mode is a K mode u other than the first K mode of extent > 1:
// tiles of kb_lo * kb_run consecutive k (kb_lo = product of the extents of
// the K modes before u, kb_run values of u) x kb_rows rows, at most
// PACK_KB_ELEMS elements. Needs runs of at least 8 along u, at most 1024 k
// per tile and whole quads of k (4 | kb_lo * kb_run).
static void kblock_tiles(int nk, const int64_t* kext, const int64_t* kstr, int32_t (&kb)[5]) {
  kb[0] = kb[1] = kb[2] = kb[3] = kb[4] = 0;
  int first = -1, u = -1;
  for (int i = 0; i < nk; ++i) {
    if (kext[i] <= 1) continue;
    if (first < 0) first = i;
    if (std::llabs(kstr[i]) == 1) u = i;
  }
  if (u < 0 || u == first || kext[u] < 8) return;
  int64_t lo = 1;
  for (int i = 0; i < u; ++i) lo *= kext[i];
  if (lo > 128) return;
  const int64_t run = std::min<int64_t>(kext[u], 1024 / lo), t = lo * run;
  if (run < 8 || t % 4 != 0) return;
  kb[0] = (int32_t)lo;
  kb[1] = (int32_t)run;
  kb[2] = (int32_t)std::max<int64_t>(1, std::min<int64_t>(32, PACK_KB_ELEMS / t));
  kb[3] = (int32_t)kext[u];
  kb[4] = kstr[u] > 0 ? 1 : -1;
}

// The k-block tiles of an operand (kblock_tiles) may move 4 consecutive u at
// once: kb_lo, the run and u's extent multiples of 4, u's stride +1, and in
// the column table every quad of u (u % 4 == 0) starts at a multiple of 4 and
// runs over 4 consecutive elements.
static bool kblock_quads(int nk, const int64_t* kext, const int64_t* kstr,
                         const std::vector<int64_t>& coff) {
  int32_t kb[5];
  kblock_tiles(nk, kext, kstr, kb);
  const int64_t lo = kb[0], run = kb[1], ext = kb[3];
  if (lo == 0 || lo % 4 != 0 || run % 4 != 0 || ext % 4 != 0 || kb[4] != 1) return false;
  const int64_t K = (int64_t)coff.size();
  for (int64_t k = 0; k < K; ++k) {
    if (((k / lo) % ext) % 4 != 0) continue;  // not the first u of a quad
    if (coff[(size_t)k] % 4 != 0) return false;
    for (int64_t j = 1; j < 4 && k + j * lo < K; ++j)
      if (coff[(size_t)(k + j * lo)] != coff[(size_t)k] + j) return false;
  }
  return true;
}

// For a K-major pack whose rows are read one per lane: if a later row mode
// has a smaller stride than the first (non-unit) mode, visit the rows with
// that mode fastest. vsrc[v] = source offset, vdst[v] = destination row of
// visit index v. Returns false (tables untouched) when no reorder helps.
static bool build_visit(int n, const int64_t* ext, const int64_t* str, std::vector<int64_t>& vsrc,
                        std::vector<int64_t>& vdst) {
  int first = -1, best = -1;
  for (int i = 0; i < n; ++i) {
    if (ext[i] <= 1) continue;
    if (first < 0) first = i;
    if (best < 0 || std::llabs(str[i]) < std::llabs(str[best])) best = i;
  }
  if (first < 0 || best == first || std::llabs(str[best]) >= std::llabs(str[first])) return false;
  std::vector<int> order{best};
  for (int i = 0; i < n; ++i)
    if (i != best) order.push_back(i);
  std::vector<int64_t> place(n);
  int64_t total = 1;
  for (int i = 0; i < n; ++i) {
    place[i] = total;
    total *= ext[i];
  }
  vsrc.assign((size_t)total, 0);
  vdst.assign((size_t)total, 0);
  std::vector<int64_t> idx(n, 0);
  int64_t so = 0, dr = 0;
  for (int64_t v = 0; v < total; ++v) {
    vsrc[(size_t)v] = so;
    vdst[(size_t)v] = dr;
    for (int j = 0; j < n; ++j) {  // odometer in visit order
      const int i = order[j];
      if (++idx[i] < ext[i]) {
        so += str[i];
        dr += place[i];
        break;
      }
      so -= (ext[i] - 1) * str[i];
      dr -= (ext[i] - 1) * place[i];
      idx[i] = 0;
    }
  }
  return true;
}

// Product of the n extents of one index class (M, N or K). Each extent must
// be >= 1 and the running product may never exceed 2^31 (checked before each
// multiplication, so that huge extents cannot wrap to a small product).
static int mode_product(const char* cls, int n, const int64_t* ext, int64_t* out) {
  int64_t p = 1;
  for (int i = 0; i < n; ++i) {
    if (ext[i] < 1) return fail(TCCG_ERR_INVALID, "%s extent %d is %lld", cls, i, (long long)ext[i]);
    if (ext[i] > ((int64_t)1 << 31) / p)
      return fail(TCCG_ERR_UNSUPPORTED, "%s (the product of its extents) must be <= 2^31", cls);
    p *= ext[i];
  }
  *out = p;
  return TCCG_OK;
}

extern "C" int tccg_plan_create(const tccg_desc* desc, int32_t dtype, int32_t precision,
                                const tccg_tuning* tuning, tccg_plan** out) {
  if (!desc || !out) return fail(TCCG_ERR_INVALID, "null descriptor or output pointer");
  *out = nullptr;
  const tccg_desc& d = *desc;
  if (d.nm < 1 || d.nn < 1 || d.nk < 1 || d.nm > TCCG_MAX_MODES || d.nn > TCCG_MAX_MODES ||
      d.nk > TCCG_MAX_MODES)
    return fail(TCCG_ERR_INVALID, "mode counts (nm=%d nn=%d nk=%d) must be in [1,%d]", d.nm, d.nn,
                d.nk, TCCG_MAX_MODES);
  if (dtype != TCCG_F32 && dtype != TCCG_F64 && dtype != TCCG_BF16)
    return fail(TCCG_ERR_INVALID, "unknown dtype %d", dtype);
  if (precision < TCCG_PREC_FP32 || precision > TCCG_PREC_BF16X3)
    return fail(TCCG_ERR_INVALID, "unknown precision %d", precision);
  if ((dtype == TCCG_F64) != (precision == TCCG_PREC_FP64))
    return fail(TCCG_ERR_UNSUPPORTED, "FP64 operands need TCCG_PREC_FP64 and vice versa");
  if (dtype == TCCG_BF16 && precision != TCCG_PREC_BF16)
    return fail(TCCG_ERR_UNSUPPORTED, "BF16 operands are supported with TCCG_PREC_BF16 only");
  int64_t M = 1, N = 1, K = 1;
  int rc0 = mode_product("M", d.nm, d.m_ext, &M);
  if (!rc0) rc0 = mode_product("N", d.nn, d.n_ext, &N);
  if (!rc0) rc0 = mode_product("K", d.nk, d.k_ext, &K);
  if (rc0) return rc0;

  tccg_plan* p = new tccg_plan();
  p->d = d;
  p->dtype = dtype;
  p->prec = precision;
  if (tuning) p->tune = *tuning;
  p->M = M;
  p->N = N;
  p->K = K;
  if (p->tune.method != TCCG_METHOD_GETT && p->tune.method != TCCG_METHOD_TTGT) {
    plan_free(p);
    return fail(TCCG_ERR_UNSUPPORTED, "method %d is not available in this build", p->tune.method);
  }
  cudaError_t e = cudaGetDevice(&p->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device);
  if (e != cudaSuccess) {
    plan_free(p);
    return fail(TCCG_ERR_CUDA, "no usable CUDA device: %s", cudaGetErrorString(e));
  }
  std::vector<int64_t> h;
  int rc = TCCG_OK;
  // row offsets that are multiples of 4 and quads of k: the 16-byte pack
  // reads (streaming pass, 16-byte k-block tiles)
  build_offsets(d.nm, d.m_ext, d.a_m_stride, h);
  const bool rows4_a = rows_by_4(h);
  if (!rc) rc = upload(h, &p->t_a_m);
  build_offsets(d.nk, d.k_ext, d.a_k_stride, h);
  p->ks_a = rows4_a && k_quads(h);
  p->kbq_a = rows4_a && kblock_quads(d.nk, d.k_ext, d.a_k_stride, h);
  if (!rc) rc = upload(h, &p->t_a_k);
  build_offsets(d.nn, d.n_ext, d.b_n_stride, h);
  const bool rows4_b = rows_by_4(h);
  if (!rc) rc = upload(h, &p->t_b_n);
  build_offsets(d.nk, d.k_ext, d.b_k_stride, h);
  p->ks_b = rows4_b && k_quads(h);
  p->kbq_b = rows4_b && kblock_quads(d.nk, d.k_ext, d.b_k_stride, h);
  if (!rc) rc = upload(h, &p->t_b_k);
  build_offsets(d.nm, d.m_ext, d.c_m_stride, h);
  // C is "already [M][N]" when its M modes are dense from stride 1 and the N
  // modes continue densely after them (TTGT then needs no C transposition).
  {
    bool dense = true;
    int64_t s = 1;
    for (int i = 0; i < d.nm; ++i) { dense &= d.c_m_stride[i] == s; s *= d.m_ext[i]; }
    for (int i = 0; i < d.nn; ++i) { dense &= d.c_n_stride[i] == s; s *= d.n_ext[i]; }
    p->c_is_mn_dense = dense;
  }
  bool m_unit = true;
  for (size_t m = 0; m < h.size() && m_unit; ++m) m_unit = h[m] == (int64_t)m;
  if (!rc) rc = upload(h, &p->t_c_m);
  build_offsets(d.nn, d.n_ext, d.c_n_stride, h);
  if (m_unit) {
    const int64_t ldc = h.size() > 1 ? h[1] : std::max<int64_t>(p->M, 1);
    bool two_d = ldc > 0;
    for (size_t n = 0; n < h.size() && two_d; ++n) two_d = h[n] == (int64_t)n * ldc;
    p->c_ldc = two_d ? ldc : 0;
  }
  if (!rc) rc = upload(h, &p->t_c_n);
  if (!rc) {
    e = cudaMalloc((void**)&p->d_status, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemset(p->d_status, 0, sizeof(int32_t));
    if (e != cudaSuccess) rc = fail(TCCG_ERR_CUDA, "status word: %s", cudaGetErrorString(e));
  }
  p->crun = (d.c_m_stride[0] == 1 && d.m_ext[0] >= 2 && d.m_ext[0] < 32 && d.n_ext[0] > 1 &&
             d.c_n_stride[0] == d.m_ext[0])
                ? (int32_t)d.m_ext[0]
                : 0;
  if (!rc) {
    // the skinny kernel: its geometry, the model's choice, its Y-space tables
    std::vector<int> ym;
    int xmode = -1;
    const bool eligible = skinny_eligible(p) && skinny_geometry(p, ym, &xmode);
    if (p->tune.skinny > 0 && !eligible) {
      plan_free(p);
      return fail(TCCG_ERR_UNSUPPORTED,
                  "the skinny kernel needs FP32 operands, FP32 or BF16X3 precision, GETT, "
                  "min(M, N) <= 256 and tensors of fewer than 2^31 elements");
    }
    if (p->tune.skinny == 2 && !skinny_tc_eligible(p)) {
      plan_free(p);
      return fail(TCCG_ERR_UNSUPPORTED,
                  "the tensor-core skinny kernel needs split-BF16x3 precision, min(M, N) <= 256 "
                  "and K <= 2^29");
    }
    const bool use_tc = eligible && skinny_tc_eligible(p) && choose_skinny_tc(p);
    p->skinny = use_tc || (eligible && choose_skinny(p));
    if (use_tc && !skinny_geometry(p, ym, &xmode, true)) {
      plan_free(p);
      return fail(TCCG_ERR_UNSUPPORTED, "the tensor-core skinny kernel's jobs do not fit one launch");
    }
    if (p->skinny) {
      const bool sn = p->sk_s_is_n;
      int64_t ext[TCCG_MAX_MODES], sp[TCCG_MAX_MODES], scc[TCCG_MAX_MODES];
      for (size_t i = 0; i < ym.size(); ++i) {
        ext[i] = sn ? d.m_ext[ym[i]] : d.n_ext[ym[i]];
        sp[i] = sn ? d.a_m_stride[ym[i]] : d.b_n_stride[ym[i]];
        scc[i] = sn ? d.c_m_stride[ym[i]] : d.c_n_stride[ym[i]];
      }
      const int nsm = sn ? d.nn : d.nm;
      const int64_t* sext = sn ? d.n_ext : d.m_ext;
      // P / C offsets of the Y space, P's k, Q's rows and k, C's rows
      std::vector<int32_t> tab;
      auto add = [&](int n, const int64_t* e, const int64_t* st, int slot) {
        build_offsets(n, e, st, h);
        p->sk_tab[slot] = tab.size();
        for (int64_t v : h) tab.push_back((int32_t)v);
        while (tab.size() % 4) tab.push_back(0);  // 16-byte aligned starts
      };
      add((int)ym.size(), ext, sp, 0);
      add((int)ym.size(), ext, scc, 1);
      add(d.nk, d.k_ext, sn ? d.a_k_stride : d.b_k_stride, 2);
      add(nsm, sext, sn ? d.b_n_stride : d.a_m_stride, 3);
      add(d.nk, d.k_ext, sn ? d.b_k_stride : d.a_k_stride, 4);
      add(nsm, sext, sn ? d.c_n_stride : d.c_m_stride, 5);
      e = cudaMalloc((void**)&p->t_sk, tab.size() * sizeof(int32_t));
      if (e == cudaSuccess)
        e = cudaMemcpy(p->t_sk, tab.data(), tab.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) rc = fail(TCCG_ERR_CUDA, "skinny tables: %s", cudaGetErrorString(e));
    }
  }
  p->simt = !p->skinny && choose_simt(p);
  p->read_k_fast_a = pick_read_k_fast(d.nm, d.m_ext, d.a_m_stride, d.nk, d.k_ext, d.a_k_stride);
  p->read_k_fast_b = pick_read_k_fast(d.nn, d.n_ext, d.b_n_stride, d.nk, d.k_ext, d.b_k_stride);
  if (!p->skinny && !simt_path(p) && p->tune.load == 2 && p->prec == TCCG_PREC_BF16X3 && p->dtype == TCCG_F32 &&
      p->tune.method == TCCG_METHOD_GETT && !p->tune.pair && p->tune.tile_n != 0 &&
      p->tune.tile_n != 128) {
    const int32_t tn = p->tune.tile_n;
    plan_free(p);
    return fail(TCCG_ERR_UNSUPPORTED, "the gather loader has 128-column tiles (tile_n %d)", tn);
  }
  if (!p->skinny && !simt_path(p) && choose_gather(p)) {
    // gather schedules: 16-byte k quads, else along the operand's faster
    // direction (k or rows)
    p->gather = true;
    p->gread_a = p->ks_a ? GATHER_KQUAD : p->read_k_fast_a ? GATHER_K : GATHER_ROWS;
    p->gread_b = p->ks_b ? GATHER_KQUAD : p->read_k_fast_b ? GATHER_K : GATHER_ROWS;
  }
  if (!rc && !p->skinny && !simt_path(p) && !p->gather) {
    // tensor-core packs: unit stride on a later K mode -> k-block tiles read
    // along it; else walk the rows along the smallest-stride row mode when
    // that beats both the first row mode and reading along k
    // (FP32 sources only: the tiles move 4-byte elements by cp.async)
    if (!p->ks_a && p->dtype != TCCG_BF16) kblock_tiles(d.nk, d.k_ext, d.a_k_stride, p->kb_a);
    if (!p->ks_b && p->dtype != TCCG_BF16) kblock_tiles(d.nk, d.k_ext, d.b_k_stride, p->kb_b);
    std::vector<int64_t> vs, vd;
    auto kstride = [&](const int64_t* kst) {
      for (int i = 0; i < d.nk; ++i)
        if (d.k_ext[i] > 1) return std::llabs(kst[i]);
      return (long long)INT64_MAX;
    };
    if (!p->ks_a && p->kb_a[0] == 0 && min_stride(d.nm, d.m_ext, d.a_m_stride) < kstride(d.a_k_stride) &&
        build_visit(d.nm, d.m_ext, d.a_m_stride, vs, vd)) {
      p->read_k_fast_a = 0;
      rc = upload(vs, &p->t_a_vsrc);
      if (!rc) rc = upload(vd, &p->t_a_vdst);
    }
    if (!rc && !p->ks_b && p->kb_b[0] == 0 && min_stride(d.nn, d.n_ext, d.b_n_stride) < kstride(d.b_k_stride) &&
        build_visit(d.nn, d.n_ext, d.b_n_stride, vs, vd)) {
      p->read_k_fast_b = 0;
      rc = upload(vs, &p->t_b_vsrc);
      if (!rc) rc = upload(vd, &p->t_b_vdst);
    }
  }
  if (!rc) rc = plan_layout(p);
  if (rc) {
    plan_free(p);
    return rc;
  }
  *out = p;
  return TCCG_OK;
}

static int plan_layout(tccg_plan* p) {
  size_t ws = 0;
  const bool ttgt = p->tune.method == TCCG_METHOD_TTGT;
  if (p->skinny) {
    const SkinnyArgs& a = p->sk;
    if (p->sk_tc) {  // packed Q: passes x spad rows x Kc bf16 (K-major, [hi | lo] per 32 k)
      p->Kc = 2 * round_up(p->K, 32);
      p->off_q = 0;
      ws = align_up((size_t)a.npass * p->sk_spad * (size_t)p->Kc * 2, 256);
    }
    if (p->sk_ksplit > 1) {  // FP32 slices [split][block][pass][row][position]
      p->off_part = ws;
      ws = align_up(ws + (size_t)p->sk_ksplit * (size_t)a.nblk * a.npass * 4 * a.rs * SK_BW * 4, 256);
    }
    static const char* pw[] = {"x", "y", "k"};
    static const char* cw[] = {"xs", "xy", "sx"};
    if (p->sk_tc) {
      snprintf(p->describe, sizeof(p->describe),
               "method=GETT prec=bf16x3 kernel=skinny_tc<BF16X3> M=%lld N=%lld K=%lld narrow=%s "
               "S=%d n=%dx%d box=%dx%d ex=%lld ey=%lld blocks=%lld kchunks=%d ksplit=%d jobs=%lld "
               "grid=%lld load=%s%s store=%s%s%s pack=q",
               (long long)p->M, (long long)p->N, (long long)p->K, p->sk_s_is_n ? "N" : "M", a.S,
               a.npass, p->sk_spad, a.tx, a.ty, (long long)a.ex, (long long)a.ey, (long long)a.nblk,
               a.nchunks, p->sk_ksplit, (long long)a.njobs,
               (long long)std::min<int64_t>(a.njobs, p->num_sms), pw[a.p_walk],
               p->sk_p_vec ? " x16B" : "", cw[a.c_walk],
               a.c_walk == SK_C_SX ? (std::string(" run=") + std::to_string(a.s_run)).c_str() : "",
               a.c_lin ? " linear" : "");
      p->ws_bytes = ws;
      return TCCG_OK;
    }
    snprintf(p->describe, sizeof(p->describe),
             "method=GETT prec=%s kernel=skinny_gett<f32> M=%lld N=%lld K=%lld narrow=%s S=%d "
             "rows=%dx%d box=%dx%d ex=%lld ey=%lld blocks=%lld kchunks=%d ksplit=%d jobs=%lld "
             "grid=%lld load=%s%s%s store=%s%s%s%s pack=none",
             p->prec == TCCG_PREC_BF16X3 ? "bf16x3" : "fp32", (long long)p->M, (long long)p->N,
             (long long)p->K, p->sk_s_is_n ? "N" : "M", a.S, a.npass, a.spr, a.tx, a.ty,
             (long long)a.ex, (long long)a.ey, (long long)a.nblk, a.nchunks, p->sk_ksplit,
             (long long)a.njobs,
             (long long)std::min<int64_t>(
                 a.njobs, (int64_t)(p->sk_reg ? SKR_CTAS_PER_SM : SK_CTAS_PER_SM) * p->num_sms),
             pw[a.p_walk], p->sk_p_vec ? " x16B" : "", a.q_kfast ? " q=k" : " q=s", cw[a.c_walk],
             a.c_walk == SK_C_SX ? (std::string(" run=") + std::to_string(a.s_run)).c_str() : "",
             a.c_lin == SK_CLIN_RUNS ? " ranges" : a.c_lin ? " linear" : "",
             p->sk_reg ? " path=registers" : "");
    p->ws_bytes = ws;
    return TCCG_OK;
  }
  if (simt_path(p)) {
    const bool dbl = p->prec == TCCG_PREC_FP64;
    // the short-K kernel keeps the square tile: a tuning that asks for it
    // settles the shape
    p->simt_shape = p->tune.shortk > 0 ? SIMT_SQUARE : choose_simt_shape(p, nullptr);
    int BM, BN, BK;
    simt_dims(dbl, p->simt_shape, &BM, &BN, &BK);
    p->simt_bm = BM;
    p->simt_bn = BN;
    const int min_blocks = p->simt_shape == SIMT_SQUARE ? SimtCfg<float>::MIN_BLOCKS
                                                        : SimtCfg<float, SIMT_NARROW_N>::MIN_BLOCKS;
    const size_t es = dbl ? 8 : 4;
    p->Mp = round_up(p->M, BM);
    p->Np = round_up(p->N, BN);
    p->Kp = round_up(p->K, BK);
    p->ktiles = (int32_t)(p->Kp / BK);
    const int64_t tiles = (p->Mp / BM) * (p->Np / BN);
    // min_blocks CTAs per SM; a slice is at least 8 k-tiles
    p->ktiles_per_split = (int32_t)choose_ksplit(p->tune.ksplit, tiles, p->ktiles,
                                                 min_blocks * (int64_t)p->num_sms, 8, &p->ksplit);
    p->direct = choose_direct(p);
    choose_gather_k(p);
    p->shortk = choose_shortk(p, tiles);
    p->off_a = 0;
    if (!p->direct) {
      ws = align_up((size_t)(p->Kp * p->Mp) * es, 256);
      p->off_b = ws;
      ws = align_up(ws + (size_t)(p->Kp * p->Np) * es, 256);
    }
    if (p->ksplit > 1) {
      p->off_part = ws;
      ws = align_up(ws + (size_t)p->ksplit * p->Np * p->Mp * es, 256);
    }
    static const char* pn[] = {"fp32", "fp64", "bf16", "bf16x3"};
    snprintf(p->describe, sizeof(p->describe),
             "method=%s prec=%s kernel=simt_%s<%s> tile=%dx%dx%d M=%lld N=%lld K=%lld "
             "ksplit=%d pack=%s%s%s(%s a=%d b=%d)",
             ttgt ? "TTGT" : "GETT", pn[p->prec], p->shortk ? "shortk" : "gett", dbl ? "f64" : "f32",
             BM, BN, BK,
             (long long)p->M, (long long)p->N, (long long)p->K, p->ksplit,
             p->direct ? "none" : "MN", p->prec == TCCG_PREC_BF16 ? " bf16-rounded" : "",
             !p->shortk ? "" : shortk_tma(p, ttgt ? p->M : p->c_ldc) ? " cblock=tma" : " cblock=cp.async",
             p->direct ? "gather_k" : "read_k_fast",
             p->direct ? (int)p->gather_k_a : p->read_k_fast_a,
             p->direct ? (int)p->gather_k_b : p->read_k_fast_b);
  } else {
    const bool x3 = p->prec == TCCG_PREC_BF16X3;
    if (x3) {
      p->Kc = 2 * round_up(p->K, 32);
      p->num_kb = (int32_t)cdiv(p->K, 32);
    } else {
      p->Kc = round_up(p->K, 8);
      p->num_kb = (int32_t)cdiv(p->K, 64);
    }
    // BF16X3 accumulates 512 k per TMEM accumulator (tuning.variant overrides,
    // in k-blocks of 32); BF16 one chunk per tile
    p->chunk_kb = x3 ? (p->tune.variant > 0 ? p->tune.variant : 16) : p->num_kb;
    if (p->chunk_kb < 1) p->chunk_kb = 1;
    const bool pair = p->tune.pair != 0;
    int stages = 0;
    if (pair) {
      p->bn = x3 ? Tc2Cfg<TC_BF16X3>::BN : Tc2Cfg<TC_BF16>::BN;
      stages = x3 ? Tc2Cfg<TC_BF16X3>::STAGES : Tc2Cfg<TC_BF16>::STAGES;
    } else {
      p->tcv = tc_variant(x3, p->gather, p->tune.tile_n);
      if (p->tcv < 0)
        return fail(TCCG_ERR_UNSUPPORTED, "tile width %d is not built for %s%s", p->tune.tile_n,
                    x3 ? "BF16X3" : "BF16", p->gather ? " with the gather loader" : "");
      with_tc_variant(p->tcv, [&](auto k) {
        p->bn = decltype(k)::Cfg::BN;
        stages = decltype(k)::Cfg::STAGES;
      });
    }
    p->tiles_m = (int32_t)cdiv(p->M, pair ? 256 : 128);
    p->tiles_n = (int32_t)cdiv(p->N, p->bn);
    // tile order: groups of `raster` tile rows (> 0, default 8) or of
    // -raster tile columns (< 0), the two GEMM loop orders
    p->raster = p->tune.raster != 0 ? p->tune.raster : 8;
    int64_t tiles = (int64_t)p->tiles_m * p->tiles_n;
    int ctas = p->tune.max_ctas > 0 ? std::min(p->tune.max_ctas, p->num_sms) : p->num_sms;
    // one CTA per SM; a slice is at least one accumulation chunk (BF16X3) or
    // 512 k (BF16). The CTA-pair kernel does not split.
    p->kb_per_split = (int32_t)choose_ksplit(pair ? 1 : p->tune.ksplit, tiles, p->num_kb, ctas,
                                             x3 ? p->chunk_kb : 8, &p->ksplit);
    tiles *= p->ksplit;
    // Tail split: whole rounds of the persistent grid plus a short tail (at
    // most half a round) -- the tail's tiles run as k slices that fill the
    // last round while the full tiles keep all of K. It saves (1 - 1/slices)
    // of a tile's time and costs the slices' partial sums (written, read back,
    // C written) and a launch, so it is taken only for long tiles: a tile at
    // about 0.52 us per k-block (BF16X3, 128 x 192) or 0.47 us (BF16,
    // 128 x 256), the partial sums at 6.5 TB/s, 5 us fixed. Automatic k-split
    // only (not with an explicit ksplit, nor for the CTA-pair kernel).
    const int64_t mn = (int64_t)p->tiles_m * p->tiles_n;
    p->full_tiles = 0;
    p->tail_split = 1;
    p->tail_kb = 0;
    if (!pair && p->ksplit == 1 && p->tune.ksplit == 0 && p->tune.tail_split >= 0 && mn > ctas) {
      const int64_t full = mn / ctas * ctas, tail = mn - full;
      const int64_t min_kb = x3 ? p->chunk_kb : 8;
      const int64_t want = tail > 0 ? std::min<int64_t>(ctas / tail, p->num_kb / min_kb) : 0;
      if (tail > 0 && 2 * tail <= ctas && want >= 2) {
        const int64_t per = cdiv(p->num_kb, want);  // no empty slice
        const int64_t splits = cdiv(p->num_kb, per);
        const double t_tile = p->num_kb * (x3 ? 0.52e-6 : 0.47e-6);
        const double t_sum =
            5e-6 + (double)tail * 128 * p->bn * 4 * (2.0 * splits + 2.0) / 6.5e12;
        if ((1.0 - 1.0 / splits) * t_tile > t_sum) {
          p->tail_kb = (int32_t)per;
          p->tail_split = (int32_t)splits;
          p->full_tiles = (int32_t)full;
          tiles = full + tail * p->tail_split;
        }
      }
    }
    if (tiles > INT32_MAX) return fail(TCCG_ERR_UNSUPPORTED, "too many tiles");
    if (pair) {  // clusters of two CTAs, one pair tile per cluster at a time
      int resident = 0;
      int rc = pair_clusters(x3, &resident);
      if (rc) return rc;
      const int clusters = std::max(1, std::min(ctas / 2, resident));
      p->grid = 2 * (int32_t)std::min<int64_t>(tiles, clusters);
    } else
      p->grid = (int32_t)std::min<int64_t>(tiles, ctas);
    p->off_a = 0;
    if (!p->gather) {  // packed operands
      ws = align_up((size_t)(p->M * p->Kc) * 2, 256);
      p->off_b = ws;
      ws = align_up(ws + (size_t)(p->N * p->Kc) * 2, 256);
    }
    if (p->ksplit > 1) {  // FP32 slices [split][N][M]
      p->off_part = ws;
      ws = align_up(ws + (size_t)p->ksplit * p->N * p->M * 4, 256);
    }
    if (p->tail_split > 1) {  // FP32 tail slices [split][tail tile][BN][128]
      p->off_tail = ws;
      ws = align_up(ws + (size_t)p->tail_split * (size_t)(mn - p->full_tiles) * p->bn * 128 * 4, 256);
    }
    static const char* gr[] = {"rows", "k", "kquad"};
    if (p->gather)
      snprintf(p->describe, sizeof(p->describe),
               "method=GETT prec=bf16x3 kernel=gett_tc<BF16X3,gather> tile=128x%d stages=%d M=%lld "
               "N=%lld K=%lld kblocks=%d chunk=%d ksplit=%d tail=%dx%d grid=%d raster=%d pack=none "
               "(gather a=%s b=%s)",
               p->bn, stages, (long long)p->M, (long long)p->N,
               (long long)p->K, p->num_kb, p->chunk_kb, p->ksplit,
               p->tail_split > 1 ? (int)((int64_t)p->tiles_m * p->tiles_n - p->full_tiles) : 0,
               p->tail_split, p->grid, p->raster, gr[p->gread_a], gr[p->gread_b]);
    else
    snprintf(p->describe, sizeof(p->describe),
             "method=%s prec=%s kernel=gett_tc%s<%s> tile=%dx%d stages=%d M=%lld N=%lld K=%lld "
             "kblocks=%d chunk=%d ksplit=%d tail=%dx%d grid=%d raster=%d pack=K-major bf16%s(read_k_fast a=%d b=%d "
             "visit a=%d b=%d kblock a=%dx%dx%d%s b=%dx%dx%d%s kstream a=%d b=%d)",
             ttgt ? "TTGT" : "GETT", x3 ? "bf16x3" : "bf16", pair ? "2" : "", x3 ? "BF16X3" : "BF16",
             pair ? 256 : 128, p->bn, stages,
             (long long)p->M, (long long)p->N, (long long)p->K, p->num_kb, p->chunk_kb, p->ksplit,
             p->tail_split > 1 ? (int)((int64_t)p->tiles_m * p->tiles_n - p->full_tiles) : 0,
             p->tail_split, p->grid, p->raster, x3 ? " hi|lo " : " ", p->read_k_fast_a, p->read_k_fast_b,
             p->t_a_vsrc ? 1 : 0, p->t_b_vsrc ? 1 : 0, p->kb_a[0], p->kb_a[1], p->kb_a[2],
             p->kb_a[0] && p->kbq_a ? " x16B" : "", p->kb_b[0], p->kb_b[1], p->kb_b[2],
             p->kb_b[0] && p->kbq_b ? " x16B" : "", p->ks_a ? 1 : 0, p->ks_b ? 1 : 0);
  }
  if (ttgt) {
    // contiguous C' = [M][N] (column-major) in the workspace, then C' -> C
    const size_t es = p->prec == TCCG_PREC_FP64 ? 8 : 4;
    std::vector<int64_t> h((size_t)p->M);
    for (int64_t i = 0; i < p->M; ++i) h[(size_t)i] = i;
    int rc = upload(h, &p->t_id_m);
    if (rc) return rc;
    h.resize((size_t)p->N);
    for (int64_t i = 0; i < p->N; ++i) h[(size_t)i] = i * p->M;
    rc = upload(h, &p->t_id_n);
    if (rc) return rc;
    if (!p->c_is_mn_dense) {
      p->off_cprime = ws;
      ws = align_up(ws + (size_t)(p->M * p->N) * es, 256);
    }
  }
  p->ws_bytes = ws;
  return TCCG_OK;
}

extern "C" int tccg_plan_workspace(const tccg_plan* p, size_t* bytes) {
  if (!p || !bytes) return fail(TCCG_ERR_INVALID, "null argument");
  *bytes = p->ws_bytes;
  return TCCG_OK;
}

// Programmatic dependent launch (launch_after) lets a kernel start while the
// one before it drains (about 2 us per kernel boundary). For the persistent
// tcgen05 grid it also moves the CTAs: they start on SMs in the order the
// previous kernel frees them instead of the hardware's own placement (pairs
// of SMs round-robin over the GPCs), so the CTAs that share operand tiles
// across the rounds of the tile order land elsewhere. Measured on
// configuration 3 (37 rounds of 148 tiles): steps 20 % slower as the power
// draw rose, while in SM order (tile positions from %smid, identical with
// and without it) the steps were the same with and without -- the placement
// is the cost. Default: on for the CUDA-core kernels (independent CTAs) and
// for tcgen05 grids of at most 4 rounds (little reuse across rounds to
// lose); TCCG_B200_PDL=1 / =0 in the environment forces it on / off.
static bool pdl_auto(const tccg_plan* p) {
  if (p->simt || p->skinny) return true;
  const int64_t mn = (int64_t)p->tiles_m * p->tiles_n;
  const int64_t tiles = p->tail_split > 1 ? p->full_tiles + (mn - p->full_tiles) * p->tail_split
                                          : mn * p->ksplit;
  return tiles <= 4 * (int64_t)std::max(p->grid, 1);
}
static int pdl_forced() {  // 1 on, 0 off, -1 the size rule
  const char* e = std::getenv("TCCG_B200_PDL");
  if (e && e[0] == '0') return 0;
  if (e && e[0] == '1') return 1;
  return -1;
}
// Whether tccg_plan_run launches this plan's kernels with programmatic
// dependent launch; tccg_plan_run_timed never does (an event sits between
// the kernels), see pdl_enabled.
static bool pdl_selected(const tccg_plan* p) {
  const int f = pdl_forced();
  return f < 0 ? pdl_auto(p) : f == 1;
}

extern "C" int tccg_plan_describe(const tccg_plan* p, char* buf, size_t len) {
  if (!p || !buf || len == 0) return fail(TCCG_ERR_INVALID, "null argument");
  snprintf(buf, len, "%s launch=%s ws=%zu", p->describe,
           pdl_selected(p) ? "dependent(plain when timed per kernel)" : "plain", p->ws_bytes);
  return TCCG_OK;
}

extern "C" double tccg_plan_flops(const tccg_plan* p, double beta) {
  if (!p) return 0.0;
  double f = 2.0 * (double)p->M * (double)p->N * (double)p->K;
  if (beta != 0.0) f += 3.0 * (double)p->M * (double)p->N;
  return f;
}

extern "C" int tccg_plan_destroy(tccg_plan* p) {
  plan_free(p);
  return TCCG_OK;
}

extern "C" int tccg_plan_status(const tccg_plan* p, int32_t* device_status) {
  if (!p || !device_status) return fail(TCCG_ERR_INVALID, "null argument");
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(device_status, p->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemset(p->d_status, 0, sizeof(int32_t)));
  return TCCG_OK;
}

// --------------------------------------------------------------------------
// kernel attributes (once per device)
// --------------------------------------------------------------------------
// cudaFuncSetAttribute acts on the current device's context, so the large
// shared-memory sizes are set once for each device the process uses.
#define TCCG_MAX_DEVICES 64
static std::once_flag g_attr_once[TCCG_MAX_DEVICES];
static cudaError_t g_attr_err[TCCG_MAX_DEVICES];

static cudaError_t set_attrs() {
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) { if (e == cudaSuccess && x != cudaSuccess) e = x; };
  chk(cudaFuncSetAttribute(simt_gett_kernel<float, SIMT_PACKED>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)simt_smem_bytes<float>()));
  chk(cudaFuncSetAttribute(simt_gett_kernel<float, SIMT_DIRECT>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)simt_smem_bytes<float>()));
  chk(cudaFuncSetAttribute(simt_gett_kernel<double, SIMT_PACKED>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)simt_smem_bytes<double>()));
  chk(cudaFuncSetAttribute(simt_gett_kernel<double, SIMT_DIRECT>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)simt_smem_bytes<double>()));
  chk(cudaFuncSetAttribute(simt_shortk_kernel<float, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SimtShortKCfg<float>::SMEM_BYTES));
  chk(cudaFuncSetAttribute(simt_shortk_kernel<float, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SimtShortKCfg<float>::SMEM_BYTES));
  chk(cudaFuncSetAttribute(simt_shortk_kernel<double, true>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SimtShortKCfg<double>::SMEM_BYTES));
  chk(cudaFuncSetAttribute(simt_shortk_kernel<double, false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SimtShortKCfg<double>::SMEM_BYTES));
  for (int v = 0; v < TCV_COUNT; ++v)
    with_tc_variant(v, [&](auto k) {
      using K = decltype(k);
      chk(cudaFuncSetAttribute(K::single, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)K::Cfg::SMEM_BYTES));
      chk(cudaFuncSetAttribute(K::group, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)K::Cfg::SMEM_BYTES));
    });
  chk(cudaFuncSetAttribute(simt_gett_group_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)simt_group_smem_bytes<float>()));
  chk(cudaFuncSetAttribute(simt_gett_group_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)simt_group_smem_bytes<double>()));
  for (int rs = 4; rs <= 12; rs += 4)
    with_skinny_rs(rs, [&](auto r) {
      chk(cudaFuncSetAttribute(skinny_gett_kernel<decltype(r)::value>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SK_SMEM_BYTES));
      chk(cudaFuncSetAttribute(skinny_group_kernel<decltype(r)::value>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SK_SMEM_BYTES));
    });
  chk(cudaFuncSetAttribute(skinny_reduce_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SK_SMEM_BYTES));
  chk(cudaFuncSetAttribute(skinny_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SKT_SMEM_BYTES));
  chk(cudaFuncSetAttribute(skinny_tc_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SKT_SMEM_BYTES));
  chk(cudaFuncSetAttribute(skinny_reg_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SKR_SMEM_BYTES));
  chk(cudaFuncSetAttribute(skinny_reg_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SKR_SMEM_BYTES));
  chk(cudaFuncSetAttribute(skinny_reg_group_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SKR_SMEM_BYTES));
  chk(cudaFuncSetAttribute(skinny_reduce_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)SK_SMEM_BYTES));
  chk(cudaFuncSetAttribute(gett_tc2_kernel<TC_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)Tc2Cfg<TC_BF16>::SMEM_BYTES));
  chk(cudaFuncSetAttribute(gett_tc2_kernel<TC_BF16X3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)Tc2Cfg<TC_BF16X3>::SMEM_BYTES));

  return e;
}

static int ensure_attrs() {
  int dev = -1;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= TCCG_MAX_DEVICES)
    return fail(TCCG_ERR_UNSUPPORTED, "device index %d (at most %d devices)", dev, TCCG_MAX_DEVICES);
  std::call_once(g_attr_once[dev], [dev] { g_attr_err[dev] = set_attrs(); });
  if (g_attr_err[dev] != cudaSuccess)
    return fail(TCCG_ERR_CUDA, "cudaFuncSetAttribute on device %d: %s", dev,
                cudaGetErrorString(g_attr_err[dev]));
  return TCCG_OK;
}

// Clusters of the CTA-pair kernel that fit on the device at once (an SM whose
// partner in the GPC is unavailable cannot host half a cluster).
static int pair_clusters(bool x3, int* clusters) {
  int rc = ensure_attrs();
  if (rc) return rc;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(x3 ? Tc2Cfg<TC_BF16X3>::NUM_THREADS : Tc2Cfg<TC_BF16>::NUM_THREADS, 1, 1);
  cfg.dynamicSmemBytes = x3 ? Tc2Cfg<TC_BF16X3>::SMEM_BYTES : Tc2Cfg<TC_BF16>::SMEM_BYTES;
  cudaError_t e = x3 ? cudaOccupancyMaxActiveClusters(clusters, gett_tc2_kernel<TC_BF16X3>, &cfg)
                     : cudaOccupancyMaxActiveClusters(clusters, gett_tc2_kernel<TC_BF16>, &cfg);
  if (e != cudaSuccess)
    return fail(TCCG_ERR_CUDA, "cudaOccupancyMaxActiveClusters: %s", cudaGetErrorString(e));
  if (*clusters < 1) return fail(TCCG_ERR_UNSUPPORTED, "the CTA-pair kernel does not fit on this device");
  return TCCG_OK;
}

// --------------------------------------------------------------------------
// tensor maps
// --------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::once_flag g_encode_once;

static int get_encode() {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  if (!g_encode) return fail(TCCG_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  return TCCG_OK;
}

// 2-D bf16 K-major operand [rows][cols], box {64, box_rows}, 128-byte swizzle.
static int encode_kmajor(CUtensorMap* tm, const void* base, int64_t rows, int64_t cols,
                         int box_rows) {
  int rc = get_encode();
  if (rc) return rc;
  if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0 || (cols * 2) % 16 != 0)
    return fail(TCCG_ERR_ALIGNMENT, "TMA operand not 16-byte aligned");
  cuuint64_t gdim[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t gstride[1] = {(cuuint64_t)(cols * 2)};
  cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), gdim,
                        gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(TCCG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return TCCG_OK;
}

// 2-D C matrix C[m + ldc * n] (FP32 or FP64), box {box_m, box_n}, no swizzle:
// the block lands in shared memory as a dense [box_n][box_m] array. Returns
// false (no map) when the base or the column stride is not 16-byte aligned.
template <typename T>
static bool encode_c2d(CUtensorMap* tm, const T* base, int64_t M, int64_t N, int64_t ldc,
                       int box_m, int box_n) {
  if (get_encode() != TCCG_OK) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0 || (ldc * (int64_t)sizeof(T)) % 16 != 0)
    return false;
  cuuint64_t gdim[2] = {(cuuint64_t)M, (cuuint64_t)N};
  cuuint64_t gstride[1] = {(cuuint64_t)(ldc * (int64_t)sizeof(T))};
  cuuint32_t box[2] = {(cuuint32_t)box_m, (cuuint32_t)box_n};
  cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt =
      sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return g_encode(tm, dt, 2, const_cast<T*>(base), gdim, gstride, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// --------------------------------------------------------------------------
// launches
// --------------------------------------------------------------------------
// Optional per-kernel timing (tccg_plan_run_timed): events[2*i], events[2*i+1]
// bracket kernel slot i (0 pack, 1 GEMM, 2 reduce/transpose) on the stream.
static thread_local cudaEvent_t* g_events = nullptr;

static void mark(int slot, int end, cudaStream_t s) {
  if (g_events) cudaEventRecord(g_events[2 * slot + end], s);
}

// Test trigger of the bounded device waits (tccg_debug_inject_timeout):
// armed per host thread, taken by the next launch of gett_tc_kernel.
static thread_local int32_t g_inject_tile1 = 0;
static thread_local uint64_t g_inject_wait_ns = 0;

static void take_injection(TcArgs& a) {
  a.skip_tile1 = g_inject_tile1;
  a.wait_ns = g_inject_wait_ns;
  g_inject_tile1 = 0;
  g_inject_wait_ns = 0;
}

extern "C" int tccg_debug_inject_timeout(int32_t tile, int32_t wait_ms) {
  if (tile < 0 || wait_ms < 1 || wait_ms > 4000)
    return fail(TCCG_ERR_INVALID, "tile must be >= 0 and wait_ms in [1, 4000]");
  g_inject_tile1 = tile + 1;
  g_inject_wait_ns = (uint64_t)wait_ms * 1000000ull;
  return TCCG_OK;
}

static int launch_check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(TCCG_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
  return TCCG_OK;
}

// Programmatic dependent launch of a kernel that directly follows one of this
// library's own kernels on the stream (packing -> GETT, GETT -> reduction):
// its CTAs may start, and set up barriers and TMEM, while that kernel drains;
// they call grid_dep_wait() before reading its output, and read nothing
// before it that an earlier kernel of the call could still be writing. When
// it is used: pdl_auto. Always off under per-kernel event timing (an event
// sits between the kernels).
static bool pdl_enabled(const tccg_plan* p) { return !g_events && pdl_selected(p); }

template <typename... P, typename... A>
static void launch_after(bool after_own_kernel, const tccg_plan* p, void (*kernel)(P...),
                         dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = after_own_kernel && pdl_enabled(p) ? 1 : 0;
  (void)cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);  // launch_check reads the error
}

static PackOperand pack_op(const void* src, const int64_t* roff, const int64_t* coff, int64_t R,
                           int64_t Kk, int64_t Rcover, int64_t Kcover, void* dst, int64_t ld,
                           int32_t kfast) {
  PackOperand o;
  o.src = src;
  o.row_off = roff;
  o.col_off = coff;
  o.R = R;
  o.Kk = Kk;
  o.Rcover = Rcover;
  o.Kcover = Kcover;
  o.dst = dst;
  o.ld = ld;
  o.read_k_fast = kfast;
  o.active = 1;
  o.row_dst = nullptr;
  o.kb_lo = o.kb_run = o.kb_rows = o.kb_ext = o.kb_step = o.kb_quad = 0;
  o.kstream = 0;
  o.ktiles = o.tiles = 0;
  return o;
}

// The read schedule of a K-major pack chosen at plan creation: the streaming
// pass (when the source is aligned for its vector loads; es = source element
// bytes) or k-block tiles, else unchanged.
static PackOperand with_kread(PackOperand o, bool kstream, const int32_t (&kb)[5], bool kb_quad,
                              size_t es) {
  const bool aligned = (reinterpret_cast<uintptr_t>(o.src) % (4 * es)) == 0;
  if (kstream && aligned) {
    o.kstream = 1;
  } else if (kb[0] > 0) {
    o.kb_lo = kb[0];
    o.kb_run = kb[1];
    o.kb_rows = kb[2];
    o.kb_ext = kb[3];
    o.kb_step = kb[4];
    o.kb_quad = kb_quad && aligned ? 1 : 0;
  }
  return o;
}

// Tile grid of one operand: k-block tiles, or 32 rows x `ktile` k.
static void pack_geometry(PackOperand& o, int ktile) {
  if (o.kstream) {  // one tile along k; 256 threads x PACK_KS_Q quads per CTA
    o.ktiles = 1;
    o.tiles = cdiv(o.Rcover * (o.Kcover / 4), 256 * PACK_KS_Q);
    return;
  }
  int64_t kt = ktile, rows = 32;
  if (o.kb_lo > 0) {
    kt = (int64_t)o.kb_lo * o.kb_run;
    rows = o.kb_rows;
  }
  o.ktiles = cdiv(o.Kcover, kt);
  o.tiles = o.ktiles * cdiv(o.Rcover, rows);
}

// Row visit order of a K-major pack (tables built at plan creation).
static PackOperand with_visit(PackOperand o, const int64_t* vsrc, const int64_t* vdst) {
  if (vsrc && vdst) {
    o.row_off = vsrc;
    o.row_dst = vdst;
  }
  return o;
}

// Read schedule of one operand (PackRead).
static int pack_read(const PackOperand& o) {
  return o.kstream ? PACK_READ_STREAM : o.kb_lo > 0 ? PACK_READ_KBLOCK : PACK_READ_WIDE;
}

// One launch for both operands, with the kernel of their common read
// schedule, or the kernel holding all schedules when they differ (a second
// launch costs more than the wider kernel's extra registers).
template <typename Tin, typename Tout, int LAYOUT>
static int launch_pack(PackArgs pa, cudaStream_t s, bool* launched = nullptr) {
  if (launched) *launched = false;
  int64_t ctas = 0;
  int read = -1;
  for (PackOperand& o : pa.op) {
    pack_geometry(o, pack_k_tile<LAYOUT>());
    if (!o.active) continue;
    ctas = std::max(ctas, o.tiles);
    read = read < 0 || read == pack_read(o) ? pack_read(o) : PACK_READ_ANY;
  }
  if (ctas > INT32_MAX) return fail(TCCG_ERR_UNSUPPORTED, "operand too large to pack (%lld tiles)", (long long)ctas);
  if (ctas == 0) return TCCG_OK;
  if (launched) *launched = true;
  const dim3 grid((unsigned)ctas, 1, 2), block(32, 8);
  constexpr bool KMAJOR = LAYOUT == PACK_K_BF16 || LAYOUT == PACK_K_BF16X3;
  mark(0, 0, s);
  if (!KMAJOR || read == PACK_READ_WIDE)
    pack_kernel<Tin, Tout, LAYOUT, PACK_READ_WIDE><<<grid, block, 0, s>>>(pa);
  else if constexpr (KMAJOR) {
    if (read == PACK_READ_STREAM)
      pack_kernel<Tin, Tout, LAYOUT, PACK_READ_STREAM><<<grid, block, 0, s>>>(pa);
    else if (read == PACK_READ_KBLOCK)
      pack_kernel<Tin, Tout, LAYOUT, PACK_READ_KBLOCK><<<grid, block, 0, s>>>(pa);
    else
      pack_kernel<Tin, Tout, LAYOUT, PACK_READ_ANY><<<grid, block, 0, s>>>(pa);
  }
  mark(0, 1, s);
  return launch_check("pack");
}

template <typename T>
static void set_direct(SimtArgs<T>& a, const tccg_plan* p, const void* GA, const void* GB) {
  a.direct = p->direct ? 1 : 0;
  a.a_kfast = p->gather_k_a ? 1 : 0;
  a.b_kfast = p->gather_k_b ? 1 : 0;
  a.K = p->K;
  a.Asrc = static_cast<const T*>(GA);
  a.Bsrc = static_cast<const T*>(GB);
  a.a_m_off = p->t_a_m;
  a.a_k_off = p->t_a_k;
  a.b_n_off = p->t_b_n;
  a.b_k_off = p->t_b_k;
}

// simt_gett_kernel with the plan's tile shape (FP32: three shapes).
template <typename T, int LOAD>
static void launch_simt_tiles(const tccg_plan* p, const SimtArgs<T>& a, dim3 grid, bool after,
                              cudaStream_t s) {
  if constexpr (sizeof(T) == 4) {
    if (p->simt_shape == SIMT_NARROW_N) {
      launch_after(after, p, simt_gett_kernel<T, LOAD, SIMT_NARROW_N>, grid, dim3(256),
                   simt_smem_bytes<T, SIMT_NARROW_N>(), s, a);
      return;
    }
    if (p->simt_shape == SIMT_NARROW_M) {
      launch_after(after, p, simt_gett_kernel<T, LOAD, SIMT_NARROW_M>, grid, dim3(256),
                   simt_smem_bytes<T, SIMT_NARROW_M>(), s, a);
      return;
    }
  }
  launch_after(after, p, simt_gett_kernel<T, LOAD>, grid, dim3(256), simt_smem_bytes<T>(), s, a);
}

template <typename T>
static int run_simt(const tccg_plan* p, const void* GA, const void* GB, T* Cout,
                    const int64_t* c_m, const int64_t* c_n, int64_t c_ldc, T alpha, T beta,
                    char* ws, cudaStream_t s) {
  using Cfg = SimtCfg<T>;
  T* Ap = reinterpret_cast<T*>(ws + p->off_a);
  T* Bp = reinterpret_cast<T*>(ws + p->off_b);
  PackArgs pa;
  pa.op[0] = pack_op(GA, p->t_a_m, p->t_a_k, p->M, p->K, p->Mp, p->Kp, Ap, p->Mp, p->read_k_fast_a);
  pa.op[1] = pack_op(GB, p->t_b_n, p->t_b_k, p->N, p->K, p->Np, p->Kp, Bp, p->Np, p->read_k_fast_b);
  int rc = TCCG_OK;
  bool packed = false;  // the packing kernel is the last launch on s
  if (p->direct) {
    // no packing pass
  } else if constexpr (sizeof(T) == 8) {
    rc = launch_pack<T, T, PACK_MN>(pa, s, &packed);
  } else {
    if (p->dtype == TCCG_BF16)
      rc = launch_pack<__nv_bfloat16, float, PACK_MN>(pa, s, &packed);
    else if (p->prec == TCCG_PREC_BF16)
      rc = launch_pack<float, float, PACK_MN_BF16>(pa, s, &packed);
    else
      rc = launch_pack<float, float, PACK_MN>(pa, s, &packed);
  }
  if (rc) return rc;
  SimtArgs<T> a;
  a.Ap = Ap;
  a.Bp = Bp;
  a.Mp = p->Mp;
  a.Np = p->Np;
  a.M = p->M;
  a.N = p->N;
  a.ktiles = p->ktiles;
  a.ktiles_per_split = p->ktiles_per_split;
  a.C = Cout;
  a.c_m_off = c_m;
  a.c_n_off = c_n;
  a.alpha = alpha;
  a.beta = beta;
  a.partial = p->ksplit > 1 ? reinterpret_cast<T*>(ws + p->off_part) : nullptr;
  set_direct(a, p, GA, GB);
  a.status = p->d_status;
  a.crun = c_m == p->t_c_m ? p->crun : 0;  // not for TTGT's contiguous C'
  dim3 grid((unsigned)(p->Mp / p->simt_bm), (unsigned)(p->Np / p->simt_bn), (unsigned)p->ksplit);
  if (grid.y > 65535u || grid.z > 65535u) return fail(TCCG_ERR_UNSUPPORTED, "grid too large");
  mark(1, 0, s);
  CUtensorMap tmC{};
  if (p->shortk && shortk_tma(p, c_ldc) &&
      encode_c2d<T>(&tmC, Cout, p->M, p->N, c_ldc, Cfg::BM, Cfg::BN))
    launch_after(packed, p, simt_shortk_kernel<T, true>, grid, dim3(256),
                 SimtShortKCfg<T>::SMEM_BYTES, s, a, tmC);
  else if (p->shortk)
    launch_after(packed, p, simt_shortk_kernel<T, false>, grid, dim3(256),
                 SimtShortKCfg<T>::SMEM_BYTES, s, a, tmC);
  else if (p->direct)
    launch_simt_tiles<T, SIMT_DIRECT>(p, a, grid, false, s);
  else
    launch_simt_tiles<T, SIMT_PACKED>(p, a, grid, packed, s);
  mark(1, 1, s);
  rc = launch_check("simt_gett");
  if (rc) return rc;
  if (p->ksplit > 1) {
    dim3 g2((unsigned)cdiv(p->M, 256), (unsigned)std::min<int64_t>(p->N, 65535));
    mark(2, 0, s);
    launch_after(true, p, simt_reduce_kernel<T>, g2, dim3(256), 0, s, a.partial, (int)p->ksplit,
                 p->Mp, p->Np, p->M, p->N, Cout, c_m, c_n, alpha, beta);
    mark(2, 1, s);
    rc = launch_check("simt_reduce");
  }
  return rc;
}

// Tile order of the persistent tcgen05 grid by SM (TcArgs::sm_order) when
// TCCG_B200_CTA_ORDER=sm in the environment; by default the launch order.
// Measured on configuration 3: the SM order makes the placement independent
// of programmatic dependent launch, but its placement (consecutive tiles on
// consecutive SM ids) ran 13 % slower than the hardware's own (launch order
// without dependent launch), which the default keeps.
static bool sm_order_enabled() {
  const char* e = std::getenv("TCCG_B200_CTA_ORDER");
  return e && std::strcmp(e, "sm") == 0;
}

// Arguments of the tcgen05 kernels common to both loaders (k-split partial
// sums and tail slices in the workspace `ws`).
static TcArgs tc_args(const tccg_plan* p, float* Cout, const int64_t* c_m, const int64_t* c_n,
                      float alpha, float beta, char* ws) {
  TcArgs a{};
  a.M = (int32_t)p->M;
  a.N = (int32_t)p->N;
  a.K = (int32_t)p->K;
  a.num_kb = p->num_kb;
  a.tiles_m = p->tiles_m;
  a.tiles_n = p->tiles_n;
  a.raster = p->raster;
  a.chunk_kb = p->chunk_kb;
  a.C = Cout;
  a.c_m_off = c_m;
  a.c_n_off = c_n;
  a.alpha = alpha;
  a.beta = beta;
  a.status = p->d_status;
  a.ksplit = p->ksplit;
  a.kb_per_split = p->kb_per_split;
  a.partial = p->ksplit > 1 ? reinterpret_cast<float*>(ws + p->off_part) : nullptr;
  a.full_tiles = p->full_tiles;
  a.tail_split = p->tail_split;
  a.tail_kb = p->tail_kb;
  a.tail_partial = p->tail_split > 1 ? reinterpret_cast<float*>(ws + p->off_tail) : nullptr;
  a.crun = c_m == p->t_c_m ? p->crun : 0;  // not for TTGT's contiguous C'
  a.sm_order = sm_order_enabled() ? 1 : 0;
  return a;
}

// Gather loader: the kernel reads GA and GB through the plan's offset tables.
// 16-byte copies need a 16-byte aligned operand; an unaligned one is read
// along k 4 bytes at a time (the same elements, the same stages).
static void set_gather(TcArgs& a, const tccg_plan* p, const void* GA, const void* GB) {
  a.gsrc[0] = static_cast<const float*>(GA);
  a.gsrc[1] = static_cast<const float*>(GB);
  a.grow[0] = p->t_a_m;
  a.grow[1] = p->t_b_n;
  a.gk[0] = p->t_a_k;
  a.gk[1] = p->t_b_k;
  const bool al_a = (reinterpret_cast<uintptr_t>(GA) & 15u) == 0;
  const bool al_b = (reinterpret_cast<uintptr_t>(GB) & 15u) == 0;
  a.gread[0] = p->gread_a == GATHER_KQUAD && !al_a ? GATHER_K : p->gread_a;
  a.gread[1] = p->gread_b == GATHER_KQUAD && !al_b ? GATHER_K : p->gread_b;
}

// Reduction after the tcgen05 kernel: tail slices or k-split slices.
static int tc_reduce(const tccg_plan* p, const TcArgs& a, float* Cout, const int64_t* c_m,
                     const int64_t* c_n, float alpha, float beta, cudaStream_t s) {
  if (p->tail_split > 1) {
    const unsigned tail = (unsigned)((int64_t)p->tiles_m * p->tiles_n - p->full_tiles);
    mark(2, 0, s);
    with_tc_variant(p->tcv, [&](auto k) {
      using K = decltype(k);
      launch_after(true, p, K::tail, dim3(tail, K::Cfg::BM * K::Cfg::BN / 256), dim3(256), 0, s, a);
    });
    mark(2, 1, s);
    return launch_check("tc_tail_reduce");
  }
  if (p->ksplit == 1) return TCCG_OK;
  dim3 g2((unsigned)cdiv(p->M, 256), (unsigned)std::min<int64_t>(p->N, 65535));
  mark(2, 0, s);
  launch_after(true, p, simt_reduce_kernel<float>, g2, dim3(256), 0, s, (const float*)a.partial,
               (int)p->ksplit, (int64_t)p->M, (int64_t)p->N, (int64_t)p->M, (int64_t)p->N, Cout, c_m,
               c_n, alpha, beta);
  mark(2, 1, s);
  return launch_check("tc_reduce");
}

static int run_tc(const tccg_plan* p, const void* GA, const void* GB, float* Cout,
                  const int64_t* c_m, const int64_t* c_n, float alpha, float beta, char* ws,
                  cudaStream_t s) {
  const bool x3 = p->prec == TCCG_PREC_BF16X3;
  TcArgs a = tc_args(p, Cout, c_m, c_n, alpha, beta, ws);
  CUtensorMap tmA, tmB;
  int rc;
  bool packed = false;  // the packing kernel is the last launch on s
  const bool pair = p->tune.pair != 0;
  if (p->gather) {
    // no packing pass: the kernel reads GA and GB through the offset tables
    set_gather(a, p, GA, GB);
    memset(&tmA, 0, sizeof(tmA));
    memset(&tmB, 0, sizeof(tmB));
  } else {
    void* Ap = ws + p->off_a;
    void* Bp = ws + p->off_b;
    PackArgs pa;
    const int64_t kcover = x3 ? round_up(p->K, 32) : p->Kc;
    const size_t es = p->dtype == TCCG_BF16 ? 2 : 4;
    pa.op[0] = with_kread(with_visit(pack_op(GA, p->t_a_m, p->t_a_k, p->M, p->K, p->M, kcover, Ap,
                                             p->Kc, p->read_k_fast_a), p->t_a_vsrc, p->t_a_vdst),
                          p->ks_a, p->kb_a, p->kbq_a, es);
    pa.op[1] = with_kread(with_visit(pack_op(GB, p->t_b_n, p->t_b_k, p->N, p->K, p->N, kcover, Bp,
                                             p->Kc, p->read_k_fast_b), p->t_b_vsrc, p->t_b_vdst),
                          p->ks_b, p->kb_b, p->kbq_b, es);
    if (x3)
      rc = launch_pack<float, __nv_bfloat16, PACK_K_BF16X3>(pa, s, &packed);
    else if (p->dtype == TCCG_BF16)
      rc = launch_pack<__nv_bfloat16, __nv_bfloat16, PACK_K_BF16>(pa, s, &packed);
    else
      rc = launch_pack<float, __nv_bfloat16, PACK_K_BF16>(pa, s, &packed);
    if (rc) return rc;
    rc = encode_kmajor(&tmA, Ap, p->M, p->Kc, 128);
    if (rc) return rc;
    rc = encode_kmajor(&tmB, Bp, p->N, p->Kc, pair ? p->bn / 2 : p->bn);
    if (rc) return rc;
  }
  mark(1, 0, s);
  if (pair && x3) {
    launch_after(packed, p, gett_tc2_kernel<TC_BF16X3>, dim3((unsigned)p->grid), dim3(Tc2Cfg<TC_BF16X3>::NUM_THREADS),
                 Tc2Cfg<TC_BF16X3>::SMEM_BYTES, s, tmA, tmB, a);
  } else if (pair) {
    launch_after(packed, p, gett_tc2_kernel<TC_BF16>, dim3((unsigned)p->grid), dim3(Tc2Cfg<TC_BF16>::NUM_THREADS),
                 Tc2Cfg<TC_BF16>::SMEM_BYTES, s, tmA, tmB, a);
  } else {
    take_injection(a);
    with_tc_variant(p->tcv, [&](auto k) {
      using K = decltype(k);
      launch_after(packed, p, K::single, dim3((unsigned)p->grid), dim3(K::Cfg::NUM_THREADS),
                   K::Cfg::SMEM_BYTES, s, tmA, tmB, a);
    });
  }
  mark(1, 1, s);
  rc = launch_check(p->gather ? "gett_tc (gather)" : "gett_tc");
  if (rc) return rc;
  return tc_reduce(p, a, Cout, c_m, c_n, alpha, beta, s);
}

// Kernel arguments of a skinny plan for one call (P / Q by the narrow side).
static SkinnyArgs skinny_args(const tccg_plan* p, const void* GA, const void* GB, float* C,
                              float alpha, float beta, char* w) {
  SkinnyArgs a = p->sk;
  const bool sn = p->sk_s_is_n;
  a.P = static_cast<const float*>(sn ? GA : GB);
  a.Q = static_cast<const float*>(sn ? GB : GA);
  a.C = C;
  a.p_y_off = p->t_sk + p->sk_tab[0];
  a.c_y_off = p->t_sk + p->sk_tab[1];
  a.p_k_off = p->t_sk + p->sk_tab[2];
  a.q_s_off = p->t_sk + p->sk_tab[3];
  a.q_k_off = p->t_sk + p->sk_tab[4];
  a.c_s_off = p->t_sk + p->sk_tab[5];
  a.alpha = alpha;
  a.beta = beta;
  a.partial = p->sk_ksplit > 1 ? reinterpret_cast<float*>(w + p->off_part) : nullptr;
  a.p_vec = p->sk_p_vec && (reinterpret_cast<uintptr_t>(a.P) & 15) == 0;
  a.c_bulk = a.c_lin == SK_CLIN_XS && beta == 0.0f && (reinterpret_cast<uintptr_t>(C) & 15) == 0;
  return a;
}

// The tensor-core skinny kernel's Q: the narrow operand packed K-major into
// the workspace (spad rows, the rows past S zeros) and its tensor map (box of
// 32 k x spad rows, 128-byte swizzle).
static PackOperand skinny_tc_q(const tccg_plan* p, const void* GA, const void* GB, char* w) {
  const bool sn = p->sk_s_is_n;
  return pack_op(sn ? GB : GA, sn ? p->t_b_n : p->t_a_m, sn ? p->t_b_k : p->t_a_k,
                 sn ? p->N : p->M, p->K, (int64_t)p->sk.npass * p->sk_spad, round_up(p->K, 32),
                 w + p->off_q, p->Kc, sn ? p->read_k_fast_b : p->read_k_fast_a);
}

static SkinnyTcArgs skinny_tc_args(const tccg_plan* p, const void* GA, const void* GB, float* C,
                                   float alpha, float beta, char* w) {
  SkinnyTcArgs t;
  t.sk = skinny_args(p, GA, GB, C, alpha, beta, w);
  t.sk.Q = nullptr;
  t.spad = p->sk_spad;
  t.chunk_kb = 16;  // the tile kernel's chunked accumulation (512 k per TMEM round)
  return t;
}

static int run_skinny_tc(const tccg_plan* p, const void* GA, const void* GB, float* C, float alpha,
                         float beta, char* w, cudaStream_t s) {
  PackArgs pa;
  memset(&pa, 0, sizeof(pa));
  pa.op[0] = skinny_tc_q(p, GA, GB, w);
  bool packed = false;
  int rc = launch_pack<float, __nv_bfloat16, PACK_K_BF16X3>(pa, s, &packed);
  if (rc) return rc;
  CUtensorMap tmQ;
  rc = encode_kmajor(&tmQ, w + p->off_q, (int64_t)p->sk.npass * p->sk_spad, p->Kc, p->sk_spad);
  if (rc) return rc;
  const SkinnyTcArgs a = skinny_tc_args(p, GA, GB, C, alpha, beta, w);
  mark(1, 0, s);
  launch_after(packed, p, skinny_tc_kernel, dim3((unsigned)std::min<int64_t>(a.sk.njobs, p->num_sms)),
               dim3(SKT_THREADS), SKT_SMEM_BYTES, s, tmQ, a, p->d_status);
  rc = launch_check("skinny_tc");
  mark(1, 1, s);
  if (rc || p->sk_ksplit == 1) return rc;
  mark(2, 0, s);
  launch_after(true, p, skinny_reduce_kernel, dim3((unsigned)(a.sk.nblk * a.sk.npass)),
               dim3(SK_THREADS), SK_SMEM_BYTES, s, a.sk);
  rc = launch_check("skinny_reduce");
  mark(2, 1, s);
  return rc;
}

static int run_skinny(const tccg_plan* p, const void* GA, const void* GB, float* C, float alpha,
                      float beta, char* w, cudaStream_t s) {
  if (p->sk_tc) return run_skinny_tc(p, GA, GB, C, alpha, beta, w, s);
  const SkinnyArgs a = skinny_args(p, GA, GB, C, alpha, beta, w);
  mark(1, 0, s);
  if (p->sk_reg) {
    const int64_t grid = std::min<int64_t>(a.njobs, (int64_t)SKR_CTAS_PER_SM * p->num_sms);
    // 8 computed rows for a narrow side of at most 8, else 16
    launch_after(false, p, a.S <= 8 ? skinny_reg_kernel<8> : skinny_reg_kernel<16>,
                 dim3((unsigned)grid), dim3(SKR_THREADS), SKR_SMEM_BYTES, s, a);
  } else {
    const int64_t grid = std::min<int64_t>(a.njobs, (int64_t)SK_CTAS_PER_SM * p->num_sms);
    with_skinny_rs(a.rs, [&](auto r) {
      launch_after(false, p, skinny_gett_kernel<decltype(r)::value>, dim3((unsigned)grid),
                   dim3(SK_THREADS), SK_SMEM_BYTES, s, a);
    });
  }
  int rc = launch_check("skinny_gett");
  mark(1, 1, s);
  if (rc || p->sk_ksplit == 1) return rc;
  mark(2, 0, s);
  launch_after(true, p, skinny_reduce_kernel, dim3((unsigned)(a.nblk * a.npass)),
               dim3(SK_THREADS), SK_SMEM_BYTES, s, a);
  rc = launch_check("skinny_reduce");
  mark(2, 1, s);
  return rc;
}

static int permute_launch(int32_t dtype, const PermArgs& pa0, cudaStream_t s);

extern "C" int tccg_plan_run(const tccg_plan* p, const void* A, const void* B, void* C,
                             double alpha, double beta, void* ws, size_t ws_bytes, void* stream) {
  if (!p) return fail(TCCG_ERR_INVALID, "null plan");
  if (!A || !B || !C) return fail(TCCG_ERR_INVALID, "null operand pointer");
  if (ws_bytes < p->ws_bytes || (p->ws_bytes > 0 && !ws))
    return fail(TCCG_ERR_WORKSPACE, "workspace of %zu bytes needed, %zu given", p->ws_bytes, ws_bytes);
  if ((reinterpret_cast<uintptr_t>(ws) & 255u) != 0)
    return fail(TCCG_ERR_ALIGNMENT, "workspace must be 256-byte aligned");
  int dev = -1;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev != p->device)
    return fail(TCCG_ERR_INVALID, "plan was created on device %d, current device is %d", p->device, dev);
  int rc = ensure_attrs();
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const void* GA = p->d.swap_ab ? B : A;
  const void* GB = p->d.swap_ab ? A : B;
  char* w = static_cast<char*>(ws);
  const bool ttgt = p->tune.method == TCCG_METHOD_TTGT;
  // TTGT: the GEMM writes the contiguous [M][N] matrix C' (or C itself when C
  // already has that layout), then one transposition applies alpha/beta.
  const bool direct = !ttgt || p->c_is_mn_dense;
  const int64_t* cm = direct && !ttgt ? p->t_c_m : p->t_id_m;
  const int64_t* cn = direct && !ttgt ? p->t_c_n : p->t_id_n;
  void* Cdst = direct ? C : (void*)(w + p->off_cprime);
  const double ga = direct ? alpha : 1.0, gb = direct ? beta : 0.0;
  // C(m, n) = Cdst[m + ldc n]: C itself (GETT on a 2-D C) or the contiguous C'
  const int64_t ldc = cm == p->t_id_m ? p->M : p->c_ldc;
  if (p->skinny)
    rc = run_skinny(p, GA, GB, static_cast<float*>(Cdst), (float)ga, (float)gb, w, s);
  else if (p->prec == TCCG_PREC_FP64)
    rc = run_simt<double>(p, GA, GB, static_cast<double*>(Cdst), cm, cn, ldc, ga, gb, w, s);
  else if (simt_path(p))
    rc = run_simt<float>(p, GA, GB, static_cast<float*>(Cdst), cm, cn, ldc, (float)ga, (float)gb,
                         w, s);
  else
    rc = run_tc(p, GA, GB, static_cast<float*>(Cdst), cm, cn, (float)ga, (float)gb, w, s);
  if (rc || direct) return rc;
  // C'[m + M n] -> C[c_m_stride . m_idx + c_n_stride . n_idx]
  PermArgs pa{};
  pa.A = Cdst;
  pa.B = C;
  pa.alpha = alpha;
  pa.beta = beta;
  int dim = 0;
  int64_t s_cp = 1;
  for (int i = 0; i < p->d.nm; ++i, ++dim) {
    pa.ext[dim] = p->d.m_ext[i];
    pa.sa[dim] = s_cp;
    pa.sb[dim] = p->d.c_m_stride[i];
    s_cp *= p->d.m_ext[i];
  }
  for (int i = 0; i < p->d.nn; ++i, ++dim) {
    pa.ext[dim] = p->d.n_ext[i];
    pa.sa[dim] = s_cp;
    pa.sb[dim] = p->d.c_n_stride[i];
    s_cp *= p->d.n_ext[i];
  }
  pa.dim = dim;
  return permute_launch(p->prec == TCCG_PREC_FP64 ? TCCG_F64 : TCCG_F32, pa, s);
}

extern "C" int tccg_plan_run_timed(const tccg_plan* p, const void* A, const void* B, void* C,
                                   double alpha, double beta, void* ws, size_t ws_bytes,
                                   void* stream, float* kernel_ms) {
  if (!kernel_ms) return fail(TCCG_ERR_INVALID, "null kernel_ms");
  cudaEvent_t ev[6];
  for (int i = 0; i < 6; ++i) CUDA_TRY(cudaEventCreate(&ev[i]));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // pre-record every event so that slots without a kernel read as 0 ms
  for (int i = 0; i < 6; ++i) cudaEventRecord(ev[i], s);
  g_events = ev;
  int rc = tccg_plan_run(p, A, B, C, alpha, beta, ws, ws_bytes, stream);
  g_events = nullptr;
  cudaError_t e = cudaStreamSynchronize(s);
  for (int i = 0; i < 3; ++i) {
    float ms = 0.f;
    if (!rc && e == cudaSuccess) cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
    kernel_ms[i] = ms;
  }
  for (int i = 0; i < 6; ++i) cudaEventDestroy(ev[i]);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(TCCG_ERR_CUDA, "stream sync: %s", cudaGetErrorString(e));
  return TCCG_OK;
}

extern "C" int tccg_plan_run_events(const tccg_plan* p, const void* A, const void* B, void* C,
                                    double alpha, double beta, void* ws, size_t ws_bytes,
                                    void* stream, void* const* events) {
  if (!events) return fail(TCCG_ERR_INVALID, "null events");
  cudaEvent_t ev[6];
  for (int i = 0; i < 6; ++i) {
    ev[i] = reinterpret_cast<cudaEvent_t>(events[i]);
    if (!ev[i]) return fail(TCCG_ERR_INVALID, "event %d is null", i);
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // pre-record every event so that slots without a kernel read as 0 ms
  for (int i = 0; i < 6; ++i) CUDA_TRY(cudaEventRecord(ev[i], s));
  g_events = ev;
  int rc = tccg_plan_run(p, A, B, C, alpha, beta, ws, ws_bytes, stream);
  g_events = nullptr;
  return rc;
}

// --------------------------------------------------------------------------
// transposition
// --------------------------------------------------------------------------
// Sorts the output dims so that dim 0 is B's stride-one dim, finds the dim of
// A's stride one and launches permute_kernel.
static int permute_launch(int32_t dtype, const PermArgs& pa0, cudaStream_t s) {
  PermArgs pa = pa0;
  if (pa.dim < 1 || pa.dim > PERM_MAX_DIMS) return fail(TCCG_ERR_INVALID, "bad dimension count");
  // drop unit extents, then fuse neighbouring output dims that are contiguous
  // in both tensors (fewer, longer dims: longer coalesced runs, less decoding)
  int n = 0;
  for (int d = 0; d < pa.dim; ++d) {
    if (pa.ext[d] == 1) continue;
    if (n > 0 && pa.sa[d] == pa.sa[n - 1] * pa.ext[n - 1] && pa.sb[d] == pa.sb[n - 1] * pa.ext[n - 1]) {
      pa.ext[n - 1] *= pa.ext[d];
      continue;
    }
    pa.ext[n] = pa.ext[d];
    pa.sa[n] = pa.sa[d];
    pa.sb[n] = pa.sb[d];
    ++n;
  }
  if (n == 0) {  // a single element
    pa.ext[0] = 1;
    pa.sa[0] = pa.sb[0] = 1;
    n = 1;
  }
  pa.dim = n;
  // the output dim with the smallest B stride first
  int b0 = 0;
  for (int d = 1; d < pa.dim; ++d)
    if (std::llabs(pa.sb[d]) < std::llabs(pa.sb[b0])) b0 = d;
  std::swap(pa.ext[0], pa.ext[b0]);
  std::swap(pa.sa[0], pa.sa[b0]);
  std::swap(pa.sb[0], pa.sb[b0]);
  int da = 0;
  for (int d = 1; d < pa.dim; ++d)
    if (std::llabs(pa.sa[d]) < std::llabs(pa.sa[da])) da = d;
  if (std::llabs(pa.sa[da]) == std::llabs(pa.sa[0])) da = 0;
  pa.da = da;
  int64_t rest = 1;
  for (int d = 1; d < pa.dim; ++d)
    if (d != da) rest *= pa.ext[d];
  pa.rest = rest;
  // tile edge: 64 unless that pads dim 0 x dim da by more than 5 % over 32
  const auto padded = [&](int64_t t) {
    return (double)(cdiv(pa.ext[0], t) * t) * (double)(cdiv(pa.ext[da], t) * t);
  };
  const bool t64 = da != 0 && padded(64) <= 1.05 * padded(32);
  const int te = t64 ? 64 : 32, rows = t64 ? 1 : 4;
  const bool along0 = !t64 && rest < 64;  // few rows: group tiles along dim 0 instead
  if (da == 0) {
    pa.nt0 = cdiv(pa.ext[0], 256 * PERM_STREAM);
    pa.nta = 1;
  } else {
    pa.nt0 = cdiv(pa.ext[0], (int64_t)te * (along0 ? rows : 1));
    pa.nta = cdiv(pa.ext[da], te);
  }
  if (pa.nt0 * pa.nta > INT32_MAX) return fail(TCCG_ERR_UNSUPPORTED, "transpose too large");
  const int64_t groups = (da == 0 || along0) ? rest : cdiv(rest, rows);
  dim3 grid;
  grid.x = (unsigned)(pa.nt0 * pa.nta);
  grid.y = (unsigned)std::min<int64_t>(groups, 65535);
  grid.z = (unsigned)std::min<int64_t>(cdiv(groups, grid.y), 1024);
  mark(2, 0, s);
  const dim3 blk(32, 8);
  if (da == 0 && pa.ext[0] < PERM_ROWS_MAX) {  // short rows: one warp per row
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const dim3 g1((unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv(rest, 8), (int64_t)sms * 8)));
    if (dtype == TCCG_F64)
      permute_rows_kernel<double><<<g1, blk, 0, s>>>(pa);
    else if (dtype == TCCG_F32)
      permute_rows_kernel<float><<<g1, blk, 0, s>>>(pa);
    else
      return fail(TCCG_ERR_UNSUPPORTED, "transpose supports TCCG_F32 and TCCG_F64");
    mark(2, 1, s);
    return launch_check("permute_rows");
  }
  if (dtype == TCCG_F64) {
    if (da == 0)
      permute_stream_kernel<double><<<grid, blk, 0, s>>>(pa);
    else if (t64)
      permute_kernel<double, 64, 1, false><<<grid, blk, 0, s>>>(pa);
    else if (along0)
      permute_kernel<double, 32, 4, true><<<grid, blk, 0, s>>>(pa);
    else
      permute_kernel<double, 32, 4, false><<<grid, blk, 0, s>>>(pa);
  } else if (dtype == TCCG_F32) {
    if (da == 0)
      permute_stream_kernel<float><<<grid, blk, 0, s>>>(pa);
    else if (t64)
      permute_kernel<float, 64, 1, false><<<grid, blk, 0, s>>>(pa);
    else if (along0)
      permute_kernel<float, 32, 4, true><<<grid, blk, 0, s>>>(pa);
    else
      permute_kernel<float, 32, 4, false><<<grid, blk, 0, s>>>(pa);
  } else {
    return fail(TCCG_ERR_UNSUPPORTED, "transpose supports TCCG_F32 and TCCG_F64");
  }
  mark(2, 1, s);
  return launch_check("permute");
}

extern "C" int tccg_transpose(int32_t dtype, int32_t dim, const int32_t* perm,
                              const int64_t* size, const int64_t* outer_a,
                              const int64_t* outer_b, double alpha, const void* A, double beta,
                              void* B, void* stream) {
  if (dim < 1 || dim > PERM_MAX_DIMS || !perm || !size || !A || !B)
    return fail(TCCG_ERR_INVALID, "bad transpose arguments");
  bool seen[PERM_MAX_DIMS] = {false};
  for (int j = 0; j < dim; ++j) {
    if (perm[j] < 0 || perm[j] >= dim || seen[perm[j]]) return fail(TCCG_ERR_INVALID, "perm is not a permutation");
    seen[perm[j]] = true;
    if (size[j] < 1) return fail(TCCG_ERR_INVALID, "size[%d] = %lld", j, (long long)size[j]);
  }
  int64_t stA[PERM_MAX_DIMS], stB[PERM_MAX_DIMS];
  int64_t s = 1;
  for (int i = 0; i < dim; ++i) {  // A strides (input order)
    stA[i] = s;
    const int64_t o = outer_a ? outer_a[i] : size[i];
    if (o < size[i]) return fail(TCCG_ERR_INVALID, "outer_a[%d] < size", i);
    s *= o;
  }
  s = 1;
  for (int j = 0; j < dim; ++j) {  // B strides (output order)
    stB[j] = s;
    const int64_t o = outer_b ? outer_b[j] : size[perm[j]];
    if (o < size[perm[j]]) return fail(TCCG_ERR_INVALID, "outer_b[%d] < size", j);
    s *= o;
  }
  PermArgs pa{};
  pa.A = A;
  pa.B = B;
  pa.dim = dim;
  pa.alpha = alpha;
  pa.beta = beta;
  for (int j = 0; j < dim; ++j) {
    pa.ext[j] = size[perm[j]];
    pa.sa[j] = stA[perm[j]];
    pa.sb[j] = stB[j];
  }
  return permute_launch(dtype, pa, reinterpret_cast<cudaStream_t>(stream));
}

// --------------------------------------------------------------------------
// grouped launches
// --------------------------------------------------------------------------
struct tccg_group {
  std::vector<const tccg_plan*> plans;
  int32_t prec = 0, dtype = 0;
  int device = 0, num_sms = 148;
  std::vector<size_t> ws_off;  // per item: start of its workspace within its wave's region
  size_t ws_bytes = 0;
  // CUDA-core lane (FP32/FP64 groups, and BF16-precision items that plan for
  // the CUDA cores): SimtGroupItem<T>[], T = double for FP64 groups else float
  void* d_simt = nullptr;
  int32_t n_simt = 0;
  PackJob* d_simt_jobs = nullptr;
  // tensor-core lane (BF16 / BF16X3 groups)
  TcGroupItem* d_tc = nullptr;
  int32_t n_tc = 0;
  PackJob* d_tc_jobs = nullptr;
  int32_t* tc_status = nullptr;
  // k-split reductions: ReduceJob<T>[] (same T as the CUDA-core lane)
  void* d_reduce = nullptr;
  // skinny lane (FP32 operands): the items' contractions and the k-split
  // reductions of those that split
  SkinnyItem* d_sk = nullptr;
  SkinnyItem* d_skr = nullptr;  // reductions of both skinny lanes
  int32_t n_sk = 0;
  // tensor-core skinny lane (split-BF16x3): items with Q's tensor maps; Q's
  // packs join the tensor-core lane's pack jobs
  SkinnyTcItem* d_sktc = nullptr;
  int32_t n_sktc = 0;
  int32_t* sktc_status = nullptr;
  // compact first-CTA / first-tile arrays of the jobs and items above (one
  // allocation): what the kernels binary-search instead of the large structs
  int64_t* d_begin = nullptr;
  int64_t *b_simt_jobs = nullptr, *b_tc_jobs = nullptr, *b_simt_items = nullptr,
          *b_tc_items = nullptr, *b_reduce = nullptr, *b_sk = nullptr, *b_skr = nullptr,
          *b_sktc = nullptr;
  // Waves: the items run in sets whose workspaces together stay within
  // kGroupWaveBytes (an item above it is a set of its own). Each wave is
  // packed and multiplied before the next one reuses the same workspace
  // region, so the group's workspace is that of its largest wave, not the sum
  // over its items. On the 256-item batched workload 4 GiB waves take the
  // time of one wave (22.0 vs 22.1 ms BF16x3) with 4.0 instead of 12.8 GiB of
  // workspace; 512 MiB waves cost 8 % more time (more, shorter launches).
  // The tensor-core items of a wave form one lane per kernel variant
  // (TcVariant): lane v holds items [lane0[v], lane0[v] + nlane[v]) of d_tc
  // and runs as one grouped launch of that variant's kernel.
  struct Wave {
    std::vector<size_t> items;  // plan indices
    int32_t simt0 = 0, n_simt = 0, red0 = 0, n_red = 0;
    int32_t lane0[TCV_COUNT] = {}, nlane[TCV_COUNT] = {};
    int64_t lane_tiles[TCV_COUNT] = {};
    int32_t tcj0 = 0, ntcj = 0;  // pack jobs of the packed-operand lanes (two per item)
    int64_t simt_tiles = 0, simt_pack_ctas = 0, tc_pack_ctas = 0, red_ctas = 0;
    // skinny lanes, one per rows-per-thread class (rs / 4 - 1: 4, 8, 12): items
    // [sk0[c], sk0[c] + nsk[c]) of d_sk with sk_jobs[c] jobs; reductions
    int32_t sk0[3] = {}, nsk[3] = {}, skr0 = 0, nskr = 0;
    int64_t sk_jobs[3] = {}, skr_ctas = 0;
    bool sk_reg[3] = {};  // the lane runs the register path
    // the tensor-core skinny lane: items [sktc0, sktc0 + nsktc) of d_sktc
    int32_t sktc0 = 0, nsktc = 0;
    int64_t sktc_jobs = 0;
  };
  std::vector<Wave> waves;
  bool bound = false;
  // concurrent lanes: two side streams (the CUDA-core skinny lanes; the
  // CUDA-core tiles with their packing) forked from and joined back into the
  // caller's stream around each wave's GETT launches, and their events
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
};

#ifndef TCCG_GROUP_WAVE_MB
#define TCCG_GROUP_WAVE_MB 4096
#endif
static constexpr size_t kGroupWaveBytes = size_t(TCCG_GROUP_WAVE_MB) << 20;

static void group_free(tccg_group* g) {
  if (!g) return;
  void* ps[] = {g->d_simt, g->d_simt_jobs, g->d_tc, g->d_tc_jobs, g->d_reduce, g->d_begin,
                g->d_sk, g->d_skr, g->d_sktc};
  for (void* q : ps)
    if (q) cudaFree(q);
  for (cudaStream_t q : g->side)
    if (q) cudaStreamDestroy(q);
  if (g->ev_fork) cudaEventDestroy(g->ev_fork);
  for (cudaEvent_t e : g->ev_join)
    if (e) cudaEventDestroy(e);
  delete g;
}

extern "C" int tccg_group_create(const tccg_plan* const* plans, int32_t count, tccg_group** out) {
  if (!plans || count < 1 || !out) return fail(TCCG_ERR_INVALID, "bad group arguments");
  *out = nullptr;
  tccg_group* g = new tccg_group();
  g->prec = plans[0]->prec;
  g->dtype = plans[0]->dtype;
  g->device = plans[0]->device;
  g->num_sms = plans[0]->num_sms;
  const bool dbl = g->prec == TCCG_PREC_FP64;
  size_t ws = 0;
  for (int i = 0; i < count; ++i) {
    const tccg_plan* p = plans[i];
    if (!p) { group_free(g); return fail(TCCG_ERR_INVALID, "plan %d is null", i); }
    if (p->prec != g->prec || p->dtype != g->dtype || p->device != g->device) {
      group_free(g);
      return fail(TCCG_ERR_UNSUPPORTED, "all plans of a group need the same precision, dtype and device");
    }
    if (p->tune.method != TCCG_METHOD_GETT || p->tune.pair) {
      group_free(g);
      return fail(TCCG_ERR_UNSUPPORTED, "grouped plans must be GETT without the CTA-pair kernel (plan %d)", i);
    }
    g->plans.push_back(p);
    if (p->sk_tc) {
      if (!g->sktc_status) g->sktc_status = p->d_status;
      ++g->n_sktc;
    } else if (p->skinny) {
      ++g->n_sk;
    } else if (simt_path(p)) {
      ++g->n_simt;
    } else {
      if (!g->tc_status) g->tc_status = p->d_status;
      ++g->n_tc;
    }
  }
  // waves, largest workspaces first (next fit under kGroupWaveBytes)
  std::vector<size_t> order(count);
  for (int i = 0; i < count; ++i) order[i] = (size_t)i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return g->plans[a]->ws_bytes > g->plans[b]->ws_bytes;
  });
  g->ws_off.assign(count, 0);
  for (size_t i : order) {
    const tccg_plan* p = g->plans[i];
    const size_t need = align_up(p->ws_bytes, 256);
    if (g->waves.empty() || ws + need > kGroupWaveBytes) {
      g->waves.emplace_back();
      ws = 0;
    }
    tccg_group::Wave& wv = g->waves.back();
    wv.items.push_back(i);
    g->ws_off[i] = ws;
    ws += need;
    g->ws_bytes = std::max(g->ws_bytes, ws);
    if (p->sk_tc) {
      wv.sktc_jobs += p->sk.njobs;
    } else if (p->skinny) {
      wv.sk_jobs[p->sk.rs / 4 - 1] += p->sk.njobs;
    } else if (simt_path(p)) {
      wv.simt_tiles += (p->Mp / p->simt_bm) * (p->Np / p->simt_bn) * p->ksplit;
    } else {
      wv.lane_tiles[p->tcv] += (int64_t)p->tiles_m * p->tiles_n * p->ksplit;
    }
    bool too_many = wv.simt_tiles > INT32_MAX || wv.sktc_jobs > INT32_MAX;
    for (int c = 0; c < 3; ++c) too_many |= wv.sk_jobs[c] > INT32_MAX;
    for (int v = 0; v < TCV_COUNT; ++v) too_many |= wv.lane_tiles[v] > INT32_MAX;
    if (too_many) {
      group_free(g);
      return fail(TCCG_ERR_UNSUPPORTED, "too many tiles");
    }
  }
  const size_t simt_item = dbl ? sizeof(SimtGroupItem<double>) : sizeof(SimtGroupItem<float>);
  cudaError_t e = cudaSuccess;
  if (g->n_simt) {
    e = cudaMalloc(&g->d_simt, simt_item * g->n_simt);
    if (e == cudaSuccess) e = cudaMalloc((void**)&g->d_simt_jobs, sizeof(PackJob) * 2 * g->n_simt);
  }
  // tensor-core pack jobs: two per tile item, Q's one per tensor-core skinny item
  const int32_t n_tcj = 2 * g->n_tc + g->n_sktc;
  if (e == cudaSuccess && n_tcj) e = cudaMalloc((void**)&g->d_tc_jobs, sizeof(PackJob) * n_tcj);
  if (e == cudaSuccess && g->n_tc) e = cudaMalloc((void**)&g->d_tc, sizeof(TcGroupItem) * g->n_tc);
  if (e == cudaSuccess && g->n_sk) e = cudaMalloc((void**)&g->d_sk, sizeof(SkinnyItem) * g->n_sk);
  if (e == cudaSuccess && g->n_sktc)
    e = cudaMalloc((void**)&g->d_sktc, sizeof(SkinnyTcItem) * g->n_sktc);
  if (e == cudaSuccess && g->n_sk + g->n_sktc)
    e = cudaMalloc((void**)&g->d_skr, sizeof(SkinnyItem) * (g->n_sk + g->n_sktc));
  if (e == cudaSuccess) e = cudaMalloc(&g->d_reduce, sizeof(ReduceJob<double>) * count);
  const size_t nbegin = 2 * (size_t)g->n_simt + n_tcj + g->n_simt + g->n_tc + count + g->n_sk +
                        (g->n_sk + g->n_sktc) + g->n_sktc;
  if (e == cudaSuccess) e = cudaMalloc((void**)&g->d_begin, sizeof(int64_t) * nbegin);
  if (e == cudaSuccess) {
    g->b_simt_jobs = g->d_begin;
    g->b_tc_jobs = g->b_simt_jobs + 2 * g->n_simt;
    g->b_simt_items = g->b_tc_jobs + n_tcj;
    g->b_tc_items = g->b_simt_items + g->n_simt;
    g->b_reduce = g->b_tc_items + g->n_tc;
    g->b_sk = g->b_reduce + count;
    g->b_skr = g->b_sk + g->n_sk;
    g->b_sktc = g->b_skr + g->n_sk + g->n_sktc;
  }
  if (e != cudaSuccess) {
    group_free(g);
    return fail(TCCG_ERR_CUDA, "group tables: %s", cudaGetErrorString(e));
  }
  *out = g;
  return TCCG_OK;
}

extern "C" int tccg_group_workspace(const tccg_group* g, size_t* bytes) {
  if (!g || !bytes) return fail(TCCG_ERR_INVALID, "null argument");
  *bytes = g->ws_bytes;
  return TCCG_OK;
}

template <typename T>
static void set_direct(SimtArgs<T>& a, const tccg_plan* p, const void* GA, const void* GB);

template <typename T>
static SimtArgs<T> simt_args_for(const tccg_plan* p, char* w, const void* GA, const void* GB,
                                 void* C, double alpha, double beta) {
  SimtArgs<T> a;
  a.Ap = reinterpret_cast<T*>(w + p->off_a);
  a.Bp = reinterpret_cast<T*>(w + p->off_b);
  a.Mp = p->Mp;
  a.Np = p->Np;
  a.M = p->M;
  a.N = p->N;
  a.ktiles = p->ktiles;
  a.ktiles_per_split = p->ktiles_per_split;
  a.C = static_cast<T*>(C);
  a.c_m_off = p->t_c_m;
  a.c_n_off = p->t_c_n;
  a.alpha = (T)alpha;
  a.beta = (T)beta;
  a.partial = p->ksplit > 1 ? reinterpret_cast<T*>(w + p->off_part) : nullptr;
  set_direct(a, p, GA, GB);
  a.status = p->d_status;
  a.crun = p->crun;
  return a;
}

// Reduction job of a k-split item: slices [split][Np][Mp] -> C.
template <typename T>
static ReduceJob<T> reduce_job_for(const T* partial, int32_t splits, int64_t Mp, int64_t Np,
                                   const tccg_plan* p, void* C, double alpha, double beta,
                                   int64_t begin) {
  ReduceJob<T> j;
  j.partial = partial;
  j.Mp = Mp;
  j.Np = Np;
  j.M = p->M;
  j.N = p->N;
  j.C = static_cast<T*>(C);
  j.c_m_off = p->t_c_m;
  j.c_n_off = p->t_c_n;
  j.alpha = (T)alpha;
  j.beta = (T)beta;
  j.begin = begin;
  j.splits = splits;
  j.mblocks = (int32_t)cdiv(p->M, 256);
  // about 256 loads per thread: many slices -> few columns per CTA
  j.ncols = (int32_t)std::max<int64_t>(1, std::min<int64_t>(64, 256 / splits));
  return j;
}

template <typename T>
static int64_t reduce_ctas(const ReduceJob<T>& j) {
  return (int64_t)j.mblocks * cdiv(j.N, j.ncols);
}

// Items of one lane, the most k-blocks per tile first: CTAs take tiles in
// index order (round robin in the persistent tensor-core kernel, launch order
// in the CUDA-core one), so the longest tiles start first and the short ones
// fill in behind them.
static std::vector<size_t> by_tile_cost(const tccg_group* g, const tccg_group::Wave& wv, bool simt,
                                        int variant = -1) {
  std::vector<size_t> idx;
  for (size_t i : wv.items)
    if (!g->plans[i]->skinny && simt_path(g->plans[i]) == simt &&
        (simt || g->plans[i]->tcv == variant))
      idx.push_back(i);
  auto cost = [&](size_t i) {
    const tccg_plan* p = g->plans[i];
    return simt ? (int64_t)p->ktiles_per_split : (int64_t)p->kb_per_split;
  };
  std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return cost(a) > cost(b); });
  return idx;
}

// Uploads the `begin` fields of `v` as a compact int64 array.
template <typename V, typename F>
static int upload_begins(const std::vector<V>& v, F field, int64_t* dst) {
  if (v.empty()) return TCCG_OK;
  std::vector<int64_t> b(v.size());
  for (size_t i = 0; i < v.size(); ++i) b[i] = field(v[i]);
  CUDA_TRY(cudaMemcpy(dst, b.data(), sizeof(int64_t) * b.size(), cudaMemcpyHostToDevice));
  return TCCG_OK;
}

// Two pack jobs (A, B) of one item; a direct item's jobs own no CTAs.
static void add_pack_jobs(std::vector<PackJob>& jobs, int64_t& ctas, const PackOperand& oa,
                          const PackOperand& ob, int ktile, bool active) {
  for (const PackOperand* o : {&oa, &ob}) {
    PackJob jb;
    jb.op = *o;
    pack_geometry(jb.op, ktile);
    jb.begin = ctas;
    if (active) ctas += jb.op.tiles;
    jobs.push_back(jb);
  }
}

// The CUDA-core lane of one wave of a bind, appended to `items` / `jobs` /
// `red` (first CTAs and tiles counted from 0 within the wave); T = the lane's
// element type.
template <typename T>
static int bind_simt(tccg_group* g, tccg_group::Wave& wv, const void* const* A,
                     const void* const* B, void* const* C, const double* alpha,
                     const double* beta, char* ws, std::vector<SimtGroupItem<T>>& items,
                     std::vector<PackJob>& jobs, std::vector<ReduceJob<T>>& red, int64_t& rctas) {
  wv.simt0 = (int32_t)items.size();
  int64_t tile = 0, pctas = 0;
  for (size_t i : by_tile_cost(g, wv, true)) {
    const tccg_plan* p = g->plans[i];
    char* w = ws + g->ws_off[i];
    const void* GA = p->d.swap_ab ? B[i] : A[i];
    const void* GB = p->d.swap_ab ? A[i] : B[i];
    add_pack_jobs(jobs, pctas,
                  pack_op(GA, p->t_a_m, p->t_a_k, p->M, p->K, p->Mp, p->Kp, w + p->off_a, p->Mp,
                          p->read_k_fast_a),
                  pack_op(GB, p->t_b_n, p->t_b_k, p->N, p->K, p->Np, p->Kp, w + p->off_b, p->Np,
                          p->read_k_fast_b),
                  pack_k_tile<PACK_MN>(), !p->direct);
    SimtGroupItem<T> it;
    it.args = simt_args_for<T>(p, w, GA, GB, C[i], alpha[i], beta[i]);
    it.tile_begin = tile;
    it.tiles_m = (int32_t)(p->Mp / p->simt_bm);
    it.tiles_n = (int32_t)(p->Np / p->simt_bn);
    it.shape = p->simt_shape;
    tile += (int64_t)it.tiles_m * it.tiles_n * p->ksplit;
    items.push_back(it);
    if (p->ksplit > 1) {
      red.push_back(reduce_job_for<T>(it.args.partial, p->ksplit, p->Mp, p->Np, p, C[i], alpha[i],
                                      beta[i], rctas));
      rctas += reduce_ctas(red.back());
    }
  }
  if (pctas > INT32_MAX) return fail(TCCG_ERR_UNSUPPORTED, "grouped packing grid too large");
  wv.n_simt = (int32_t)items.size() - wv.simt0;
  wv.simt_pack_ctas = pctas;
  return TCCG_OK;
}

static int bind_tc(tccg_group* g, tccg_group::Wave& wv, const void* const* A, const void* const* B,
                   void* const* C, const double* alpha, const double* beta, char* ws,
                   std::vector<TcGroupItem>& items, std::vector<PackJob>& jobs,
                   std::vector<ReduceJob<float>>& red, int64_t& rctas) {
  int64_t pctas = 0;
  wv.tcj0 = (int32_t)jobs.size();
  for (int lane = 0; lane < TCV_COUNT; ++lane) {  // one lane per kernel variant
    const bool gather = lane == TCV_X3_GATHER;
    wv.lane0[lane] = (int32_t)items.size();
    int64_t tile = 0;
    for (size_t i : by_tile_cost(g, wv, false, lane)) {
      const tccg_plan* p = g->plans[i];
      char* w = ws + g->ws_off[i];
      const void* GA = p->d.swap_ab ? B[i] : A[i];
      const void* GB = p->d.swap_ab ? A[i] : B[i];
      TcGroupItem it;
      memset(&it, 0, sizeof(it));
      it.args = tc_args(p, static_cast<float*>(C[i]), p->t_c_m, p->t_c_n, (float)alpha[i],
                        (float)beta[i], w);
      // grouped tiles run over all of K or their k-split slices, never a tail split
      it.args.full_tiles = 0;
      it.args.tail_split = 1;
      it.args.tail_kb = 0;
      it.args.tail_partial = nullptr;
      if (gather) {
        set_gather(it.args, p, GA, GB);
      } else {
        const int64_t kcover = p->prec == TCCG_PREC_BF16X3 ? round_up(p->K, 32) : p->Kc;
        const size_t es = p->dtype == TCCG_BF16 ? 2 : 4;
        add_pack_jobs(jobs, pctas,
                      with_kread(with_visit(pack_op(GA, p->t_a_m, p->t_a_k, p->M, p->K, p->M, kcover,
                                                    w + p->off_a, p->Kc, p->read_k_fast_a),
                                            p->t_a_vsrc, p->t_a_vdst), p->ks_a, p->kb_a, p->kbq_a, es),
                      with_kread(with_visit(pack_op(GB, p->t_b_n, p->t_b_k, p->N, p->K, p->N, kcover,
                                                    w + p->off_b, p->Kc, p->read_k_fast_b),
                                            p->t_b_vsrc, p->t_b_vdst), p->ks_b, p->kb_b, p->kbq_b, es),
                      pack_k_tile<PACK_K_BF16>(), true);
        int rc = encode_kmajor(&it.tmA, w + p->off_a, p->M, p->Kc, 128);
        if (!rc) rc = encode_kmajor(&it.tmB, w + p->off_b, p->N, p->Kc, p->bn);
        if (rc) return rc;
      }
      it.tile_begin = tile;
      tile += (int64_t)p->tiles_m * p->tiles_n * p->ksplit;
      items.push_back(it);
      if (p->ksplit > 1) {
        red.push_back(reduce_job_for<float>(it.args.partial, p->ksplit, p->M, p->N, p, C[i],
                                            alpha[i], beta[i], rctas));
        rctas += reduce_ctas(red.back());
      }
    }
    wv.nlane[lane] = (int32_t)items.size() - wv.lane0[lane];
  }
  if (pctas > INT32_MAX) return fail(TCCG_ERR_UNSUPPORTED, "grouped packing grid too large");
  wv.ntcj = (int32_t)jobs.size() - wv.tcj0;
  wv.tc_pack_ctas = pctas;
  return TCCG_OK;
}

// The skinny lanes of one wave (one per rows-per-thread class; in each the
// items with the longest k slices first: a CTA takes jobs in index order)
// and the reductions of the items with a k-split; job and CTA indices
// counted from 0 within the lane.
static void bind_skinny(tccg_group* g, tccg_group::Wave& wv, const void* const* A,
                        const void* const* B, void* const* C, const double* alpha,
                        const double* beta, char* ws, std::vector<SkinnyItem>& items,
                        std::vector<SkinnyItem>& red) {
  wv.skr0 = (int32_t)red.size();
  int64_t rctas = 0;
  for (int cls = 0; cls < 3; ++cls) {
    wv.sk0[cls] = (int32_t)items.size();
    std::vector<size_t> idx;
    for (size_t i : wv.items)
      if (g->plans[i]->skinny && !g->plans[i]->sk_tc && g->plans[i]->sk.rs / 4 - 1 == cls)
        idx.push_back(i);
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
      return g->plans[a]->sk.chunks_per_split > g->plans[b]->sk.chunks_per_split;
    });
    int64_t jobs = 0;
    for (size_t i : idx) {
      const tccg_plan* p = g->plans[i];
      const void* GA = p->d.swap_ab ? B[i] : A[i];
      const void* GB = p->d.swap_ab ? A[i] : B[i];
      SkinnyItem it;
      memset(&it, 0, sizeof(it));
      it.args = skinny_args(p, GA, GB, static_cast<float*>(C[i]), (float)alpha[i],
                            (float)beta[i], ws + g->ws_off[i]);
      it.begin = jobs;
      jobs += p->sk.njobs;
      items.push_back(it);
      if (p->sk_ksplit > 1) {
        SkinnyItem r = it;
        r.begin = rctas;
        rctas += (int64_t)p->sk.nblk * p->sk.npass;
        red.push_back(r);
      }
    }
    wv.nsk[cls] = (int32_t)items.size() - wv.sk0[cls];
    wv.sk_jobs[cls] = jobs;
    wv.sk_reg[cls] = !idx.empty() && g->plans[idx[0]]->sk_reg;
  }
  wv.nskr = (int32_t)red.size() - wv.skr0;
  wv.skr_ctas = rctas;
}

// The tensor-core skinny lane of one wave: its items (Q's tensor map on the
// item's workspace, longest k slices first), Q's pack jobs appended to the
// tensor-core lane's (the same packing launch) and the k-split reductions
// next to the CUDA-core skinny lane's.
static int bind_sktc(tccg_group* g, tccg_group::Wave& wv, const void* const* A,
                     const void* const* B, void* const* C, const double* alpha,
                     const double* beta, char* ws, std::vector<SkinnyTcItem>& items,
                     std::vector<PackJob>& jobs, std::vector<SkinnyItem>& red) {
  wv.sktc0 = (int32_t)items.size();
  std::vector<size_t> idx;
  for (size_t i : wv.items)
    if (g->plans[i]->sk_tc) idx.push_back(i);
  std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
    return g->plans[a]->sk.chunks_per_split > g->plans[b]->sk.chunks_per_split;
  });
  int64_t jobs_n = 0, pctas = wv.tc_pack_ctas, rctas = wv.skr_ctas;
  for (size_t i : idx) {
    const tccg_plan* p = g->plans[i];
    char* w = ws + g->ws_off[i];
    const void* GA = p->d.swap_ab ? B[i] : A[i];
    const void* GB = p->d.swap_ab ? A[i] : B[i];
    SkinnyTcItem it;
    memset(&it, 0, sizeof(it));
    int rc = encode_kmajor(&it.tmQ, w + p->off_q, (int64_t)p->sk.npass * p->sk_spad, p->Kc,
                           p->sk_spad);
    if (rc) return rc;
    it.args = skinny_tc_args(p, GA, GB, static_cast<float*>(C[i]), (float)alpha[i], (float)beta[i], w);
    it.begin = jobs_n;
    jobs_n += p->sk.njobs;
    items.push_back(it);
    PackJob jb;
    jb.op = skinny_tc_q(p, GA, GB, w);
    pack_geometry(jb.op, pack_k_tile<PACK_K_BF16>());
    jb.begin = pctas;
    pctas += jb.op.tiles;
    jobs.push_back(jb);
    if (p->sk_ksplit > 1) {
      SkinnyItem r;
      memset(&r, 0, sizeof(r));
      r.args = it.args.sk;
      r.begin = rctas;
      rctas += (int64_t)p->sk.nblk * p->sk.npass;
      red.push_back(r);
    }
  }
  if (pctas > INT32_MAX) return fail(TCCG_ERR_UNSUPPORTED, "grouped packing grid too large");
  wv.nsktc = (int32_t)items.size() - wv.sktc0;
  wv.sktc_jobs = jobs_n;
  wv.ntcj = (int32_t)jobs.size() - wv.tcj0;
  wv.tc_pack_ctas = pctas;
  wv.nskr = (int32_t)red.size() - wv.skr0;
  wv.skr_ctas = rctas;
  return TCCG_OK;
}

extern "C" int tccg_group_bind(tccg_group* g, const void* const* A, const void* const* B,
                               void* const* C, const double* alpha, const double* beta, void* ws,
                               size_t ws_bytes) {
  if (!g || !A || !B || !C || !alpha || !beta) return fail(TCCG_ERR_INVALID, "null argument");
  if (ws_bytes < g->ws_bytes || (g->ws_bytes && !ws))
    return fail(TCCG_ERR_WORKSPACE, "group workspace of %zu bytes needed, %zu given", g->ws_bytes, ws_bytes);
  if ((reinterpret_cast<uintptr_t>(ws) & 255u) != 0) return fail(TCCG_ERR_ALIGNMENT, "workspace must be 256-byte aligned");
  for (size_t i = 0; i < g->plans.size(); ++i)
    if (!A[i] || !B[i] || !C[i]) return fail(TCCG_ERR_INVALID, "null operand pointer for item %zu", i);
  g->bound = false;
  if (!g->ev_fork) {  // the concurrent lanes' streams and events, once per group
    for (cudaStream_t& q : g->side) CUDA_TRY(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming));
    for (cudaEvent_t& e : g->ev_join) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  char* w = static_cast<char*>(ws);
  int rc;
  // all waves' items, jobs and reductions in one array per kind, wave after
  // wave; each wave's kernels see their slice (first CTAs from 0)
  auto bind_all = [&](auto tag, auto& simt_items, auto& red) -> int {
    using T = decltype(tag);
    std::vector<PackJob> sjobs, tjobs;
    std::vector<TcGroupItem> titems;
    std::vector<SkinnyItem> kitems, kred;
    std::vector<SkinnyTcItem> ktc;
    int r = TCCG_OK;
    for (tccg_group::Wave& wv : g->waves) {
      int64_t rctas = 0;
      wv.red0 = (int32_t)red.size();
      r = bind_simt<T>(g, wv, A, B, C, alpha, beta, w, simt_items, sjobs, red, rctas);
      if (r) return r;
      if constexpr (sizeof(T) == 4) {
        r = bind_tc(g, wv, A, B, C, alpha, beta, w, titems, tjobs, red, rctas);
        if (r) return r;
        bind_skinny(g, wv, A, B, C, alpha, beta, w, kitems, kred);
        r = bind_sktc(g, wv, A, B, C, alpha, beta, w, ktc, tjobs, kred);
        if (r) return r;
      }
      if (rctas > INT32_MAX) return fail(TCCG_ERR_UNSUPPORTED, "grouped reduction grid too large");
      wv.n_red = (int32_t)red.size() - wv.red0;
      wv.red_ctas = rctas;
    }
    if (!simt_items.empty()) {
      CUDA_TRY(cudaMemcpy(g->d_simt, simt_items.data(), sizeof(simt_items[0]) * simt_items.size(),
                          cudaMemcpyHostToDevice));
      CUDA_TRY(cudaMemcpy(g->d_simt_jobs, sjobs.data(), sizeof(PackJob) * sjobs.size(),
                          cudaMemcpyHostToDevice));
    }
    if (!titems.empty())
      CUDA_TRY(cudaMemcpy(g->d_tc, titems.data(), sizeof(TcGroupItem) * titems.size(),
                          cudaMemcpyHostToDevice));
    if (!tjobs.empty())
      CUDA_TRY(cudaMemcpy(g->d_tc_jobs, tjobs.data(), sizeof(PackJob) * tjobs.size(),
                          cudaMemcpyHostToDevice));
    if (!red.empty())
      CUDA_TRY(cudaMemcpy(g->d_reduce, red.data(), sizeof(red[0]) * red.size(), cudaMemcpyHostToDevice));
    if (!kitems.empty())
      CUDA_TRY(cudaMemcpy(g->d_sk, kitems.data(), sizeof(SkinnyItem) * kitems.size(),
                          cudaMemcpyHostToDevice));
    if (!kred.empty())
      CUDA_TRY(cudaMemcpy(g->d_skr, kred.data(), sizeof(SkinnyItem) * kred.size(),
                          cudaMemcpyHostToDevice));
    if (!ktc.empty())
      CUDA_TRY(cudaMemcpy(g->d_sktc, ktc.data(), sizeof(SkinnyTcItem) * ktc.size(),
                          cudaMemcpyHostToDevice));
    auto item_begin = [](const auto& x) { return x.tile_begin; };
    auto job_begin = [](const auto& x) { return x.begin; };
    r = upload_begins(simt_items, item_begin, g->b_simt_items);
    if (!r) r = upload_begins(sjobs, job_begin, g->b_simt_jobs);
    if (!r) r = upload_begins(titems, item_begin, g->b_tc_items);
    if (!r) r = upload_begins(tjobs, job_begin, g->b_tc_jobs);
    if (!r) r = upload_begins(red, job_begin, g->b_reduce);
    if (!r) r = upload_begins(kitems, job_begin, g->b_sk);
    if (!r) r = upload_begins(kred, job_begin, g->b_skr);
    if (!r) r = upload_begins(ktc, job_begin, g->b_sktc);
    return r;
  };
  if (g->prec == TCCG_PREC_FP64) {
    std::vector<SimtGroupItem<double>> items;
    std::vector<ReduceJob<double>> red;
    rc = bind_all(double(0), items, red);
  } else {
    std::vector<SimtGroupItem<float>> items;
    std::vector<ReduceJob<float>> red;
    rc = bind_all(float(0), items, red);
  }
  if (rc) return rc;
  g->bound = true;
  return TCCG_OK;
}

// Launches of a group run, wave by wave. The lanes run concurrently: the
// tensor-core lanes (their packing, the tcgen05 tiles, the tensor-core
// skinny kernel) on the caller's stream, the CUDA-core skinny lanes on one
// side stream and the CUDA-core tiles (with their packing) on another, forked
// from the caller's stream and joined back before the k-split reductions --
// so that a lane's last CTAs share the GPU with the next lane's first
// instead of leaving SMs idle (in a CUDA graph the streams become parallel
// branches). Each launch only when the wave has work for it.
template <typename T>
static int run_wave(const tccg_group* g, const tccg_group::Wave& wv, cudaStream_t s) {
  int rc;
  const dim3 blk(32, 8);
  const int sj = 2 * wv.n_simt, tj = wv.ntcj;
  bool skinny_side = false;
  for (int cls = 0; cls < 3; ++cls) skinny_side |= wv.nsk[cls] > 0;
  const bool simt_side = wv.n_simt > 0;
  cudaStream_t s_sk = skinny_side ? g->side[0] : s, s_simt = simt_side ? g->side[1] : s;
  if (skinny_side || simt_side) {
    CUDA_TRY(cudaEventRecord(g->ev_fork, s));
    if (skinny_side) CUDA_TRY(cudaStreamWaitEvent(s_sk, g->ev_fork, 0));
    if (simt_side) CUDA_TRY(cudaStreamWaitEvent(s_simt, g->ev_fork, 0));
  }
  // CUDA-core tiles: packing and GETT on their stream
  const PackJob* sjobs = g->d_simt_jobs + 2 * wv.simt0;
  const int64_t* sb = g->b_simt_jobs + 2 * wv.simt0;
  if (wv.simt_pack_ctas > 0) {
    const dim3 pg((unsigned)wv.simt_pack_ctas);
    if (g->prec == TCCG_PREC_FP64)
      pack_group_kernel<double, double, PACK_MN><<<pg, blk, 0, s_simt>>>(sjobs, sb, sj);
    else if (g->dtype == TCCG_BF16)
      pack_group_kernel<__nv_bfloat16, float, PACK_MN><<<pg, blk, 0, s_simt>>>(sjobs, sb, sj);
    else if (g->prec == TCCG_PREC_BF16)
      pack_group_kernel<float, float, PACK_MN_BF16><<<pg, blk, 0, s_simt>>>(sjobs, sb, sj);
    else
      pack_group_kernel<float, float, PACK_MN><<<pg, blk, 0, s_simt>>>(sjobs, sb, sj);
    if ((rc = launch_check("pack_group"))) return rc;
  }
  if (wv.n_simt > 0) {
    simt_gett_group_kernel<T><<<(unsigned)wv.simt_tiles, 256, simt_group_smem_bytes<T>(), s_simt>>>(
        static_cast<const SimtGroupItem<T>*>(g->d_simt) + wv.simt0, g->b_simt_items + wv.simt0,
        wv.n_simt);
    if ((rc = launch_check("simt_gett_group"))) return rc;
  }
  // CUDA-core skinny lanes on theirs
  if constexpr (sizeof(T) == 4) {
    for (int cls = 0; cls < 3; ++cls) {
      if (wv.nsk[cls] == 0) continue;
      if (wv.sk_reg[cls]) {  // the register path (its items all take it)
        // one launch of 16 computed rows for all of them: splitting the lane
        // into an 8-row launch (narrow sides <= 8) and a 16-row one measured
        // slower on the 256-item batched workload (10.95 against 10.78 ms:
        // two launch tails), though the 8-row kernel is faster for such an
        // item alone
        const unsigned grid =
            (unsigned)std::min<int64_t>(wv.sk_jobs[cls], (int64_t)SKR_CTAS_PER_SM * g->num_sms);
        skinny_reg_group_kernel<16><<<grid, SKR_THREADS, SKR_SMEM_BYTES, s_sk>>>(
            g->d_sk + wv.sk0[cls], g->b_sk + wv.sk0[cls], wv.nsk[cls], (int)wv.sk_jobs[cls]);
      } else {
        const unsigned grid =
            (unsigned)std::min<int64_t>(wv.sk_jobs[cls], (int64_t)SK_CTAS_PER_SM * g->num_sms);
        with_skinny_rs(4 * (cls + 1), [&](auto r) {
          skinny_group_kernel<decltype(r)::value><<<grid, SK_THREADS, SK_SMEM_BYTES, s_sk>>>(
              g->d_sk + wv.sk0[cls], g->b_sk + wv.sk0[cls], wv.nsk[cls], wv.sk_jobs[cls]);
        });
      }
      if ((rc = launch_check("skinny_group"))) return rc;
    }
  }
  // tensor-core lanes on the caller's stream
  const bool x3 = g->prec == TCCG_PREC_BF16X3;
  const PackJob* tjobs = g->d_tc_jobs + wv.tcj0;
  const int64_t* tb = g->b_tc_jobs + wv.tcj0;
  if (wv.tc_pack_ctas > 0) {
    const dim3 pg((unsigned)wv.tc_pack_ctas);
    if (x3)
      pack_group_kernel<float, __nv_bfloat16, PACK_K_BF16X3><<<pg, blk, 0, s>>>(tjobs, tb, tj);
    else if (g->dtype == TCCG_BF16)
      pack_group_kernel<__nv_bfloat16, __nv_bfloat16, PACK_K_BF16><<<pg, blk, 0, s>>>(tjobs, tb, tj);
    else
      pack_group_kernel<float, __nv_bfloat16, PACK_K_BF16><<<pg, blk, 0, s>>>(tjobs, tb, tj);
    if ((rc = launch_check("pack_group"))) return rc;
  }
  for (int v = 0; v < TCV_COUNT; ++v) {
    if (wv.nlane[v] == 0) continue;
    TcGroup tg;
    tg.items = g->d_tc + wv.lane0[v];
    tg.tile_begin = g->b_tc_items + wv.lane0[v];
    tg.n_items = wv.nlane[v];
    tg.total_tiles = (int32_t)wv.lane_tiles[v];
    const unsigned grid = (unsigned)std::min<int64_t>(wv.lane_tiles[v], g->num_sms);
    with_tc_variant(v, [&](auto k) {
      using K = decltype(k);
      K::group<<<grid, K::Cfg::NUM_THREADS, K::Cfg::SMEM_BYTES, s>>>(tg, g->tc_status);
    });
    if ((rc = launch_check("gett_tc_group"))) return rc;
  }
  if constexpr (sizeof(T) == 4) {
    if (wv.nsktc > 0) {
      const unsigned grid = (unsigned)std::min<int64_t>(wv.sktc_jobs, g->num_sms);
      skinny_tc_group_kernel<<<grid, SKT_THREADS, SKT_SMEM_BYTES, s>>>(
          g->d_sktc + wv.sktc0, g->b_sktc + wv.sktc0, wv.nsktc, (int)wv.sktc_jobs, g->sktc_status);
      if ((rc = launch_check("skinny_tc_group"))) return rc;
    }
  }
  // join, then the k-split reductions of every lane
  if (skinny_side) {
    CUDA_TRY(cudaEventRecord(g->ev_join[0], s_sk));
    CUDA_TRY(cudaStreamWaitEvent(s, g->ev_join[0], 0));
  }
  if (simt_side) {
    CUDA_TRY(cudaEventRecord(g->ev_join[1], s_simt));
    CUDA_TRY(cudaStreamWaitEvent(s, g->ev_join[1], 0));
  }
  if constexpr (sizeof(T) == 4) {
    if (wv.nskr > 0) {
      skinny_reduce_group_kernel<<<(unsigned)wv.skr_ctas, SK_THREADS, SK_SMEM_BYTES, s>>>(
          g->d_skr + wv.skr0, g->b_skr + wv.skr0, wv.nskr);
      if ((rc = launch_check("skinny_reduce_group"))) return rc;
    }
  }
  if (wv.n_red > 0) {
    reduce_group_kernel<T><<<(unsigned)wv.red_ctas, 256, 0, s>>>(
        static_cast<const ReduceJob<T>*>(g->d_reduce) + wv.red0, g->b_reduce + wv.red0, wv.n_red);
    if ((rc = launch_check("reduce_group"))) return rc;
  }
  return TCCG_OK;
}

extern "C" int tccg_group_run(const tccg_group* g, void* stream) {
  if (!g) return fail(TCCG_ERR_INVALID, "null group");
  if (!g->bound) return fail(TCCG_ERR_INVALID, "tccg_group_bind must be called before tccg_group_run");
  int rc = ensure_attrs();
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  for (const tccg_group::Wave& wv : g->waves) {
    rc = g->prec == TCCG_PREC_FP64 ? run_wave<double>(g, wv, s) : run_wave<float>(g, wv, s);
    if (rc) return rc;
  }
  return TCCG_OK;
}

extern "C" int tccg_group_destroy(tccg_group* g) {
  group_free(g);
  return TCCG_OK;
}

// --------------------------------------------------------------------------
// allocation-free split-BF16x3 GETT
// --------------------------------------------------------------------------
// For callers that must not allocate device memory: a process whose HBM is
// already reserved up front by a framework's caching allocator (cudaMalloc
// would fail or fragment its pool), or a latency-critical serving loop that
// cannot afford cudaMalloc/cudaFree, which may synchronise the device. This
// entry point runs the same packing and tcgen05 kernels as tccg_plan_run with
// PREC_BF16X3, but everything it needs besides the caller's A, B and C -- the
// offset tables, the packed operands and the status word -- lives in the
// static device array below: TCCG_NOALLOC_SCRATCH_BYTES (64 MiB) on every GPU
// that loads the library, held until the process exits. The status word is
// read (and cleared) by tccg_gett_bf16x3_noalloc_status.
#define TCCG_NOALLOC_SCRATCH_BYTES (64ull << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[TCCG_NOALLOC_SCRATCH_BYTES];

#define TCCG_NOALLOC_MAX_DEVICES 64
static void* g_noalloc_ptr[TCCG_NOALLOC_MAX_DEVICES];
static int g_noalloc_sms[TCCG_NOALLOC_MAX_DEVICES];
static cudaError_t g_noalloc_err[TCCG_NOALLOC_MAX_DEVICES];
static std::once_flag g_noalloc_once[TCCG_NOALLOC_MAX_DEVICES];

// The host-side name g_noalloc_scratch is only a stand-in for the device
// array; its device address comes from cudaGetSymbolAddress, once per device,
// with that device current (the first call on each device does this).
static int noalloc_setup(int dev) {
  std::call_once(g_noalloc_once[dev], [dev] {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e == cudaSuccess)
      e = cudaDeviceGetAttribute(&g_noalloc_sms[dev], cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaMemset(ptr, 0, sizeof(int32_t));  // the status word
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    g_noalloc_ptr[dev] = (e == cudaSuccess) ? ptr : nullptr;
    g_noalloc_err[dev] = e;
  });
  if (g_noalloc_err[dev] != cudaSuccess || !g_noalloc_ptr[dev])
    return fail(TCCG_ERR_CUDA, "scratch address of device %d: %s", dev,
                cudaGetErrorString(g_noalloc_err[dev]));
  return TCCG_OK;
}

// The six offset tables of a descriptor, computed on the device (so that no
// host buffer or host-to-device copy is needed). Table t, entry l:
// sum_i idx_i(l) * stride_i with the modes of that table, first mode fastest.
__global__ void __launch_bounds__(256) noalloc_tables_kernel(const tccg_desc d, int64_t* a_m,
                                                             int64_t* a_k, int64_t* b_n,
                                                             int64_t* b_k, int64_t* c_m,
                                                             int64_t* c_n, int64_t M, int64_t N,
                                                             int64_t K) {
  const int64_t total = 2 * (M + N + K);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t l = t;
    int n;
    const int64_t *ext, *str;
    int64_t* out;
    if (l < M) { n = d.nm; ext = d.m_ext; str = d.a_m_stride; out = a_m; }
    else if ((l -= M) < K) { n = d.nk; ext = d.k_ext; str = d.a_k_stride; out = a_k; }
    else if ((l -= K) < N) { n = d.nn; ext = d.n_ext; str = d.b_n_stride; out = b_n; }
    else if ((l -= N) < K) { n = d.nk; ext = d.k_ext; str = d.b_k_stride; out = b_k; }
    else if ((l -= K) < M) { n = d.nm; ext = d.m_ext; str = d.c_m_stride; out = c_m; }
    else { l -= M; n = d.nn; ext = d.n_ext; str = d.c_n_stride; out = c_n; }
    int64_t rem = l, off = 0;
    for (int i = 0; i < n; ++i) {
      off += (rem % ext[i]) * str[i];
      rem /= ext[i];
    }
    out[l] = off;
  }
}

extern "C" int tccg_gett_bf16x3_noalloc(const tccg_desc* desc, const float* A, const float* B,
                                        float* C, double alpha, double beta, void* stream) {
  if (!desc || !A || !B || !C) return fail(TCCG_ERR_INVALID, "null argument");
  const tccg_desc& d = *desc;
  if (d.nm < 1 || d.nn < 1 || d.nk < 1 || d.nm > TCCG_MAX_MODES || d.nn > TCCG_MAX_MODES ||
      d.nk > TCCG_MAX_MODES)
    return fail(TCCG_ERR_INVALID, "mode counts (nm=%d nn=%d nk=%d) must be in [1,%d]", d.nm, d.nn,
                d.nk, TCCG_MAX_MODES);
  int64_t M = 1, N = 1, K = 1;
  int rc0 = mode_product("M", d.nm, d.m_ext, &M);
  if (!rc0) rc0 = mode_product("N", d.nn, d.n_ext, &N);
  if (!rc0) rc0 = mode_product("K", d.nk, d.k_ext, &K);
  if (rc0) return rc0;
  // scratch layout: status | a_m | a_k | b_n | b_k | c_m | c_n | A' | B'
  const int64_t Kc = 2 * round_up(K, 32);
  size_t off = 256;
  const size_t o_am = off; off = align_up(off + (size_t)M * 8, 256);
  const size_t o_ak = off; off = align_up(off + (size_t)K * 8, 256);
  const size_t o_bn = off; off = align_up(off + (size_t)N * 8, 256);
  const size_t o_bk = off; off = align_up(off + (size_t)K * 8, 256);
  const size_t o_cm = off; off = align_up(off + (size_t)M * 8, 256);
  const size_t o_cn = off; off = align_up(off + (size_t)N * 8, 256);
  const size_t o_pa = off; off = align_up(off + (size_t)(M * Kc) * 2, 256);
  const size_t o_pb = off; off = align_up(off + (size_t)(N * Kc) * 2, 256);
  if (off > TCCG_NOALLOC_SCRATCH_BYTES)
    return fail(TCCG_ERR_WORKSPACE,
                "contraction needs %zu bytes of scratch; the allocation-free entry point has a "
                "fixed %llu-byte static scratch (use tccg_plan_run with a workspace instead)",
                off, (unsigned long long)TCCG_NOALLOC_SCRATCH_BYTES);
  int dev = -1;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= TCCG_NOALLOC_MAX_DEVICES) return fail(TCCG_ERR_UNSUPPORTED, "device index %d", dev);
  int rc = noalloc_setup(dev);
  if (rc) return rc;
  rc = ensure_attrs();
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  char* w = static_cast<char*>(g_noalloc_ptr[dev]);
  int32_t* status = reinterpret_cast<int32_t*>(w);
  int64_t* t_am = reinterpret_cast<int64_t*>(w + o_am);
  int64_t* t_ak = reinterpret_cast<int64_t*>(w + o_ak);
  int64_t* t_bn = reinterpret_cast<int64_t*>(w + o_bn);
  int64_t* t_bk = reinterpret_cast<int64_t*>(w + o_bk);
  int64_t* t_cm = reinterpret_cast<int64_t*>(w + o_cm);
  int64_t* t_cn = reinterpret_cast<int64_t*>(w + o_cn);
  // the status word keeps the first code a kernel recorded (from this or an
  // earlier call) until tccg_gett_bf16x3_noalloc_status reads and clears it
  const int64_t ntab = 2 * (M + N + K);
  noalloc_tables_kernel<<<(unsigned)std::min<int64_t>(cdiv(ntab, 256), 4096), 256, 0, s>>>(
      d, t_am, t_ak, t_bn, t_bk, t_cm, t_cn, M, N, K);
  if ((rc = launch_check("noalloc_tables"))) return rc;
  const void* GA = d.swap_ab ? (const void*)B : (const void*)A;
  const void* GB = d.swap_ab ? (const void*)A : (const void*)B;
  PackArgs pa;
  const int64_t kcover = round_up(K, 32);
  pa.op[0] = pack_op(GA, t_am, t_ak, M, K, M, kcover, w + o_pa, Kc,
                     pick_read_k_fast(d.nm, d.m_ext, d.a_m_stride, d.nk, d.k_ext, d.a_k_stride));
  pa.op[1] = pack_op(GB, t_bn, t_bk, N, K, N, kcover, w + o_pb, Kc,
                     pick_read_k_fast(d.nn, d.n_ext, d.b_n_stride, d.nk, d.k_ext, d.b_k_stride));
  if ((rc = launch_pack<float, __nv_bfloat16, PACK_K_BF16X3>(pa, s))) return rc;
  using Cfg = TcCfgT<TC_BF16X3>;
  CUtensorMap tmA, tmB;
  if ((rc = encode_kmajor(&tmA, w + o_pa, M, Kc, Cfg::BM))) return rc;
  if ((rc = encode_kmajor(&tmB, w + o_pb, N, Kc, Cfg::BN))) return rc;
  TcArgs a{};
  a.M = (int32_t)M;
  a.N = (int32_t)N;
  a.K = (int32_t)K;
  a.num_kb = (int32_t)cdiv(K, 32);
  a.tiles_m = (int32_t)cdiv(M, Cfg::BM);
  a.tiles_n = (int32_t)cdiv(N, Cfg::BN);
  a.raster = 8;
  a.chunk_kb = 16;
  a.C = C;
  a.c_m_off = t_cm;
  a.c_n_off = t_cn;
  a.alpha = (float)alpha;
  a.beta = (float)beta;
  a.status = status;
  a.ksplit = 1;  // no k-split: C written directly
  a.kb_per_split = a.num_kb;
  a.partial = nullptr;
  const int64_t tiles = (int64_t)a.tiles_m * a.tiles_n;
  if (tiles > INT32_MAX) return fail(TCCG_ERR_UNSUPPORTED, "too many tiles");
  const int grid = (int)std::min<int64_t>(tiles, g_noalloc_sms[dev]);
  take_injection(a);
  gett_tc_kernel<TC_BF16X3><<<grid, Cfg::NUM_THREADS, Cfg::SMEM_BYTES, s>>>(tmA, tmB, a);
  return launch_check("gett_tc (allocation-free)");
}

extern "C" int tccg_gett_bf16x3_noalloc_status(int32_t* device_status) {
  if (!device_status) return fail(TCCG_ERR_INVALID, "null argument");
  int dev = -1;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= TCCG_NOALLOC_MAX_DEVICES) return fail(TCCG_ERR_UNSUPPORTED, "device index %d", dev);
  int rc = noalloc_setup(dev);
  if (rc) return rc;
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(device_status, g_noalloc_ptr[dev], sizeof(int32_t), cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemset(g_noalloc_ptr[dev], 0, sizeof(int32_t)));
  CUDA_TRY(cudaDeviceSynchronize());
  return TCCG_OK;
}
