/*
 * tccg_b200 -- C ABI of the B200 tensor-contraction library.
 *
 * Computes  C = alpha * contract(A, B) + beta * C  for dense or strided
 * tensors on one NVIDIA B200 (sm_100a). All pointers are device pointers
 * owned by the caller; every call is stream-ordered on the given stream
 * (a cudaStream_t passed as void*; NULL = legacy default stream).
 *
 * Every function returns 0 on success or a negative TCCG_ERR_* code and never
 * aborts the process; tccg_last_error() returns a thread-local message.
 *
 * Boundary with the reference (HPAC/tccg), which emits one specialised C++
 * function per contraction:
 *
 *   void gett(float* A, float* B, float* C, const float alpha, const float beta)
 *       -- tccg/gett.py:342-344 (the name is `gett` for the fastest candidate,
 *          gett.py:1240-1241; `double` for --floatType=d). Extents and strides
 *          are compile-time constants there; here they are a tccg_desc bound
 *          once into a tccg_plan (tccg_plan_create), which plays the role of
 *          the specialised function, and tccg_plan_run is the call.
 *   int ttgemmt_<cand>(cublasHandle_t, const T* A, const T* B, T* C, T alpha,
 *                      T beta, T* work_)
 *       -- tccg/ttgemmt.py:212-214, 296-300 (returns the workspace size when
 *          work_ == NULL). Replaced by tccg_plan_create with
 *          TCCG_METHOD_TTGT plus tccg_plan_workspace / tccg_plan_run.
 *   int LoG_<...>(cublasHandle_t, const T* A, const T* B, T* C, T alpha, T beta)
 *       -- tccg/gemm_loop.py:94-97. Replaced by TCCG_METHOD_LOG.
 *   hptt::create_plan(perm, dim, alpha, A, size, outerSizeA, beta, B,
 *                     outerSizeB, ...)->execute()
 *       -- the transposition TCCG's TTGT and GETT packing call
 *          (tccg/transpose.py:140-141). Replaced by tccg_transpose.
 *
 * The emitted per-contraction artifact (python -m tccg_b200 file.tccg) wraps
 * a plan behind TCCG's exact `gett(A, B, C, alpha, beta)` signature.
 */
#ifndef TCCG_B200_H
#define TCCG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TCCG_MAX_MODES 12 /* per index class (M, N or K) after index fusion */

/* error codes */
#define TCCG_OK 0
#define TCCG_ERR_INVALID (-1)      /* bad argument or descriptor */
#define TCCG_ERR_UNSUPPORTED (-2)  /* valid request this build cannot run */
#define TCCG_ERR_WORKSPACE (-3)    /* workspace missing or too small */
#define TCCG_ERR_CUDA (-4)         /* a CUDA runtime call failed */
#define TCCG_ERR_ALIGNMENT (-5)    /* pointer alignment requirement not met */
#define TCCG_ERR_DEVICE (-6)       /* a kernel reported an error (e.g. a bounded wait ran out) */

/* operand element types */
#define TCCG_F32 0
#define TCCG_F64 1
#define TCCG_BF16 2

/* arithmetic of the contraction */
#define TCCG_PREC_FP32 0   /* FP32 FFMA on the CUDA cores */
#define TCCG_PREC_FP64 1   /* FP64 DFMA; k-split partial sums and alpha/beta in FP64 */
#define TCCG_PREC_BF16 2   /* BF16 products on tcgen05 tensor cores, FP32 accumulation in TMEM */
#define TCCG_PREC_BF16X3 3 /* split-BF16x3: a*b ~ ah*bh + ah*bl + al*bh on tcgen05, FP32 accumulation */

/* method (TCCG's three code styles, tccg/tccg.py:121-130) */
#define TCCG_METHOD_GETT 0
#define TCCG_METHOD_TTGT 1
#define TCCG_METHOD_LOG 2

/*
 * A contraction in GETT form (TCCG's classification, tccg/tccg_util.py:212-296,
 * 597-611): M = indices of C that are in the operand holding C's stride-one
 * index ("GA"), N = indices of C in the other operand ("GB"), K = contracted
 * indices. Strides are in elements; the M, N and K modes are listed in the
 * linearisation order the kernels use (first = fastest). swap_ab != 0 says
 * that GA is the caller's B: tccg_plan_run then reads its B argument as GA
 * (the operand swap of tccg/gett.py:70-76), so callers always pass (A, B) in
 * file order.
 */
typedef struct tccg_desc {
  int32_t nm, nn, nk;
  int32_t swap_ab;
  int64_t m_ext[TCCG_MAX_MODES];
  int64_t n_ext[TCCG_MAX_MODES];
  int64_t k_ext[TCCG_MAX_MODES];
  int64_t a_m_stride[TCCG_MAX_MODES]; /* GA stride of each M mode */
  int64_t a_k_stride[TCCG_MAX_MODES]; /* GA stride of each K mode */
  int64_t b_n_stride[TCCG_MAX_MODES]; /* GB stride of each N mode */
  int64_t b_k_stride[TCCG_MAX_MODES]; /* GB stride of each K mode */
  int64_t c_m_stride[TCCG_MAX_MODES]; /* C stride of each M mode */
  int64_t c_n_stride[TCCG_MAX_MODES]; /* C stride of each N mode */
} tccg_desc;

/* Kernel choices the autotuner searches over; zero-initialised = defaults. */
typedef struct tccg_tuning {
  int32_t method;      /* TCCG_METHOD_* */
  int32_t variant;     /* BF16/BF16X3 kernel family: 0 = chosen by a bandwidth/compute model,
                          > 0 = tensor cores (BF16X3: k-blocks of 32 per TMEM accumulation
                          chunk, default 16), < 0 = CUDA cores (operands rounded to bf16 for
                          BF16, FP32 FFMA) */
  int32_t ksplit;      /* k-split factor: 0 = automatic (split K over CTAs when the C tiles
                          cannot fill the GPU), 1 = none, > 1 = that many slices
                          (the CTA-pair kernel never splits) */
  int32_t raster;      /* tile order of the persistent tcgen05 kernel (TCCG's two loop orders,
                          tccg/gett.py:52-55): > 0 = groups of that many tile rows, m fastest;
                          < 0 = groups of -raster tile columns, n fastest; 0 = default (8) */
  int32_t max_ctas;    /* persistent grid size cap (0 = one CTA per SM) */
  int32_t pair;        /* tensor-core precisions: 1 = CTA-pair kernel (cta_group::2, 256-row tiles) */
  int32_t direct;      /* CUDA-core kernels: 0 = automatic (no packing pass when K <= 256 and the
                          operand loads stay coalesced), 1 = always, -1 = never (GETT only) */
  int32_t shortk;      /* CUDA-core kernels, K <= 32 (FP64: 16): the kernel that prefetches each
                          tile's C block under its FMA phase. 0 = automatic (C a 2-D matrix
                          moved by TMA, at least two tiles per SM), 1 = always, -1 = never */
  int32_t simt_tile;   /* CUDA-core tile shape, FP32 accumulation: 0 = the least padded work
                          (narrow tiles counted at 1.6x), 1 = 128x128, 2 = 128x32 (small N),
                          3 = 32x128 (small M); FP64 always 128x64 */
  int32_t tail_split;  /* tcgen05, automatic k-split: 0 = run the tiles of a short last round of
                          the persistent grid as k slices where that pays, -1 = never (grouped
                          runs never split that way) */
  int32_t load;        /* tcgen05 BF16X3 with FP32 operands: 0 = chosen by the model, 1 = packing
                          pass + TMA loads (128x192 tiles), 2 = gather: producer warps read the
                          caller's tensors through the offset tables and split them into the
                          swizzled bf16 stages themselves (128x128 tiles, no packing pass) */
  int32_t tile_n;      /* tcgen05 tile width (columns of C per tile): 0 = the loader's default
                          (BF16 256, BF16X3 192, gather 128); 128, 192 or 256 (BF16), 128 or
                          192 (BF16X3 with the packing pass) */
  int32_t skinny;      /* FP32 operands, FP32 or BF16X3 precision, GETT, min(M, N) <= 256,
                          tensors of fewer than 2^31 elements: the skinny kernel -- chunks of
                          the narrow operand in shared memory, the wide one streamed once in
                          place, C written once. 0 = chosen by the model, 1 = always (an
                          error where it does not apply), -1 = never; 2 = its tensor-core
                          form (BF16X3, K <= 2^29, passes of 64 rows: the wide operand split
                          into bf16 hi / lo on the fly, tcgen05 MMAs; 0 picks it for K > 32
                          and at least 48 blocks of positions) */
} tccg_tuning;

typedef struct tccg_plan tccg_plan; /* opaque */

/* Library version string and the build's target ("sm_100a"). */
const char* tccg_version(void);

/* Thread-local message of the last failing call on this thread. */
const char* tccg_last_error(void);

/*
 * Bind a contraction to a plan: validates the descriptor, builds the offset
 * tables (uploaded to the current device) and picks kernels.
 * dtype: element type of A and B (TCCG_F32, TCCG_BF16 or TCCG_F64); C is
 * float for TCCG_F32/TCCG_BF16 and double for TCCG_F64. tuning may be NULL.
 */
int tccg_plan_create(const tccg_desc* desc, int32_t dtype, int32_t precision,
                     const tccg_tuning* tuning, tccg_plan** out);

/* Bytes of device workspace tccg_plan_run needs (ws_bytes >= this). */
int tccg_plan_workspace(const tccg_plan* plan, size_t* bytes);

/*
 * C = alpha * contract(A, B) + beta * C on `stream`. A and B are in the
 * caller's (file) order; ws must be 256-byte aligned when ws_bytes > 0.
 * With beta == 0, C is written without being read (as TCCG's update=0 path).
 * The kernels after the first one use programmatic dependent launch (they
 * start while the kernel before them drains) on the CUDA cores, and on the
 * tensor cores when the persistent grid runs at most four rounds of tiles;
 * TCCG_B200_PDL=1 or =0 in the environment forces it on or off.
 */
int tccg_plan_run(const tccg_plan* plan, const void* A, const void* B, void* C, double alpha,
                  double beta, void* ws, size_t ws_bytes, void* stream);

/*
 * tccg_plan_run with CUDA-event timing of each kernel it launches, for
 * benchmarks and the autotuner: kernel_ms[0] = operand packing,
 * kernel_ms[1] = the GEMM kernel (SIMT or tcgen05), kernel_ms[2] = k-split
 * reduction or TTGT output transposition (0 if none). Synchronises `stream`.
 */
int tccg_plan_run_timed(const tccg_plan* plan, const void* A, const void* B, void* C,
                        double alpha, double beta, void* ws, size_t ws_bytes, void* stream,
                        float* kernel_ms);

/*
 * tccg_plan_run that records caller-created CUDA events around each kernel it
 * launches, without synchronising: events[2*i] / events[2*i+1] bracket kernel
 * slot i (0 = operand packing, 1 = the GEMM kernel, 2 = k-split reduction or
 * TTGT output transposition; all six are recorded first, so a slot without a
 * kernel measures 0 ms). For timing every kernel of a run inside a loop of
 * runs; the kernels are launched as by tccg_plan_run_timed (never with
 * programmatic dependent launch).
 */
int tccg_plan_run_events(const tccg_plan* plan, const void* A, const void* B, void* C,
                         double alpha, double beta, void* ws, size_t ws_bytes, void* stream,
                         void* const* events);

/* Human-readable plan summary (method, kernels, tiles, launch=dependent|plain
 * for programmatic dependent launch as the environment now selects it,
 * workspace). */
int tccg_plan_describe(const tccg_plan* plan, char* buf, size_t len);

/* FLOPs of one run by TCCG's count (tccg/tccg.py:1230-1234): 2MNK (+3MN if beta != 0). */
double tccg_plan_flops(const tccg_plan* plan, double beta);

int tccg_plan_destroy(tccg_plan* plan);

/*
 * Device-side status of the plan's kernels since the last call: 0, or the
 * TCCG_DEVSTAT_* code a kernel recorded (a bounded wait that ran out, ...).
 * Synchronises the device, reads and clears the word.
 */
#define TCCG_DEVSTAT_TIMEOUT_PRODUCER 1
#define TCCG_DEVSTAT_TIMEOUT_MMA 2
#define TCCG_DEVSTAT_TIMEOUT_EPILOGUE 3
int tccg_plan_status(const tccg_plan* plan, int32_t* device_status);

/*
 * Allocation-free split-BF16x3 GETT. This entry point has no counterpart in
 * the reference. It is for callers that must not allocate device memory --
 * a process whose HBM a framework's caching allocator has already reserved,
 * or a latency-critical loop that cannot afford cudaMalloc/cudaFree (which may
 * synchronise the device) -- and it allocates nothing: no plan, no workspace.
 * Its scratch (offset tables, packed operands, status word) is a static
 * 64 MiB device array that every GPU loading the library holds until the
 * process exits; a contraction needing more is rejected with
 * TCCG_ERR_WORKSPACE and a message (use tccg_plan_run then). The first call
 * on each device looks up the array's device address with that device
 * current (and clears the status word); make that first call before any
 * stream capture. All calls share the array (each call rebuilds the tables
 * and packed operands it reads), so calls whose kernels overlap on the GPU --
 * e.g. on two streams -- race; serialise them.
 * A, B, C: device pointers, float, in the caller's (file) order as for
 * tccg_plan_run; desc as for tccg_plan_create.
 */
int tccg_gett_bf16x3_noalloc(const tccg_desc* desc, const float* A, const float* B, float* C,
                             double alpha, double beta, void* stream);

/*
 * Device-side status of the allocation-free entry point on the current
 * device: 0, or the first TCCG_DEVSTAT_* code one of its kernels recorded
 * since the last query (a bounded wait that ran out means C is incomplete).
 * The word lives in the same static scratch array; calls do not clear it, so
 * a code stays until this query. Synchronises the device, reads and clears
 * the word. No counterpart in the reference (its calls return void).
 */
int tccg_gett_bf16x3_noalloc_status(int32_t* device_status);

/*
 * Testing of the bounded device waits (no counterpart in the reference).
 * Arms a one-shot trigger on the calling host thread: the next tcgen05 GETT
 * launch this thread makes (tccg_plan_run of a tensor-core plan without the
 * CTA-pair kernel, or tccg_gett_bf16x3_noalloc) bounds every device wait by
 * wait_ms instead of 4 s, and its producer does not load the first k-block of
 * tile `tile` of the tile order. The MMA warp's wait for that block runs out,
 * the CTA that owns the tile records TCCG_DEVSTAT_TIMEOUT_* and winds down
 * (in-flight copies and MMAs are waited for, tensor memory is released), and
 * the launch leaves that CTA's tiles of C unwritten. Nothing faults and no
 * wait is unbounded; tccg_plan_status / tccg_gett_bf16x3_noalloc_status then
 * report the code. tile >= 0 (a tile past the last one skips nothing),
 * wait_ms in [1, 4000].
 */
int tccg_debug_inject_timeout(int32_t tile, int32_t wait_ms);

/*
 * HPTT-style out-of-place transposition (the call TCCG emits at
 * tccg/transpose.py:140-141):  B[perm(i)] = alpha * A[i] + beta * B[perm(i)],
 * where dimension j of B is dimension perm[j] of A. size[] are A's extents,
 * outer_a / outer_b the padded extents (NULL = dense). beta == 0 does not read B.
 */
int tccg_transpose(int32_t dtype, int32_t dim, const int32_t* perm, const int64_t* size,
                   const int64_t* outer_a, const int64_t* outer_b, double alpha, const void* A,
                   double beta, void* B, void* stream);

/*
 * Grouped launch: many plans of the same precision run by a few launches per
 * wave (waves of at most 4 GiB of workspace): grouped packing, one grouped
 * GETT kernel per kernel family (CUDA-core tiles, tcgen05 tiles, the skinny
 * kernels) and the grouped k-split reductions, each only when it has work.
 * The tensor-core lanes run on the given stream, the CUDA-core skinny lanes
 * and the CUDA-core tiles on two side streams of the group forked from it and
 * joined back before the reductions. tccg_group_bind fixes the operand
 * pointers and workspace (it uploads the work lists, synchronously, and
 * creates the side streams), after which tccg_group_run only launches kernels
 * and can be captured in a CUDA graph. Groups run a plan's tcgen05 tiles
 * without its tail split (tuning.tail_split); plans made with tail_split = -1
 * give the same sums in a group as alone.
 */
typedef struct tccg_group tccg_group; /* opaque */
int tccg_group_create(const tccg_plan* const* plans, int32_t count, tccg_group** out);
int tccg_group_workspace(const tccg_group* group, size_t* bytes);
int tccg_group_bind(tccg_group* group, const void* const* A, const void* const* B,
                    void* const* C, const double* alpha, const double* beta, void* ws,
                    size_t ws_bytes);
int tccg_group_run(const tccg_group* group, void* stream);
int tccg_group_destroy(tccg_group* group);

#ifdef __cplusplus
}
#endif

#endif /* TCCG_B200_H */
