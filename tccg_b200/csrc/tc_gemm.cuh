// tcgen05 GETT kernel (sm_100a): BF16 and split-BF16x3 products on the 5th
// generation tensor cores with FP32 accumulation in tensor memory.
//
// Operands arrive packed K-major by pack_kernel: GA as [M][Kc] and GB as
// [N][Kc] bf16 rows. In BF16 mode a 128-byte row chunk holds 64 consecutive k;
// in BF16X3 mode it holds [hi(k..k+31) | lo(k..k+31)], so both modes load the
// same TMA boxes (64 x 128 rows for GA, 64 x 256 rows for GB, 128-byte
// swizzle) and only the MMA schedule differs:
//   BF16  : 4 MMAs (k-steps of 16) per stage
//   BF16X3: per k-step of 16, D += ah*bh, D += ah*bl, D += al*bh
// (al*bl, ~2^-16 relative, is dropped).
//
// Accumulation in chunks of K: the tensor cores add each MMA's result into the
// FP32 accumulator with truncation, so a long sum in one accumulator drifts
// (normwise ~1.5e-5 at K = 4096 on N(0,1) data). The MMA warp therefore
// accumulates each chunk of `chunk_kb` k-blocks (512 k by default in BF16X3
// mode) into a fresh TMEM accumulator, and the epilogue adds the chunk sums in
// registers with IEEE round-to-nearest FP32 adds (~5e-6 at K = 4096). The two
// 256-column accumulators ping-pong between chunks (and tiles), so the MMAs of
// one chunk overlap the epilogue's read of the previous one. BF16 mode uses
// one chunk per tile.
//
// Structure: one persistent CTA per SM, 10 warps.
//   warp 0     TMA producer (one lane): STAGES-deep smem ring, mbarrier full/empty
//   warp 1     TMEM owner + MMA issuer (one lane): 128x256 UMMA tiles into one of
//              two 256-column FP32 accumulators (double buffering)
//   warps 2-9  epilogue: warp w reads TMEM lane quadrant w%4, columns
//              [128*h, 128*h+128) with h = (w-2)/4, sums the chunks, then writes
//              C[c_m_off[m] + c_n_off[n]] = alpha*acc (+ beta*C) straight into
//              C's own layout (GETT: no transposition of C).
// With a k-split (contractions whose C tiles cannot fill the GPU), tile
// indices run over (split, tile) and each split's epilogue writes raw sums to
// a workspace slice; simt_reduce_kernel adds the slices in split order.
// Every mbarrier wait is bounded (TcArgs::wait_ns, by default
// TCCG_DEVICE_WAIT_NS = 4 s); a wait that runs out records an error code in
// *status and the CTA winds down: in-flight TMA loads and MMAs are waited for
// (bounded) and TMEM is released before returning.
#pragma once
#include <cuda.h>
#include "common.cuh"

namespace tccg {

enum TcMode : int { TC_BF16 = 0, TC_BF16X3 = 1 };

// How the operand stages are filled.
//   TC_LOAD_TMA   : one thread issues 2-D TMA loads of operands packed K-major
//                   by pack_kernel (a separate pass through HBM before the GETT).
//   TC_LOAD_GATHER: four producer warps gather FP32 elements straight from the
//                   caller's tensors through the offset tables (cp.async into
//                   an FP32 staging ring), split them into bf16 hi/lo and write
//                   the same 128-byte-swizzled K-major stage TMA would deliver
//                   -- no packing pass, each operand element crosses HBM once
//                   per tile that reads it. BF16X3 only.
enum TcLoad : int { TC_LOAD_TMA = 0, TC_LOAD_GATHER = 1 };

// Gather read schedule of one operand (chosen at plan creation).
enum GatherRead : int {
  GATHER_ROWS = 0,   // lanes along rows, 4-byte copies (rows have the smallest stride)
  GATHER_K = 1,      // lanes along k, 4-byte copies
  GATHER_KQUAD = 2,  // lanes along k, 16-byte copies of 4 consecutive, aligned k
};

// Tile configuration per mode. BF16X3 uses 128x192 tiles so that each of the 8
// epilogue warps keeps its 96-column running chunk sum in registers (a 10-warp
// CTA has at most 168 registers per thread: 3 warps share one SM sub-partition).
// The gather variant has 13 warps (4 producers, the MMA warp, 8 epilogue
// warps: at most 152 registers each), so its tiles are 128x128 (64 running
// sums per epilogue warp).
//
// BNV != 0 sets the tile width of the TMA loader (a blocking the autotuner
// searches: 128, 192 or 256 columns for BF16, 128 or 192 for BF16X3); the
// operand ring then has as many stages as fit in shared memory (at most 6).
template <int MODE, int LOAD = TC_LOAD_TMA, int BNV = 0>
struct TcCfgT {
  static constexpr bool GATHER = LOAD == TC_LOAD_GATHER;
  static_assert(!GATHER || MODE == TC_BF16X3, "the gather loader serves split-BF16x3");
  static_assert(!GATHER || BNV == 0 || BNV == 128, "the gather loader has 128-column tiles");
  static_assert(BNV == 0 || BNV == 128 || BNV == 192 || (BNV == 256 && MODE == TC_BF16),
                "tile widths: 128, 192 (and 256 for BF16)");
  static constexpr int BM = 128;
  static constexpr int BN = BNV ? BNV : GATHER ? 128 : (MODE == TC_BF16X3) ? 192 : 256;
  static constexpr int ROW_BYTES = 128;  // one swizzle row per operand row per stage
  static constexpr int A_STAGE = BM * ROW_BYTES;   // 16 KB
  static constexpr int B_STAGE = BN * ROW_BYTES;   // 16 / 24 / 32 KB
  static constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
  // default shapes keep their measured ring depths (BF16X3 5 x 40 KB, BF16
  // 4 x 48 KB); other widths take what fits next to the epilogue staging
  static constexpr int STAGES = GATHER ? 2
                                : BNV == 0 ? ((MODE == TC_BF16X3) ? 5 : 4)
                                : (200 * 1024 / STAGE_BYTES > 6 ? 6 : 200 * 1024 / STAGE_BYTES);
  static constexpr int ACC_STRIDE = BN <= 128 ? 128 : 256;  // accumulator b starts at column ACC_STRIDE*b
  static constexpr int TMEM_COLS = 2 * ACC_STRIDE;       // two accumulators of BN columns
  static constexpr int PRODUCER_WARPS = GATHER ? 4 : 1;
  static constexpr int MMA_WARP = PRODUCER_WARPS;
  static constexpr int EPI_WARP0 = PRODUCER_WARPS + 1;
  static constexpr int EPI_WARPS = 8;
  static constexpr int NUM_THREADS = 32 * (PRODUCER_WARPS + 1 + EPI_WARPS);
  // gather: FP32 staging ring of STG_SLOTS k-blocks (copies run STG_SLOTS - 1
  // k-blocks ahead of the conversion); a staging row holds the 32 source
  // elements of one operand row, 36 floats apart (16-byte copies stay
  // aligned, conversion reads are bank-conflict free) or 33 (4-byte copies
  // along rows are bank-conflict free)
  static constexpr int KB_ELEMS = 32;
  static constexpr int STG_LD = 36;
  static constexpr int STG_SLOTS = GATHER ? 3 : 0;
  static constexpr int STG_SLOT_BYTES = (BM + BN) * STG_LD * 4;
  static constexpr int ROWCACHE_BYTES = GATHER ? (BM + BN) * 8 : 0;
  // staged C stores (TcArgs::crun): 32 rows x 16 columns per epilogue warp
  static constexpr int EPI_LD = 33;
  static constexpr int EPI_STG_BYTES = EPI_WARPS * 16 * EPI_LD * 4;
  static constexpr size_t SMEM_BYTES = 1024 + (size_t)STAGES * STAGE_BYTES +
                                       (size_t)STG_SLOTS * STG_SLOT_BYTES + ROWCACHE_BYTES +
                                       EPI_STG_BYTES + 256;
};

struct TcArgs {
  int32_t M, N, K;
  int32_t num_kb;           // 128-byte k-chunks per row: BF16 ceil(K/64), BF16X3 ceil(K/32)
  int32_t tiles_m, tiles_n;
  int32_t raster;           // tiles along m per raster group
  int32_t chunk_kb;         // k-blocks accumulated per TMEM accumulator (>= 1)
  float* C;
  const int64_t* c_m_off;
  const int64_t* c_n_off;
  float alpha, beta;
  int32_t* status;
  // k-split: the tiles of split z cover k-blocks [z*kb_per_split, ...) and
  // write raw FP32 sums to partial[z][n][M]; a reduction kernel applies
  // alpha/beta. ksplit == 1 writes C directly.
  int32_t ksplit, kb_per_split;
  float* partial;
  // Tail split (ksplit == 1, tail_split > 1): tiles [0, full_tiles) of the
  // tile order run over all of K; each of the remaining tail = tiles -
  // full_tiles tiles runs as tail_split slices of tail_kb k-blocks (tile index
  // full_tiles + z * tail + t) that write raw sums to
  // tail_partial[((z * tail + t) * BN + n_local) * 128 + m_local];
  // tc_tail_reduce_kernel adds the slices and applies alpha/beta. It fills the
  // last round of the persistent grid instead of leaving it mostly idle.
  int32_t full_tiles, tail_split, tail_kb;
  float* tail_partial;
  // Bound of every mbarrier wait of the launch (0 = TCCG_DEVICE_WAIT_NS).
  uint64_t wait_ns;
  // Position of a CTA in the tile order: 0 = its launch index (blockIdx.x);
  // 1 = the SM it runs on (%smid), when the grid has one CTA per SM id
  // (%nsmid == gridDim.x, so the ids are exactly 0 .. grid-1). With the SM
  // order, consecutive tiles -- which share operand rows -- run on
  // consecutive SMs whatever order the CTAs were launched in (programmatic
  // dependent launch places them as the previous kernel frees SMs).
  int32_t sm_order;
  // Testing of the abort path (0 = off): the producer does not load the
  // first k-block of tile skip_tile1 - 1, so the MMA warp's wait for it runs
  // out and the CTA winds down with a status code.
  int32_t skip_tile1;
  // TC_LOAD_GATHER: operand o (0 = GA, rows m; 1 = GB, rows n) element (r, k)
  // is gsrc[o][grow[o][r] + gk[o][k]] (FP32), read with schedule gread[o]
  const float* gsrc[2];
  const int64_t* grow[2];
  const int64_t* gk[2];
  int32_t gread[2];
  // C layout: 0 = the epilogue's lanes store along m (C's stride-one run
  // along m is >= 32 elements, or partial sums); e0 in [2, 31] = C's
  // stride-one index is the first M mode, of extent e0, directly followed in
  // C by the first N mode: stores go through shared memory in runs of e0 m
  // by 32 / e0 columns, which are consecutive addresses of C
  int32_t crun;
};

// Grouped launch: one entry per contraction, in device memory. The tensor maps
// live here (64-byte aligned) and are read by TMA from global memory.
struct __align__(64) TcGroupItem {
  CUtensorMap tmA;
  CUtensorMap tmB;
  TcArgs args;
  int64_t tile_begin;  // first global tile of this item
};

struct TcGroup {
  const TcGroupItem* items;
  const int64_t* tile_begin;  // items[i].tile_begin, compact, for the tile search
  int32_t n_items;
  int32_t total_tiles;
};

// Tile order of the persistent grid (TCCG's two GEMM loop orders,
// tccg/gett.py:52-55): raster > 0 walks groups of `raster` tile rows (m),
// m fastest inside a group and the group's columns after each other -- the
// group's A rows stay in L2 while B streams (matrix-panel); raster < 0 walks
// groups of -raster tile columns (n), n fastest -- B's rows stay (panel-matrix).
__device__ __forceinline__ void tile_coords(int tile, const TcArgs& a, int& tm, int& tn) {
  if (a.raster < 0) {
    const int R = -a.raster;
    const int group = R * a.tiles_m;
    const int gid = tile / group;
    const int first_n = gid * R;
    int gn = a.tiles_n - first_n;
    if (gn > R) gn = R;
    const int r = tile - gid * group;
    tn = first_n + r % gn;
    tm = r / gn;
    return;
  }
  const int group = a.raster * a.tiles_n;
  const int gid = tile / group;
  const int first_m = gid * a.raster;
  int gm = a.tiles_m - first_m;
  if (gm > a.raster) gm = a.raster;
  const int r = tile - gid * group;
  tm = first_m + r % gm;
  tn = r / gm;
}

// Resolves a global tile index to (item arguments, tensor maps, tile coords,
// k-split slice). Splits are the outermost tile dimension.
struct TileRef {
  const TcArgs* a;
  const CUtensorMap* tA;
  const CUtensorMap* tB;
  int tm, tn;
  int z, kb_begin, kb_end;
  int tail;  // index among the tail tiles (a slice of it), or -1
};

__device__ __forceinline__ void split_coords(int local, const TcArgs& a, TileRef& r) {
  const int mn = a.tiles_m * a.tiles_n;
  r.tail = -1;
  if (a.tail_split > 1 && local >= a.full_tiles) {
    const int tail = mn - a.full_tiles, u = local - a.full_tiles;
    r.z = u / tail;
    r.tail = u - r.z * tail;
    tile_coords(a.full_tiles + r.tail, a, r.tm, r.tn);
    r.kb_begin = r.z * a.tail_kb;
    r.kb_end = r.kb_begin + a.tail_kb < a.num_kb ? r.kb_begin + a.tail_kb : a.num_kb;
    return;
  }
  r.z = local / mn;
  tile_coords(local - r.z * mn, a, r.tm, r.tn);
  r.kb_begin = r.z * a.kb_per_split;
  r.kb_end = r.kb_begin + a.kb_per_split < a.num_kb ? r.kb_begin + a.kb_per_split : a.num_kb;
}

template <bool GROUPED>
__device__ __forceinline__ TileRef resolve_tile(int tile, const CUtensorMap* tmA,
                                                const CUtensorMap* tmB, const TcArgs* a1,
                                                const TcGroup& g) {
  TileRef r;
  if constexpr (GROUPED) {
    const TcGroupItem& it = g.items[find_segment(g.tile_begin, g.n_items, tile)];
    r.a = &it.args;
    r.tA = &it.tmA;
    r.tB = &it.tmB;
    split_coords(tile - (int)it.tile_begin, it.args, r);
  } else {
    r.a = a1;
    r.tA = tmA;
    r.tB = tmB;
    split_coords(tile, *a1, r);
  }
  return r;
}

// Staged C store of one epilogue warp (TcArgs::crun = e0): stg holds the
// warp's 32 rows (m0 ...) x ncols <= 16 columns as [column][row], 33 floats
// per column; cm_lane / cn_lane are C's offsets of row m0 + lane and of
// column lane (lane < ncols) of the block, passed around by warp shuffles (no
// memory access on the store path). For each run of e0 consecutive m
// (clipped to the warp's rows and to M, length L) the block of L x ncols
// elements is stored in C's address order, element f = i + L * j (row ma +
// i, column j) by lane f % 32: a store instruction covers 32 consecutive
// positions of the block -- one contiguous stretch of C for a whole run.
// Every lane runs the same number of steps (the shuffles need the whole
// warp), stepping (i, j) by 32 positions without dividing. Same arithmetic
// as the register epilogue (alpha * acc, fmaf with beta).
__device__ __forceinline__ void store_runs(const float* stg, const TcArgs& a, int64_t m0,
                                           int ncols, int e0, float alpha, float beta, int lane,
                                           int64_t cm_lane, int64_t cn_lane) {
  // fields read once: in a grouped launch a is the item in global memory,
  // which the compiler must otherwise read again after every store
  float* const Cb = a.C;
  int64_t mlim = a.M - m0;  // rows of this warp inside M
  if (mlim > 32) mlim = 32;
#pragma unroll 1
  for (int rs = (int)((m0 / e0) * e0 - m0); rs < (int)mlim; rs += e0) {  // run starts, warp-relative
    const int ma = rs > 0 ? rs : 0;
    const int mb = rs + e0 < (int)mlim ? rs + e0 : (int)mlim;
    const int L = mb - ma;
    if (L <= 0) continue;  // warp-uniform
    const int total = L * ncols;
    int i = lane % L, j = lane / L;
    const int di = 32 % L, dj = 32 / L;
#pragma unroll 2
    for (int f0 = 0; f0 < total; f0 += 32) {
      const int64_t cm = __shfl_sync(0xffffffffu, cm_lane, (ma + i) & 31);
      const int64_t cn = __shfl_sync(0xffffffffu, cn_lane, j & 31);
      if (f0 + lane < total) {
        float* dst = Cb + cm + cn;
        const float v = alpha * stg[j * 33 + ma + i];
        *dst = beta != 0.0f ? fmaf(beta, *dst, v) : v;
      }
      i += di;
      j += dj;
      if (i >= L) {
        i -= L;
        ++j;
      }
    }
  }
}

// ---- gather loader (TC_LOAD_GATHER) ------------------------------------------
// The producer warps walk this CTA's (tile, k-block) jobs in the order the MMA
// warp consumes them, twice: copies run STG_SLOTS - 1 jobs ahead of the
// conversion into MMA stages.
// The fields a job's copies and conversion use are read from the kernel
// arguments once per tile, into registers (the copy loops then touch no
// argument memory).
struct GatherJob {
  int tile, kb;
  bool valid;
  TileRef t;
  int K;
  const float* src[2];
  const int64_t* gk[2];
  int read[2];
  int nr[2];       // rows of the tile inside the operand (0..128)
  int64_t r0[2];   // first row of the tile
};

template <int BM, int BN, bool GROUPED>
__device__ __forceinline__ void gjob_seek(GatherJob& j, int num_tiles, const TcArgs* a1,
                                          const TcGroup& g) {
  while (j.tile < num_tiles) {
    j.t = resolve_tile<GROUPED>(j.tile, nullptr, nullptr, a1, g);
    if (j.t.kb_begin < j.t.kb_end) {
      const TcArgs& a = *j.t.a;
      j.kb = j.t.kb_begin;
      j.valid = true;
      j.K = a.K;
#pragma unroll
      for (int o = 0; o < 2; ++o) {
        j.src[o] = a.gsrc[o];
        j.gk[o] = a.gk[o];
        j.read[o] = a.gread[o];
        const int64_t R = o ? a.N : a.M;
        j.r0[o] = o ? (int64_t)j.t.tn * BN : (int64_t)j.t.tm * BM;
        const int rows = o ? BN : BM;
        j.nr[o] = R - j.r0[o] < rows ? (int)(R - j.r0[o]) : rows;
      }
      return;
    }
    j.tile += gridDim.x;
  }
  j.valid = false;
}

template <int BM, int BN, bool GROUPED>
__device__ __forceinline__ void gjob_next(GatherJob& j, int num_tiles, const TcArgs* a1,
                                          const TcGroup& g) {
  if (++j.kb < j.t.kb_end) return;
  j.tile += gridDim.x;
  gjob_seek<BM, BN, GROUPED>(j, num_tiles, a1, g);
}

// Staging row stride of an operand (floats): 33 for copies along rows (the 32
// lanes' 4-byte writes land in 32 banks), 36 for copies along k (16-byte
// aligned rows; the conversion reads 8 rows x 32 bytes per phase conflict free).
__device__ __forceinline__ int gather_ld(int read) { return read == GATHER_ROWS ? 33 : 36; }

// Producer barrier over the 128 producer threads (named barrier 1) that also
// ANDs a flag across them, so that every producer takes the same branch.
__device__ __forceinline__ bool producers_and(bool v) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, 1, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)v)
      : "memory");
  return out != 0;
}

// Row offsets of the job's tile (A rows then B rows) into the shared cache.
template <int BM, int BN>
__device__ __forceinline__ void gather_rows(const GatherJob& j, int64_t* rowc, int ptid) {
  const TcArgs& a = *j.t.a;
  for (int r = ptid; r < BM + BN; r += 128) {
    const int o = r >= BM;
    const int64_t row = o ? (int64_t)j.t.tn * BN + (r - BM) : (int64_t)j.t.tm * BM + r;
    const int64_t R = o ? a.N : a.M;
    rowc[r] = row < R ? __ldg(a.grow[o] + row) : 0;
  }
}

// Asynchronous copies of one job's source elements into a staging slot:
// operand o's element (r, k) of the k-block goes to slot_o[r * ld + k]. The
// k-block's 32 k offsets are loaded once per lane and broadcast with warp
// shuffles, row offsets come from the shared cache; the copy loops are
// unrolled so that many copies of a thread are in flight at once.
template <int BM, int BN>
__device__ __forceinline__ void gather_issue(const GatherJob& j, float* slot, const int64_t* rowc,
                                             int ptid) {
  static_assert(BM == 128 && BN == 128, "one row per producer thread along rows");
  const int pw = ptid >> 5, lane = ptid & 31;
  const int k0 = j.kb * 32;
  const int kn = j.K - k0 < 32 ? j.K - k0 : 32;  // k of this block inside K
#pragma unroll
  for (int o = 0; o < 2; ++o) {
    const float* src = j.src[o];
    const int nr = j.nr[o];
    const int64_t* rc = rowc + (o ? BM : 0);
    const int read = j.read[o];
    const int ld = gather_ld(read);
    float* dst = slot + (o ? BM * 36 : 0);
    // k offset of k = lane (0 past K)
    const int64_t ko_lane = lane < kn ? __ldg(j.gk[o] + k0 + lane) : 0;
    if (read == GATHER_ROWS) {
      // lanes along rows: thread ptid copies row ptid (every tile has <= 128 rows)
      const int r = ptid;
      const bool ok = r < nr;
      const float* srow = src + (ok ? rc[r] : 0);
      float* drow = dst + r * ld;
#pragma unroll 8
      for (int k = 0; k < 32; ++k) {
        const int64_t ko = __shfl_sync(0xffffffffu, ko_lane, k);
        if (ok && k < kn) cp_async_elem<4>(drow + k, srow + ko);
      }
    } else if (read == GATHER_K) {
      if (lane < kn) {
#pragma unroll 8
        for (int r = pw; r < nr; r += 4) cp_async_elem<4>(dst + r * ld + lane, src + rc[r] + ko_lane);
      }
    } else {  // GATHER_KQUAD: lane -> (row sub = lane / 8, quad = lane % 8)
      const int kq = 4 * (lane & 7), sub = lane >> 3;
      int64_t koq[4];  // offsets of the quad's 4 k (every lane shuffles, before any branch)
#pragma unroll
      for (int e = 0; e < 4; ++e) koq[e] = __shfl_sync(0xffffffffu, ko_lane, kq + e);
      if (kq + 3 < kn) {
#pragma unroll 8
        for (int r = pw * 4 + sub; r < nr; r += 16) cp_async_16(dst + r * ld + kq, src + rc[r] + koq[0]);
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (kq + e < kn)
            for (int r = pw * 4 + sub; r < nr; r += 16)
              cp_async_elem<4>(dst + r * ld + kq + e, src + rc[r] + koq[e]);
      }
    }
  }
}

// Converts one job's staging slot into an MMA stage: element (r, k) becomes
// hi = bf16(x), lo = bf16(x - hi) in the K-major [hi(32 k) | lo(32 k)] row r,
// 16-byte chunk c stored at chunk c ^ (r & 7) (the 128-byte swizzle TMA
// applies); rows past the operand and k past K are zero, as TMA's
// out-of-bounds fill and the packing pass leave them.
template <int BM, int BN>
__device__ __forceinline__ void gather_convert(const GatherJob& j, const float* slot, uint8_t* stA,
                                               uint8_t* stB, int ptid) {
  static_assert(BM == 128 && BN == 128, "the conversion walks 16 groups of 8 rows per operand");
  const int pw = ptid >> 5, lane = ptid & 31;
  const int k0 = j.kb * 32;
  const int kn = j.K - k0 < 32 ? j.K - k0 : 32;
  const int k8 = lane >> 3;
#pragma unroll
  for (int o = 0; o < 2; ++o) {
    const int ld = gather_ld(j.read[o]);
    const int nr = j.nr[o];
    const float* sop = slot + (o ? BM * 36 : 0);
    uint8_t* stage = o ? stB : stA;
    constexpr int GROUPS = 16;  // 8-row groups per operand (128 rows)
#pragma unroll 1
    for (int rg = pw; rg < GROUPS; rg += 4) {
      const int rr = rg * 8 + (lane & 7);
      const bool row_ok = rr < nr;
      const float* srow = sop + rr * ld + k8 * 8;
      float v[8];
      if (ld == 36) {
        const float4 x0 = *reinterpret_cast<const float4*>(srow);
        const float4 x1 = *reinterpret_cast<const float4*>(srow + 4);
        v[0] = x0.x; v[1] = x0.y; v[2] = x0.z; v[3] = x0.w;
        v[4] = x1.x; v[5] = x1.y; v[6] = x1.z; v[7] = x1.w;
      } else {
#pragma unroll
        for (int e = 0; e < 8; ++e) v[e] = srow[e];
      }
      uint32_t hw[4], lw[4];
#pragma unroll
      for (int e = 0; e < 8; e += 2) {
        const float x0 = (row_ok && k8 * 8 + e < kn) ? v[e] : 0.0f;
        const float x1 = (row_ok && k8 * 8 + e + 1 < kn) ? v[e + 1] : 0.0f;
        split_bf16x2(x0, x1, hw[e / 2], lw[e / 2]);
      }
      uint8_t* drow = stage + rr * 128;
      const int sw = rr & 7;
      *reinterpret_cast<uint4*>(drow + ((k8 ^ sw) << 4)) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
      *reinterpret_cast<uint4*>(drow + (((4 + k8) ^ sw) << 4)) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
  }
}

// The four producer warps of the gather variant.
template <int MODE, bool GROUPED>
__device__ __forceinline__ void gather_producer(const TcArgs* a1, const TcGroup& g, int num_tiles,
                                                int cta, uint8_t* sA, uint8_t* sB, float* stg,
                                                int64_t* rowc, uint64_t* full, uint64_t* empty,
                                                uint64_t wait_ns, int skip_tile1,
                                                int32_t* status) {
  using Cfg = TcCfgT<MODE, TC_LOAD_GATHER>;
  constexpr int S = Cfg::STG_SLOTS;
  constexpr int SLOT = Cfg::STG_SLOT_BYTES / 4;  // floats per staging slot
  const int ptid = threadIdx.x;                  // 0..127
  GatherJob ji, jc;                              // issue / conversion iterators
  ji.tile = jc.tile = cta;
  gjob_seek<Cfg::BM, Cfg::BN, GROUPED>(ji, num_tiles, a1, g);
  gjob_seek<Cfg::BM, Cfg::BN, GROUPED>(jc, num_tiles, a1, g);
  int cached = -1;  // tile whose row offsets are in rowc
  auto issue = [&](int slot) {
    if (ji.valid) {
      if (ji.tile != cached) {  // every producer is past its copies of the old tile
        named_barrier_sync(1, 128);
        gather_rows<Cfg::BM, Cfg::BN>(ji, rowc, ptid);
        named_barrier_sync(1, 128);
        cached = ji.tile;
      }
      gather_issue<Cfg::BM, Cfg::BN>(ji, stg + slot * SLOT, rowc, ptid);
      gjob_next<Cfg::BM, Cfg::BN, GROUPED>(ji, num_tiles, a1, g);
    }
    cp_async_commit();  // one group per job (empty past the last), so waits count jobs
  };
  int islot = 0;
  for (int d = 0; d < S - 1; ++d) {
    issue(islot);
    islot = islot + 1 == S ? 0 : islot + 1;
  }
  int stage = 0, cslot = 0;
  uint32_t phase = 0;
  while (jc.valid) {
    const bool free_stage = mbar_wait(&empty[stage], phase ^ 1, wait_ns);
    cp_async_wait<S - 2>();  // this thread's copies of job jc landed
    // all producers' copies of jc landed, their previous conversion is done
    if (!producers_and(free_stage)) {
      record_error(status, 1);
      break;
    }
    issue(islot);
    islot = islot + 1 == S ? 0 : islot + 1;
    if (jc.tile + 1 != skip_tile1 || jc.kb != jc.t.kb_begin) {
      gather_convert<Cfg::BM, Cfg::BN>(jc, stg + cslot * SLOT, sA + stage * Cfg::A_STAGE,
                                       sB + stage * Cfg::B_STAGE, ptid);
      fence_proxy_async_smem();  // the stage is read by the tensor cores (async proxy)
      mbar_arrive(&full[stage]);
    }
    cslot = cslot + 1 == S ? 0 : cslot + 1;
    if (++stage == Cfg::STAGES) {
      stage = 0;
      phase ^= 1;
    }
    gjob_next<Cfg::BM, Cfg::BN, GROUPED>(jc, num_tiles, a1, g);
  }
  cp_async_wait<0>();  // no copy in flight when the producers leave
}

template <int MODE, int LOAD, int BNV, bool GROUPED>
__device__ __forceinline__ void gett_tc_body(const CUtensorMap* tmA, const CUtensorMap* tmB,
                                             const TcArgs* a1, const TcGroup& g,
                                             int32_t* status) {
  using Cfg = TcCfgT<MODE, LOAD, BNV>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + (((raw_addr + 1023u) & ~1023u) - raw_addr);
  uint8_t* sA = smem;                                   // STAGES x 16 KB
  uint8_t* sB = smem + Cfg::STAGES * Cfg::A_STAGE;      // STAGES x B_STAGE
  // gather: FP32 staging slots and the row-offset cache after the stages
  float* stg = reinterpret_cast<float*>(smem + Cfg::STAGES * Cfg::STAGE_BYTES);
  int64_t* rowc = reinterpret_cast<int64_t*>(smem + Cfg::STAGES * Cfg::STAGE_BYTES +
                                             Cfg::STG_SLOTS * Cfg::STG_SLOT_BYTES);
  float* epi_stg = reinterpret_cast<float*>(smem + Cfg::STAGES * Cfg::STAGE_BYTES +
                                            Cfg::STG_SLOTS * Cfg::STG_SLOT_BYTES +
                                            Cfg::ROWCACHE_BYTES);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Cfg::STAGES * Cfg::STAGE_BYTES +
                                               Cfg::STG_SLOTS * Cfg::STG_SLOT_BYTES +
                                               Cfg::ROWCACHE_BYTES + Cfg::EPI_STG_BYTES);
  uint64_t* full = bars;                   // [STAGES]
  uint64_t* empty = bars + Cfg::STAGES;    // [STAGES]
  uint64_t* accf = bars + 2 * Cfg::STAGES; // [2] accumulator ready
  uint64_t* acce = accf + 2;               // [2] accumulator drained
  uint64_t* drain = acce + 2;              // MMA completion on the abort path
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int num_tiles =
      GROUPED ? g.total_tiles
              : (a1->tail_split > 1
                     ? a1->full_tiles + (a1->tiles_m * a1->tiles_n - a1->full_tiles) * a1->tail_split
                     : a1->tiles_m * a1->tiles_n * a1->ksplit);
  const uint64_t wait_ns = (GROUPED || a1->wait_ns == 0) ? TCCG_DEVICE_WAIT_NS : a1->wait_ns;
  const int skip_tile1 = GROUPED ? 0 : a1->skip_tile1;
  int cta = (int)blockIdx.x;  // position in the tile order (TcArgs::sm_order)
  if (!GROUPED && a1->sm_order) {
    uint32_t smid, nsmid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    asm volatile("mov.u32 %0, %%nsmid;" : "=r"(nsmid));
    if (nsmid == gridDim.x) cta = (int)smid;
  }

  if (threadIdx.x == 0) {
    for (int s = 0; s < Cfg::STAGES; ++s) {
      mbar_init(&full[s], Cfg::GATHER ? 32 * Cfg::PRODUCER_WARPS : 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], Cfg::EPI_WARPS);
    }
    mbar_init(drain, 1);
    fence_mbar_init();
    if (!GROUPED && !Cfg::GATHER) {
      tma_prefetch_desc(tmA);
      tma_prefetch_desc(tmB);
    }
  }
  if (warp == Cfg::MMA_WARP) tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;
  // barriers and TMEM were set up while the packing kernel may still run:
  // its operands (and nothing else this kernel reads) come from it
  grid_dep_wait();

  if (Cfg::GATHER && warp < Cfg::PRODUCER_WARPS) {
    // ---------------- gather producers (4 warps) ----------------
    if constexpr (Cfg::GATHER)
      gather_producer<MODE, GROUPED>(a1, g, num_tiles, cta, sA, sB, stg, rowc, full, empty,
                                     wait_ns, skip_tile1, status);
  } else if (!Cfg::GATHER && warp == 0 && lane == 0) {
    // ---------------- TMA producer ----------------
    int stage = 0;
    uint32_t phase = 0;
    int issued_phase[Cfg::STAGES];
    for (int s = 0; s < Cfg::STAGES; ++s) issued_phase[s] = -1;
    bool ok = true;
    for (int tile = cta; tile < num_tiles && ok; tile += gridDim.x) {
      const TileRef t = resolve_tile<GROUPED>(tile, tmA, tmB, a1, g);
      for (int kb = t.kb_begin; kb < t.kb_end; ++kb) {
        if (!mbar_wait(&empty[stage], phase ^ 1, wait_ns)) {
          record_error(status, 1);
          ok = false;
          break;
        }
        if (tile + 1 != skip_tile1 || kb != t.kb_begin) {
          mbar_arrive_expect_tx(&full[stage], Cfg::STAGE_BYTES);
          tma_load_2d(sA + stage * Cfg::A_STAGE, t.tA, kb * 64, t.tm * Cfg::BM, &full[stage]);
          tma_load_2d(sB + stage * Cfg::B_STAGE, t.tB, kb * 64, t.tn * Cfg::BN, &full[stage]);
          issued_phase[stage] = (int)phase;
        }
        if (++stage == Cfg::STAGES) {
          stage = 0;
          phase ^= 1;
        }
      }
    }
    if (!ok) {  // let in-flight copies land before the CTA's smem goes away
      for (int s = 0; s < Cfg::STAGES; ++s)
        if (issued_phase[s] >= 0) (void)mbar_wait(&full[s], (uint32_t)issued_phase[s], wait_ns);
    }
  } else if (warp == Cfg::MMA_WARP && lane == 0) {
    // ---------------- MMA issuer ----------------
    int stage = 0;
    uint32_t phase = 0;
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true, issued_any = false;
    for (int tile = cta; tile < num_tiles && ok; tile += gridDim.x) {
      const TileRef t = resolve_tile<GROUPED>(tile, tmA, tmB, a1, g);
      const int nkb = t.kb_end, K = t.a->K, ckb = t.a->chunk_kb;
      // the MMAs stop at the tile's last column of C, rounded up to 32 (the
      // epilogue reads no further): a narrow C, or the last column tile,
      // costs only the tensor work its columns need
      const int64_t ncols = t.a->N - (int64_t)t.tn * Cfg::BN;
      const uint32_t idesc =
          idesc_bf16_f32(Cfg::BM, ncols >= Cfg::BN ? Cfg::BN : (int)((ncols + 31) / 32) * 32);
      for (int kb0 = t.kb_begin; kb0 < nkb && ok; kb0 += ckb) {
        if (!mbar_wait(&acce[acc], acc_phase ^ 1, wait_ns)) {
          record_error(status, 2);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d_tmem = tbase + (uint32_t)(acc * Cfg::ACC_STRIDE);
        uint32_t accumulate = 0;
        const int kend = (kb0 + ckb < nkb) ? kb0 + ckb : nkb;
        for (int kb = kb0; kb < kend; ++kb) {
          if (!mbar_wait(&full[stage], phase, wait_ns)) {
            record_error(status, 2);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t ad = umma_desc_k128(smem_u32(sA + stage * Cfg::A_STAGE));
          const uint64_t bd = umma_desc_k128(smem_u32(sB + stage * Cfg::B_STAGE));
          if constexpr (MODE == TC_BF16) {
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
              if (kb * 64 + ks * 16 < K) {
                tc_mma_f16(d_tmem, ad + 2 * ks, bd + 2 * ks, idesc, accumulate);
                accumulate = 1;
              }
            }
          } else {
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
              if (kb * 32 + ks * 16 < K) {
                // descriptor start address is in 16-byte units: +2 = 32 B (16 bf16),
                // +4 = 64 B (the lo half of the 128-byte row)
                tc_mma_f16(d_tmem, ad + 2 * ks, bd + 2 * ks, idesc, accumulate);  // ah*bh
                tc_mma_f16(d_tmem, ad + 2 * ks, bd + 4 + 2 * ks, idesc, 1);       // ah*bl
                tc_mma_f16(d_tmem, ad + 4 + 2 * ks, bd + 2 * ks, idesc, 1);       // al*bh
                accumulate = 1;
              }
            }
          }
          issued_any = true;
          tc_commit(&empty[stage]);  // frees the smem stage when these MMAs finish
          if (++stage == Cfg::STAGES) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (!ok) break;
        tc_commit(&accf[acc]);  // chunk sum ready for the epilogue
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1;
        }
      }
    }
    if (!ok && issued_any) {  // wait for outstanding MMAs before TMEM is released
      tc_commit(drain);
      (void)mbar_wait(drain, 0, wait_ns);
    }
  } else if (warp >= Cfg::EPI_WARP0) {
    // ---------------- epilogue ----------------
    const int q = warp & 3;             // TMEM lanes [32q, 32q+32) are accessible to this warp
    const int h = (warp - Cfg::EPI_WARP0) >> 2;  // column half of the tile
    constexpr int HC = Cfg::BN / 2;     // columns per epilogue warp
    float* wstg = epi_stg + (warp - Cfg::EPI_WARP0) * 16 * Cfg::EPI_LD;  // staged C stores
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    for (int tile = cta; tile < num_tiles && ok; tile += gridDim.x) {
      const TileRef t = resolve_tile<GROUPED>(tile, tmA, tmB, a1, g);
      const TcArgs& a = *t.a;
      const int64_t m = (int64_t)t.tm * Cfg::BM + q * 32 + lane;
      const bool m_ok = m < a.M;
      const int64_t cmo = m_ok ? a.c_m_off[m] : 0;
      const int64_t n0 = (int64_t)t.tn * Cfg::BN + h * HC;
      const int64_t nlim = a.N - n0;
      const float alpha = a.alpha, beta = a.beta;
      // C read once: in a grouped launch a is the item in global memory,
      // which the compiler must otherwise read again after every store
      float* const Cb = a.C;
      const int64_t* const cno = a.c_n_off + n0;
      // k-split slice: raw sums to partial[z][n][M], a tail slice to its
      // tile's block of tail_partial (both coalesced along m): element
      // (m, column c of this warp's half) at part[(pc0 + c) * pld]
      float* part = nullptr;
      int64_t pld = 0, pc0 = 0;
      if (t.tail >= 0) {
        const int tail = a.tiles_m * a.tiles_n - a.full_tiles;
        part = a.tail_partial + ((size_t)(t.z * tail + t.tail) * Cfg::BN) * Cfg::BM + q * 32 + lane;
        pld = Cfg::BM;
        pc0 = h * HC;
      } else if (a.partial) {
        part = a.partial + (size_t)t.z * a.N * a.M + m;
        pld = a.M;
        pc0 = n0;
      }
      if constexpr (MODE == TC_BF16) {
        // one accumulator per tile: stream TMEM -> C
        if (!mbar_wait(&accf[acc], acc_phase, wait_ns)) {
          record_error(status, 3);
          break;
        }
        tc_fence_after();
        const uint32_t tsrc = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * Cfg::ACC_STRIDE + h * HC);
        // columns of this warp's half that exist in C (warp-uniform): the
        // TMEM reads stop at the last 32-column group holding one of them
        const int last = nlim >= HC ? HC - 32 : (nlim > 0 ? (int)((nlim - 1) / 32) * 32 : -32);
        if (last < 0) {  // nothing to store: hand the accumulator straight back
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acce[acc]);
        }
#pragma unroll 1
        for (int cc = 0; cc <= last; cc += 32) {
          uint32_t r[32];
          tmem_ld_32x32b_x32(tsrc + (uint32_t)cc, r);
          tmem_ld_wait();
          if (cc == last) {  // accumulator read: hand it back to the MMA warp
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[acc]);
          }
          if (m_ok && part) {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (cc + j < nlim) part[(size_t)(pc0 + cc + j) * pld] = __uint_as_float(r[j]);
          } else if (a.crun > 0 && !part) {
#pragma unroll
            for (int hh = 0; hh < 32; hh += 16) {
              if (cc + hh < nlim) {  // warp-uniform
                __syncwarp();
#pragma unroll
                for (int j = 0; j < 16; ++j) wstg[j * Cfg::EPI_LD + lane] = __uint_as_float(r[hh + j]);
                __syncwarp();
                const int64_t left = nlim - cc - hh;
                const int64_t cn_lane =
                    lane < 16 && cc + hh + lane < nlim ? __ldg(cno + cc + hh + lane) : 0;
                store_runs(wstg, a, (int64_t)t.tm * Cfg::BM + q * 32, left < 16 ? (int)left : 16,
                           a.crun, alpha, beta, lane, cmo, cn_lane);
              }
            }
          } else if (m_ok) {
            if (beta != 0.0f) {
              float old[32];
#pragma unroll
              for (int j = 0; j < 32; ++j)
                old[j] = (cc + j < nlim) ? Cb[cmo + __ldg(cno + cc + j)] : 0.0f;
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (cc + j < nlim)
                  Cb[cmo + __ldg(cno + cc + j)] =
                      fmaf(beta, old[j], alpha * __uint_as_float(r[j]));
            } else {
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (cc + j < nlim)
                  Cb[cmo + __ldg(cno + cc + j)] = alpha * __uint_as_float(r[j]);
            }
          }
        }
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1;
        }
      } else {
        // chunked accumulation: sum the chunk accumulators in registers (RN adds)
        const int nchunks = (t.kb_end - t.kb_begin + a.chunk_kb - 1) / a.chunk_kb;
        // C's offsets of this warp's columns, column 32 i + lane in lane's
        // cn[i] (loaded while the MMAs run; passed around by shuffles when
        // storing, so no store waits on a table load)
        int64_t cn[HC / 32];
#pragma unroll
        for (int i = 0; i < HC / 32; ++i)
          cn[i] = 32 * i + lane < nlim ? __ldg(cno + 32 * i + lane) : 0;
        float sum[HC];
        for (int ch = 0; ch < nchunks; ++ch) {
          if (!mbar_wait(&accf[acc], acc_phase, wait_ns)) {
            record_error(status, 3);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t tsrc = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * Cfg::ACC_STRIDE + h * HC);
#pragma unroll
          for (int cc = 0; cc < HC; cc += 16) {
            if (cc < nlim) {  // warp-uniform: groups past C's last column are not read
              uint32_t r[16];
              tmem_ld_32x32b_x16(tsrc + (uint32_t)cc, r);
              tmem_ld_wait();
#pragma unroll
              for (int j = 0; j < 16; ++j)
                sum[cc + j] = (ch == 0) ? __uint_as_float(r[j])
                                        : __fadd_rn(sum[cc + j], __uint_as_float(r[j]));
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acce[acc]);  // accumulator free for the MMA warp
          if (++acc == 2) {
            acc = 0;
            acc_phase ^= 1;
          }
        }
        if (!ok) break;
        if (part) {  // warp-uniform, like the branches below
          if (m_ok) {
#pragma unroll
            for (int j = 0; j < HC; ++j)
              if (j < nlim) part[(size_t)(pc0 + j) * pld] = sum[j];
          }
        } else if (a.crun > 0) {
#pragma unroll
          for (int cc = 0; cc < HC; cc += 16) {
            if (cc < nlim) {  // warp-uniform
              __syncwarp();
#pragma unroll
              for (int j = 0; j < 16; ++j) wstg[j * Cfg::EPI_LD + lane] = sum[cc + j];
              __syncwarp();
              const int64_t left = nlim - cc;
              const int64_t cn_lane =
                  lane < 16 && cc + lane < nlim ? __ldg(cno + cc + lane) : 0;
              store_runs(wstg, a, (int64_t)t.tm * Cfg::BM + q * 32, left < 16 ? (int)left : 16,
                         a.crun, alpha, beta, lane, cmo, cn_lane);
            }
          }
        } else {
          // every lane takes part in the shuffles; rows past M store nothing
          if (beta != 0.0f) {
#pragma unroll
            for (int cc = 0; cc < HC; cc += 8) {
              int64_t o[8];
              float old[8];
#pragma unroll
              for (int j = 0; j < 8; ++j) {
                o[j] = cmo + __shfl_sync(0xffffffffu, cn[(cc + j) / 32], (cc + j) % 32);
                old[j] = m_ok && cc + j < nlim ? Cb[o[j]] : 0.0f;
              }
#pragma unroll
              for (int j = 0; j < 8; ++j)
                if (m_ok && cc + j < nlim) Cb[o[j]] = fmaf(beta, old[j], alpha * sum[cc + j]);
            }
          } else {
#pragma unroll
            for (int j = 0; j < HC; ++j) {
              const int64_t o = cmo + __shfl_sync(0xffffffffu, cn[j / 32], j % 32);
              if (m_ok && j < nlim) Cb[o] = alpha * sum[j];
            }
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == Cfg::MMA_WARP) {
    tc_fence_after();
    tmem_dealloc(tbase, Cfg::TMEM_COLS);
  }
}

template <int MODE, int LOAD = TC_LOAD_TMA, int BNV = 0>
__global__ void __launch_bounds__(TcCfgT<MODE, LOAD, BNV>::NUM_THREADS, 1)
    gett_tc_kernel(const __grid_constant__ CUtensorMap tmA,
                   const __grid_constant__ CUtensorMap tmB, const TcArgs a) {
  TcGroup g{nullptr, nullptr, 0, 0};
  gett_tc_body<MODE, LOAD, BNV, false>(&tmA, &tmB, &a, g, a.status);
}

template <int MODE, int LOAD = TC_LOAD_TMA, int BNV = 0>
__global__ void __launch_bounds__(TcCfgT<MODE, LOAD, BNV>::NUM_THREADS, 1)
    gett_tc_group_kernel(const TcGroup g, int32_t* status) {
  gett_tc_body<MODE, LOAD, BNV, true>(nullptr, nullptr, nullptr, g, status);
}

// Tail split: C = alpha * (slice 0 + slice 1 + ...) + beta * C over the tail
// tiles (RN adds in slice order). grid = (tail tiles, BM * BN / 256), block
// 256: thread e of a tile takes element (m_local = e % BM, n_local = e / BM).
template <int MODE, int LOAD = TC_LOAD_TMA, int BNV = 0>
__global__ void __launch_bounds__(256) tc_tail_reduce_kernel(const TcArgs a) {
  using Cfg = TcCfgT<MODE, LOAD, BNV>;
  grid_dep_wait();  // partial sums written by the GETT kernel before
  const int tail = a.tiles_m * a.tiles_n - a.full_tiles;
  const int tl = blockIdx.x;
  const int e = blockIdx.y * 256 + threadIdx.x;
  if (tl >= tail || e >= Cfg::BM * Cfg::BN) return;
  const int ml = e % Cfg::BM, nl = e / Cfg::BM;
  int tm, tn;
  tile_coords(a.full_tiles + tl, a, tm, tn);
  const int64_t m = (int64_t)tm * Cfg::BM + ml, n = (int64_t)tn * Cfg::BN + nl;
  if (m >= a.M || n >= a.N) return;
  const float* p = a.tail_partial + ((size_t)tl * Cfg::BN + nl) * Cfg::BM + ml;
  const size_t slice = (size_t)tail * Cfg::BN * Cfg::BM;
  float s = p[0];
  for (int z = 1; z < a.tail_split; ++z) s = __fadd_rn(s, p[z * slice]);
  float* c = a.C + a.c_m_off[m] + a.c_n_off[n];
  *c = a.beta != 0.0f ? fmaf(a.beta, *c, a.alpha * s) : a.alpha * s;
}

}  // namespace tccg
