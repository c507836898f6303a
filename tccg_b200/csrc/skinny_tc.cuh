// Skinny GETT on the tensor cores (split-BF16x3): the skinny kernel's boxes,
// jobs, k slices and C stores, with tcgen05 MMAs in place of its FP32 FMAs.
//
// For a narrow side S <= 64 and long K the FP32 FMAs of the skinny kernel
// (S x K per position) cost more than streaming P; the tile kernel instead
// pays a packing pass over P (read, written, read again) and pads S to its
// tile width. Here P crosses HBM once, as in the skinny kernel, and the
// products run on the tensor cores:
//
//   warps 0-7   (256 threads): copy P's chunks of 32 k from the caller's
//               tensor into a ring of FP32 staging slots ([k][position],
//               the skinny kernel's copies, cp.async) as fast as slots free
//               up; each thread's copies arrive on the slot's barrier as
//               they land (cp.async.mbarrier.arrive);
//   warps 8-15  (256 threads, thread = box position = TMEM lane of its
//               half): per chunk, split the position's 32 staged values into
//               bf16 hi / lo and write them to its TMEM lane of the chunk's A
//               stage (tcgen05.st: 16 columns of hi, 16 of lo) -- the MMAs
//               read the wide operand from TMEM, so it takes no shared-memory
//               stage; thread 0 first loads the matching chunk of the narrow
//               operand Q, packed once per call into the K-major layout, by
//               TMA;
//   warp 16     one thread issues per chunk and half box (128 positions)
//               the three products hi*hi + hi*lo + lo*hi of both k16 steps
//               (tcgen05.mma kind::f16, M = 128, N = S rounded up to 16)
//               into a TMEM accumulator; a job's chunks go into TMEM rounds
//               of chunk_kb chunks, two accumulators alternating;
//   warps 17-24 (256 threads, thread = position = TMEM lane of its half)
//               add each round into the job's running sums, kept in TMEM
//               (RN adds: the tile kernel's chunked accumulation), then
//               store the C block by the skinny kernel's store walks or
//               linear copies, or its raw sums to the job's k slice (four
//               warps, each thread both halves, measured 1.2-1.4x slower on
//               items whose C stores dominate).
//
// Copies, conversion and MMAs run in separate warps: with one set of warps
// issuing a chunk's copies, its Q load and its conversion in turn, a chunk
// took 1.7-2.8 us against the 0.7 us of its HBM bytes (the copy pattern
// alone streams at 4.9-6.6 TB/s).
//
// One CTA per SM (216 KB of shared memory: five 33 KB staging slots, two
// 8 KB Q stages, the 33 KB epilogue staging and the offset tables; 25
// warps); TMEM 512 columns (accumulators, running sums, A stages). Every
// wait is bounded (TCCG_DEVICE_WAIT_NS): a wait that runs out records a
// status code and the CTA winds down.
#pragma once

#include <cuda.h>

#include "skinny_gett.cuh"

namespace tccg {

constexpr int SKT_COPY_THREADS = SK_THREADS;             // 256, warps 0-7
constexpr int SKT_CONV_WARP0 = SKT_COPY_THREADS / 32;    // 8
constexpr int SKT_CONV_THREADS = SK_BW;                  // 256, warps 8-15
constexpr int SKT_MMA_WARP = SKT_CONV_WARP0 + SKT_CONV_THREADS / 32;  // 16
constexpr int SKT_EPI_WARP0 = SKT_MMA_WARP + 1;          // 17
constexpr int SKT_EPI_THREADS = SK_BW;  // one position each: TMEM lane of its half
constexpr int SKT_THREADS = SKT_COPY_THREADS + SKT_CONV_THREADS + 32 + SKT_EPI_THREADS;  // 800
constexpr int SKT_SMAX = 64;   // rows per pass (a narrow side above 64 runs passes of 64)
constexpr int SKT_HALF = 128;  // MMA rows: positions per half box
constexpr int SKT_SLOTS = 5;   // FP32 staging ring
constexpr int SKT_STAGES = 2;  // MMA operand stages (P in TMEM, Q in shared memory)
constexpr size_t SKT_B_STAGE = (size_t)SKT_SMAX * 128;  // up to 64 Q rows x 128 B
constexpr size_t SKT_SLOT = (size_t)SK_KC * SK_LDP * 4;
constexpr size_t SKT_OFF_B = 0;
constexpr size_t SKT_OFF_SLOT = SKT_OFF_B + SKT_STAGES * SKT_B_STAGE;
constexpr size_t SKT_OFF_OS = SKT_OFF_SLOT + SKT_SLOTS * SKT_SLOT;
constexpr size_t SKT_OFF_TAB = SKT_OFF_OS + (size_t)SK_SUB * SK_LDP * 4;
// tables: pw[2][BW] (copy warps), cw[BW] and cs[SMAX] (epilogue)
constexpr size_t SKT_OFF_BAR = SKT_OFF_TAB + (size_t)(3 * SK_BW + SKT_SMAX) * 4;
constexpr size_t SKT_SMEM_BYTES = 1024 + SKT_OFF_BAR + 24 * 8;
// TMEM columns: accumulator b of half h at b * 2 SMAX + h SMAX, the job's
// running sums of half h at SKT_SUMCOL + h SMAX, and the converted P (the
// MMAs' A operand) of stage s, half h at SKT_ACOL + s * 64 + h * 32: 16
// columns of hi then 16 of lo (two bf16 of k per column)
constexpr int SKT_SUMCOL = 4 * SKT_SMAX;
constexpr int SKT_ACOL = SKT_SUMCOL + 2 * SKT_SMAX;
constexpr uint32_t SKT_TMEM_COLS = 512;
static_assert(SKT_ACOL + SKT_STAGES * 64 <= (int)SKT_TMEM_COLS, "TMEM columns");
static_assert(SK_BW == 2 * SKT_HALF, "a box is two MMA halves");
static_assert(SKT_SMEM_BYTES <= 227 * 1024, "one CTA per SM");
static_assert(SKT_OFF_B % 1024 == 0 && SKT_B_STAGE % 1024 == 0, "swizzled stages 1024-byte aligned");

struct SkinnyTcArgs {
  SkinnyArgs sk;     // P, C, tables, boxes, jobs (rs = spad / 4); Q unused
  int32_t spad;      // MMA N = rows per pass: S rounded up to 16, or 64 (S > 64, passes)
  int32_t chunk_kb;  // chunks accumulated per TMEM round
};

// A grouped launch's item: Q's tensor map (64-byte aligned, read by TMA from
// global memory), the arguments and the item's first global job.
struct __align__(64) SkinnyTcItem {
  CUtensorMap tmQ;
  SkinnyTcArgs args;
  int64_t begin;
};

struct SktRef {
  const SkinnyTcArgs* a;
  const CUtensorMap* tq;
  int J;
};

// Whether box position w of block b is inside the tensor.
__device__ __forceinline__ bool skt_inside(const SkinnyArgs& a, int b, int w) {
  const int ix = a.bxn == 1 ? 0 : b % a.bxn, iy = a.bxn == 1 ? b : b / a.bxn;
  const int xl = a.p_walk == SK_P_Y ? w / a.ty : w % a.tx;
  const int yl = a.p_walk == SK_P_Y ? w % a.ty : w / a.tx;
  return w < a.tx * a.ty && ix * a.tx + xl < a.ex && iy * a.ty + yl < a.ey;
}

// Box position w's P offset (loaders) / C offset (epilogue); SK_NONE outside.
__device__ __forceinline__ int32_t skt_box(const SkinnyArgs& a, int b, int w, bool c) {
  const int ix = a.bxn == 1 ? 0 : b % a.bxn, iy = a.bxn == 1 ? b : b / a.bxn;
  int xl, yl;
  if (a.p_walk == SK_P_Y) {
    yl = w % a.ty;
    xl = w / a.ty;
  } else {
    xl = w % a.tx;
    yl = w / a.tx;
  }
  const int x = ix * a.tx + xl, y = iy * a.ty + yl;
  const bool ok = w < a.tx * a.ty && x < a.ex && y < a.ey;
  return !ok ? SK_NONE : c ? x * a.cx + __ldg(a.c_y_off + y) : x * a.px + __ldg(a.p_y_off + y);
}

__device__ __forceinline__ void skt_epi_sync() { named_barrier_sync(2, SKT_EPI_THREADS); }

// Barrier over the 256 epilogue threads (named barrier 2) that ANDs a flag:
// after a wait that ran out in any of them, all leave before the next
// barrier of the store path.
__device__ __forceinline__ bool skt_epi_and(bool v) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, 2, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)v), "n"(SKT_EPI_THREADS)
      : "memory");
  return out != 0;
}

// Converts position w's column of a staging slot ([k][position], k < kc
// valid) into its TMEM lane of an A stage (ta: the warp's lane quarter, the
// stage and half's first column): hi = bf16(x) in 16 columns, then lo =
// bf16(x - hi) in 16, two k per column (the lower k in the low half); k past
// kc, and every k of a position outside the tensor (kc = 0: the copies skip
// it), are zeros. Warp-collective (tcgen05.st).
__device__ __forceinline__ void skt_convert(const float* slot, uint32_t ta, int w, int kc) {
  // shared-window addresses: the reads stay shared-memory loads
  const uint32_t src = smem_u32(slot + w);
  uint32_t hw[16], lw[16];
#pragma unroll
  for (int e = 0; e < SK_KC; e += 2) {
    float x0 = 0.0f, x1 = 0.0f;
    if (e < kc) asm volatile("ld.shared.f32 %0, [%1];" : "=f"(x0) : "r"(src + e * SK_LDP * 4));
    if (e + 1 < kc)
      asm volatile("ld.shared.f32 %0, [%1];" : "=f"(x1) : "r"(src + (e + 1) * SK_LDP * 4));
    split_bf16x2(x0, x1, hw[e / 2], lw[e / 2]);
  }
  tmem_st_32x32b_x16(ta, hw);
  tmem_st_32x32b_x16(ta + 16, lw);
}

// The end of job j in the epilogue, its sums in TMEM (tsum(g): columns g *
// 16 .. + 15 of the thread's half in its warp's lane quarter): raw sums to
// its k slice, or the C block of its pass's rows (staged in os, then the
// skinny kernel's store walks or linear copies). Thread etid (0..255) holds
// position w.
template <typename TSum>
__device__ __forceinline__ void skt_finish(const SkinnyArgs& a, const SkJob& j, int spad,
                                           TSum&& tsum, float* os, int32_t* cw, int32_t* cs,
                                           int w, int etid) {
  const int r0 = j.p * spad;  // the pass's first row
  const int S = a.S - r0 < spad ? a.S - r0 : spad;  // rows of this pass
  if (a.partial) {  // the skinny layout, passes of spad (= 4 rs) rows
    {
      float* dst = a.partial + (((size_t)j.z * a.nblk + j.b) * a.npass + j.p) * (size_t)spad * SK_BW + w;
#pragma unroll
      for (int g = 0; g < SKT_SMAX / 16; ++g) {
        if (g * 16 < S) {  // warp-uniform
          uint32_t v[16];
          tmem_ld_32x32b_x16(tsum(g), v);
          tmem_ld_wait();
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (g * 16 + i < S) dst[(size_t)(g * 16 + i) * SK_BW] = __uint_as_float(v[i]);
        }
      }
    }
    return;
  }
  skt_epi_sync();  // the previous job's stores are done with os, cw, cs
  cw[w] = skt_box(a, j.b, w, true);
  if (etid < S) cs[etid] = __ldg(a.c_s_off + r0 + etid);
  const bool py = a.p_walk == SK_P_Y;
  const int tx = a.tx, ty = a.ty;
  const float sc = a.c_bulk ? a.alpha : 1.0f;
  // staging index of row 0 of position w and the distance between rows:
  // [y][x][s] (SX), [y][s][x] (XS, 32-row steps) or [s][position]
  auto base = [&](int w, int& step) {
    const int xl = py ? w / ty : w % tx, yl = py ? w % ty : w / tx;
    if (a.c_lin == SK_CLIN_SX) {
      step = 1;
      return yl * tx * S + xl * S;
    }
    if (a.c_lin == SK_CLIN_XS) {
      step = tx;
      return yl * tx * SK_SUB + xl;
    }
    step = SK_LDP;
    return w;
  };
#pragma unroll
  for (int hh = 0; hh < SKT_SMAX; hh += SK_SUB) {
    // SX stages all of S (<= 32 rows) in one step
    if (hh < S && (hh == 0 || a.c_lin != SK_CLIN_SX)) {
      const int ns = a.c_lin == SK_CLIN_SX ? S : (S - hh < SK_SUB ? S - hh : SK_SUB);
      skt_epi_sync();  // the staging's last reader is done
      {
        int rstep;
        const int o = base(w, rstep);
        const bool in = a.c_lin == SK_CLIN_NONE || w < tx * ty;
#pragma unroll
        for (int g = 0; g < SK_SUB / 16; ++g) {
          if (g * 16 < ns) {  // warp-uniform
            uint32_t v[16];
            tmem_ld_32x32b_x16(tsum(hh / 16 + g), v);
            tmem_ld_wait();
#pragma unroll
            for (int i = 0; i < 16; ++i)
              if (in && g * 16 + i < ns) os[o + (g * 16 + i) * rstep] = sc * __uint_as_float(v[i]);
          }
        }
      }
      if (a.c_bulk) fence_proxy_async_smem();  // the bulk copies read the staging
      skt_epi_sync();
      if (a.c_lin == SK_CLIN_SX) {
        const int ix = a.bxn == 1 ? 0 : j.b % a.bxn;
        const int xn = a.ex - ix * tx < tx ? a.ex - ix * tx : tx;
        skinny_copy_rows<SKT_EPI_THREADS>(a, os, tx * S, cw, cs[0], xn * S, etid);
      } else if (a.c_lin == SK_CLIN_XS) {
        skinny_copy_rows<SKT_EPI_THREADS>(a, os, tx * SK_SUB, cw, cs[hh], tx * ns, etid);
      } else {
        skinny_store<SKT_EPI_THREADS>(a, os, cw, cs + hh, r0 + hh, ns, etid);
      }
    }
  }
}

// The kernel body over global jobs j0, j0 + jstep, ... < njobs; resolve(J)
// gives the job's item (its arguments and Q's tensor map) and its index in
// the item.
template <typename Resolve>
__device__ __forceinline__ void skinny_tc_body(int njobs, Resolve&& resolve, int32_t* status) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + (((raw_addr + 1023u) & ~1023u) - raw_addr);
  uint8_t* sB = smem + SKT_OFF_B;
  float* slots = reinterpret_cast<float*>(smem + SKT_OFF_SLOT);
  float* os = reinterpret_cast<float*>(smem + SKT_OFF_OS);
  int32_t* pw = reinterpret_cast<int32_t*>(smem + SKT_OFF_TAB);  // [2][BW]
  int32_t* cw = pw + 2 * SK_BW;                                  // [BW]
  int32_t* cs = cw + SK_BW;                                      // [SMAX]
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + SKT_OFF_BAR);
  uint64_t* full = bars;                    // [STAGES] P stage converted + Q landed
  uint64_t* empty = bars + SKT_STAGES;      // [STAGES] the stage's MMAs done
  uint64_t* accf = bars + 2 * SKT_STAGES;   // [2] TMEM round ready
  uint64_t* acce = accf + 2;                // [2] TMEM round drained
  uint64_t* drain = acce + 2;               // MMA completion on the abort path
  uint64_t* sfull = drain + 1;              // [SLOTS] the slot's copies landed
  uint64_t* sempty = sfull + SKT_SLOTS;     // [SLOTS] the slot was converted
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sempty + SKT_SLOTS);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t wait_ns = TCCG_DEVICE_WAIT_NS;
  const int j0 = (int)blockIdx.x, js = (int)gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < SKT_STAGES; ++s) {
      mbar_init(&full[s], SKT_CONV_THREADS + 1);  // the converters + thread 0's expect_tx
      mbar_init(&empty[s], 1);
    }
    for (int s = 0; s < SKT_SLOTS; ++s) {
      mbar_init(&sfull[s], SKT_COPY_THREADS);  // each copy thread, when its copies landed
      mbar_init(&sempty[s], SKT_CONV_THREADS);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], SKT_EPI_THREADS / 32);
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == SKT_MMA_WARP) tmem_alloc(tmem_slot, SKT_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;
  // barriers and TMEM were set up while the packing kernel may still run:
  // Q comes from it
  grid_dep_wait();

  if (warp < SKT_CONV_WARP0) {
    // ---------------- copy warps ----------------
    const int tid = threadIdx.x;
    // job ig, chunk ic of [.., ic1), its box offsets slot and the k offset
    // its next copies start from (loaded a chunk ahead: the copies would
    // otherwise wait for the table load)
    int ig = j0, ic = 0, ic1 = 0, ib = 0, ipw = 1;
    int32_t iko = 0;
    bool inew = false;
    const SkinnyArgs* ia = nullptr;
    SkPFields ipf{};  // ia's fields the copies of each chunk read
    auto iseek = [&]() {
      if (ig < njobs) {
        const SktRef r = resolve(ig);
        ia = &r.a->sk;
        ipf = skinny_p_fields(*ia);
        const SkJob jb = skinny_job(*ia, r.J);
        ic = jb.c0;
        ic1 = jb.c1;
        ib = jb.b;
        inew = true;
      }
    };
    iseek();
    if (ig < njobs) iko = skinny_p_ko(ipf, ic);
    int slot = 0;
    uint32_t sphase = 0;
    while (ig < njobs) {
      if (!mbar_wait(&sempty[slot], sphase ^ 1, wait_ns)) {
        record_error(status, 1);
        break;
      }
      if (inew) {  // the other box slot is no longer read: its job's copies were issued
        ipw ^= 1;
        pw[ipw * SK_BW + tid] = skt_box(*ia, ib, tid, false);
        named_barrier_sync(1, SKT_COPY_THREADS);  // walks read other threads' offsets
        inew = false;
      }
      skinny_issue_p<true>(ipf, ic, slots + slot * (SKT_SLOT / 4), pw + ipw * SK_BW, iko);
      cp_async_mbar_arrive(&sfull[slot]);
      if (++slot == SKT_SLOTS) {
        slot = 0;
        sphase ^= 1;
      }
      if (++ic >= ic1) {
        ig += js;
        iseek();
      }
      if (ig < njobs) iko = skinny_p_ko(ipf, ic);
    }
    cp_async_wait<0>();  // no copy in flight when the copy warps leave
  } else if (warp < SKT_MMA_WARP) {
    // ---------------- converters ----------------
    const int w = threadIdx.x - SKT_COPY_THREADS;  // the thread's box position
    int cg = j0, cc = 0, cc1 = 0, cq = 0;  // cq: the job's first Q row (its pass)
    int cK = 0, cspad = 0;  // the item's K and rows per pass, read once per job
    bool inside = false;  // the position is inside the tensor (else the copies skip it)
    SktRef cr{};
    auto cseek = [&]() {
      if (cg < njobs) {
        cr = resolve(cg);
        const SkJob jb = skinny_job(cr.a->sk, cr.J);
        cc = jb.c0;
        cc1 = jb.c1;
        cK = cr.a->sk.K;
        cspad = cr.a->spad;
        cq = jb.p * cspad;
        inside = skt_inside(cr.a->sk, jb.b, w);
      }
    };
    cseek();
    int stage = 0, slot = 0;
    uint32_t phase = 0, sphase = 0;
    while (cg < njobs) {
      if (!mbar_wait(&empty[stage], phase ^ 1, wait_ns)) {
        record_error(status, 1);
        break;
      }
      if (w == 0) {  // Q's chunk, in flight while the copies are waited for
        mbar_arrive_expect_tx(&full[stage], (uint32_t)cspad * 128u);
        tma_load_2d(sB + stage * SKT_B_STAGE, cr.tq, cc * 64, cq, &full[stage]);
      }
      if (!mbar_wait(&sfull[slot], sphase, wait_ns)) {
        record_error(status, 1);
        break;
      }
      tc_fence_after();  // the stage's MMAs (waited for above) are done with its TMEM columns
      skt_convert(slots + slot * (SKT_SLOT / 4),
                  tbase + ((uint32_t)((warp & 3) * 32) << 16) +
                      (uint32_t)(SKT_ACOL + stage * 64 + (w / SKT_HALF) * 32),
                  w, inside ? (cK - cc * SK_KC < SK_KC ? cK - cc * SK_KC : SK_KC) : 0);
      mbar_arrive(&sempty[slot]);
      tmem_st_wait();    // the stage's TMEM columns are written ...
      tc_fence_before();  // ... before the MMA warp learns of it
      mbar_arrive(&full[stage]);
      if (++slot == SKT_SLOTS) {
        slot = 0;
        sphase ^= 1;
      }
      if (++stage == SKT_STAGES) {
        stage = 0;
        phase ^= 1;
      }
      if (++cc >= cc1) {
        cg += js;
        cseek();
      }
    }
  } else if (warp == SKT_MMA_WARP) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int stage = 0, acc = 0;
      uint32_t phase = 0, acc_phase = 0;
      bool ok = true, issued = false;
      for (int jg = j0; jg < njobs && ok; jg += js) {
        const SktRef r = resolve(jg);
        const SkinnyArgs& a = r.a->sk;
        const SkJob jb = skinny_job(a, r.J);
        const uint32_t idesc = idesc_bf16_f32(SKT_HALF, r.a->spad);
        const int ckb = r.a->chunk_kb;
        const int K = a.K;  // read once (the waits below clobber memory)
        for (int c0 = jb.c0; c0 < jb.c1 && ok; c0 += ckb) {
          if (!mbar_wait(&acce[acc], acc_phase ^ 1, wait_ns)) {
            record_error(status, 2);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d0 = tbase + (uint32_t)(acc * 2 * SKT_SMAX);
          uint32_t accumulate = 0;
          const int ce = c0 + ckb < jb.c1 ? c0 + ckb : jb.c1;
          for (int c = c0; c < ce; ++c) {
            if (!mbar_wait(&full[stage], phase, wait_ns)) {
              record_error(status, 2);
              ok = false;
              break;
            }
            tc_fence_after();
            const uint64_t bd = umma_desc_k128(smem_u32(sB + stage * SKT_B_STAGE));
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
              if (c * SK_KC + ks * 16 < K) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                  // A in TMEM: k step ks at column + 8 ks (16 bf16), lo 16 columns on
                  const uint32_t ah = tbase + (uint32_t)(SKT_ACOL + stage * 64 + h * 32 + 8 * ks);
                  const uint32_t d = d0 + (uint32_t)(h * SKT_SMAX);
                  // B descriptor start addresses in 16-byte units: +2 = 32 B (16
                  // bf16), +4 = 64 B (the lo half of the 128-byte row)
                  tc_mma_f16_ts(d, ah, bd + 2 * ks, idesc, accumulate);       // hi * hi
                  tc_mma_f16_ts(d, ah, bd + 4 + 2 * ks, idesc, 1);            // hi * lo
                  tc_mma_f16_ts(d, ah + 16, bd + 2 * ks, idesc, 1);           // lo * hi
                }
                accumulate = 1;
              }
            }
            issued = true;
            tc_commit(&empty[stage]);  // frees the stage when these MMAs finish
            if (++stage == SKT_STAGES) {
              stage = 0;
              phase ^= 1;
            }
          }
          if (!ok) break;
          tc_commit(&accf[acc]);  // the round's sums are ready for the epilogue
          if (++acc == 2) {
            acc = 0;
            acc_phase ^= 1;
          }
        }
      }
      if (!ok && issued) {  // outstanding MMAs finish before TMEM is released
        tc_commit(drain);
        (void)mbar_wait(drain, 0, wait_ns);
      }
    }
    __syncwarp();
  } else {
    // ---------------- epilogue ----------------
    const int etid = threadIdx.x - SKT_EPI_WARP0 * 32;  // 0..255
    const int q = warp & 3;       // TMEM lanes [32 q, 32 q + 32) are this warp's
    const int h = etid >> 7;      // its half box
    const int w = h * SKT_HALF + q * 32 + lane;  // the thread's position
    const uint32_t tq = tbase + ((uint32_t)(q * 32) << 16);
    auto tsum = [&](int g) { return tq + (uint32_t)(SKT_SUMCOL + h * SKT_SMAX + g * 16); };
    int acc = 0;
    uint32_t acc_phase = 0;
    for (int jg = j0; jg < njobs; jg += js) {
      const SktRef r = resolve(jg);
      const SkinnyArgs& a = r.a->sk;
      const SkJob jb = skinny_job(a, r.J);
      const int spad = r.a->spad, ckb = r.a->chunk_kb;
      const int rounds = (jb.c1 - jb.c0 + ckb - 1) / ckb;
      bool ok = true;
      for (int rd = 0; rd < rounds; ++rd) {
        if (!mbar_wait(&accf[acc], acc_phase, wait_ns)) {
          record_error(status, 3);
          ok = false;
          break;
        }
        tc_fence_after();
        // running sums (TMEM) = round 0, then + each round (RN adds)
#pragma unroll
        for (int g = 0; g < SKT_SMAX / 16; ++g) {
          if (g * 16 < spad) {  // warp-uniform
            uint32_t v[16];
            tmem_ld_32x32b_x16(tq + (uint32_t)(acc * 2 * SKT_SMAX + h * SKT_SMAX + g * 16), v);
            if (rd > 0) {
              uint32_t u[16];
              tmem_ld_32x32b_x16(tsum(g), u);
              tmem_ld_wait();
#pragma unroll
              for (int i = 0; i < 16; ++i)
                v[i] = __float_as_uint(__fadd_rn(__uint_as_float(u[i]), __uint_as_float(v[i])));
            } else {
              tmem_ld_wait();
            }
            tmem_st_32x32b_x16(tsum(g), v);
          }
        }
        tmem_st_wait();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acce[acc]);  // the accumulator is free for the MMA warp
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1;
        }
      }
      if (!skt_epi_and(ok)) break;  // every epilogue thread takes the same branch
      skt_finish(a, jb, spad, tsum, os, cw, cs, w, etid);
    }
    bulk_wait_all();  // bulk C copies complete before the CTA exits
  }

  tc_fence_before();
  __syncthreads();
  if (warp == SKT_MMA_WARP) {
    tc_fence_after();
    tmem_dealloc(tbase, SKT_TMEM_COLS);
  }
}

// One plan: a persistent grid of at most one CTA per SM over the plan's jobs.
__global__ void __launch_bounds__(SKT_THREADS, 1)
    skinny_tc_kernel(const __grid_constant__ CUtensorMap tmQ, const __grid_constant__ SkinnyTcArgs a,
                     int32_t* status) {
  // the arguments in shared memory, read through the job references (items
  // 46 / 47 of the 256-item batched workload: 0.83 / 0.28 ms against 1.04 /
  // 0.37 ms reading them in the parameter space); the tensor map stays a
  // parameter (TMA reads it there)
  __shared__ SkinnyTcArgs sa;
  if (threadIdx.x == 0) sa = a;
  __syncthreads();
  auto resolve = [&](int J) { return SktRef{&sa, &tmQ, J}; };
  skinny_tc_body(a.sk.njobs, resolve, status);
}

// Grouped: item i owns the global jobs [begin[i], begin[i + 1]).
__global__ void __launch_bounds__(SKT_THREADS, 1)
    skinny_tc_group_kernel(const SkinnyTcItem* items, const int64_t* begin, int n, int njobs,
                           int32_t* status) {
  auto resolve = [&](int J) {
    const SkinnyTcItem& it = items[find_segment(begin, n, J)];
    return SktRef{&it.args, &it.tmQ, (int)(J - it.begin)};
  };
  skinny_tc_body(njobs, resolve, status);
}

}  // namespace tccg
