// tcgen05 GETT kernel on CTA pairs (cta_group::2): one UMMA covers a 256-row
// tile whose rows are split over the two SMs of a cluster, and the B operand
// tile is split too, so each SM stages and reads only half of B. Compared with
// the one-SM kernel (tc_gemm.cuh) this lowers the shared-memory traffic per SM
// by about 30 % for split-BF16x3 (its bound there) at the same tile area.
//
// Per pair tile (256 x BN) and k-block:
//   CTA r loads rows [128r, 128r+128) of the A' tile and rows
//   [r*BN/2, (r+1)*BN/2) of the B' tile into its own shared memory; both TMA
//   loads complete on the barrier of the even CTA (the address with the peer
//   bit cleared), whose producer arrives with the byte count of the pair;
//   the even CTA's MMA thread issues tcgen05.mma.cta_group::2 (M = 256),
//   which reads the halves from both SMs and writes D rows [128r, 128r+128)
//   into CTA r's TMEM; each of its commits is issued once per CTA's barrier.
// Each CTA's epilogue drains its own TMEM rows; the odd CTA's epilogue warps
// release the accumulator with remote arrives on the even CTA's barrier.
// K is accumulated in chunks (as in tc_gemm.cuh) for BF16X3.
//
// Every CTA loads its own operand halves with its own TMA loads (no load is
// shared between the two CTAs of a pair).
#pragma once
#include "tc_gemm.cuh"

namespace tccg {

__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}

// Arrive on the mbarrier at the same shared offset in CTA `rank` of the cluster.
__device__ __forceinline__ void mbar_arrive_remote(uint64_t* bar, uint32_t rank) {
  asm volatile(
      "{\n\t.reg .b32 ra;\n\t"
      "mapa.shared::cluster.u32 ra, %0, %1;\n\t"
      "mbarrier.arrive.release.cluster.shared::cluster.b64 _, [ra];\n\t}" ::"r"(smem_u32(bar)),
      "r"(rank)
      : "memory");
}

// 2-D TMA load into this CTA's smem, completing on the even CTA's barrier.
__device__ __forceinline__ void tma_load_2d_pair(void* smem_dst, const void* tmap, int32_t c0,
                                                 int32_t c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(smem_u32(bar) & 0xFEFFFFFFu)
      : "memory");
}

__device__ __forceinline__ void tmem_alloc_pair(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tc_mma_f16_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                                uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive on `bar` in both CTAs of the pair once the prior MMAs completed:
// one commit per barrier (this CTA's, then the peer's at the same offset,
// addressed through mapa); each commit tracks all prior MMAs of this thread.
__device__ __forceinline__ void tc_commit_pair(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
  asm volatile(
      "{\n\t.reg .b32 ra;\n\t"
      "mapa.shared::cluster.u32 ra, %0, 1;\n\t"
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [ra];\n\t}" ::"r"(
          smem_u32(bar))
      : "memory");
}

template <int MODE>
struct Tc2Cfg {
  static constexpr int BM = 128;  // rows per CTA (256 per pair)
  static constexpr int BN = (MODE == TC_BF16X3) ? 192 : 256;
  static constexpr int BNH = BN / 2;  // B rows staged per CTA
  static constexpr int STAGES = (MODE == TC_BF16X3) ? 7 : 6;
  static constexpr int A_STAGE = BM * 128;
  static constexpr int B_STAGE = BNH * 128;
  static constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
  static constexpr int TMEM_COLS = 512;
  static constexpr int ACC_STRIDE = 256;
  static constexpr int NUM_THREADS = 320;
  static constexpr int EPI_WARPS = 8;
  static constexpr size_t SMEM_BYTES = 1024 + (size_t)STAGES * STAGE_BYTES + 256;
};

// tile_coords over pair tiles of 256 x BN (a.tiles_m counts 256-row tiles)
template <int MODE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(Tc2Cfg<MODE>::NUM_THREADS, 1)
    gett_tc2_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    const TcArgs a) {
  using Cfg = Tc2Cfg<MODE>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  uint8_t* smem = smem_raw + (((raw_addr + 1023u) & ~1023u) - raw_addr);
  uint8_t* sA = smem;
  uint8_t* sB = smem + Cfg::STAGES * Cfg::A_STAGE;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Cfg::STAGES * Cfg::STAGE_BYTES);
  uint64_t* full = bars;
  uint64_t* empty = bars + Cfg::STAGES;
  uint64_t* accf = bars + 2 * Cfg::STAGES;
  uint64_t* acce = accf + 2;
  uint64_t* drain = acce + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  const int num_tiles = a.tiles_m * a.tiles_n;
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  int32_t* status = a.status;

  if (threadIdx.x == 0) {
    for (int s = 0; s < Cfg::STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 2 * Cfg::EPI_WARPS);  // both CTAs' epilogue warps (used on the leader)
    }
    mbar_init(drain, 1);
    fence_mbar_init();
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
  }
  if (warp == 1) tmem_alloc_pair(tmem_slot, Cfg::TMEM_COLS);
  tc_fence_before();
  __syncwarp();
  cluster_sync();  // barriers of both CTAs initialised, TMEM allocated
  tc_fence_after();
  const uint32_t tbase = *tmem_slot;
  grid_dep_wait();  // packed operands written by the kernel before

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int tile = pair; tile < num_tiles && ok; tile += npairs) {
      int tm, tn;
      tile_coords(tile, a, tm, tn);
      for (int kb = 0; kb < a.num_kb; ++kb) {
        if (!mbar_wait(&empty[stage], phase ^ 1)) {
          record_error(status, 1);
          ok = false;
          break;
        }
        if (leader) mbar_arrive_expect_tx(&full[stage], 2 * Cfg::STAGE_BYTES);
        tma_load_2d_pair(sA + stage * Cfg::A_STAGE, &tmA, kb * 64, tm * 2 * Cfg::BM + rank * Cfg::BM,
                         &full[stage]);
        tma_load_2d_pair(sB + stage * Cfg::B_STAGE, &tmB, kb * 64, tn * Cfg::BN + rank * Cfg::BNH,
                         &full[stage]);
        if (++stage == Cfg::STAGES) {
          stage = 0;
          phase ^= 1;
        }
      }
    }
    // drain: the last MMA commits of every stage must have landed here
    // before this CTA may exit
    for (int s = 0; s < Cfg::STAGES; ++s) {
      (void)mbar_wait(&empty[stage], phase ^ 1);
      if (++stage == Cfg::STAGES) {
        stage = 0;
        phase ^= 1;
      }
    }
  } else if (warp == 1 && lane == 0 && leader) {
    // ---------------- MMA issuer (even CTA) ----------------
    constexpr uint32_t idesc = idesc_bf16_f32(2 * Cfg::BM, Cfg::BN);
    int stage = 0;
    uint32_t phase = 0;
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true, issued_any = false;
    for (int tile = pair; tile < num_tiles && ok; tile += npairs) {
      const int nkb = a.num_kb, K = a.K, ckb = a.chunk_kb;
      for (int kb0 = 0; kb0 < nkb && ok; kb0 += ckb) {
        if (!mbar_wait(&acce[acc], acc_phase ^ 1)) {
          record_error(status, 2);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d_tmem = tbase + (uint32_t)(acc * Cfg::ACC_STRIDE);
        uint32_t accumulate = 0;
        const int kend = (kb0 + ckb < nkb) ? kb0 + ckb : nkb;
        for (int kb = kb0; kb < kend; ++kb) {
          if (!mbar_wait(&full[stage], phase)) {
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
                tc_mma_f16_pair(d_tmem, ad + 2 * ks, bd + 2 * ks, idesc, accumulate);
                accumulate = 1;
              }
            }
          } else {
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
              if (kb * 32 + ks * 16 < K) {
                tc_mma_f16_pair(d_tmem, ad + 2 * ks, bd + 2 * ks, idesc, accumulate);  // ah*bh
                tc_mma_f16_pair(d_tmem, ad + 2 * ks, bd + 4 + 2 * ks, idesc, 1);       // ah*bl
                tc_mma_f16_pair(d_tmem, ad + 4 + 2 * ks, bd + 2 * ks, idesc, 1);       // al*bh
                accumulate = 1;
              }
            }
          }
          issued_any = true;
          tc_commit_pair(&empty[stage]);  // frees this stage in both CTAs
          if (++stage == Cfg::STAGES) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (!ok) break;
        tc_commit_pair(&accf[acc]);  // chunk ready for both CTAs' epilogues
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1;
        }
      }
    }
    if (!ok && issued_any) {
      tc_commit_pair(drain);
      (void)mbar_wait(drain, 0);
    }
  } else if (warp >= 2) {
    // ---------------- epilogue (both CTAs, own TMEM rows) ----------------
    const int q = warp & 3;
    const int h = (warp - 2) >> 2;
    constexpr int HC = Cfg::BN / 2;
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    auto release = [&](int b) {  // accumulator b free again (arrive on the even CTA)
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        if (leader)
          mbar_arrive(&acce[b]);
        else
          mbar_arrive_remote(&acce[b], 0);
      }
    };
    for (int tile = pair; tile < num_tiles && ok; tile += npairs) {
      int tm, tn;
      tile_coords(tile, a, tm, tn);
      const int64_t m = (int64_t)tm * 2 * Cfg::BM + rank * Cfg::BM + q * 32 + lane;
      const bool m_ok = m < a.M;
      const int64_t cmo = m_ok ? a.c_m_off[m] : 0;
      const int64_t n0 = (int64_t)tn * Cfg::BN + h * HC;
      const int64_t nlim = a.N - n0;
      const float alpha = a.alpha, beta = a.beta;
      if constexpr (MODE == TC_BF16) {
        if (!mbar_wait(&accf[acc], acc_phase)) {
          record_error(status, 3);
          break;
        }
        tc_fence_after();
        const uint32_t tsrc = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * Cfg::ACC_STRIDE + h * HC);
#pragma unroll 1
        for (int cc = 0; cc < HC; cc += 32) {
          uint32_t r[32];
          tmem_ld_32x32b_x32(tsrc + (uint32_t)cc, r);
          tmem_ld_wait();
          if (cc == HC - 32) release(acc);
          if (m_ok) {
            if (beta != 0.0f) {
              float old[32];
#pragma unroll
              for (int j = 0; j < 32; ++j)
                old[j] = (cc + j < nlim) ? a.C[cmo + __ldg(a.c_n_off + n0 + cc + j)] : 0.0f;
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (cc + j < nlim)
                  a.C[cmo + __ldg(a.c_n_off + n0 + cc + j)] =
                      fmaf(beta, old[j], alpha * __uint_as_float(r[j]));
            } else {
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (cc + j < nlim)
                  a.C[cmo + __ldg(a.c_n_off + n0 + cc + j)] = alpha * __uint_as_float(r[j]);
            }
          }
        }
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1;
        }
      } else {
        const int nchunks = (a.num_kb + a.chunk_kb - 1) / a.chunk_kb;
        float sum[HC];
        for (int ch = 0; ch < nchunks; ++ch) {
          if (!mbar_wait(&accf[acc], acc_phase)) {
            record_error(status, 3);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t tsrc = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * Cfg::ACC_STRIDE + h * HC);
#pragma unroll
          for (int cc = 0; cc < HC; cc += 16) {
            uint32_t r[16];
            tmem_ld_32x32b_x16(tsrc + (uint32_t)cc, r);
            tmem_ld_wait();
#pragma unroll
            for (int j = 0; j < 16; ++j)
              sum[cc + j] = (ch == 0) ? __uint_as_float(r[j])
                                      : __fadd_rn(sum[cc + j], __uint_as_float(r[j]));
          }
          release(acc);
          if (++acc == 2) {
            acc = 0;
            acc_phase ^= 1;
          }
        }
        if (!ok) break;
        if (m_ok) {
          if (beta != 0.0f) {
#pragma unroll
            for (int cc = 0; cc < HC; cc += 8) {
              float old[8];
#pragma unroll
              for (int j = 0; j < 8; ++j)
                old[j] = (cc + j < nlim) ? a.C[cmo + __ldg(a.c_n_off + n0 + cc + j)] : 0.0f;
#pragma unroll
              for (int j = 0; j < 8; ++j)
                if (cc + j < nlim)
                  a.C[cmo + __ldg(a.c_n_off + n0 + cc + j)] = fmaf(beta, old[j], alpha * sum[cc + j]);
            }
          } else {
#pragma unroll
            for (int j = 0; j < HC; ++j)
              if (j < nlim) a.C[cmo + __ldg(a.c_n_off + n0 + j)] = alpha * sum[j];
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncwarp();    // the .aligned cluster barrier needs converged warps
  cluster_sync();  // no CTA leaves while its peer may still signal its barriers
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tbase, Cfg::TMEM_COLS);
  }
}

}  // namespace tccg
