"""CPU replay of the tcgen05 gather loader's index arithmetic
(tccg_b200/csrc/tc_gemm.cuh: gather_issue, gather_convert) over whole
k-blocks of random operand shapes, for each read schedule:

* every copy lands inside its staging slot, no staging element is written
  twice, and exactly the elements (r < rows in the operand, k < K) are copied,
  each from src[row_off[r] + k_off[k]];
* 16-byte copies start on 16-byte boundaries of the slot;
* the conversion reads each (row, 8-k group) of the slot once and writes
  every 16-byte chunk of the 128-row x 128-byte stage exactly once, at chunk
  c ^ (row & 7) of its row (the 128-byte swizzle of a TMA load into a
  1024-byte aligned stage), hi halves in chunks 0-3 and lo halves in 4-7;
* each 8-lane phase of a conversion store touches 8 distinct 16-byte bank
  groups (no shared-memory bank conflict).
"""
import numpy as np
import pytest

BM = BN = 128
STG_LD = 36
ROWS, K_, KQUAD = 0, 1, 2


def gather_ld(read):
    return 33 if read == ROWS else 36


def replay_issue(read, nr, kn, rows):
    """Staging element index -> (row, k) copied there, following gather_issue
    for one operand (rows = BM or BN; nr valid rows; kn valid k)."""
    ld = gather_ld(read)
    written = {}
    quads = []
    for ptid in range(128):
        pw, lane = ptid >> 5, ptid & 31
        if read == ROWS:
            for k in range(kn):
                for r in range(ptid, nr, 128):
                    written.setdefault(r * ld + k, []).append((r, k))
        elif read == K_:
            if lane < kn:
                for r in range(pw, nr, 4):
                    written.setdefault(r * ld + lane, []).append((r, lane))
        else:
            kq, sub = 4 * (lane & 7), lane >> 3
            if kq + 3 < kn:
                for r in range(pw * 4 + sub, nr, 16):
                    quads.append(r * ld + kq)
                    for e in range(4):
                        written.setdefault(r * ld + kq + e, []).append((r, kq + e))
            else:
                e = 0
                while e < 4 and kq + e < kn:
                    for r in range(pw * 4 + sub, nr, 16):
                        written.setdefault(r * ld + kq + e, []).append((r, kq + e))
                    e += 1
    return written, quads, ld


@pytest.mark.parametrize("read", [ROWS, K_, KQUAD])
@pytest.mark.parametrize("nr,kn", [(128, 32), (37, 32), (128, 13), (5, 7), (1, 1), (100, 30)])
def test_issue_copies_each_element_once(read, nr, kn):
    written, quads, ld = replay_issue(read, nr, kn, BM)
    assert all(len(v) == 1 for v in written.values())
    got = {v[0] for v in written.values()}
    assert got == {(r, k) for r in range(nr) for k in range(kn)}
    # inside the operand's part of the slot (rows x 36 floats)
    assert max(written) < BM * STG_LD and min(written) >= 0
    for off, ((r, k),) in written.items():
        assert off == r * ld + k and k < 32
    # 16-byte copies: the slot base is 16-byte aligned, so the float offset
    # must be a multiple of 4
    assert all(q % 4 == 0 for q in quads)


def test_operand_b_region_does_not_overlap_a():
    # B's staging rows start at float BM * 36 of the slot; A's last element
    # is below that for both row strides
    for read in (ROWS, K_, KQUAD):
        written, _, _ = replay_issue(read, BM, 32, BM)
        assert max(written) < BM * 36


def replay_convert():
    """(row, k8) read from the slot and the stage byte offsets written, per
    conversion unit, following gather_convert (BM + BN rows, 8 k per unit)."""
    reads, writes, phases = [], [], []
    for ptid in range(128):
        pw, lane = ptid >> 5, ptid & 31
        k8 = lane >> 3
        for rg in range(pw, (BM + BN) // 8, 4):
            r = rg * 8 + (lane & 7)
            o = 1 if r >= BM else 0
            rr = r - (BM if o else 0)
            reads.append((o, rr, k8))
            sw = rr & 7
            hi = rr * 128 + ((k8 ^ sw) << 4)
            lo = rr * 128 + (((4 + k8) ^ sw) << 4)
            writes.append((o, hi, rr, k8))
            writes.append((o, lo, rr, 4 + k8))
            phases.append((pw, rg, lane, o, hi, lo))
    return reads, writes, phases


def test_convert_covers_the_stage_in_tma_swizzle_order():
    reads, writes, _ = replay_convert()
    assert sorted(reads) == sorted((o, r, k8) for o in (0, 1) for r in range(128) for k8 in range(4))
    for o in (0, 1):
        offs = sorted(w[1] for w in writes if w[0] == o)
        assert offs == list(range(0, 128 * 128, 16))  # every 16-byte chunk once
    # TMA's 128-byte swizzle: logical chunk c of row r at physical chunk
    # c ^ (r % 8) of that row (address bits 4-6 XOR bits 7-9, base 1024-aligned)
    for o, off, r, c in writes:
        assert off // 128 == r
        assert (off % 128) // 16 == c ^ (r % 8)


def test_convert_stores_are_bank_conflict_free():
    _, _, phases = replay_convert()
    by_instr = {}
    for pw, rg, lane, o, hi, lo in phases:
        by_instr.setdefault((pw, rg), []).append((lane, hi, lo))
    for lanes in by_instr.values():
        lanes.sort()
        for which in (1, 2):
            for ph in range(4):  # 8 lanes per phase of a 16-byte store
                groups = {(lanes[ph * 8 + i][which] % 128) // 16 for i in range(8)}
                assert len(groups) == 8


def test_convert_reads_are_bank_conflict_free():
    """Scalar reads (row stride 33) and 16-byte reads (row stride 36) of one
    8-lane phase spread over distinct banks."""
    for ld in (33, 36):
        for rg in range(32):
            for ph in range(4):
                lanes = range(ph * 8, ph * 8 + 8)
                if ld == 36:
                    # lanes of a phase: rows rg*8 + (lane & 7) with one k8
                    # per 8 lanes; each reads 4 consecutive words
                    banks = []
                    for lane in lanes:
                        r, k8 = (rg * 8 + (lane & 7)) % 128, lane >> 3
                        w = r * ld + k8 * 8
                        banks += [(w + e) % 32 for e in range(4)]
                    assert len(set(banks)) == 32
            if ld == 33:
                for e in range(8):
                    banks = [((rg * 8 + (lane & 7)) % 128 * 33 + (lane >> 3) * 8 + e) % 32
                             for lane in range(32)]
                    assert len(set(banks)) == 32


def test_smem_budget():
    stages, slots = 2, 3
    total = 1024 + stages * (BM + BN) * 128 + slots * (BM + BN) * STG_LD * 4 + (BM + BN) * 8 + 256
    assert total <= 227 * 1024
