"""CPU replay of the tcgen05 epilogue's staged C stores
(tccg_b200/csrc/tc_gemm.cuh: store_runs), used when C's stride-one index is
the tile's first M mode of extent e0 < 32 directly followed in C by the first
N mode. Over a warp's 32 rows x 16 columns, at every m0 (multiple of 32) and
edge of M and N:

* every element (m, n) of the block inside C is stored exactly once, read
  from its own staging slot ([column][row], 33 floats per column);
* the lanes of one store instruction write consecutive C addresses in runs
  (one run of e0 * q addresses per full instruction, q = 32 // e0).
"""
import pytest


def store_runs(m0, nb, ncols, e0, M, N):
    """[(instruction, lane, m, n, staging index)] in issue order."""
    q = 32 // e0
    out = []
    for lane in range(32):
        i, j = lane % e0, lane // e0
        if j >= q:
            continue
        step = 0
        rs = (m0 // e0) * e0
        while rs < m0 + 32:
            m = rs + i
            if m0 <= m < m0 + 32 and m < M:
                c = j
                k = 0
                while c < ncols:
                    n = nb + c
                    if n < N:  # the kernel's column count already stops at N
                        out.append(((rs, k), lane, m, n, c * 33 + (m - m0)))
                    c += q
                    k += 1
            rs += e0
            step += 1
    return out


@pytest.mark.parametrize("e0", [2, 3, 5, 10, 16, 19, 31])
@pytest.mark.parametrize("m0,M", [(0, 4096), (32, 4096), (96, 100), (128, 150), (4064, 4070)])
@pytest.mark.parametrize("nb,ncols,N", [(0, 16, 1000), (48, 16, 60), (64, 7, 71)])
def test_each_element_once_from_its_slot(e0, m0, M, nb, ncols, N):
    ncols = min(ncols, N - nb)
    st = store_runs(m0, nb, ncols, e0, M, N)
    got = [(m, n) for _, _, m, n, _ in st]
    want = [(m, n) for m in range(m0, min(m0 + 32, M)) for n in range(nb, nb + ncols)]
    assert sorted(got) == sorted(want)
    for _, _, m, n, idx in st:
        assert idx == (n - nb) * 33 + (m - m0) and 0 <= idx < 16 * 33


@pytest.mark.parametrize("e0", [2, 3, 5, 10, 16, 19, 31])
def test_store_instructions_are_contiguous(e0):
    """C[m + e0 * n] layout (the first M mode of extent e0, then the first N
    mode): a full instruction's lanes cover e0 * q consecutive addresses."""
    q = 32 // e0
    m_ext0 = e0

    def addr(m, n):  # first M mode of extent e0 at stride 1, then N at stride e0,
        # the rest of M after all of N (N = 64 columns)
        return (m % m_ext0) + e0 * n + e0 * 64 * (m // m_ext0)

    st = store_runs(0, 0, 16, e0, 4096, 64)
    by_instr = {}
    for ins, lane, m, n, _ in st:
        by_instr.setdefault(ins, []).append(addr(m, n))
    full = 0
    for addrs in by_instr.values():
        addrs.sort()
        if len(addrs) == e0 * q:
            full += 1
            assert addrs == list(range(addrs[0], addrs[0] + e0 * q))
    assert full > 0
