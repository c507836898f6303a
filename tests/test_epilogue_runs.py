"""CPU replay of the tcgen05 epilogue's staged C stores
(tccg_b200/csrc/tc_gemm.cuh: store_runs), used when C's stride-one index is
the tile's first M mode of extent e0 < 32 directly followed in C by the first
N mode. Over a warp's 32 rows x 16 columns, at every m0 (multiple of 32) and
edge of M and N:

* every element (m, n) of the block inside C is stored exactly once, read
  from its own staging slot ([column][row], 33 floats per column);
* the lanes of one store instruction write 32 consecutive C addresses when
  the run is whole (rows ma + i of a run of e0, columns j, element i + e0 j),
  stepping (i, j) by 32 positions without a division.
"""
import pytest


def store_runs(m0, nb, ncols, e0, M, N):
    """[(instruction, lane, m, n, staging index)] in issue order, following
    the kernel's incremental (i, j) walk."""
    out = []
    rs = (m0 // e0) * e0
    while rs < m0 + 32:
        ma = max(rs, m0)
        mb = min(rs + e0, m0 + 32, M)
        L = mb - ma
        if L > 0:
            total = L * ncols
            di, dj = 32 % L, 32 // L
            for lane in range(32):
                i, j = lane % L, lane // L
                f, k = lane, 0
                while f < total:
                    assert (i, j) == (f % L, f // L)  # the division-free walk
                    n = nb + j
                    out.append(((rs, k, L), lane, ma + i, n, j * 33 + (ma - m0) + i))
                    i += di
                    j += dj
                    if i >= L:
                        i -= L
                        j += 1
                    f += 32
                    k += 1
        rs += e0
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
    mode): a full instruction's 32 lanes cover 32 consecutive addresses."""
    m_ext0 = e0

    def addr(m, n):  # first M mode of extent e0 at stride 1, then N at stride e0,
        # the rest of M after all of N (N = 64 columns)
        return (m % m_ext0) + e0 * n + e0 * 64 * (m // m_ext0)

    st = store_runs(0, 0, 16, e0, 4096, 64)
    by_instr = {}
    for ins, lane, m, n, _ in st:
        by_instr.setdefault(ins, []).append(addr(m, n))
    full = 0
    for (rs, k, L), addrs in by_instr.items():
        addrs.sort()
        if len(addrs) == 32 and L == e0:  # a whole run (partial runs sit at block edges)
            full += 1
            assert addrs == list(range(addrs[0], addrs[0] + 32))
    assert full > 0
