"""TMEM columns of the tcgen05 GETT kernel, on the CPU. The MMAs of a tile
stop at the tile's last column of C rounded up to 32 (N of the per-tile
instruction descriptor, tc_gemm.cuh). This restates that width and the two
epilogues' TMEM reads -- BF16: 32-column loads up to the warp's last group
that holds a column of C; BF16x3: 16-column loads below the warp's last
column -- and checks, for every count of columns left in a tile: the MMA
shape is one tcgen05.mma kind::f16 takes with M = 128 (N a multiple of 16,
16..256) and the descriptor's fields hold it; no epilogue load reads a column
the MMAs did not write; every column of C is read; an accumulator stays in
its 256-column half of the 512 allocated. The kernel itself is checked on a
B200 by the parity tests, whose N tails cover these widths."""
import pytest

BM = 128
ACC_STRIDE, TMEM_COLS = 256, 512
TILE_N = {"bf16": 256, "bf16x3": 192}


def idesc_bf16_f32(m, n):  # the descriptor built by common.cuh's idesc_bf16_f32
    return (1 << 4) | (1 << 7) | (1 << 10) | ((n >> 3) << 17) | ((m >> 4) << 24)


def mma_n(ncols, bn):
    return bn if ncols >= bn else (ncols + 31) // 32 * 32


def epilogue_reads(mode, ncols, bn):
    """TMEM columns each of the two column halves loads, per tile."""
    hc = bn // 2
    cols = set()
    for h in range(2):
        nlim = ncols - h * hc
        if mode == "bf16":
            last = hc - 32 if nlim >= hc else ((nlim - 1) // 32 * 32 if nlim > 0 else -32)
            for cc in range(0, last + 1, 32):
                cols.update(h * hc + cc + j for j in range(32))
        else:
            for cc in range(0, hc, 16):
                if cc < nlim:
                    cols.update(h * hc + cc + j for j in range(16))
    return cols


@pytest.mark.parametrize("mode", sorted(TILE_N))
def test_mma_width_covers_the_epilogue(mode):
    bn = TILE_N[mode]
    for ncols in range(1, bn + 40):
        n = mma_n(ncols, bn)
        assert n % 16 == 0 and 16 <= n <= 256
        d = idesc_bf16_f32(BM, n)
        assert (d >> 17) & 0x3F == n >> 3 and (d >> 24) & 0x1F == BM >> 4
        assert (d >> 23) & 1 == 0  # reserved bit between N and M stays clear
        reads = epilogue_reads(mode, ncols, bn)
        assert max(reads) < n, (ncols, n, max(reads))  # only columns the MMAs wrote
        assert set(range(min(ncols, bn))) <= reads  # every column of C is read
        for acc in range(2):  # both ping-pong accumulators inside the allocation
            assert acc * ACC_STRIDE + n <= min((acc + 1) * ACC_STRIDE, TMEM_COLS)


def test_full_tiles_keep_the_tile_width():
    for mode, bn in TILE_N.items():
        assert mma_n(bn, bn) == bn and mma_n(10 * bn, bn) == bn
        assert epilogue_reads(mode, bn, bn) == set(range(bn))
