"""Tile mapping of the tcgen05 tail split, on the CPU. A restatement of the
plan-time choice (tccg_abi.cu, the tail split in the tcgen05 layout step:
full rounds, tail tiles, slices of ``tail_kb`` k-blocks) and of the
kernel's ``tile_coords`` / ``split_coords`` (tc_gemm.cuh), replayed on fixed
and random shapes: every (C tile, k-block) pair is computed exactly once, no
slice is empty, every slice's partial-sum block lies inside the workspace,
the slices of the tail fill at most one round of the persistent grid, and
the tiles split are the ones the raster order puts last. The kernel itself is
checked against the FP64 loop nest on a B200 by test_tail_split.py; the
cost check that decides whether the split pays does not change the mapping
and is left out here."""
import random

import pytest


def cdiv(a, b):
    return -(-a // b)


def tile_coords(tile, tiles_m, tiles_n, raster):
    if raster < 0:  # groups of -raster tile columns, n fastest
        R = -raster
        group = R * tiles_m
        gid = tile // group
        first_n = gid * R
        gn = min(tiles_n - first_n, R)
        r = tile - gid * group
        return r // gn, first_n + r % gn
    group = raster * tiles_n
    gid = tile // group
    first_m = gid * raster
    gm = min(tiles_m - first_m, raster)
    r = tile - gid * group
    return first_m + r % gm, r // gm


def plan(M, N, K, x3=True, ctas=148, chunk_kb=16, raster=8):
    bn = 192 if x3 else 256
    num_kb = cdiv(K, 32) if x3 else cdiv(K, 64)
    tiles_m, tiles_n = cdiv(M, 128), cdiv(N, bn)
    mn = tiles_m * tiles_n
    p = dict(tiles_m=tiles_m, tiles_n=tiles_n, mn=mn, num_kb=num_kb, bn=bn, raster=raster,
             ctas=ctas, full=0, split=1, tail_kb=0)
    if mn > ctas:
        full = mn // ctas * ctas
        tail = mn - full
        min_kb = chunk_kb if x3 else 8
        want = min(ctas // tail, num_kb // min_kb) if tail > 0 else 0
        if tail > 0 and 2 * tail <= ctas and want >= 2:
            per = cdiv(num_kb, want)
            p.update(full=full, split=cdiv(num_kb, per), tail_kb=per)
    return p


def replay(p):
    """(tm, tn) -> sorted k-block ranges, over every tile index of the grid."""
    mn, full, split, tail_kb, num_kb = p["mn"], p["full"], p["split"], p["tail_kb"], p["num_kb"]
    tail = mn - full
    num_tiles = full + tail * split if split > 1 else mn
    partial_elems = split * tail * p["bn"] * 128
    cover = {}
    for local in range(num_tiles):
        if split > 1 and local >= full:
            u = local - full
            z, t = u // tail, u % tail
            tm, tn = tile_coords(full + t, p["tiles_m"], p["tiles_n"], p["raster"])
            kb0 = z * tail_kb
            kb1 = min(kb0 + tail_kb, num_kb)
            assert kb1 > kb0, "empty slice"
            block = (z * tail + t) * p["bn"] * 128  # the slice's tile-compact partial sums
            assert 0 <= block and block + p["bn"] * 128 <= partial_elems
        else:
            tm, tn = tile_coords(local, p["tiles_m"], p["tiles_n"], p["raster"])
            kb0, kb1 = 0, num_kb
        cover.setdefault((tm, tn), []).append((kb0, kb1))
    return cover


def check(p):
    cover = replay(p)
    assert len(cover) == p["mn"]
    assert all(0 <= tm < p["tiles_m"] and 0 <= tn < p["tiles_n"] for tm, tn in cover)
    for key, ranges in cover.items():
        ranges.sort()
        pos = 0
        for a, b in ranges:
            assert a == pos, (key, ranges)
            pos = b
        assert pos == p["num_kb"], (key, ranges)
    if p["split"] > 1:
        tail = p["mn"] - p["full"]
        assert tail * p["split"] <= p["ctas"]  # the slices fill at most one round
        last = {tile_coords(p["full"] + t, p["tiles_m"], p["tiles_n"], p["raster"])
                for t in range(tail)}
        assert last == {k for k, r in cover.items() if len(r) > 1}
    return p["split"] > 1


def test_backward_gemms_of_configuration_4():
    # dA / dB of configuration 4 (M = 1024, N = K = 4096): 176 tiles of
    # 128 x 192 on 148 SMs, the 28 tail tiles in 5 slices of 26 k-blocks
    p = plan(1024, 4096, 4096)
    assert (p["mn"] - p["full"], p["split"], p["tail_kb"]) == (28, 5, 26) and check(p)
    # transposed: 192 tiles, 44 tail tiles in 3 slices
    p = plan(4096, 1024, 4096)
    assert (p["mn"] - p["full"], p["split"]) == (44, 3) and check(p)
    # BF16 (128 x 256 tiles): 128 tiles fit one round, no split
    p = plan(1024, 4096, 4096, x3=False)
    assert p["split"] == 1 and not check(p)


def test_tail_split_test_shapes():
    # the GPU test's cases: 150 tiles, 2 tail tiles in 2 (BF16x3) or 4 (BF16) slices
    p = plan(1280, 2880, 1024)
    assert (p["mn"] - p["full"], p["split"]) == (2, 2) and check(p)
    p = plan(1280, 3840, 2048, x3=False)
    assert (p["mn"] - p["full"], p["split"]) == (2, 4) and check(p)
    p = plan(1250, 2800, 1100)  # K = 1100: 35 k-blocks, slices of 18
    assert (p["split"], p["tail_kb"]) == (2, 18) and check(p)


@pytest.mark.parametrize("seed", range(4))
def test_random_shapes(seed):
    rng = random.Random(seed)
    split = 0
    for _ in range(600):
        p = plan(rng.randint(1, 5000), rng.randint(1, 9000), rng.randint(1, 20000),
                 x3=rng.random() < 0.5, raster=rng.choice([1, 4, 8, 16]),
                 ctas=rng.choice([148, 132, 100]))
        split += check(p)
    assert split > 20  # the split case is exercised, not just the plain tile order


@pytest.mark.parametrize("raster", [8, 1, 5, 16, -8, -1, -3])
@pytest.mark.parametrize("tiles_m,tiles_n", [(1, 1), (7, 3), (13, 40), (64, 9), (3, 100)])
def test_tile_order_is_a_permutation(raster, tiles_m, tiles_n):
    """Both loop orders (groups of tile rows, raster > 0; groups of tile
    columns, raster < 0) visit every (tm, tn) of the grid exactly once, and
    a group's tiles are consecutive in the order."""
    seen = [tile_coords(t, tiles_m, tiles_n, raster) for t in range(tiles_m * tiles_n)]
    assert sorted(seen) == [(m, n) for m in range(tiles_m) for n in range(tiles_n)]
    R = abs(raster)
    key = (lambda mn: mn[0] // R) if raster > 0 else (lambda mn: mn[1] // R)
    groups = [key(x) for x in seen]
    assert groups == sorted(groups)
