"""Narrow CUDA-core tiles (FP32 accumulation): 128 x 32 for contractions with
a small N and 32 x 128 for a small M, 4 x 4 per thread. Same k order and
epilogue arithmetic as the 128 x 128 tile, so without a k-split the results
are bitwise equal to it; all against the FP64 loop nest. Cases: packed and
pack-free loads (gathered along rows or, where an operand's unit stride is a
K mode, along k), tails in M, N and K, k-splits, beta, the automatic choice,
and a grouped run that mixes the three shapes."""
import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Plan, Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

# (C, A, B, extents, alpha, beta, tile) -- tile = Tuning.simt_tile
CASES = {
    # small N, long K, N below the tile (20 of 32)
    "narrow_n": ("mn", "mk", "kn", dict(m=1000, n=20, k=700), 1.0, 0.0, 2),
    # small N spread over two modes, beta, C's stride-one index in M
    "narrow_n_modes": ("abn", "akb", "nk", dict(a=37, b=29, n=45, k=300), 0.5, -1.0, 2),
    # small N, A's unit stride along k (pack-free: A gathered along k)
    "narrow_n_kfast": ("mn", "km", "kn", dict(m=1000, n=20, k=700), 1.0, 0.0, 2),
    # small M, N over several tiles with a tail (pack-free: both along k)
    "narrow_m": ("mn", "km", "kn", dict(m=11, n=900, k=500), 1.0, 0.5, 3),
    # small M from two modes, K a product of two modes with a tail
    "narrow_m_modes": ("abnp", "akbl", "nlkp", dict(a=5, b=4, n=60, p=7, k=13, l=9), 2.0, 0.0, 3),
}


# pack-free narrow tiles: which operands are gathered along k
GATHER_K = {"narrow_n": "gather_k a=0 b=1", "narrow_n_kfast": "gather_k a=1 b=1",
            "narrow_m": "gather_k a=1 b=1", "narrow_n_modes": "gather_k a=0 b=0"}


def _data(lc, la, lb, sizes, seed):
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, seed).astype(np.float32)
    B = seeded_normal(ln.size_b, seed + 1).astype(np.float32)
    C = seeded_normal(ln.size_c, seed + 2).astype(np.float32)
    return ln, A, B, C


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("direct", [-1, 1])
@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_narrow_tile_matches_square_and_oracle(cuda, name, direct, precision):
    lc, la, lb, sizes, alpha, beta, tile = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln, A, B, C = _data(lc, la, lb, sizes, 151)
    v = -1 if precision == "bf16x3" else 0  # bf16x3 on the CUDA cores
    narrow, pn = run_gpu(con, precision, A, B, C,
                         tuning=Tuning(variant=v, simt_tile=tile, ksplit=1, direct=direct))
    square, ps = run_gpu(con, precision, A, B, C,
                         tuning=Tuning(variant=v, simt_tile=1, ksplit=1, direct=direct))
    want = "tile=128x32x16" if tile == 2 else "tile=32x128x16"
    assert want in pn.describe() and "tile=128x128x16" in ps.describe(), pn.describe()
    if direct == 1 and name in GATHER_K:
        assert GATHER_K[name] in pn.describe(), pn.describe()
    assert np.array_equal(narrow, square)
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(narrow, ref)["normwise"] <= 1e-6


@pytest.mark.parametrize("name", ["narrow_n", "narrow_m"])
def test_narrow_tile_with_k_split(cuda, name):
    lc, la, lb, sizes, alpha, beta, tile = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln, A, B, C = _data(lc, la, lb, sizes, 152)
    out, p = run_gpu(con, "fp32", A, B, C, tuning=Tuning(simt_tile=tile, ksplit=5))
    assert "ksplit=5" in p.describe()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(out, ref)["normwise"] <= 1e-6


def test_automatic_shape(cuda):
    # the tile kernel's own choice (the skinny kernel, which may take these
    # shapes, held off)
    off = Tuning(skinny=-1)
    small_n = make_contraction("mn", "mk", "kn", dict(m=4096, n=16, k=1024))
    assert "tile=128x32x16" in Plan(small_n, precision="fp32", tuning=off).describe()
    small_m = make_contraction("mn", "mk", "kn", dict(m=24, n=4096, k=1024))
    assert "tile=32x128x16" in Plan(small_m, precision="fp32", tuning=off).describe()
    square = make_contraction("mn", "mk", "kn", dict(m=1000, n=1000, k=64))
    assert "tile=128x128x16" in Plan(square, precision="fp32").describe()
    # FP64 keeps its one tile
    assert "tile=128x64x8" in Plan(small_n, precision="fp64").describe()


def test_group_mixing_shapes(cuda):
    import torch
    from tccg_b200.grouped import Group
    items = [make_contraction(*CASES[n][:4], CASES[n][4], CASES[n][5]) for n in sorted(CASES)]
    items.append(make_contraction("mn", "mk", "kn", dict(m=300, n=260, k=200), 1.0, 0.0))
    tunings = [Tuning(simt_tile=CASES[n][6]) for n in sorted(CASES)] + [Tuning(simt_tile=1)]
    g = torch.Generator(device="cuda").manual_seed(7)
    As = [torch.randn(c.A0.num_elements(), generator=g, device="cuda") for c in items]
    Bs = [torch.randn(c.B0.num_elements(), generator=g, device="cuda") for c in items]
    Cs = [torch.randn(c.C0.num_elements(), generator=g, device="cuda") for c in items]
    C0 = [c.clone() for c in Cs]
    grp = Group(items, "fp32", tunings=tunings)
    descs = [p.describe() for p in grp.plans]
    assert any("128x32x16" in d for d in descs) and any("32x128x16" in d for d in descs)
    assert any("128x128x16" in d for d in descs)
    grp.bind(As, Bs, Cs)
    grp.run()
    torch.cuda.synchronize()
    grouped = [c.clone() for c in Cs]
    for c, c0 in zip(Cs, C0):
        c.copy_(c0)
    grp.run_per_item()
    torch.cuda.synchronize()
    for con, gr, pi, a, b, c0 in zip(items, grouped, Cs, As, Bs, C0):
        assert torch.equal(gr, pi)
        ln = LoopNest(con.C0.labels, con.A0.labels, con.B0.labels,
                      {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices})
        ref = ln.run(a.double().cpu().numpy(), b.double().cpu().numpy(), c0.double().cpu().numpy(),
                     con.alpha, con.beta)
        assert error_metrics(gr.double().cpu().numpy(), ref)["normwise"] <= 1e-6
