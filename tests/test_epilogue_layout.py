"""The epilogues' staged C stores for a C whose stride-one index is the
first M mode, of extent e0 < 32, directly followed in C by the first N mode:
stores go through shared memory in runs of e0 m by 32 // e0 columns, in the
tcgen05 kernel (both loaders) and in the CUDA-core tile kernel.

With alpha = 1 and beta = 0 the result must equal, bit for bit, the same
contraction through TTGT, whose GEMM writes the contiguous C' with the
register epilogue (lanes along m) and whose transposition copies it exactly;
with beta != 0 it must be within the split-BF16x3 bound of the FP64 oracle.
Both tcgen05 loaders and both tensor-core precisions are covered.
"""
import numpy as np
import pytest

from helpers import seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Plan, Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

CASES = {
    # e0 = 10, one N mode at C-stride 10, K = 64
    "e10": ("ajb", "akb", "kj", dict(a=10, j=50, b=300, k=64)),
    # e0 = 19, N modes (j at C-stride 19, then l), K = 16 (one k-block)
    "e19_shortk": ("ajbl", "akb", "kjl", dict(a=19, j=7, b=40, l=30, k=16)),
    # e0 = 3 (a run of 3 by 10 columns per store)
    "e3": ("ajb", "akb", "kj", dict(a=3, j=200, b=500, k=40)),
}


def _data(ln, seed):
    return (seeded_normal(ln.size_a, seed).astype(np.float32),
            seeded_normal(ln.size_b, seed + 1).astype(np.float32),
            seeded_normal(ln.size_c, seed + 2).astype(np.float32))


def _run(con, A, B, C, precision, tuning, alpha, beta):
    import torch
    dt = torch.float64 if precision == "fp64" else torch.float32
    p = Plan(con, precision=precision, tuning=tuning, dtype="f64" if precision == "fp64" else "f32")
    dC = torch.from_numpy(C).cuda().to(dt)
    p.run(torch.from_numpy(A).cuda().to(dt), torch.from_numpy(B).cuda().to(dt), dC, alpha, beta)
    torch.cuda.synchronize()
    assert p.status() == 0
    return dC, p


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision,load", [("bf16x3", 1), ("bf16x3", 2), ("bf16", 0)])
def test_staged_stores_equal_ttgt(cuda, name, precision, load):
    import torch
    lc, la, lb, sizes = CASES[name]
    con = make_contraction(lc, la, lb, sizes)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 3)
    tc = 16 if precision == "bf16x3" else 1
    base = dict(variant=tc, ksplit=1, tail_split=-1)
    cg, pg = _run(con, A, B, C, precision, Tuning(load=load, **base), 1.0, 0.0)
    ct, pt = _run(con, A, B, C, precision, Tuning(method="ttgt", **base), 1.0, 0.0)
    assert "method=GETT" in pg.describe() and "method=TTGT" in pt.describe()
    assert torch.equal(cg, ct)
    if precision == "bf16x3":
        ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), 1.0, 0.0)
        assert error_metrics(cg.double().cpu().numpy(), ref)["normwise"] <= 1e-5


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("load", [1, 2])
def test_staged_stores_with_beta(cuda, name, load):
    lc, la, lb, sizes = CASES[name]
    con = make_contraction(lc, la, lb, sizes, 0.5, -1.25)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 4)
    cg, _ = _run(con, A, B, C, "bf16x3", Tuning(load=load, variant=16), 0.5, -1.25)
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), 0.5, -1.25)
    assert error_metrics(cg.double().cpu().numpy(), ref)["normwise"] <= 1e-5


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision,tuning", [("fp32", dict(shortk=-1)), ("fp32", dict(simt_tile=3)),
                                              ("fp64", dict(shortk=-1))])
def test_cuda_core_staged_stores_equal_ttgt(cuda, name, precision, tuning):
    """CUDA-core tile kernel: the staged run stores of GETT equal TTGT (whose
    GEMM writes the contiguous C' with quads along m) bit for bit, beta = 0;
    with beta != 0 they match the FP64 oracle at the FP32 / FP64 bound."""
    import torch
    lc, la, lb, sizes = CASES[name]
    con = make_contraction(lc, la, lb, sizes)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 5)
    t = dict(tuning, ksplit=1)
    cg, pg = _run(con, A, B, C, precision, Tuning(**t), 1.0, 0.0)
    ct, pt = _run(con, A, B, C, precision, Tuning(method="ttgt", **t), 1.0, 0.0)
    assert "simt_gett" in pg.describe(), pg.describe()
    assert torch.equal(cg, ct)
    con2 = make_contraction(lc, la, lb, sizes, 0.5, -1.25)
    cb, _ = _run(con2, A, B, C, precision, Tuning(**t), 0.5, -1.25)
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), 0.5, -1.25)
    tol = 1e-6 if precision == "fp32" else 1e-13
    assert error_metrics(cb.double().cpu().numpy(), ref)["normwise"] <= tol
