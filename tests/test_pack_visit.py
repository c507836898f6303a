"""Tensor-core packing with a row visit order: when an operand's unit-stride
mode is not the first mode of its row order (M for the operand holding C's
stride-one index, N for the other), the pack walks the rows along the
unit-stride mode and writes each K-major row to its place. Parity with the
FP64 loop nest and with the CUDA-core kernel (which packs without it)."""
import dataclasses

import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Tuning, gett_view
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu


def _data(lc, la, lb, sizes, seed):
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, seed).astype(np.float32)
    B = seeded_normal(ln.size_b, seed + 1).astype(np.float32)
    C = seeded_normal(ln.size_c, seed + 2).astype(np.float32)
    return ln, A, B, C


@pytest.mark.parametrize("precision", ["bf16x3", "bf16"])
def test_visit_order_for_the_m_operand(cuda, precision):
    import torch
    # C's stride-one index a is M's first mode; A's stride-one index is b
    lc, la, lb, sizes = "abn", "bak", "kn", dict(a=37, b=45, n=70, k=300)
    con = make_contraction(lc, la, lb, sizes, 1.5, 0.5)
    ln, A, B, C = _data(lc, la, lb, sizes, 101)
    if precision == "bf16":
        A = torch.from_numpy(A).bfloat16().float().numpy()
        B = torch.from_numpy(B).bfloat16().float().numpy()
    out, p = run_gpu(con, precision, A, B, C, tuning=Tuning(variant=16))
    assert "visit a=1" in p.describe(), p.describe()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), 1.5, 0.5)
    assert error_metrics(out, ref)["normwise"] <= 1e-5
    cc, _ = run_gpu(con, precision, A, B, C, tuning=Tuning(variant=-1))
    assert error_metrics(out, cc)["normwise"] <= 1e-5


def test_visit_order_for_the_n_operand(cuda):
    # a hand-made view whose N order does not start with B's stride-one mode
    lc, la, lb, sizes = "anp", "ak", "pnk", dict(a=64, n=33, p=29, k=200)
    con = make_contraction(lc, la, lb, sizes, 1.0, 0.0)
    v = gett_view(con)
    assert v.b_n[0] == 1  # the library's own order starts with B's stride-one mode p
    v = dataclasses.replace(v, n=v.n[::-1], b_n=v.b_n[::-1], c_n=v.c_n[::-1])
    ln, A, B, C = _data(lc, la, lb, sizes, 102)
    out, p = run_gpu(con, "bf16x3", A, B, C, view=v, tuning=Tuning(variant=16))
    assert "visit a=0 b=1" in p.describe(), p.describe()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), 1.0, 0.0)
    assert error_metrics(out, ref)["normwise"] <= 1e-5
