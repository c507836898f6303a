"""K-split (TCCG's k-parallel GETT with one private C per k-group and a final
sum, tccg/gett.py:755-781): slices of K on separate CTAs write FP32/FP64
partial sums, a reduction applies alpha/beta. Explicit split counts and the
automatic choice (few C tiles, long K) on both kernel families."""
import re

import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-6, "fp64": 1e-13, "bf16x3": 1e-5, "bf16": 1e-5}


def _case(lc, la, lb, sizes, alpha, beta, precision, tuning, seed):
    import torch
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    dt = np.float64 if precision == "fp64" else np.float32
    A = seeded_normal(ln.size_a, seed).astype(dt)
    B = seeded_normal(ln.size_b, seed + 1).astype(dt)
    C = seeded_normal(ln.size_c, seed + 2).astype(dt)
    if precision == "bf16":
        A = torch.from_numpy(A).bfloat16().float().numpy()
        B = torch.from_numpy(B).bfloat16().float().numpy()
    out, p = run_gpu(con, precision, A, B, C, tuning=tuning)
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    ks = int(re.search(r"ksplit=(\d+)", p.describe()).group(1))
    return out, ref, ks, p


@pytest.mark.parametrize("precision", ["bf16", "bf16x3", "fp32", "fp64"])
def test_explicit_split_matches_oracle(cuda, precision):
    # 300 x 200 C, K = 5000 in three slices; beta != 0 goes through the reduction
    out, ref, ks, _ = _case("mn", "mk", "kn", dict(m=300, n=200, k=5000), 1.25, -0.75,
                            precision, Tuning(ksplit=3), seed=81)
    assert ks == 3
    assert error_metrics(out, ref)["normwise"] <= TOL[precision]


@pytest.mark.parametrize("precision", ["bf16", "bf16x3", "fp32", "fp64"])
def test_automatic_split_for_long_k(cuda, precision):
    # a 20 x 30 C with K = 60000 (K spread over two modes): one C tile, so
    # the plan splits K over the idle SMs
    out, ref, ks, p = _case("ab", "akl", "lkb", dict(a=20, b=30, k=300, l=200), 1.0, 0.5,
                            precision, None, seed=82)
    assert ks > 1, p.describe()
    assert error_metrics(out, ref)["normwise"] <= TOL[precision]


def test_no_split_when_tiles_fill_the_gpu(cuda):
    _, _, ks, p = _case("mn", "mk", "kn", dict(m=4096, n=4096, k=256), 1.0, 0.0, "bf16x3",
                        None, seed=83)
    assert ks == 1, p.describe()


def test_split_with_ttgt(cuda):
    out, ref, ks, _ = _case("acbd", "aebk", "kedc", dict(a=8, b=6, c=5, d=4, e=50, k=60), 1.5,
                            0.5, "bf16x3", Tuning(method="ttgt", ksplit=2), seed=84)
    assert ks == 2
    assert error_metrics(out, ref)["normwise"] <= 1e-5
