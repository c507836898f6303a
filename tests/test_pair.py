"""The CTA-pair tensor-core kernel (tcgen05 cta_group::2, 256-row tiles):
parity with the FP64 loop nest and with the one-SM kernel on shapes that
exercise partial pair tiles (rows of only the even CTA valid), partial B
halves, K tails, several K chunks, the persistent tile loop and alpha/beta."""
import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

CASES = {
    # plain GEMM with tails in M (700 = 2*256 + 188), N and K
    "gemm_tails": ("mn", "mk", "kn", dict(m=700, n=500, k=1100), 1.0, 0.0, 0),
    # the same on two clusters only: every cluster walks several pair tiles
    "persistent": ("mn", "mk", "kn", dict(m=700, n=500, k=1100), 1.5, -0.5, 4),
    # only rows of the even CTA valid (M = 100)
    "short_m": ("mn", "mk", "kn", dict(m=100, n=300, k=200), 1.0, 1.0, 0),
    # the benchmark's index pattern at reduced extents
    "cfg3_small": ("abcijk", "ambnc", "minjk",
                   dict(a=16, b=8, c=4, i=16, j=4, k=8, m=32, n=24), 2.4, 1.1, 0),
    # operand swap (B holds C's stride-one index), odd extents
    "odd_swap": ("pqr", "qs", "spr", dict(p=37, q=29, r=11, s=53), 0.75, -0.5, 0),
}


def _run(name, precision, seed):
    import torch
    lc, la, lb, sizes, alpha, beta, max_ctas = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, seed).astype(np.float32)
    B = seeded_normal(ln.size_b, seed + 1).astype(np.float32)
    C = seeded_normal(ln.size_c, seed + 2).astype(np.float32)
    if precision == "bf16":  # exact products on the tensor cores
        A = torch.from_numpy(A).bfloat16().float().numpy()
        B = torch.from_numpy(B).bfloat16().float().numpy()
    pair, p = run_gpu(con, precision, A, B, C, tuning=Tuning(pair=1, max_ctas=max_ctas))
    assert "kernel=gett_tc2<" in p.describe(), p.describe()
    assert p.status() == 0
    single, _ = run_gpu(con, precision, A, B, C, tuning=Tuning(max_ctas=max_ctas))
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    return pair, single, ref


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", ["bf16", "bf16x3"])
def test_pair_kernel_vs_fp64(cuda, name, precision):
    pair, single, ref = _run(name, precision, seed=71)
    m = error_metrics(pair, ref)
    assert m["normwise"] <= 1e-5, m
    # same tile arithmetic as the one-SM kernel: equal up to the order in
    # which the tensor cores sum within a k-block
    scale = np.abs(ref).max()
    assert np.abs(pair - single).max() <= 1e-5 * max(scale, 1.0)
