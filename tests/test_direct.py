"""The CUDA-core kernel without a packing pass ("direct": operands gathered
from the user's tensors through the offset tables): parity with the packed
schedule and with the FP64 loop nest, on coalesced and strided layouts, K
tails, k-splits and alpha/beta; the automatic choice for short K."""
import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

CASES = {
    # configuration 2's pattern at reduced extents: short K, beta = 1
    "cfg2_small": ("abcd", "aeb", "edc", dict(a=40, b=24, c=32, d=20, e=16), 1.0, 1.0),
    # skinny N, K spread over two modes, odd extents
    "skinny": ("vqub", "qeu", "ebv", dict(v=37, q=11, u=29, b=5, e=13), 0.5, 0.0),
    # A's stride-one index is contracted (strided gather along m)
    "a_k_fast": ("mn", "km", "kn", dict(m=300, n=70, k=45), 1.0, -1.0),
    # swap: B holds C's stride-one index
    "swap": ("pqr", "qs", "spr", dict(p=37, q=29, r=11, s=53), 0.75, -0.5),
    # longer K with a tail (K = 1000 is not a multiple of the k-tile)
    "long_k": ("mn", "mk", "kn", dict(m=200, n=150, k=1000), 1.0, 0.0),
}


def _inputs(lc, la, lb, sizes, dt, seed):
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, seed).astype(dt)
    B = seeded_normal(ln.size_b, seed + 1).astype(dt)
    C = seeded_normal(ln.size_c, seed + 2).astype(dt)
    return ln, A, B, C


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp32", "fp64", "bf16x3"])
def test_direct_matches_packed_and_oracle(cuda, name, precision):
    lc, la, lb, sizes, alpha, beta = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    dt = np.float64 if precision == "fp64" else np.float32
    ln, A, B, C = _inputs(lc, la, lb, sizes, dt, seed=91)
    # bf16x3 reaches the CUDA-core kernel through variant < 0
    v = -1 if precision == "bf16x3" else 0
    direct, pd = run_gpu(con, precision, A, B, C, tuning=Tuning(direct=1, variant=v))
    packed, pp = run_gpu(con, precision, A, B, C, tuning=Tuning(direct=-1, variant=v))
    assert "pack=none" in pd.describe() and "pack=MN" in pp.describe()
    # same k order and tile arithmetic: identical results
    assert np.array_equal(direct, packed)
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    tol = 1e-13 if precision == "fp64" else 1e-6
    assert error_metrics(direct, ref)["normwise"] <= tol


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_direct_with_k_split(cuda, precision):
    lc, la, lb, sizes, alpha, beta = "ab", "akl", "lkb", dict(a=20, b=30, k=30, l=40), 1.0, 0.5
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    dt = np.float64 if precision == "fp64" else np.float32
    ln, A, B, C = _inputs(lc, la, lb, sizes, dt, seed=92)
    out, p = run_gpu(con, precision, A, B, C, tuning=Tuning(direct=1, ksplit=4))
    assert "ksplit=4" in p.describe() and "pack=none" in p.describe()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(out, ref)["normwise"] <= (1e-13 if precision == "fp64" else 1e-6)


def test_automatic_choice(cuda):
    from tccg_b200.plan import Plan
    # skinny C, short K: the operands are a large share of the traffic
    skinny = make_contraction("abn", "abk", "kn", dict(a=300, b=400, n=12, k=20))
    assert "pack=none" in Plan(skinny, precision="fp32").describe()
    # configuration 2: C dominates, packing the small operands costs nothing
    cfg2 = make_contraction("abcd", "aeb", "edc", dict(a=96, b=96, c=96, d=96, e=16))
    assert "pack=MN" in Plan(cfg2, precision="fp32").describe()
    long_k = make_contraction("mn", "mk", "kn", dict(m=512, n=512, k=4096))
    assert "pack=MN" in Plan(long_k, precision="fp32").describe()
    # BF16 rounding needs the pack
    assert "pack=MN" in Plan(skinny, precision="bf16", tuning=Tuning(variant=-1)).describe()
