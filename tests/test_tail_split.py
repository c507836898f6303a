"""Tail split of the tcgen05 tile order: when the C tiles fill the persistent
grid a whole number of times plus a short tail, the tail's tiles run as k
slices (tile-compact FP32 partial sums, added by tc_tail_reduce_kernel with
alpha/beta) while the other tiles keep all of K. Against the FP64 loop nest
and the same contraction without the split (tuning ksplit = 1), with M, N and
K tails and beta != 0. The shapes assume 148 SMs (B200)."""
import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Plan, Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

# (C, A, B, extents, alpha, beta, precision, describe tag "tail=<tiles>x<slices>")
CASES = {
    # BF16x3, 10 x 15 = 150 tiles of 128 x 192: 2 tail tiles in 2 slices
    "x3_even": ("mn", "mk", "kn", dict(m=1280, n=2880, k=1024), 1.0, 0.0, "bf16x3", "tail=2x2"),
    # tails in M, N and K (K = 1100: 35 k-blocks, slices of 18)
    "x3_tails": ("mn", "km", "kn", dict(m=1250, n=2800, k=1100), 0.75, -0.5, "bf16x3", "tail=2x2"),
    # BF16, 10 x 15 = 150 tiles of 128 x 256: 2 tail tiles in 4 slices
    "bf16": ("mn", "mk", "nk", dict(m=1280, n=3840, k=2048), 1.5, 0.5, "bf16", "tail=2x4"),
    # multi-mode C and operands
    "modes": ("abnp", "akb", "kpn", dict(a=40, b=32, n=48, p=60, k=1024), 1.0, 1.0, "bf16x3",
              "tail=2x2"),
}


def _inputs(lc, la, lb, sizes, seed):
    import torch
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, seed).astype(np.float32)
    B = seeded_normal(ln.size_b, seed + 1).astype(np.float32)
    C = seeded_normal(ln.size_c, seed + 2).astype(np.float32)
    return ln, A, B, C


@pytest.mark.parametrize("name", sorted(CASES))
def test_tail_split(cuda, name):
    import torch
    lc, la, lb, sizes, alpha, beta, precision, tag = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln, A, B, C = _inputs(lc, la, lb, sizes, 161)
    if precision == "bf16":  # exact products on the tensor cores
        A = torch.from_numpy(A).bfloat16().float().numpy()
        B = torch.from_numpy(B).bfloat16().float().numpy()
    v = 16 if precision == "bf16x3" else 1  # the tensor cores
    split, ps = run_gpu(con, precision, A, B, C, tuning=Tuning(variant=v))
    whole, pw = run_gpu(con, precision, A, B, C, tuning=Tuning(variant=v, ksplit=1))
    assert tag in ps.describe() and "tail=0x1" in pw.describe(), ps.describe()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(split, ref)["normwise"] <= 1e-5
    # the split only regroups the k sums of the tail tiles
    assert error_metrics(split, whole)["normwise"] <= 1e-5


def test_no_tail_split_when_rounds_are_full(cuda):
    # 148 tiles exactly, and 300 tiles (tail 4 of 148 but K too short to split)
    full = make_contraction("mn", "mk", "kn", dict(m=128 * 4, n=192 * 37, k=1024))
    assert "tail=0x1" in Plan(full, precision="bf16x3", tuning=Tuning(variant=16)).describe()
    short_k = make_contraction("mn", "mk", "kn", dict(m=128 * 10, n=192 * 15, k=256))
    assert "tail=0x1" in Plan(short_k, precision="bf16x3", tuning=Tuning(variant=16)).describe()
