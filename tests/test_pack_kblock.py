"""Tensor-core packing with k-block tiles: when an operand's unit-stride mode
is a K mode other than the first one of the contraction's K order, the pack
reads runs along that mode (kb_lo * kb_run consecutive k per tile, kb_rows
rows), reorders them in shared memory and writes K-major rows. Parity with
the FP64 loop nest and with the CUDA-core kernel (which packs without them)
for BF16x3 and BF16, on either operand, with K tails, runs that wrap into
the next value of the higher K modes, and row tails; element-wise and
16-byte (4 consecutive u per copy) tiles."""
import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

CASES = {
    # configuration 4's pattern at reduced extents: B = B[k1, j1, k0, j0]
    # has unit stride on k1, the second K mode (K order k0, k1: A's, the
    # larger operand, leads)
    "cfg4_small": (["i0", "j0", "j1", "i1"], ["k0", "i0", "k1", "i1"], ["k1", "j1", "k0", "j0"],
                   dict(i0=16, i1=24, j0=8, j1=40, k0=32, k1=32), "b=32x32x4"),
    # three K modes with odd extents: tiles of 5 x 24 = 120 k, K = 360 (BF16x3
    # pads to 384: the last tile runs past K), 32 rows per tile over M = 70
    "odd": (["m", "n"], ["k0", "m", "k1", "k2"], ["k1", "n", "k0", "k2"],
            dict(m=70, n=50, k0=5, k1=24, k2=3), "b=5x24x32"),
    # runs of 64 over an extent of 100: tiles wrap into the next k2
    "wrap": (["m", "n"], ["k0", "k1", "m", "k2"], ["k1", "k0", "k2", "n"],
             dict(m=300, n=130, k0=16, k1=100, k2=2), "b=16x64x4"),
    # B larger: K order k1, k0, k2 and A's unit-stride k0 comes second, after
    # 100 values of k1 (runs of 10)
    "long_lo": (["m", "n"], ["k0", "k1", "m", "k2"], ["k1", "k0", "k2", "n"],
                dict(m=60, n=130, k0=16, k1=100, k2=2), "a=100x10x4"),
    # unit stride on the third K mode
    "third": (["m", "n"], ["k1", "m", "k0", "k2"], ["k2", "k0", "k1", "n"],
              dict(m=90, n=75, k0=4, k1=16, k2=12), "b=64x12x5"),
}


# tiles that move 16-byte quads along u (kb_lo, run and u's extent multiples
# of 4, u's stride +1, aligned quads)
QUAD = {"cfg4_small": True, "odd": False, "wrap": True, "long_lo": False, "third": True}


def _run(name, precision, seed):
    import torch
    lc, la, lb, sizes, tag = CASES[name]
    con = make_contraction(lc, la, lb, sizes, 1.25, 0.5)
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, seed).astype(np.float32)
    B = seeded_normal(ln.size_b, seed + 1).astype(np.float32)
    C = seeded_normal(ln.size_c, seed + 2).astype(np.float32)
    if precision == "bf16":  # exact products on the tensor cores
        A = torch.from_numpy(A).bfloat16().float().numpy()
        B = torch.from_numpy(B).bfloat16().float().numpy()
    out, p = run_gpu(con, precision, A, B, C, tuning=Tuning(variant=16))
    assert "kernel=gett_tc<" in p.describe(), p.describe()
    assert "kblock " in p.describe() and tag in p.describe(), p.describe()
    assert (" x16B" in p.describe()) == QUAD[name], p.describe()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), 1.25, 0.5)
    cc, _ = run_gpu(con, precision, A, B, C, tuning=Tuning(variant=-1))
    return out, ref, cc


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", ["bf16x3", "bf16"])
def test_kblock_pack(cuda, name, precision):
    out, ref, cc = _run(name, precision, seed=141)
    assert error_metrics(out, ref)["normwise"] <= 1e-5
    assert error_metrics(out, cc)["normwise"] <= 1e-5

