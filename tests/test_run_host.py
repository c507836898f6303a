"""``Compiled.run_host``: end-to-end calls on host buffers, in one piece and
pipelined over slabs of C's last index (copies overlapping compute on two
copy streams). Results against the FP64 loop nest and the device call."""
import numpy as np
import pytest

from helpers import seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.api import Compiled
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

CASES = {
    # the benchmark's pattern: C's last index k is B's last index (B slabs
    # stream up with the compute)
    "cfg3_small": ("abcijk", "ambnc", "minjk", dict(a=16, b=8, c=8, i=16, j=4, k=6, m=32, n=16),
                   1.0, 0.0),
    # beta != 0: C slabs go up as well; C's last index d is in B but not last
    "beta": ("abcd", "aeb", "edc", dict(a=40, b=24, c=32, d=7, e=16), 1.5, 0.5),
    # C's last index belongs to A
    "in_a": ("nm", "km", "kn", dict(m=5, n=300, k=200), 1.0, -1.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
@pytest.mark.parametrize("slabs", [1, 3])
def test_run_host(cuda, name, precision, slabs):
    import torch
    lc, la, lb, sizes, alpha, beta = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, 111).astype(np.float32)
    B = seeded_normal(ln.size_b, 112).astype(np.float32)
    C = seeded_normal(ln.size_c, 113).astype(np.float32)
    c = Compiled(con, precision)
    Ah, Bh = torch.from_numpy(A).pin_memory(), torch.from_numpy(B).pin_memory()
    Ch = torch.from_numpy(C.copy()).pin_memory()
    for _ in range(2):  # twice: the cached device buffers and slab plans are reused
        Ch.copy_(torch.from_numpy(C))
        h2d, d2h = c.run_host(Ah, Bh, Ch, slabs=slabs)
        torch.cuda.synchronize()
    assert d2h == C.nbytes and h2d == A.nbytes + B.nbytes + (C.nbytes if beta else 0)
    out = Ch.double().numpy()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    tol = 1e-6 if precision == "fp32" else 1e-5
    assert error_metrics(out, ref)["normwise"] <= tol
    dev = c(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), torch.from_numpy(C).cuda())
    assert error_metrics(out, dev.double().cpu().numpy())["normwise"] <= tol
