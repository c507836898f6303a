"""The tcgen05 gather loader (tuning.load = 2): split-BF16x3 with the
producer warps reading the caller's FP32 tensors through the offset tables
(no packing pass).

Each case runs the same contraction with the gather loader and with the
packing pass + TMA loads (tuning.load = 1) at the same accumulation chunk:
both feed the tensor cores bitwise identical bf16 hi/lo stages and add the
same MMAs in the same order, so C must be equal bit for bit; and C must be
within the split-BF16x3 bound (normwise 1e-5) of the FP64 oracle. Cases cover
the three read schedules (along rows, along k, 16-byte k quads), odd extents
and tile edges, the operand swap, beta != 0, K tails, several accumulation
chunks, k-split and tail split, an operand that is not 16-byte aligned, and
a grouped run mixing gather and packed items.
"""
import numpy as np
import pytest

from helpers import seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Plan, Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

CASES = {
    # A's stride-one index is an M index (rows), B's is a K index (k quads)
    "cfg1": ("abij", "ima", "mjb", dict(a=48, b=48, i=48, j=48, m=48), 1.0, 0.0),
    # odd extents, operand swap, beta != 0, K = 53 (tail of a k-block)
    "odd_swap": ("pqr", "qs", "spr", dict(p=37, q=29, r=11, s=53), 0.75, -0.5),
    # configuration 4 pattern: the unit stride of both operands is a K mode
    "cfg4": ("xyzw", "pxqw", "qzpy", dict(x=24, w=16, y=20, z=16, p=16, q=40), 1.0, 0.0),
    # long K over several accumulation chunks, N a single column tile
    "longk": ("mn", "km", "kn", dict(m=300, n=70, k=1700), 1.0, 0.0),
    # K extents not a multiple of 4 on the unit-stride K mode (no k quads)
    "k_odd": ("abij", "mnai", "jbmn", dict(a=40, b=36, i=9, j=7, m=13, n=7), 1.0, 0.25),
    # matrix-vector and outer product
    "matvec": ("a", "ak", "k", dict(a=300, k=77), 1.0, 0.0),
    "outer": ("ab", "a", "b", dict(a=33, b=65), 1.5, 0.0),
}


def _data(ln, seed):
    A = seeded_normal(ln.size_a, seed).astype(np.float32)
    B = seeded_normal(ln.size_b, seed + 1).astype(np.float32)
    C = seeded_normal(ln.size_c, seed + 2).astype(np.float32)
    return A, B, C


def _run(con, A, B, C, tuning, alpha, beta, offset=0):
    import torch
    p = Plan(con, precision="bf16x3", tuning=tuning)
    dA = torch.zeros(A.size + offset, device="cuda")
    dA[offset:] = torch.from_numpy(A).cuda()
    dA = dA[offset:]
    dB = torch.from_numpy(B).cuda()
    dC = torch.from_numpy(C).cuda()
    p.run(dA, dB, dC, alpha, beta)
    torch.cuda.synchronize()
    assert p.status() == 0
    return dC, p


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("chunk", [16, 3])
def test_gather_equals_packed_and_oracle(cuda, name, chunk):
    import torch
    lc, la, lb, sizes, alpha, beta = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 61)
    base = dict(variant=chunk, ksplit=1, tail_split=-1)
    cg, pg = _run(con, A, B, C, Tuning(load=2, **base), alpha, beta)
    cp, pp = _run(con, A, B, C, Tuning(load=1, **base), alpha, beta)
    assert "gather" in pg.describe() and "gather" not in pp.describe()
    assert torch.equal(cg, cp), (pg.describe(), pp.describe())
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(cg.double().cpu().numpy(), ref)["normwise"] <= 1e-5


@pytest.mark.parametrize("tuning", [dict(ksplit=3), dict(ksplit=0)])
def test_gather_k_splits(cuda, tuning):
    """Explicit k-split (partial sums + reduction) and the automatic choice
    (k-split or tail split) with the gather loader: equal to the packed path
    under the same split."""
    import torch
    lc, la, lb, sizes, alpha, beta = CASES["longk"]
    sizes = dict(sizes, m=700, n=900, k=3000)
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 71)
    cg, pg = _run(con, A, B, C, Tuning(load=2, variant=16, **tuning), alpha, beta)
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(cg.double().cpu().numpy(), ref)["normwise"] <= 1e-5, pg.describe()


def test_gather_unaligned_operand(cuda):
    """An operand 4 bytes off a 16-byte boundary: the k-quad schedule falls
    back to 4-byte copies along k, with the same result."""
    import torch
    lc, la, lb, sizes, alpha, beta = CASES["cfg1"]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 81)
    t = Tuning(load=2, variant=16, ksplit=1, tail_split=-1)
    c0, _ = _run(con, A, B, C, t, alpha, beta)
    c1, _ = _run(con, A, B, C, t, alpha, beta, offset=1)
    assert torch.equal(c0, c1)


def test_grouped_mixes_gather_and_packed_items(cuda):
    """A group whose items use both tensor-core loaders (and the CUDA cores):
    each item equal to its own plan run bit for bit."""
    import torch
    from tccg_b200.grouped import Group
    from tccg_b200.workloads import batched_workload
    items = batched_workload(48, seed=3)
    g = torch.Generator(device="cuda").manual_seed(9)
    As = [torch.randn(c.A0.num_elements(), generator=g, device="cuda") for c in items]
    Bs = [torch.randn(c.B0.num_elements(), generator=g, device="cuda") for c in items]
    Cs = [torch.zeros(c.C0.num_elements(), device="cuda") for c in items]
    cycle = [Tuning(load=2), Tuning(load=1), Tuning(variant=-1), Tuning()]
    grp = Group(items, "bf16x3", tunings=[cycle[i % 4] for i in range(len(items))])
    kinds = {("gather" in p.describe(), "simt" in p.describe()) for p in grp.plans}
    assert {(True, False), (False, False), (False, True)} <= kinds, kinds
    grp.bind(As, Bs, Cs)
    grp.run()
    torch.cuda.synchronize()
    grouped = [c.clone() for c in Cs]
    grp.run_per_item()
    torch.cuda.synchronize()
    for con, a, b in zip(items, grouped, Cs):
        assert torch.equal(a, b), str(con)
