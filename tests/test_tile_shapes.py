"""tcgen05 tile widths (tuning.tile_n, the autotuner's tile-shape choice):
every width computes each C element from the same bf16 stages with the same
MMAs in the same order, so results are equal bit for bit across widths, and
within the precision's bound of the FP64 oracle; a grouped run mixing
widths equals its per-item runs."""
import numpy as np
import pytest

from helpers import seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Plan, Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

CASES = {
    "cfg4_small": ("xyzw", "pxqw", "qzpy", dict(x=48, w=16, y=24, z=40, p=16, q=40)),
    "odd": ("pqr", "qs", "spr", dict(p=37, q=29, r=23, s=333)),
}


def _run(con, A, B, precision, tuning):
    import torch
    dt = torch.bfloat16 if precision == "bf16" else torch.float32
    p = Plan(con, precision=precision, tuning=tuning, dtype="bf16" if precision == "bf16" else None)
    C = torch.zeros(con.C0.num_elements(), device="cuda")
    p.run(torch.from_numpy(A).cuda().to(dt), torch.from_numpy(B).cuda().to(dt), C)
    torch.cuda.synchronize()
    assert p.status() == 0
    return C, p


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision,widths", [("bf16x3", (0, 128, 192)), ("bf16", (0, 128, 192, 256))])
def test_tile_widths_agree_bitwise(cuda, name, precision, widths):
    import torch
    lc, la, lb, sizes = CASES[name]
    con = make_contraction(lc, la, lb, sizes)
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, 7).astype(np.float32)
    B = seeded_normal(ln.size_b, 8).astype(np.float32)
    tc = 16 if precision == "bf16x3" else 1
    outs = []
    for w in widths:
        c, p = _run(con, A, B, precision, Tuning(variant=tc, ksplit=1, tail_split=-1, load=1 if precision == "bf16x3" else 0, tile_n=w))
        assert ("x%d " % (w or (192 if precision == "bf16x3" else 256))) in p.describe(), p.describe()
        outs.append(c)
    for c in outs[1:]:
        assert torch.equal(c, outs[0])
    if precision == "bf16x3":
        ref = ln.run(A.astype(np.float64), B.astype(np.float64), np.zeros(ln.size_c), 1.0, 0.0)
        assert error_metrics(outs[0].double().cpu().numpy(), ref)["normwise"] <= 1e-5


def test_unbuilt_width_is_an_error(cuda):
    from tccg_b200 import _native as N
    lc, la, lb, sizes = CASES["odd"]
    con = make_contraction(lc, la, lb, sizes)
    with pytest.raises(N.TccgError):
        Plan(con, precision="bf16x3", tuning=Tuning(variant=16, load=1, tile_n=256))
    with pytest.raises(N.TccgError):
        Plan(con, precision="bf16x3", tuning=Tuning(load=2, tile_n=192))


def test_grouped_run_mixes_widths(cuda):
    import torch
    from tccg_b200.grouped import Group
    from tccg_b200.workloads import batched_workload
    items = batched_workload(24, seed=13, fmax=3e8)
    cycle = [Tuning(load=1, tile_n=128), Tuning(load=1), Tuning(load=2), Tuning(variant=-1)]
    grp = Group(items, "bf16x3", tunings=[cycle[i % 4] for i in range(len(items))])
    g = torch.Generator(device="cuda").manual_seed(4)
    As = [torch.randn(c.A0.num_elements(), generator=g, device="cuda") for c in items]
    Bs = [torch.randn(c.B0.num_elements(), generator=g, device="cuda") for c in items]
    Cs = [torch.zeros(c.C0.num_elements(), device="cuda") for c in items]
    grp.bind(As, Bs, Cs)
    grp.run()
    torch.cuda.synchronize()
    grouped = [c.clone() for c in Cs]
    grp.run_per_item()
    torch.cuda.synchronize()
    for a, b in zip(grouped, Cs):
        assert torch.equal(a, b)
