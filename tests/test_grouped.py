"""Grouped launch (configuration 5 pattern): many contractions of uneven
extents in one persistent launch, captured in a CUDA graph, against one
launch per contraction and the FP64 oracle."""
import numpy as np
import pytest

from oracle import LoopNest, error_metrics
from tccg_b200.workloads import batched_workload


def test_workload_generator_properties():
    items = batched_workload(64, seed=3)
    for c in items:
        c.validate()
        assert not c.loop_indices and len(c.k_indices) >= 1
        assert 2 <= len(c.C0.indices) <= 6
        assert all(8 <= i.size <= 128 for t in (c.A0, c.B0, c.C0) for i in t.indices)
        assert 1e6 / 2 <= c.flop_count(0.0) <= 1e10 * 2


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x3", "fp32", "bf16"])
def test_group_matches_oracle_and_per_item(cuda, precision):
    import torch
    from tccg_b200.grouped import Group
    items = batched_workload(24, seed=11, fmax=3e8)
    g = torch.Generator(device="cuda").manual_seed(5)
    As = [torch.randn(c.A0.num_elements(), generator=g, device="cuda") for c in items]
    Bs = [torch.randn(c.B0.num_elements(), generator=g, device="cuda") for c in items]
    Cs = [torch.empty(c.C0.num_elements(), device="cuda") for c in items]
    grp = Group(items, precision)
    grp.bind(As, Bs, Cs)
    grp.run()
    torch.cuda.synchronize()
    grouped = [c.clone() for c in Cs]
    for c in Cs:
        c.zero_()
    grp.run_per_item()
    torch.cuda.synchronize()
    for a, b in zip(grouped, Cs):
        assert torch.equal(a, b)
    # graph replay gives the same result
    for c in Cs:
        c.zero_()
    grp.capture()
    grp.replay()
    torch.cuda.synchronize()
    for a, b in zip(grouped, Cs):
        assert torch.equal(a, b)
    # FP64 oracle on sampled entries
    for con, A, B, C in zip(items, As, Bs, grouped):
        # FP32 summation error grows like 2^-24 sqrt(K) (K reaches ~1e6 here)
        tol = {"bf16x3": 1e-5, "fp32": 2 * 2.0 ** -24 * max(8.0, np.sqrt(con.sizeK)),
               "bf16": 1e-2}[precision]
        ln = LoopNest(con.C0.labels, con.A0.labels, con.B0.labels,
                      {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices})
        lins = np.linspace(0, ln.size_c - 1, 512).astype(np.int64)
        An, Bn = A.cpu().numpy(), B.cpu().numpy()
        if precision == "bf16":
            An = torch.from_numpy(An).bfloat16().float().numpy()
            Bn = torch.from_numpy(Bn).bfloat16().float().numpy()
        ref = ln.sample64(An, Bn, None, 1.0, 0.0, lins)
        m = error_metrics(C.cpu().double().numpy()[lins], ref)
        assert m["normwise"] <= tol, (str(con), m)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x3", "bf16", "fp64"])
def test_group_with_both_lanes_and_k_splits(cuda, precision):
    """Items forced onto both kernel families (BF16 precisions: CUDA-core
    lane and tensor-core lane in one group), with long-K items that split K
    and short-K items that skip the pack; grouped results equal the per-item
    plan runs bit for bit and match the FP64 oracle."""
    import torch
    from tccg_b200.grouped import Group
    from tccg_b200.plan import Tuning
    from tccg_b200.spec import make_contraction
    shapes = [
        ("ab", "akl", "lkb", dict(a=20, b=30, k=300, l=200)),          # long K, one tile: split
        ("abn", "abk", "kn", dict(a=300, b=40, n=12, k=20)),           # short K, skinny: direct
        ("mn", "mk", "kn", dict(m=700, n=500, k=1100)),
        ("pqr", "qs", "spr", dict(p=37, q=29, r=11, s=53)),
    ]
    items = [make_contraction(lc, la, lb, sz, 1.0, 0.0) for lc, la, lb, sz in shapes] * 2
    if precision == "fp64":
        tunings = None
    else:
        tunings = [Tuning(variant=-1)] * 4 + [Tuning(variant=16 if precision == "bf16x3" else 1)] * 4
    dt = torch.float64 if precision == "fp64" else torch.float32
    g = torch.Generator(device="cuda").manual_seed(9)
    As = [torch.randn(c.A0.num_elements(), generator=g, device="cuda", dtype=dt) for c in items]
    Bs = [torch.randn(c.B0.num_elements(), generator=g, device="cuda", dtype=dt) for c in items]
    if precision == "bf16":  # exact products on either kernel family
        As = [a.bfloat16().float() for a in As]
        Bs = [b.bfloat16().float() for b in Bs]
    Cs = [torch.zeros(c.C0.num_elements(), device="cuda", dtype=dt) for c in items]
    grp = Group(items, precision, tunings=tunings)
    descs = [p.describe() for p in grp.plans]
    if precision != "fp64":
        assert any("simt_gett" in d for d in descs) and any("gett_tc" in d for d in descs)
    assert any("ksplit=1 " not in d for d in descs)
    grp.bind(As, Bs, Cs)
    grp.capture()
    grp.replay()
    torch.cuda.synchronize()
    grouped = [c.clone() for c in Cs]
    for c in Cs:
        c.zero_()
    grp.run_per_item()
    torch.cuda.synchronize()
    for a, b in zip(grouped, Cs):
        assert torch.equal(a, b)
    tol = 1e-13 if precision == "fp64" else 1e-5
    for con, A, B, C in zip(items, As, Bs, grouped):
        ln = LoopNest(con.C0.labels, con.A0.labels, con.B0.labels,
                      {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices})
        ref = ln.run(A.double().cpu().numpy(), B.double().cpu().numpy(),
                     np.zeros(ln.size_c), 1.0, 0.0)
        assert error_metrics(C.double().cpu().numpy(), ref)["normwise"] <= tol, str(con)


@pytest.mark.gpu
def test_group_autotune_consults_the_cache_per_item(cuda, tmp_path):
    """Group(autotune=True): the first group tunes every item (GETT, no tail
    split) and stores the winners in the SQLite cache; a second group over
    the same items finds every item in the cache, builds the same plans, and
    its grouped run equals its per-item runs bit for bit."""
    import torch
    from tccg_b200.autotune import TuningDB, gpu_signature, tuning_key
    from tccg_b200.grouped import Group
    items = batched_workload(6, seed=21, fmax=2e8)
    db = str(tmp_path / "group.db")
    g1 = Group(items, "bf16x3", autotune=True, max_implementations=4, cache_path=db)
    assert g1.tune_stats == {"tuned": len(items)}
    g2 = Group(items, "bf16x3", autotune=True, max_implementations=4, cache_path=db)
    assert g2.tune_stats == {"hits": len(items)}
    store = TuningDB(db)
    for con, p1, p2 in zip(items, g1.plans, g2.plans):
        hit = store.lookup(tuning_key(con, "bf16x3", "f32", gpu_signature()) + "|grouped")
        assert hit is not None and hit[0].tail_split == -1
        assert p1.describe() == p2.describe()
        assert p2.tuning.key() == hit[0].key()
    g = torch.Generator(device="cuda").manual_seed(2)
    As = [torch.randn(c.A0.num_elements(), generator=g, device="cuda") for c in items]
    Bs = [torch.randn(c.B0.num_elements(), generator=g, device="cuda") for c in items]
    Cs = [torch.zeros(c.C0.num_elements(), device="cuda") for c in items]
    g2.bind(As, Bs, Cs)
    g2.run()
    torch.cuda.synchronize()
    grouped = [c.clone() for c in Cs]
    g2.run_per_item()
    torch.cuda.synchronize()
    for a, b in zip(grouped, Cs):
        assert torch.equal(a, b)
