"""Grouped launch (configuration 5 pattern): many contractions of uneven
extents in one persistent launch, captured in a CUDA graph, against one
launch per contraction and the FP64 oracle."""
import random

import numpy as np
import pytest

from oracle import LoopNest, error_metrics
from tccg_b200.workloads import batched_workload, random_contraction


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
