"""The allocation-free split-BF16x3 entry point (tccg_gett_bf16x3_noalloc).

It exists for callers that must not allocate device memory (HBM reserved up
front by a framework's caching allocator, or a latency-critical loop that
cannot afford cudaMalloc's device synchronisation): its scratch is a static
device array of the library. These tests call it through the C ABI and check
its output against the regular entry point (tccg_plan_run with a workspace)
and the FP64 oracle, on two calls in a row (the second call must not be
affected by what the first left in the shared scratch), and check that a
contraction larger than the static scratch is refused with an error code.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from helpers import seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200 import _native as N
from tccg_b200.plan import Plan, Tuning, gett_view, native_desc
from tccg_b200.spec import make_contraction

CASES = [
    # configuration 1 pattern (all 48), beta = 0
    ("abij", "ima", "mjb", dict(a=48, b=48, i=48, j=48, m=48), 1.0, 0.0),
    # odd extents, operand swap, beta != 0 (C is read), K spanning 3 chunks
    ("pqr", "qs", "spr", dict(p=37, q=29, r=11, s=1200), 0.75, -0.5),
]


def _noalloc(con, dA, dB, dC, alpha, beta):
    import torch
    d = native_desc(gett_view(con))
    rc = N.lib().tccg_gett_bf16x3_noalloc(ctypes.byref(d), ctypes.c_void_p(dA.data_ptr()),
                                          ctypes.c_void_p(dB.data_ptr()),
                                          ctypes.c_void_p(dC.data_ptr()), alpha, beta,
                                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc)


@pytest.mark.gpu
def test_noalloc_matches_plan_run_twice(cuda):
    import torch
    for i, (lc, la, lb, sizes, alpha, beta) in enumerate(CASES):
        con = make_contraction(lc, la, lb, sizes, alpha, beta)
        ln = LoopNest(lc, la, lb, sizes)
        A = seeded_normal(ln.size_a, 31 + i).astype(np.float32)
        B = seeded_normal(ln.size_b, 41 + i).astype(np.float32)
        C = seeded_normal(ln.size_c, 51 + i).astype(np.float32)
        dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
        c_plan = torch.from_numpy(C).cuda()
        c_free = torch.from_numpy(C).cuda()
        # the allocation-free entry point never splits K and always runs the
        # tensor-core kernel: compare with the plan's schedule of the same kind
        Plan(con, precision="bf16x3", tuning=Tuning(ksplit=1, variant=16)).run(dA, dB, c_plan,
                                                                               alpha, beta)
        _noalloc(con, dA, dB, c_free, alpha, beta)
        torch.cuda.synchronize()
        out_plan = c_plan.double().cpu().numpy()
        out_free = c_free.double().cpu().numpy()
        ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
        assert error_metrics(out_free, ref)["normwise"] <= 1e-5
        # same kernels on the same data: agreement far inside the 1e-5 bound
        assert error_metrics(out_free, out_plan)["normwise"] <= 1e-7


@pytest.mark.gpu
def test_noalloc_rejects_oversized(cuda):
    con = make_contraction("mn", "km", "kn", dict(m=32768, n=32768, k=4096))
    d = native_desc(gett_view(con))
    rc = N.lib().tccg_gett_bf16x3_noalloc(ctypes.byref(d), ctypes.c_void_p(16), ctypes.c_void_p(16),
                                          ctypes.c_void_p(16), 1.0, 0.0, None)
    assert rc == N.ERR_WORKSPACE
    assert b"static scratch" in N.lib().tccg_last_error()
