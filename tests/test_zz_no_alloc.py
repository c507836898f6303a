"""The allocation-free split-BF16x3 entry point (tccg_gett_bf16x3_noalloc).

It exists for callers that must not allocate device memory (HBM reserved up
front by a framework's caching allocator, or a latency-critical loop that
cannot afford cudaMalloc's device synchronisation): its scratch is a static
device array of the library. These tests call it through the C ABI and check
its output against the regular entry point (tccg_plan_run with a workspace)
and the FP64 oracle, on two calls in a row (the second call must not be
affected by what the first left in the shared scratch, and must not change
the device's free memory), check that its status query reports a device
wait that was made to run out, and check that a contraction larger than the
static scratch is refused with an error code.
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


def _case_data(i):
    lc, la, lb, sizes, alpha, beta = CASES[i]
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, 31 + i).astype(np.float32)
    B = seeded_normal(ln.size_b, 41 + i).astype(np.float32)
    C = seeded_normal(ln.size_c, 51 + i).astype(np.float32)
    return make_contraction(lc, la, lb, sizes, alpha, beta), ln, A, B, C, alpha, beta


def _status():
    s = ctypes.c_int32(-1)
    N.check(N.lib().tccg_gett_bf16x3_noalloc_status(ctypes.byref(s)))
    return int(s.value)


@pytest.mark.gpu
def test_noalloc_matches_plan_run_twice(cuda):
    """Each case against the plan path and the FP64 oracle; then both cases
    once more in the same order, so that each second call follows a call of
    a different size that left its own tables and packed operands in the
    shared scratch: the outputs are bitwise equal to the first ones, the
    status word stays 0, and the device's free memory does not move (the
    entry point allocates nothing)."""
    import torch
    data = [_case_data(i) for i in range(len(CASES))]
    dev = [(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), torch.from_numpy(C).cuda())
           for _, _, A, B, C, _, _ in data]
    first = []
    for (con, ln, A, B, C, alpha, beta), (dA, dB, dC0) in zip(data, dev):
        c_plan = dC0.clone()
        c_free = dC0.clone()
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
        first.append(c_free)
    assert _status() == 0
    again = [dC0.clone() for _, _, dC0 in dev]
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for (con, _, _, _, _, alpha, beta), (dA, dB, _), c in zip(data, dev, again):
        _noalloc(con, dA, dB, c, alpha, beta)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    for a, b in zip(first, again):
        assert torch.equal(a, b)
    assert _status() == 0


@pytest.mark.gpu
def test_noalloc_status_reports_a_wait_that_ran_out(cuda):
    """A bounded device wait made to run out (tccg_debug_inject_timeout: one
    tile's first k-block is not loaded, waits bounded by 100 ms): the call
    returns, the status query reports the timeout code once, and the next
    call on the same scratch is bitwise equal to an undisturbed one."""
    import torch
    con, _, A, B, C, alpha, beta = _case_data(0)
    dA, dB, dC0 = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), torch.from_numpy(C).cuda()
    good = dC0.clone()
    _noalloc(con, dA, dB, good, alpha, beta)
    assert _status() == 0
    bad = dC0.clone()
    N.check(N.lib().tccg_debug_inject_timeout(0, 100))
    _noalloc(con, dA, dB, bad, alpha, beta)
    code = _status()
    assert code in (1, 2, 3), code  # TCCG_DEVSTAT_TIMEOUT_*
    assert not torch.equal(bad, good)  # the aborting CTA's tiles were not written
    assert _status() == 0  # read and cleared
    after = dC0.clone()
    _noalloc(con, dA, dB, after, alpha, beta)
    torch.cuda.synchronize()
    assert _status() == 0
    assert torch.equal(after, good)


@pytest.mark.gpu
def test_noalloc_rejects_oversized(cuda):
    con = make_contraction("mn", "km", "kn", dict(m=32768, n=32768, k=4096))
    d = native_desc(gett_view(con))
    rc = N.lib().tccg_gett_bf16x3_noalloc(ctypes.byref(d), ctypes.c_void_p(16), ctypes.c_void_p(16),
                                          ctypes.c_void_p(16), 1.0, 0.0, None)
    assert rc == N.ERR_WORKSPACE
    assert b"static scratch" in N.lib().tccg_last_error()
