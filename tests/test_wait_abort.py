"""The abort path of the tcgen05 kernel's bounded waits, made to run out on
purpose without any fault: tccg_debug_inject_timeout arms a one-shot trigger
under which the producer does not load one k-block of one tile and every
device wait is bounded by a short limit. The MMA warp's wait for that block
runs out, the CTA records a status code, waits for its copies and MMAs in
flight, releases its tensor memory and returns.

Checked: the run returns (no hang), tccg_plan_status reports a
TCCG_DEVSTAT_TIMEOUT_* code, and the next ordinary run on the same plan and
device is bitwise equal to a run made before the trigger (the device context
and the SM's tensor memory are usable again).
"""
import numpy as np
import pytest

from tccg_b200 import _native as N
from tccg_b200.plan import Plan, Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

TIMEOUT_CODES = {1, 2, 3}  # TCCG_DEVSTAT_TIMEOUT_PRODUCER / _MMA / _EPILOGUE


@pytest.mark.parametrize("precision,tile", [("bf16x3", 0), ("bf16x3", 150), ("bf16", 3)])
def test_wait_runs_out_and_plan_recovers(cuda, precision, tile):
    import torch
    # configuration 1 pattern at 64: M = N = 4096, K = 64 -> 32 x 22 tiles of
    # 128 x 192 (BF16x3) or 32 x 16 of 128 x 256 (BF16): several rounds of
    # the persistent grid
    sizes = dict(a=64, b=64, i=64, j=64, m=64)
    con = make_contraction("abij", "ima", "mjb", sizes)
    g = torch.Generator(device="cuda").manual_seed(7)
    A = torch.randn(64 ** 3, generator=g, device="cuda")
    B = torch.randn(64 ** 3, generator=g, device="cuda")
    tc = 16 if precision == "bf16x3" else 1  # tensor cores (default BF16x3 chunk)
    p = Plan(con, precision=precision, tuning=Tuning(ksplit=1, tail_split=-1, variant=tc))
    assert "gett_tc<" in p.describe()
    ws = torch.empty(p.workspace_bytes, dtype=torch.uint8, device="cuda")
    C_good = torch.zeros(64 ** 4, device="cuda")
    p.run(A, B, C_good, workspace=ws)
    torch.cuda.synchronize()
    assert p.status() == 0

    C_bad = torch.full((64 ** 4,), float("nan"), device="cuda")
    N.check(N.lib().tccg_debug_inject_timeout(tile, 100))
    p.run(A, B, C_bad, workspace=ws)
    torch.cuda.synchronize()
    code = p.status()
    assert code in TIMEOUT_CODES, code
    # the aborting CTA left its tiles unwritten (NaN), the others wrote theirs
    assert torch.isnan(C_bad).any()
    written = ~torch.isnan(C_bad)
    assert written.any()
    assert torch.equal(C_bad[written], C_good[written])
    assert p.status() == 0  # read and cleared

    C_again = torch.zeros(64 ** 4, device="cuda")
    p.run(A, B, C_again, workspace=ws)
    torch.cuda.synchronize()
    assert p.status() == 0
    assert torch.equal(C_again, C_good)
    assert np.isfinite(C_again.cpu().numpy()).all()
