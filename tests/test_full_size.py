"""The five workload configurations at their full sizes on the GPU: sampled
entries against the FP64 oracle, plus size-independent properties (exact
scaling by powers of two, beta = 1 accumulation, agreement of the grouped
and per-item runs of the 256-item workload).

Configuration 1: C[a,b,i,j] = A[i,m,a] * B[m,j,b], all 48.
Configuration 2: C[a,b,c,d] = A[a,e,b] * B[e,d,c] + C, 96 / e = 16.
Configuration 3: C[a,b,c,i,j,k] = A[a,m,b,n,c] * B[m,i,n,j,k], 32 / m = n = 64.
Configuration 4: C[i0,j0,j1,i1] = A[k0,i0,k1,i1] * B[k1,j1,k0,j0], 64 / k = 32.
Configuration 5: 256 mixed contractions (tccg_b200.workloads.batched_workload).
"""
import numpy as np
import pytest

from oracle import LoopNest, error_metrics
from tccg_b200 import parse_text

pytestmark = pytest.mark.gpu

CFG = {
    1: "C[a,b,i,j] = A[i,m,a] * B[m,j,b]\na=48\nb=48\ni=48\nj=48\nm=48\n",
    2: "C[a,b,c,d] = A[a,e,b] * B[e,d,c] + C[a,b,c,d]\na=96\nb=96\nc=96\nd=96\ne=16\n",
    3: ("C[a,b,c,i,j,k] = A[a,m,b,n,c] * B[m,i,n,j,k]\n"
        "a = 32\nb = 32\nc = 32\ni = 32\nj = 32\nk = 32\nm = 64\nn = 64\n"),
    4: "C[i0,j0,j1,i1] = A[k0,i0,k1,i1] * B[k1,j1,k0,j0]\ni0=64\ni1=64\nj0=64\nj1=64\nk0=32\nk1=32\n",
}
TOL = {"fp32": 1e-6, "bf16x3": 1e-5, "fp64": 1e-13}


def _loopnest(con):
    return LoopNest(con.C0.labels, con.A0.labels, con.B0.labels,
                    {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices})


def _data(con, dt, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn(con.A0.num_elements(), generator=g, device="cuda", dtype=dt)
    B = torch.randn(con.B0.num_elements(), generator=g, device="cuda", dtype=dt)
    C = torch.randn(con.C0.num_elements(), generator=g, device="cuda", dtype=dt)
    return A, B, C


@pytest.mark.parametrize("cfg", [1, 2, 3, 4])
@pytest.mark.parametrize("precision", ["bf16x3", "fp32"])
def test_configuration_sampled_vs_fp64(cuda, cfg, precision):
    import torch
    from tccg_b200.api import Compiled
    con = parse_text(CFG[cfg])
    A, B, C0 = _data(con, torch.float32, 200 + cfg)
    c = Compiled(con, precision)
    C = C0.clone()
    c(A, B, C)
    torch.cuda.synchronize()
    assert c.plan.status() == 0
    ln = _loopnest(con)
    lins = np.unique(np.linspace(0, ln.size_c - 1, 4096).astype(np.int64))
    An, Bn = A.cpu().numpy(), B.cpu().numpy()
    Cn = C0.cpu().numpy() if con.beta != 0 else None
    ref = ln.sample64(An, Bn, Cn, con.alpha, con.beta, lins)
    m = error_metrics(C.cpu().double().numpy()[lins], ref)
    # FP32 sums grow their error like 2^-24 sqrt(K) (K = 4096 at configuration 3)
    tol = TOL[precision] if precision != "fp32" else 2 * 2.0 ** -24 * max(8.0, np.sqrt(con.sizeK))
    assert m["normwise"] <= tol, m


def _sampled_metrics(con, A, B, C0, out, n=4096):
    """error_metrics of ``out`` on n entries spread over C against the FP64
    oracle evaluated on the values of A, B (and C0 when beta != 0) as given
    (bf16 operands are widened exactly to FP32 first)."""
    import torch
    ln = _loopnest(con)
    lins = np.unique(np.linspace(0, ln.size_c - 1, n).astype(np.int64))
    wide = lambda t: (t.float() if t.dtype == torch.bfloat16 else t).cpu().numpy()
    Cn = wide(C0) if con.beta != 0 else None
    ref = ln.sample64(wide(A), wide(B), Cn, con.alpha, con.beta, lins)
    return error_metrics(out[torch.from_numpy(lins).to(out.device)].double().cpu().numpy(), ref)


# BF16 products of bf16 operands are exact in FP32; what remains is the FP32
# accumulation. On the tensor cores each MMA (16 k) adds into the FP32
# accumulator with truncation, up to one ulp (2^-23 relative) per add,
# biased toward zero, so over K/16 adds the normwise error stays below
# (K/16) * 2^-23; on the CUDA cores it is FP32 round-to-nearest FFMA.
def _bf16_bound(K):
    return max(1e-5, (K / 16) * 2.0 ** -23)


@pytest.mark.parametrize("method", ["gett", "ttgt"])
def test_configuration2_bf16_inputs(cuda, method):
    """Configuration 2 with BF16 operands (bf16 precision: bf16 products,
    FP32 accumulation; beta = 1 with C preloaded), GETT and TTGT: 4096
    entries against the FP64 oracle of the same bf16 values."""
    import torch
    from tccg_b200.api import Compiled
    from tccg_b200.plan import Tuning
    con = parse_text(CFG[2])
    A, B, C0 = _data(con, torch.float32, 210)
    Ab, Bb = A.bfloat16(), B.bfloat16()
    c = Compiled(con, "bf16", Tuning(method=method), dtype="bf16")
    C = C0.clone()
    c(Ab, Bb, C)
    torch.cuda.synchronize()
    assert c.plan.status() == 0
    m = _sampled_metrics(con, Ab, Bb, C0, C)
    assert m["normwise"] <= _bf16_bound(con.sizeK), m
    assert m["tccg_equal_pass"], m


@pytest.mark.parametrize("precision", ["bf16", "fp64"])
def test_configuration3_bf16_fp64_vs_oracle(cuda, precision):
    """Configuration 3 at full size (M = N = 32768, K = 4096) in BF16 (bf16
    operands, tensor cores) and in FP64 (DFMA): 4096 entries against the FP64
    oracle. FP64 sums of 4096 products: normwise within 1e-13, and TCCG's
    equal() at its double tolerance 1e-9 (tccg.py:869-873)."""
    import torch
    from tccg_b200.api import Compiled
    con = parse_text(CFG[3])
    if precision == "fp64":
        A, B, _ = _data(con, torch.float64, 220)
        c = Compiled(con, "fp64")
    else:
        A, B, _ = _data(con, torch.float32, 221)
        A, B = A.bfloat16(), B.bfloat16()
        c = Compiled(con, "bf16", dtype="bf16")
    C = c(A, B)
    torch.cuda.synchronize()
    assert c.plan.status() == 0
    m = _sampled_metrics(con, A, B, None, C)
    del C
    if precision == "fp64":
        assert m["normwise"] <= 1e-13, m
        assert m["tccg_equal_worst"] <= 1e-9, m
    else:
        assert m["normwise"] <= _bf16_bound(con.sizeK), m


@pytest.mark.parametrize("precision", ["bf16x3", "fp32", "fp64"])
def test_configuration3_scaling_is_exact(cuda, precision):
    """Scaling A by 4 and B by 0.5 scales every product by exactly 2 (powers
    of two pass through the bf16 hi/lo split and every FP32/FP64 operation
    exactly), so C(4A, B/2) == 2 C(A, B) bit for bit."""
    import torch
    from tccg_b200.api import Compiled
    con = parse_text(CFG[3])
    dt = torch.float64 if precision == "fp64" else torch.float32
    A, B, _ = _data(con, dt, 300)
    c = Compiled(con, precision)
    C1 = c(A, B)
    C2 = c(A * 4, B * 0.5)
    torch.cuda.synchronize()
    assert torch.equal(C2, 2 * C1)


def test_configuration2_beta_accumulates(cuda):
    """Configuration 2 has beta = 1: running it twice on the same C adds the
    product twice (equal to C0 + 2 A*B up to rounding)."""
    import torch
    from tccg_b200.api import Compiled
    con = parse_text(CFG[2])
    A, B, C0 = _data(con, torch.float32, 400)
    c = Compiled(con, "fp32")
    C = C0.clone()
    c(A, B, C)
    c(A, B, C)
    P = c(A, B, torch.zeros_like(C0), beta=0.0)
    torch.cuda.synchronize()
    ref = C0.double() + 2 * P.double()
    err = torch.linalg.vector_norm(C.double() - ref) / torch.linalg.vector_norm(ref)
    assert err.item() <= 1e-6


def test_configuration5_grouped_full(cuda):
    """All 256 items, one grouped launch in a CUDA graph: equal to the
    per-item plan runs bit for bit, and 64 sampled entries per item within
    1e-5 of the FP64 oracle."""
    import torch
    from tccg_b200.grouped import Group
    from tccg_b200.workloads import batched_workload
    items = batched_workload(256, seed=0)
    g = torch.Generator(device="cuda").manual_seed(5)
    As = [torch.randn(c.A0.num_elements(), generator=g, device="cuda") for c in items]
    Bs = [torch.randn(c.B0.num_elements(), generator=g, device="cuda") for c in items]
    Cs = [torch.empty(c.C0.num_elements(), device="cuda") for c in items]
    grp = Group(items, "bf16x3")
    grp.bind(As, Bs, Cs)
    grp.capture()
    grp.replay()
    torch.cuda.synchronize()
    grouped = [c.clone() for c in Cs]
    grp.run_per_item()
    torch.cuda.synchronize()
    for a, b in zip(grouped, Cs):
        assert torch.equal(a, b)
    for con, A, B, C in zip(items, As, Bs, grouped):
        ln = _loopnest(con)
        lins = np.unique(np.linspace(0, ln.size_c - 1, 64).astype(np.int64))
        ref = ln.sample64(A.cpu().numpy(), B.cpu().numpy(), None, 1.0, 0.0, lins)
        m = error_metrics(C[torch.from_numpy(lins).cuda()].double().cpu().numpy(), ref)
        assert m["normwise"] <= 1e-5, (str(con), m)
