"""Programmatic dependent launch: the GETT kernel of a plan run may start
while the packing kernel before it drains (and a reduction while its GETT
kernel drains); each waits for that kernel's writes before reading them.
It is automatic for the CUDA-core kernels and for tcgen05 grids of at most
four rounds of tiles; these tests force it on (TCCG_B200_PDL=1) and off (=0). Results must be bitwise equal either way on
every launch path that uses it -- CUDA-core tiles (square, narrow), the short-K
kernel with TMA and cp.async C blocks, the skinny kernel's k-split reduction,
tcgen05 (BF16x3, BF16, CTA pairs), k-split and tail-split reductions -- and for back-to-back runs captured in
one CUDA graph, where each run's beta reads the C of the run before."""
import numpy as np
import pytest

from helpers import seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Plan, Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

# (C, A, B, extents, beta, precision, tuning, describe tag)
CASES = {
    "simt": ("mn", "mk", "kn", dict(m=1000, n=900, k=300), 0.5, "fp32", Tuning(ksplit=1),
             "kernel=simt_gett<"),
    "simt_ksplit": ("mn", "mk", "kn", dict(m=500, n=400, k=3000), 0.5, "fp32", Tuning(ksplit=4),
                    "ksplit=4"),
    "narrow": ("mn", "mk", "kn", dict(m=1000, n=20, k=700), 1.0, "fp32",
               Tuning(simt_tile=2, ksplit=1, direct=-1), "tile=128x32x16"),
    "shortk_tma": ("mn", "mk", "kn", dict(m=2048, n=2048, k=16), 1.0, "fp32", Tuning(shortk=1),
                   "cblock=tma"),
    "shortk_cp": ("acbd", "aeb", "edc", dict(a=40, b=24, c=36, d=20, e=16), 1.0, "fp32",
                  Tuning(shortk=1), "cblock=cp.async"),
    "skinny_ksplit": ("cdn", "dnxy", "yxc", dict(c=8, d=23, n=20, x=60, y=41), 0.5, "fp32",
                      Tuning(skinny=1, ksplit=3), "kernel=skinny_gett<"),
    "tc_x3": ("mn", "mk", "kn", dict(m=1000, n=900, k=700), 0.5, "bf16x3", Tuning(variant=16),
              "kernel=gett_tc<"),
    "tc_bf16": ("mn", "km", "kn", dict(m=700, n=1100, k=500), -1.0, "bf16", Tuning(variant=16),
                "kernel=gett_tc<"),
    "tc_ksplit": ("mn", "mk", "kn", dict(m=256, n=384, k=8192), 0.5, "bf16x3",
                  Tuning(variant=16, ksplit=3), "ksplit=3"),
    "tc_tail": ("mn", "mk", "kn", dict(m=1280, n=2880, k=1024), 0.0, "bf16x3", Tuning(variant=16),
                "tail=2x2"),
    "tc_pair": ("mn", "mk", "kn", dict(m=1000, n=1500, k=600), 1.0, "bf16x3",
                Tuning(variant=16, pair=1), "kernel=gett_tc2<"),
}


def _setup(name, seed):
    import torch
    lc, la, lb, sizes, beta, precision, tuning, tag = CASES[name]
    con = make_contraction(lc, la, lb, sizes, 1.25, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, seed).astype(np.float32)
    B = seeded_normal(ln.size_b, seed + 1).astype(np.float32)
    C = seeded_normal(ln.size_c, seed + 2).astype(np.float32)
    if precision == "bf16":  # exact products on the tensor cores
        A = torch.from_numpy(A).bfloat16().float().numpy()
        B = torch.from_numpy(B).bfloat16().float().numpy()
    p = Plan(con, precision=precision, tuning=tuning)
    assert tag in p.describe(), p.describe()
    dev = torch.device("cuda")
    dA, dB = torch.from_numpy(A).to(dev), torch.from_numpy(B).to(dev)
    ws = torch.empty(max(p.workspace_bytes, 1), dtype=torch.uint8, device=dev)
    return con, ln, p, dA, dB, C, ws, beta


def _run(p, dA, dB, C, ws, times=1):
    import torch
    dC = torch.from_numpy(C).to("cuda")
    for _ in range(times):
        p.run(dA, dB, dC, workspace=ws)
    torch.cuda.synchronize()
    assert p.status() == 0
    return dC.cpu().numpy()


@pytest.mark.parametrize("name", sorted(CASES))
def test_dependent_launch_bitwise(cuda, monkeypatch, name):
    con, ln, p, dA, dB, C, ws, beta = _setup(name, 171)
    monkeypatch.setenv("TCCG_B200_PDL", "0")
    plain = _run(p, dA, dB, C, ws, times=3)
    monkeypatch.setenv("TCCG_B200_PDL", "1")
    dep = _run(p, dA, dB, C, ws, times=3)
    assert np.array_equal(plain, dep)
    # one run against the FP64 loop nest
    one = _run(p, dA, dB, C, ws)
    ref = ln.run(dA.double().cpu().numpy(), dB.double().cpu().numpy(), C.astype(np.float64),
                 1.25, beta)
    assert error_metrics(one.astype(np.float64), ref)["normwise"] <= 1e-5


@pytest.mark.parametrize("name", ["shortk_tma", "tc_tail", "tc_ksplit", "simt", "skinny_ksplit"])
def test_dependent_launch_in_cuda_graph(cuda, monkeypatch, name):
    import torch
    con, ln, p, dA, dB, C, ws, beta = _setup(name, 172)
    monkeypatch.setenv("TCCG_B200_PDL", "0")
    eager = _run(p, dA, dB, C, ws, times=3)
    monkeypatch.setenv("TCCG_B200_PDL", "1")
    dC = torch.from_numpy(C).to("cuda")
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # warm-up on the capture stream
        p.run(dA, dB, dC, workspace=ws)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(3):
            p.run(dA, dB, dC, workspace=ws)
    dC.copy_(torch.from_numpy(C).to("cuda"))
    g.replay()
    torch.cuda.synchronize()
    assert p.status() == 0
    assert np.array_equal(eager, dC.cpu().numpy())
    del g


def test_describe_reports_the_launch(cuda, monkeypatch):
    small = Plan(make_contraction("mn", "mk", "kn", dict(m=1024, n=1024, k=1024)), "bf16x3")
    # configuration 3's size (8.8e12 FLOP): ordinary launches by default
    big = Plan(make_contraction("abcijk", "ambnc", "minjk",
                                dict(a=32, b=32, c=32, i=32, j=32, k=32, m=64, n=64)), "bf16x3")
    big32 = Plan(big.con, "fp32")
    monkeypatch.delenv("TCCG_B200_PDL", raising=False)
    # a tcgen05 grid of one round: dependent; of 37 rounds: plain; the
    # CUDA-core kernels (independent CTAs): dependent at any size
    assert "launch=dependent" in small.describe() and "launch=plain" in big.describe()
    assert "launch=dependent" in big32.describe()
    monkeypatch.setenv("TCCG_B200_PDL", "1")
    assert "launch=dependent" in big.describe()
    monkeypatch.setenv("TCCG_B200_PDL", "0")
    assert "launch=plain" in small.describe()


@pytest.mark.parametrize("name,pdl", [("tc_x3", "1"), ("tc_x3", "0"), ("tc_bf16", "1"),
                                      ("tc_tail", "1")])
def test_sm_tile_order_bitwise(cuda, monkeypatch, name, pdl):
    """The persistent tcgen05 grid takes tiles in SM order (%smid, when the
    grid has one CTA per SM id) or in launch order
    (TCCG_B200_CTA_ORDER=launch): the same tiles with the same sums, only on
    other SMs -- bitwise equal, with and without dependent launch. The
    shapes are widened so that the grid fills every SM for several rounds."""
    import torch
    lc, la, lb, sizes, beta, precision, tuning, tag = CASES[name]
    big = dict(sizes, m=sizes["m"] * 8, n=sizes["n"] * 2)
    con = make_contraction(lc, la, lb, big, 1.25, beta)
    ln = LoopNest(lc, la, lb, big)
    A = seeded_normal(ln.size_a, 5).astype(np.float32)
    B = seeded_normal(ln.size_b, 6).astype(np.float32)
    C = seeded_normal(ln.size_c, 7).astype(np.float32)
    if precision == "bf16":
        A = torch.from_numpy(A).bfloat16().float().numpy()
        B = torch.from_numpy(B).bfloat16().float().numpy()
    p = Plan(con, precision=precision, tuning=tuning)
    assert "grid=148" in p.describe() or "grid=" in p.describe()
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    ws = torch.empty(max(p.workspace_bytes, 1), dtype=torch.uint8, device="cuda")
    monkeypatch.setenv("TCCG_B200_PDL", pdl)
    outs = []
    for order in ("sm", "launch"):  # TCCG_B200_CTA_ORDER=sm: tile positions from %smid
        monkeypatch.setenv("TCCG_B200_CTA_ORDER", order)
        outs.append(_run(p, dA, dB, C, ws))
    assert np.array_equal(outs[0], outs[1])
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), 1.25, beta)
    assert error_metrics(outs[0], ref)["normwise"] <= 1e-5
