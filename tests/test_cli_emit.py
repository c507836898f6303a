"""CLI surface and the emitted per-contraction artifact (TCCG's
tccg_implementations/gett.cpp, tccg.py:158-186)."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from tccg_b200.cli import build_parser, main
from tccg_b200.emit import emit, source
from tccg_b200.plan import Tuning
from tccg_b200.spec import parse_text

EXAMPLE = "C[a,b,i,j] = A[i,m,a] * B[m,j,b]\na = 24\nb = 24\ni = 24\nj = 24\nm = 24\n"


def test_flags_of_the_reference_are_accepted():
    a = build_parser().parse_args(["x.tccg", "--floatType=d", "--maxImplementations=-1",
                                   "--numThreads=8", "--noTTGT", "--ignoreDatabase", "--testing"])
    assert a.floatType == "d" and a.maxImplementations == -1 and a.noTTGT


def test_bad_float_type_and_tcl(tmp_path):
    f = tmp_path / "e.tccg"
    f.write_text(EXAMPLE)
    assert main([str(f), "--floatType=z"]) == 2
    assert main([str(f), "--useTCL"]) == 2
    assert main([str(f), "--floatType=d", "--precision=bf16x3"]) == 2


def test_syntax_error_is_reported(tmp_path, capsys):
    f = tmp_path / "bad.tccg"
    f.write_text("C[a,b] += A[a,k] * B[k,b]\na=2\nb=2\nk=2\n")
    assert main([str(f), "--generateOnly"]) == 1


def test_emitted_source_compiles_and_exports_tccg_signature(tmp_path):
    con = parse_text(EXAMPLE)
    src = source(con, "bf16x3", Tuning(), "s")
    assert "void gett(float* A, float* B, float* C, const float alpha, const float beta)" in src
    paths = emit(con, "fp32", Tuning(), "s", str(tmp_path / "impl"))
    L = ctypes.CDLL(paths["so"])
    for sym in ("gett", "gett_stream", "gett_workspace_bytes", "gett_last_status"):
        assert hasattr(L, sym)
    hdr = open(paths["h"]).read()
    assert "void gett(float* A, float* B, float* C, const float alpha, const float beta);" in hdr


def test_double_signature():
    con = parse_text(EXAMPLE)
    assert "void gett(double* A, double* B, double* C, const double alpha, const double beta)" in \
        source(con, "fp64", Tuning(), "d")


@pytest.mark.gpu
def test_cli_end_to_end(cuda, tmp_path):
    """tune (2 candidates, fresh DB), --testing, emit, then call the emitted
    gett() with device pointers and compare with the FP64 oracle."""
    import torch
    from oracle import LoopNest, error_metrics
    f = tmp_path / "example.tccg"
    f.write_text(EXAMPLE)
    env = dict(os.environ, TCCG_B200_DB=str(tmp_path / "t.db"))
    out = subprocess.run([sys.executable, "-m", "tccg_b200", str(f), "--precision=bf16x3",
                          "--maxImplementations=2", "--testing", "--outdir", str(tmp_path / "impl")],
                         capture_output=True, text=True, env=env,
                         cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert out.returncode == 0, out.stdout + out.stderr
    assert "testing: worst" in out.stdout
    L = ctypes.CDLL(str(tmp_path / "impl" / "libgett.so"))
    L.gett.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_float] * 2
    L.gett_last_status.restype = ctypes.c_int
    ln = LoopNest("abij", "ima", "mjb", dict(a=24, b=24, i=24, j=24, m=24))
    rng = np.random.default_rng(1)
    A, B = rng.standard_normal(ln.size_a).astype(np.float32), rng.standard_normal(ln.size_b).astype(np.float32)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    dC = torch.zeros(ln.size_c, device="cuda")
    torch.cuda.synchronize()
    L.gett(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), 1.0, 0.0)
    assert L.gett_last_status() == 0
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), np.zeros(ln.size_c), 1.0, 0.0)
    assert error_metrics(dC.double().cpu().numpy(), ref)["normwise"] <= 1e-5
    # second invocation: the database lookup skips the search
    out2 = subprocess.run([sys.executable, "-m", "tccg_b200", str(f), "--precision=bf16x3",
                           "--maxImplementations=2", "--verbose", "--outdir", str(tmp_path / "impl2")],
                          capture_output=True, text=True, env=env,
                          cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert out2.returncode == 0 and "tuning cache hit" in out2.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("spec,precision", [
    (EXAMPLE, "fp32"),
    # configuration 2 (beta = 1, C of 340 MB: 16 slabs of its last index d,
    # B copied whole, C copied up and down per slab)
    ("C[a,b,c,d] = A[a,e,b] * B[e,d,c] + C[a,b,c,d]\na=96\nb=96\nc=96\nd=96\ne=16\n", "bf16x3"),
])
def test_emitted_gett_with_host_buffers(cuda, tmp_path, spec, precision):
    """TCCG's callers pass host buffers (tccg.py:910-919, 1040): the emitted
    gett() called with numpy arrays copies them to the GPU and back (in slabs
    when C is large) and matches the FP64 oracle; called again with device
    pointers it gives the same C (bit for bit when no slabs are used)."""
    import torch
    from oracle import LoopNest, error_metrics
    con = parse_text(spec)
    paths = emit(con, precision, Tuning(), "s", str(tmp_path / "impl"))
    src = open(paths["cu"]).read()
    L = ctypes.CDLL(paths["so"])
    L.gett.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_float] * 2
    L.gett_last_status.restype = ctypes.c_int
    sizes = {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices}
    ln = LoopNest(con.C0.labels, con.A0.labels, con.B0.labels, sizes)
    rng = np.random.default_rng(5)
    A = rng.standard_normal(ln.size_a, dtype=np.float32)
    B = rng.standard_normal(ln.size_b, dtype=np.float32)
    C0 = rng.standard_normal(ln.size_c, dtype=np.float32)
    C = C0.copy()
    L.gett(A.ctypes.data, B.ctypes.data, C.ctypes.data, con.alpha, con.beta)
    assert L.gett_last_status() == 0
    big = ln.size_c * 4 >= (256 << 20)
    assert ("#define NSLAB 16" in src) == big
    lins = np.unique(np.linspace(0, ln.size_c - 1, 4096).astype(np.int64))
    ref = ln.sample64(A, B, C0 if con.beta != 0 else None, con.alpha, con.beta, lins)
    tol = 1e-5 if precision == "bf16x3" else 1e-6
    assert error_metrics(C[lins], ref)["normwise"] <= tol
    dA, dB, dC = (torch.from_numpy(x).cuda() for x in (A, B, C0))
    torch.cuda.synchronize()
    L.gett(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), con.alpha, con.beta)
    assert L.gett_last_status() == 0
    if not big:  # the same plan on the same data
        assert np.array_equal(dC.cpu().numpy(), C)
    else:  # slab plans and the whole-tensor plan may tile differently
        assert error_metrics(dC.cpu().numpy()[lins], ref)["normwise"] <= tol
