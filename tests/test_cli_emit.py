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
