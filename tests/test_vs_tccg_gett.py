"""GPU results against TCCG's OWN generated GETT (AVX2, host cores) on the two
configurations TCCG's generator can tile (1 and 2), with TCCG's
deterministic inputs (tccg.py:957-971) and seeded ones: FP32 at TCCG's equal()
tolerance of 1e-4 (tccg.py:869-873, sign-aware), split-BF16x3 at normwise 1e-5. The generated code is
built in the container that holds the reference checkout (oracle/ref_build.py
build_all) and travels as oracle/_ref/tccg_gett_cfg{1,2}.so."""
import ctypes
import os

import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, aligned_copy, error_metrics, tccg_inputs
from tccg_b200.spec import parse_text

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref")
CFG = {
    "cfg1": ("C[a,b,i,j] = A[i,m,a] * B[m,j,b]\na=48\nb=48\ni=48\nj=48\nm=48\n",
             ("abij", "ima", "mjb", dict(a=48, b=48, i=48, j=48, m=48))),
    "cfg2": ("C[a,b,c,d] = A[a,e,b] * B[e,d,c] + C[a,b,c,d]\na=96\nb=96\nc=96\nd=96\ne=16\n",
             ("abcd", "aeb", "edc", dict(a=96, b=96, c=96, d=96, e=16))),
}


def _tccg_gett(name):
    so = os.path.join(REF, "tccg_gett_%s.so" % name)
    if not os.path.exists(so):
        pytest.skip("%s was not built (needs the reference checkout)" % so)
    L = ctypes.CDLL(so)
    L.tccg_gett_count.restype = ctypes.c_int
    L.tccg_gett_name.restype = ctypes.c_char_p
    L.tccg_gett_run.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 3 + [ctypes.c_float] * 2
    return L


@pytest.mark.parametrize("inputs", ["tccg", "seeded"])
@pytest.mark.parametrize("name", sorted(CFG))
def test_gpu_matches_tccg_generated_gett(cuda, name, inputs):
    text, (lc, la, lb, sizes) = CFG[name]
    con = parse_text(text)
    ln = LoopNest(lc, la, lb, sizes)
    if inputs == "tccg":
        A, B, C = (tccg_inputs(ln.size_a, "A"), tccg_inputs(ln.size_b, "B"),
                   tccg_inputs(ln.size_c, "C"))
    else:
        A, B, C = (seeded_normal(ln.size_a, 121).astype(np.float32),
                   seeded_normal(ln.size_b, 122).astype(np.float32),
                   seeded_normal(ln.size_c, 123).astype(np.float32))
    L = _tccg_gett(name)
    Aa, Ba, Cc = aligned_copy(A), aligned_copy(B), aligned_copy(C)  # 64-byte aligned, kept alive
    L.tccg_gett_run(0, Aa.ctypes.data, Ba.ctypes.data, Cc.ctypes.data, con.alpha, con.beta)
    ref64 = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), con.alpha,
                   con.beta)
    # TCCG's own result is itself right (its --testing check)
    assert error_metrics(Cc, ref64, tol_tccg=1e-4)["tccg_equal_pass"]
    # FP32: TCCG's per-element equal() at 1e-4; split-BF16x3 (not a TCCG
    # precision): its own bound, normwise 1e-5
    out, p = run_gpu(con, "fp32", A, B, C)
    m = error_metrics(out, Cc.astype(np.float64), tol_tccg=1e-4)
    assert m["tccg_equal_pass"], (p.describe(), m)
    out, p = run_gpu(con, "bf16x3", A, B, C)
    m = error_metrics(out, Cc.astype(np.float64))
    assert m["normwise"] <= 1e-5, (p.describe(), m)
