"""TCCG's OWN generated GETT (AVX2, from its generator via oracle/ref_build.py,
with oracle/hptt_standin for HPTT) against the reference loop nest on TCCG's
deterministic inputs -- the check TCCG's --testing performs
(tccg.py:1010-1050, equal() at 1e-4) -- on configuration 1. This validates the
CPU baseline the benchmark times next to the GPU numbers."""
import ctypes
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import ref_build  # noqa: E402
from oracle import LoopNest, aligned_copy, aligned_empty, error_metrics, tccg_inputs  # noqa: E402

pytestmark = pytest.mark.skipif(not ref_build.reference_present(),
                                reason="building TCCG's GETT needs the reference checkout")


def _load(threads):
    so = ref_build.build_tccg_gett(ref_build.CFG1, "tccg_gett_cfg1_t%d" % threads, threads=threads,
                                   max_impl=2)
    L = ctypes.CDLL(so)
    L.tccg_gett_count.restype = ctypes.c_int
    L.tccg_gett_name.restype = ctypes.c_char_p
    L.tccg_gett_run.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 3 + [ctypes.c_float] * 2
    return L


def test_tccg_generated_gett_matches_loop_nest():
    threads = min(8, os.cpu_count() or 1)
    L = _load(threads)
    assert L.tccg_gett_count() >= 1
    ln = LoopNest("abij", "ima", "mjb", dict(a=48, b=48, i=48, j=48, m=48))
    A, B = aligned_copy(tccg_inputs(ln.size_a, "A")), aligned_copy(tccg_inputs(ln.size_b, "B"))
    ref = ln.run(A.copy(), B.copy(), np.zeros(ln.size_c, dtype=np.float32), 1.0, 0.0)
    for i in range(L.tccg_gett_count()):
        C = aligned_empty(ln.size_c)
        C[:] = np.nan  # beta = 0: C is not read
        L.tccg_gett_run(i, A.ctypes.data, B.ctypes.data, C.ctypes.data, 1.0, 0.0)
        m = error_metrics(C, ref)
        assert m["tccg_equal_pass"], (L.tccg_gett_name(i), m)
