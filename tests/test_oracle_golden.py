"""The oracle pinned to the reference: its C loop nest reproduces, bit for bit,
the loop nest TCCG emits (tccg/tccg.py:686-723) compiled and run on the same
inputs (fixtures from tests/golden/make_golden.py); its FP64 einsum agrees
with the loop nest; TCCG's deterministic inputs (tccg.py:957-971)."""
import glob
import json
import os

import numpy as np
import pytest

from helpers import splitmix_uniform
from oracle import LoopNest, error_metrics, tccg_inputs

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "loopnest_*.npz")))


def _labels(summary, t):
    return [l for l, _ in summary[t]["indices"]]


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[9:-4] for p in GOLD])
def test_loopnest_bitexact_vs_reference(path):
    z = np.load(path)
    s = json.loads(str(z["summary"]))
    sizes = {l: e for t in ("A", "B", "C") for l, e in s[t]["indices"]}
    # the reference loops over the FUSED indices, so the oracle gets the fused spec
    ln = LoopNest(_labels(s, "C"), _labels(s, "A"), _labels(s, "B"), sizes)
    dt = np.float32 if str(z["float_type"]) == "float" else np.float64
    for family in ("tccg", "seeded"):
        if family == "tccg":
            A, B, C = (tccg_inputs(ln.size_a, "A", dt), tccg_inputs(ln.size_b, "B", dt),
                       tccg_inputs(ln.size_c, "C", dt))
        else:
            A = splitmix_uniform(ln.size_a, 11).astype(dt)
            B = splitmix_uniform(ln.size_b, 12).astype(dt)
            C = splitmix_uniform(ln.size_c, 13).astype(dt)
        R = ln.run(A, B, C.copy(), s["alpha"], s["beta"])
        if family + "_C" in z:
            assert np.array_equal(R, z[family + "_C"]), family
        else:
            assert np.array_equal(R[z[family + "_lins"]], z[family + "_vals"]), family
        cs = np.array([R.astype(np.float64).sum(), np.abs(R.astype(np.float64)).sum(),
                       (R.astype(np.float64) ** 2).sum()])
        assert np.array_equal(cs, z[family + "_checksum"]), family


def test_einsum64_agrees_with_loopnest():
    ln = LoopNest("abij", "ima", "mjb", dict(a=6, b=5, i=4, j=3, m=7))
    A, B, C = splitmix_uniform(ln.size_a, 1), splitmix_uniform(ln.size_b, 2), splitmix_uniform(ln.size_c, 3)
    r = ln.run(A.copy(), B.copy(), C.copy(), 1.5, -0.5)
    e = ln.einsum64(A, B, C, 1.5, -0.5).ravel(order="F")
    assert error_metrics(r, e)["normwise"] < 1e-15


def test_sample64_matches_loopnest():
    ln = LoopNest("pqr", "qs", "spr", dict(p=7, q=6, r=5, s=9))
    A, B, C = splitmix_uniform(ln.size_a, 4), splitmix_uniform(ln.size_b, 5), splitmix_uniform(ln.size_c, 6)
    r = ln.run(A.copy(), B.copy(), C.copy(), 2.0, 0.5)
    lins = np.array([0, 3, 17, ln.size_c - 1])
    assert np.allclose(ln.sample64(A, B, C, 2.0, 0.5, lins), r[lins], rtol=0, atol=1e-14)


def test_tccg_init_formula():
    a = tccg_inputs(5, "A")
    assert np.array_equal(a, np.array([(10 + ((i + 1) * 17) % 100) / 110.0 for i in range(5)], dtype=np.float32))


def test_error_metrics_sign_aware():
    """TCCG's equal() compared |x| - |y| and missed sign errors
    (tccg.py:862-866); the oracle's criterion does not."""
    m = error_metrics(np.array([-1.0, 2.0]), np.array([1.0, 2.0]))
    assert not m["tccg_equal_pass"]
