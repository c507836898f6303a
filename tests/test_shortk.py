"""The short-K CUDA-core kernel (simt_shortk_kernel: the whole K panel of A
and B and the tile's C block prefetched into shared memory, the C read
running under the FMA phase). Same k order and epilogue arithmetic as the
general tile kernel (simt_gett_kernel), so the two must agree bit for bit;
both against the FP64 loop nest. Cases cover the C block moved by TMA (C a
2-D matrix) and by cp.async, 16-byte and element accesses (M quads that are
not contiguous in C), M/N/K tails, two k-tiles, beta = 0, many tiles and
TTGT's C' buffer."""
import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Plan, Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

CASES = {
    # configuration 2's pattern at reduced extents: K = 16, beta = 1
    "cfg2_small": ("abcd", "aeb", "edc", dict(a=40, b=24, c=64, d=40, e=16), 1.0, 1.0),
    # M = (a, b) not adjacent in C: quads of m cross a's extent (element path)
    "split_m": ("anb", "akb", "kn", dict(a=6, b=50, n=300, k=16), 0.5, -1.0),
    # K tail (13 -> 16), odd M and N, beta = 0 (C not read)
    "k_tail": ("mn", "mk", "kn", dict(m=1000, n=700, k=13), 1.0, 0.0),
    # many tiles: the automatic choice
    "many_tiles": ("mn", "mk", "kn", dict(m=3000, n=2900, k=16), 1.25, 0.75),
    # 2-D C whose column stride (1001 elements) is not 16-byte aligned: no TMA
    "odd_ldc": ("mn", "mk", "kn", dict(m=1001, n=300, k=16), 1.0, -0.5),
}
# two k-tiles of the FP32 kernel (K = 30 -> 32); FP64 takes K <= 16
TWO_KTILES = ("bna", "kab", "nk", dict(a=33, b=40, n=500, k=30), 1.0, 0.5)
# TTGT computes into a contiguous C' (M = b c = 560) and permutes it into C
TTGT = ("bac", "ak", "kbc", dict(a=300, b=70, c=8, k=16), 1.0, 0.5)
# how each case moves its C block (FP32 and FP64 alike)
CBLOCK = {"cfg2_small": "tma", "split_m": "cp.async", "k_tail": "tma", "many_tiles": "tma",
          "odd_ldc": "cp.async", "two_ktiles": "cp.async", "ttgt": "tma"}


def _inputs(lc, la, lb, sizes, dt, seed):
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, seed).astype(dt)
    B = seeded_normal(ln.size_b, seed + 1).astype(dt)
    C = seeded_normal(ln.size_c, seed + 2).astype(dt)
    return ln, A, B, C


def _check(name, case, precision, method="gett"):
    lc, la, lb, sizes, alpha, beta = case
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    dt = np.float64 if precision == "fp64" else np.float32
    ln, A, B, C = _inputs(lc, la, lb, sizes, dt, seed=131)
    v = -1 if precision == "bf16x3" else 0  # bf16x3 on the CUDA cores
    shortk, ps = run_gpu(con, precision, A, B, C,
                         tuning=Tuning(method, variant=v, shortk=1, ksplit=1))
    tiles, pt = run_gpu(con, precision, A, B, C,
                        tuning=Tuning(method, variant=v, shortk=-1, direct=-1, ksplit=1))
    assert "kernel=simt_shortk<" in ps.describe(), ps.describe()
    assert "cblock=" + CBLOCK[name] in ps.describe(), ps.describe()
    assert "kernel=simt_gett<" in pt.describe(), pt.describe()
    assert np.array_equal(shortk, tiles), name
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    tol = 1e-13 if precision == "fp64" else 1e-6
    assert error_metrics(shortk, ref)["normwise"] <= tol


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp32", "fp64", "bf16x3"])
def test_shortk_matches_tile_kernel_and_oracle(cuda, name, precision):
    _check(name, CASES[name], precision)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_shortk_two_ktiles(cuda, precision):
    _check("two_ktiles", TWO_KTILES, precision)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_shortk_ttgt(cuda, precision):
    _check("ttgt", TTGT, precision, "ttgt")


def test_automatic_choice(cuda):
    cfg2 = make_contraction("abcd", "aeb", "edc", dict(a=96, b=96, c=96, d=96, e=16), 1.0, 1.0)
    assert "kernel=simt_shortk<f32>" in Plan(cfg2, precision="fp32").describe()
    assert "kernel=simt_shortk<f64>" in Plan(cfg2, precision="fp64").describe()
    # K beyond the panel, or too few tiles: the general tile kernel
    long_k = make_contraction("mn", "mk", "kn", dict(m=4096, n=4096, k=64))
    assert "kernel=simt_gett<f32>" in Plan(long_k, precision="fp32").describe()
    few = make_contraction("mn", "mk", "kn", dict(m=512, n=512, k=16))
    assert "kernel=simt_gett<f32>" in Plan(few, precision="fp32").describe()
    # no 2-D C (the cp.async C block is no faster than the tile kernel)
    split = make_contraction("anb", "akb", "kn", dict(a=6, b=1000, n=8000, k=16), 1.0, 1.0)
    assert "kernel=simt_gett<f32>" in Plan(split, precision="fp32").describe()
    # TTGT's C' is 2-D
    ttgt = Plan(cfg2, precision="fp32", tuning=Tuning("ttgt"))
    assert "kernel=simt_shortk<f32>" in ttgt.describe() and "cblock=tma" in ttgt.describe()
    assert "kernel=simt_gett<f32>" in Plan(cfg2, precision="fp32",
                                           tuning=Tuning(shortk=-1)).describe()
