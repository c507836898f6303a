"""Parity of the CUDA GETT path with the oracle (GPU).

Each case runs a contraction through the C ABI (tccg_plan_run) and compares
C with the oracle on the same inputs:

* FP32 against TCCG's loop-nest reference restated in C (float accumulator,
  tccg/tccg.py:686-723) with TCCG's own ``equal()`` tolerance, 1e-4
  (tccg.py:869-873), sign-aware; and against FP64 (normwise <= 1e-6).
* FP64 against the FP64 loop nest (TCCG's 1e-9 double tolerance; normwise
  <= 1e-13).
* BF16x3 against FP64: normwise <= 1e-5; BF16 against
  FP64 of the bf16-rounded inputs: normwise <= 1e-5.
"""
import numpy as np
import pytest

from helpers import labels, run_gpu, seeded_normal, splitmix_uniform
from oracle import LoopNest, error_metrics, tccg_inputs
from tccg_b200.plan import Tuning
from tccg_b200.spec import make_contraction, parse_text

pytestmark = pytest.mark.gpu

CASES = {
    # configuration 1 (all extents 48), FP32, U[-1,1], alpha=1 beta=0
    "cfg1": ("abij", "ima", "mjb", dict(a=48, b=48, i=48, j=48, m=48), 1.0, 0.0),
    # configuration 2 at reduced extents (bandwidth-bound pattern), beta=1
    "cfg2_small": ("abcd", "aeb", "edc", dict(a=40, b=24, c=32, d=20, e=16), 1.0, 1.0),
    # configuration 3 pattern, reduced extents
    "cfg3_small": ("abcijk", "ambnc", "minjk", dict(a=8, b=8, c=4, i=8, j=4, k=8, m=16, n=8), 1.0, 0.0),
    # configuration 4 pattern, reduced extents
    "cfg4_small": ("xyzw", "pxqw", "qzpy", dict(x=16, w=16, y=16, z=16, p=8, q=8), 1.0, 0.0),
    # alpha/beta as in the reference's transC benchmark (2.4 / 1.1)
    "transc": ("ujv", "ukv", "jk", dict(u=24, v=12, j=40, k=24), 2.4, 1.1),
    # odd extents everywhere, B holds C's stride-one index (operand swap)
    "odd_swap": ("pqr", "qs", "spr", dict(p=37, q=29, r=11, s=53), 0.75, -0.5),
    # matrix-vector (no N index) and outer product (no K index)
    "matvec": ("a", "ak", "k", dict(a=300, k=77), 1.0, 0.0),
    "outer": ("ab", "a", "b", dict(a=33, b=65), 1.5, 0.0),
}


def _inputs(lc, la, lb, sizes, seed, dist="uniform"):
    ln = LoopNest(lc, la, lb, sizes)
    gen = splitmix_uniform if dist == "uniform" else (lambda n, s: seeded_normal(n, s))
    A = gen(ln.size_a, seed)
    B = gen(ln.size_b, seed + 100)
    C = gen(ln.size_c, seed + 200)
    return ln, A, B, C


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp32_vs_loopnest(cuda, name):
    lc, la, lb, sizes, alpha, beta = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln, A, B, C = _inputs(lc, la, lb, sizes, seed=1)
    A32, B32, C32 = A.astype(np.float32), B.astype(np.float32), C.astype(np.float32)
    out, _ = run_gpu(con, "fp32", A32, B32, C32)
    ref32 = ln.run(A32.copy(), B32.copy(), C32.copy(), alpha, beta)
    m = error_metrics(out, ref32, tol_tccg=1e-4)
    assert m["tccg_equal_pass"], m
    ref64 = ln.run(A32.astype(np.float64), B32.astype(np.float64), C32.astype(np.float64), alpha, beta)
    m64 = error_metrics(out, ref64)
    assert m64["normwise"] <= 1e-6, m64


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_vs_loopnest(cuda, name):
    lc, la, lb, sizes, alpha, beta = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln, A, B, C = _inputs(lc, la, lb, sizes, seed=2, dist="normal")
    out, _ = run_gpu(con, "fp64", A, B, C)
    ref = ln.run(A.copy(), B.copy(), C.copy(), alpha, beta)
    m = error_metrics(out, ref, tol_tccg=1e-9)
    assert m["tccg_equal_pass"], m
    assert m["normwise"] <= 1e-13, m


# BF16 precisions: the library's own kernel choice and the tensor-core kernel
# forced (tuning.variant > 0), so both paths are checked on every case
KERNELS = {"auto": 0, "tensor_core": 16}


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("name", sorted(CASES))
def test_bf16x3_vs_fp64(cuda, name, kernel):
    lc, la, lb, sizes, alpha, beta = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln, A, B, C = _inputs(lc, la, lb, sizes, seed=3, dist="normal")
    A32, B32, C32 = A.astype(np.float32), B.astype(np.float32), C.astype(np.float32)
    out, p = run_gpu(con, "bf16x3", A32, B32, C32, tuning=Tuning(variant=KERNELS[kernel]))
    if kernel == "tensor_core":
        assert "gett_tc<BF16X3" in p.describe()  # either tcgen05 loader
    ref = ln.run(A32.astype(np.float64), B32.astype(np.float64), C32.astype(np.float64), alpha, beta)
    m = error_metrics(out, ref)
    assert m["normwise"] <= 1e-5, m


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("name", sorted(CASES))
def test_bf16_vs_fp64(cuda, name, kernel):
    import torch
    lc, la, lb, sizes, alpha, beta = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln, A, B, C = _inputs(lc, la, lb, sizes, seed=4, dist="normal")
    # bf16-rounded operands: the tensor cores then compute exact products
    Ab = torch.from_numpy(A.astype(np.float32)).bfloat16().float().numpy()
    Bb = torch.from_numpy(B.astype(np.float32)).bfloat16().float().numpy()
    C32 = C.astype(np.float32)
    # the same kernel for f32 and bf16 operand tensors (the automatic choice
    # looks at the operand bytes): forced with variant -1 or 1
    t = Tuning(variant=1 if kernel == "tensor_core" else -1)
    out, _ = run_gpu(con, "bf16", Ab, Bb, C32, tuning=t)
    ref = ln.run(Ab.astype(np.float64), Bb.astype(np.float64), C32.astype(np.float64), alpha, beta)
    m = error_metrics(out, ref)
    assert m["normwise"] <= 1e-5, m
    # and with bf16 tensors as inputs
    out2, _ = run_gpu(con, "bf16", Ab, Bb, C32, dtype="bf16", tuning=t)
    assert np.array_equal(out, out2)
    out3, _ = run_gpu(con, "bf16", Ab, Bb, C32)
    assert error_metrics(out3, ref)["normwise"] <= 1e-5


def test_tccg_formula_inputs_example(cuda):
    """The reference's example.tccg with TCCG's deterministic inputs
    (tccg.py:957-971) and its equal() check at 1e-4."""
    con = parse_text("C[a,b,i,j] = A[i,m,a] * B[m,j,b]\na = 24\nb = 24\ni = 24\nj = 24\nm = 24\n")
    lc, la, lb, sizes = labels(con)
    ln = LoopNest(lc, la, lb, sizes)
    A = tccg_inputs(ln.size_a, "A")
    B = tccg_inputs(ln.size_b, "B")
    C = tccg_inputs(ln.size_c, "C")
    out, _ = run_gpu(con, "fp32", A, B, C)
    ref = ln.run(A.copy(), B.copy(), C.copy(), 1.0, 0.0)
    assert error_metrics(out, ref)["tccg_equal_pass"]


def test_beta_zero_ignores_nan_in_c(cuda):
    """beta == 0 writes C without reading it (TCCG's update=0 path)."""
    lc, la, lb, sizes, alpha, _ = CASES["cfg2_small"]
    con = make_contraction(lc, la, lb, sizes, alpha, 0.0)
    ln, A, B, C = _inputs(lc, la, lb, sizes, seed=5)
    Cn = np.full(ln.size_c, np.nan, dtype=np.float32)
    for prec, t in (("fp32", None), ("bf16x3", None), ("bf16x3", Tuning(variant=16))):
        out, _ = run_gpu(con, prec, A.astype(np.float32), B.astype(np.float32), Cn, tuning=t)
        assert np.isfinite(out).all(), prec


@pytest.mark.parametrize("chunk_kb", [1, 3, 16, 1000])
def test_bf16x3_k_chunks(cuda, chunk_kb):
    """Chunked accumulation (TMEM accumulators ping-pong every chunk_kb
    k-blocks of 32): odd K over many chunks, partial 128x192 tiles."""
    from tccg_b200.plan import Tuning
    sizes = dict(m=300, n=500, k=1000)
    con = make_contraction("mn", "km", "kn", sizes)
    ln = LoopNest("mn", "km", "kn", sizes)
    A = seeded_normal(ln.size_a, 21).astype(np.float32)
    B = seeded_normal(ln.size_b, 22).astype(np.float32)
    C = np.zeros(ln.size_c, dtype=np.float32)
    out, p = run_gpu(con, "bf16x3", A, B, C, tuning=Tuning(variant=chunk_kb))
    assert "chunk=%d" % chunk_kb in p.describe()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), 1.0, 0.0)
    m = error_metrics(out, ref)
    assert m["normwise"] <= 1e-5, m
