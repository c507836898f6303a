"""TTGT (transpose-transpose-GEMM-transpose, tccg/ttgemmt.py, transpose.py)
and the HPTT-style transposition entry point; FP64 k-split."""
import ctypes

import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Tuning
from tccg_b200.spec import make_contraction

CASES = [
    ("abcd", "aeb", "edc", dict(a=40, b=24, c=32, d=20, e=16), 1.0, 1.0),   # C already [M][N]
    ("acbd", "aeb", "edc", dict(a=40, b=24, c=32, d=20, e=16), 1.5, 0.5),   # C needs a transposition
    ("abij", "ima", "mjb", dict(a=24, b=24, i=24, j=24, m=24), 1.0, 0.0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("precision", ["fp32", "bf16x3", "fp64"])
def test_ttgt_matches_gett(cuda, case, precision):
    lc, la, lb, sizes, alpha, beta = CASES[case]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    dt = np.float64 if precision == "fp64" else np.float32
    A = seeded_normal(ln.size_a, 61).astype(dt)
    B = seeded_normal(ln.size_b, 62).astype(dt)
    C = seeded_normal(ln.size_c, 63).astype(dt)
    gett, _ = run_gpu(con, precision, A, B, C)
    ttgt, p = run_gpu(con, precision, A, B, C, tuning=Tuning(method="ttgt"))
    assert "method=TTGT" in p.describe()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    tol = {"fp32": 1e-6, "bf16x3": 1e-5, "fp64": 1e-13}[precision]
    assert error_metrics(ttgt, ref)["normwise"] <= tol
    assert error_metrics(gett, ref)["normwise"] <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("ksplit", [2, 5])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_ksplit(cuda, ksplit, precision):
    sizes = dict(a=50, b=70, k=900)
    con = make_contraction("ab", "ka", "kb", sizes, 2.0, -1.0)
    ln = LoopNest("ab", "ka", "kb", sizes)
    dt = np.float64 if precision == "fp64" else np.float32
    A, B, C = (seeded_normal(n, s).astype(dt) for n, s in ((ln.size_a, 71), (ln.size_b, 72), (ln.size_c, 73)))
    out, p = run_gpu(con, precision, A, B, C, tuning=Tuning(ksplit=ksplit))
    assert "ksplit=%d" % ksplit in p.describe()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), 2.0, -1.0)
    assert error_metrics(out, ref)["normwise"] <= (1e-13 if precision == "fp64" else 1e-6)


PERMS = {
    "mixed": ([5, 7, 3, 4], [2, 0, 3, 1], True),
    "reverse": ([70, 9, 33, 66], [3, 2, 1, 0], False),
    "stream": ([130, 6, 5, 70], [0, 1, 3, 2], False),      # dim 0 stays first: streaming copy
    "identity": ([17, 3, 1, 40], [0, 1, 2, 3], False),     # fuses to one dimension
    "padded_stream": ([65, 3, 4, 2], [0, 2, 1, 3], True),  # padding blocks fusion
    "few_rows": ([300, 70, 2, 1], [1, 0, 2, 3], False),    # tiles grouped along dim 0
    "wide_tiles": ([128, 128, 3, 2], [1, 0, 3, 2], False), # 64 x 64 tiles
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(PERMS))
@pytest.mark.parametrize("dtype", ["f32", "f64"])
def test_transpose_entry_point(cuda, dtype, case):
    """tccg_transpose: B[perm] = alpha * A + beta * B with outer (padded) sizes,
    HPTT's semantics (dimension j of B is dimension perm[j] of A)."""
    import torch
    from tccg_b200 import _native as N
    tdt = torch.float32 if dtype == "f32" else torch.float64
    size, perm, padded = PERMS[case]
    outer_a = [e + (1 if padded and i % 2 == 0 else 0) for i, e in enumerate(size)]
    outer_b = [size[perm[j]] + (1 if padded and j == 1 else 0) for j in range(4)]
    g = torch.Generator(device="cuda").manual_seed(1)
    A = torch.randn(int(np.prod(outer_a)), generator=g, device="cuda", dtype=tdt)
    B = torch.randn(int(np.prod(outer_b)), generator=g, device="cuda", dtype=tdt)
    B0 = B.clone()
    i32 = (ctypes.c_int32 * 4)(*perm)
    i64 = lambda v: (ctypes.c_int64 * 4)(*v)
    rc = N.lib().tccg_transpose(N.F32 if dtype == "f32" else N.F64, 4, i32, i64(size), i64(outer_a),
                                i64(outer_b), 2.0, ctypes.c_void_p(A.data_ptr()), 0.5,
                                ctypes.c_void_p(B.data_ptr()), None)
    N.check(rc)
    torch.cuda.synchronize()
    # reference in numpy: column-major views
    An = A.cpu().numpy().reshape(outer_a[::-1]).transpose()[:size[0], :size[1], :size[2], :size[3]]
    Bv = B0.cpu().numpy().reshape(outer_b[::-1]).transpose()
    want = Bv.copy()
    sl = tuple(slice(0, size[perm[j]]) for j in range(4))
    want[sl] = 2.0 * np.transpose(An, perm) + 0.5 * Bv[sl]
    got = B.cpu().numpy().reshape(outer_b[::-1]).transpose()
    assert np.allclose(got, want, rtol=1e-6, atol=1e-6)
    # beta == 0 never reads B (NaN there stays out of the result)
    B.fill_(float("nan"))
    N.check(N.lib().tccg_transpose(N.F32 if dtype == "f32" else N.F64, 4, i32, i64(size),
                                   i64(outer_a), i64(outer_b), 2.0, ctypes.c_void_p(A.data_ptr()),
                                   0.0, ctypes.c_void_p(B.data_ptr()), None))
    torch.cuda.synchronize()
    got = B.cpu().numpy().reshape(outer_b[::-1]).transpose()[sl]
    assert np.allclose(got, 2.0 * np.transpose(An, perm), rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
@pytest.mark.parametrize("case", [
    ("abij", "ima", "mjb", dict(a=24, b=20, i=6, j=5, m=24), 1.0, 0.0),     # loops over i, j
    ("pqr", "qs", "spr", dict(p=37, q=29, r=11, s=53), 0.75, -0.5),         # swap, loop over r
    ("ab", "ak", "kb", dict(a=70, b=50, k=90), 1.0, 0.0),                    # plain GEMM: one item
])
def test_loops_over_gemm(cuda, precision, case):
    """LoG (tccg/gemm_loop.py) as one batched launch matches the oracle."""
    import torch
    from tccg_b200.loops import LoG
    lc, la, lb, sizes, alpha, beta = case
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, 81).astype(np.float32)
    B = seeded_normal(ln.size_b, 82).astype(np.float32)
    C = seeded_normal(ln.size_c, 83).astype(np.float32)
    log = LoG(con, precision)
    dA, dB, dC = (torch.from_numpy(x).cuda() for x in (A, B, C))
    log.run(dA, dB, dC)
    torch.cuda.synchronize()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    tol = {"fp32": 1e-6, "bf16x3": 1e-5}[precision]
    assert error_metrics(dC.double().cpu().numpy(), ref)["normwise"] <= tol, log.describe()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,dtype", [("bf16", "f32"), ("bf16", "bf16"), ("bf16x3", "f32")])
def test_cuda_core_variant_of_bf16_precisions(cuda, precision, dtype):
    """variant < 0: BF16 precisions on the CUDA-core kernel (bandwidth-bound
    shapes); BF16 keeps its semantics (operands rounded to bf16). BF16
    operands go with the bf16 precision only."""
    import torch
    lc, la, lb, sizes, alpha, beta = CASES[0]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A = seeded_normal(ln.size_a, 91).astype(np.float32)
    B = seeded_normal(ln.size_b, 92).astype(np.float32)
    C = seeded_normal(ln.size_c, 93).astype(np.float32)
    out, p = run_gpu(con, precision, A, B, C, tuning=Tuning(variant=-1), dtype=dtype)
    assert "simt_gett<f32>" in p.describe()
    if precision == "bf16":
        A = torch.from_numpy(A).bfloat16().float().numpy()
        B = torch.from_numpy(B).bfloat16().float().numpy()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(out, ref)["normwise"] <= 1e-6
