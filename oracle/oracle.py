"""ORACLE -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker: the product (tccg_b200/) never imports,
links or runs anything under oracle/.

Contents:

* ``LoopNest``: ctypes front end of oracle/loopnest.c, the C restatement of
  TCCG's emitted correctness reference ``referenceVersion``
  (tccg/tccg.py:686-723). Its contraction description is built here from
  plain index strings, independently of the product's parser: C's modes in
  C order, the contracted modes in getContractedIndices order (indices of A,
  in A's order, that are in B and not in C; tccg/tccg_util.py:597-611).
* ``einsum64``: the FP64 einsum oracle (numpy).
* ``tccg_inputs``: TCCG's deterministic operand values (tccg.py:957-971).
* ``error_metrics``: max abs, normwise, max relative error over entries with
  |ref| > 1e-3 max|ref|, and TCCG's ``equal()`` criterion
  (tccg.py:843-881) with its sign blindness fixed (it compared |x| - |y|).

Parity of this oracle is pinned by tests/test_oracle_golden.py against
fixtures produced by running the reference's own generator
(tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from typing import Dict, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lock = threading.Lock()
_lib = None


def build(force: bool = False) -> str:
    """Compile oracle/loopnest.c with the system gcc (OpenMP)."""
    src = os.path.join(_HERE, "loopnest.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(_LIB_PATH), exist_ok=True)
        cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
        # -ffp-contract=off: every multiply and add rounds separately (IEEE), so
        # the loop nest matches the reference's emitted code compiled the same
        # way bit for bit
        cmd = [cc, "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC",
               "-std=c11", "-shared",
               "-o", _LIB_PATH + ".tmp", src]
        subprocess.run(cmd, check=True, capture_output=True, text=True)
        os.replace(_LIB_PATH + ".tmp", _LIB_PATH)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(_LIB_PATH)
            i64p = ctypes.POINTER(ctypes.c_int64)
            for name, T in (("oracle_loopnest_f32", ctypes.c_float),
                            ("oracle_loopnest_f64", ctypes.c_double),
                            ("oracle_loopnest_f32_acc64", ctypes.c_float)):
                f = getattr(L, name)
                f.restype = ctypes.c_int
                f.argtypes = [ctypes.c_int, i64p, i64p, i64p, i64p, ctypes.c_int, i64p, i64p, i64p,
                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, T, T,
                              ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
            L.oracle_sample_f64.restype = ctypes.c_int
            L.oracle_sample_f64.argtypes = [ctypes.c_int, i64p, i64p, i64p, i64p, ctypes.c_int, i64p,
                                            i64p, i64p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int64, i64p,
                                            ctypes.POINTER(ctypes.c_double), ctypes.c_int]
            L.oracle_tccg_init_f32.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int64]
            L.oracle_tccg_init_f64.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int64]
            L.oracle_max_threads.restype = ctypes.c_int
            _lib = L
    return _lib


def _arr(v: Sequence[int]):
    a = (ctypes.c_int64 * max(1, len(v)))(*[int(x) for x in v])
    return a


def _colmajor_strides(labels: str, sizes: Dict[str, int]) -> Dict[str, int]:
    st, s = {}, 1
    for l in labels:
        st[l] = s
        s *= int(sizes[l])
    return st


class LoopNest:
    """The contraction ``C[c] = alpha * A[a] * B[b] (+ beta * C[c])`` over
    dense column-major tensors, with labels given as sequences of strings
    (single-character strings or lists of multi-character labels)."""

    def __init__(self, c: Sequence[str], a: Sequence[str], b: Sequence[str], sizes: Dict[str, int]):
        self.c, self.a, self.b = list(c), list(a), list(b)
        self.sizes = {k: int(v) for k, v in sizes.items()}
        sa = _colmajor_strides(self.a, self.sizes)
        sb = _colmajor_strides(self.b, self.sizes)
        sc = _colmajor_strides(self.c, self.sizes)
        self.c_ext = [self.sizes[l] for l in self.c]
        self.c_sa = [sa.get(l, 0) for l in self.c]
        self.c_sb = [sb.get(l, 0) for l in self.c]
        self.c_sc = [sc[l] for l in self.c]
        # getContractedIndices: A's indices, in A's order, in B and not in C
        self.k = [l for l in self.a if l in self.b and l not in self.c]
        self.k_ext = [self.sizes[l] for l in self.k]
        self.k_sa = [sa[l] for l in self.k]
        self.k_sb = [sb[l] for l in self.k]
        self.size_a = int(np.prod([self.sizes[l] for l in self.a]))
        self.size_b = int(np.prod([self.sizes[l] for l in self.b]))
        self.size_c = int(np.prod(self.c_ext))
        self.size_k = int(np.prod(self.k_ext)) if self.k else 1

    def shape(self, which: str) -> Tuple[int, ...]:
        labs = {"A": self.a, "B": self.b, "C": self.c}[which]
        return tuple(self.sizes[l] for l in labs)

    def _args(self):
        return (len(self.c), _arr(self.c_ext), _arr(self.c_sa), _arr(self.c_sb), _arr(self.c_sc),
                len(self.k), _arr(self.k_ext), _arr(self.k_sa), _arr(self.k_sb))

    def run(self, A: np.ndarray, B: np.ndarray, C: np.ndarray, alpha: float, beta: float,
            c_begin: int = 0, c_end: int = -1, threads: int = 0, acc64: bool = False) -> np.ndarray:
        """Run the loop nest in place on flat Fortran-order buffers; returns C.
        float32 arrays use a float accumulator (the reference's ``tmp``) unless
        ``acc64``; float64 arrays use double."""
        threads = threads or lib().oracle_max_threads()
        for x in (A, B, C):
            assert x.flags["F_CONTIGUOUS"] or x.ndim <= 1
        if C.dtype == np.float64:
            f = lib().oracle_loopnest_f64
        else:
            f = lib().oracle_loopnest_f32_acc64 if acc64 else lib().oracle_loopnest_f32
        rc = f(*self._args(), A.ctypes.data, B.ctypes.data, C.ctypes.data, float(alpha),
               float(beta), int(c_begin), int(c_end), int(threads))
        if rc != 0:
            raise RuntimeError("oracle loop nest failed (%d)" % rc)
        return C

    def sample64(self, A: np.ndarray, B: np.ndarray, C: np.ndarray, alpha: float, beta: float,
                 lins: np.ndarray, threads: int = 0) -> np.ndarray:
        """FP64 values of C at the column-major linear indices ``lins`` (C is
        read only when beta != 0)."""
        threads = threads or lib().oracle_max_threads()
        lins = np.ascontiguousarray(lins, dtype=np.int64)
        out = np.empty(len(lins), dtype=np.float64)
        is_double = 1 if A.dtype == np.float64 else 0
        assert A.dtype == B.dtype and (C is None or C.dtype == A.dtype)
        rc = lib().oracle_sample_f64(
            *self._args(), A.ctypes.data, B.ctypes.data, (C.ctypes.data if C is not None else None),
            is_double, float(alpha), float(beta), len(lins),
            lins.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(threads))
        if rc != 0:
            raise RuntimeError("oracle sample failed (%d)" % rc)
        return out

    def einsum_spec(self) -> str:
        letters, pool = {}, iter("abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ")
        for l in self.a + self.b + self.c:
            if l not in letters:
                letters[l] = next(pool)
        f = lambda ls: "".join(letters[l] for l in ls)
        return "%s,%s->%s" % (f(self.a), f(self.b), f(self.c))

    def einsum64(self, A: np.ndarray, B: np.ndarray, C: np.ndarray, alpha: float,
                 beta: float) -> np.ndarray:
        """FP64 einsum oracle; arrays are shaped (Fortran order) or flat."""
        A64 = np.asarray(A, dtype=np.float64).reshape(self.shape("A"), order="F")
        B64 = np.asarray(B, dtype=np.float64).reshape(self.shape("B"), order="F")
        R = alpha * np.einsum(self.einsum_spec(), A64, B64, optimize=True)
        if beta != 0:
            R = R + beta * np.asarray(C, dtype=np.float64).reshape(self.shape("C"), order="F")
        return np.asfortranarray(R)


def aligned_empty(n: int, dtype=np.float32, align: int = 64) -> np.ndarray:
    """Uninitialised 1-D array whose data is ``align``-byte aligned (TCCG's
    generated code uses aligned AVX loads/stores and its harness allocates
    with posix_memalign(64), tccg.py:910-919)."""
    itemsize = np.dtype(dtype).itemsize
    raw = np.empty(n * itemsize + align, dtype=np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off:off + n * itemsize].view(dtype)


def aligned_copy(x: np.ndarray, align: int = 64) -> np.ndarray:
    y = aligned_empty(x.size, x.dtype, align)
    y[:] = x.ravel()
    return y


def tccg_inputs(n: int, which: str, dtype=np.float32) -> np.ndarray:
    """TCCG's deterministic values for operand ``which`` in {'A','B','C'}
    (tccg.py:957-971)."""
    x = np.empty(n, dtype=dtype)
    w = "ABC".index(which)
    if dtype == np.float32:
        lib().oracle_tccg_init_f32(w, x.ctypes.data, n)
    else:
        lib().oracle_tccg_init_f64(w, x.ctypes.data, n)
    return x


def error_metrics(out: np.ndarray, ref: np.ndarray, tol_tccg: float = 1e-4) -> Dict[str, float]:
    """Errors of ``out`` against the FP64 reference ``ref`` (same shape)."""
    o = np.asarray(out, dtype=np.float64).ravel()
    r = np.asarray(ref, dtype=np.float64).ravel()
    d = np.abs(o - r)
    rmax = float(np.max(np.abs(r))) if r.size else 0.0
    nr = float(np.linalg.norm(r))
    m = np.abs(r) > 1e-3 * rmax
    rel = d[m] / np.abs(r[m]) if m.any() else np.zeros(0)
    # TCCG equal(): per element min(abs, rel) with rel = diff / max(|x|,|y|),
    # compared with 1e-4 (float) / 1e-9 (double); sign-aware diff here.
    mx = np.maximum(np.abs(o), np.abs(r))
    with np.errstate(divide="ignore", invalid="ignore"):
        crit = np.where(d > 0, np.minimum(d, d / np.where(mx > 0, mx, 1.0)), 0.0)
    return {
        "max_abs": float(d.max()) if d.size else 0.0,
        "normwise": float(np.linalg.norm(o - r) / nr) if nr > 0 else float(np.linalg.norm(o - r)),
        "max_rel": float(rel.max()) if rel.size else 0.0,
        "max_abs_over_max_ref": float(d.max() / rmax) if rmax > 0 else 0.0,
        "tccg_equal_worst": float(crit.max()) if crit.size else 0.0,
        "tccg_equal_pass": bool((crit <= tol_tccg).all()) if crit.size else True,
    }
