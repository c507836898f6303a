"""Loops-over-GEMM (LoG), TCCG's third method (tccg/gemm_loop.py:76-348), as
ONE batched launch.

TCCG picks GEMM indices (m, n, k), loops over the remaining free indices and
calls a (batched) BLAS GEMM per loop iteration (gemm_loop.py:141-192). Here the
GEMM is the strided sub-contraction C[m0, n0] = A[m0, K] * B[n0, K] (m0 = C's
stride-one index, n0 = the first N index in C's order, all contracted
indices as k); every value of the other free indices is one item of a grouped
launch (one plan, item pointers offset into the full tensors), so the whole
loop nest is a single packing launch plus a single GEMM launch -- the batch
index is the work-list position. Unlike TCCG's BLAS-based LoG, the GEMM
indices need not be stride-one: the kernels read through offset tables.
"""
from __future__ import annotations

import ctypes
import itertools
from typing import Dict, List

from . import _native as N
from .plan import Plan
from .spec import Contraction, make_contraction


def _dense(labels, sizes) -> Dict[str, int]:
    st, s = {}, 1
    for l in labels:
        st[l] = s
        s *= sizes[l]
    return st


class LoG:
    def __init__(self, con: Contraction, precision: str = "fp32"):
        con.validate()
        self.con = con
        self.precision = precision
        sizes = {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices}
        ga = con.A0 if con.A0.has(con.C0.labels[0]) else con.B0
        m_all = [l for l in con.C0.labels if ga.has(l)]
        n_all = [l for l in con.C0.labels if not ga.has(l)]
        self.m0 = m_all[0]
        self.n0 = n_all[0] if n_all else None
        self.loop = [l for l in con.C0.labels if l not in (self.m0, self.n0)]
        self.k = [l for l in con.A0.labels if con.B0.has(l) and not con.C0.has(l)]
        full = {"A": _dense(con.A0.labels, sizes), "B": _dense(con.B0.labels, sizes),
                "C": _dense(con.C0.labels, sizes)}
        keep = lambda T: [l for l in T.labels if l not in self.loop]
        sub = {l: sizes[l] for l in keep(con.A0) + keep(con.B0) + keep(con.C0)}
        self.gemm = make_contraction(keep(con.C0), keep(con.A0), keep(con.B0), sub, con.alpha,
                                     con.beta, fuse=False)
        self.plan = Plan(self.gemm, precision=precision, strides=full)
        # one item per value of the loop indices
        self.offsets: List[Dict[str, int]] = []
        for vals in itertools.product(*[range(sizes[l]) for l in self.loop]):
            off = {t: sum(v * full[t][l] for l, v in zip(self.loop, vals) if l in full[t])
                   for t in ("A", "B", "C")}
            self.offsets.append(off)
        self._lib = N.lib()
        n = len(self.offsets)
        arr = (ctypes.c_void_p * n)(*([self.plan._h.value] * n))
        h = ctypes.c_void_p()
        N.check(self._lib.tccg_group_create(arr, n, ctypes.byref(h)))
        self._h = h
        ws = ctypes.c_size_t()
        N.check(self._lib.tccg_group_workspace(self._h, ctypes.byref(ws)))
        self.workspace_bytes = int(ws.value)
        self._ws = None
        self._key = None

    @property
    def batch(self) -> int:
        return len(self.offsets)

    def describe(self) -> str:
        return "LoG: GEMM over (%s, %s, %s), %d items looped over %s; %s" % (
            self.m0, self.n0, ",".join(self.k), self.batch, ",".join(self.loop) or "-",
            self.plan.describe())

    def run(self, A, B, C, alpha=None, beta=None, stream=None):
        import torch
        alpha = self.con.alpha if alpha is None else alpha
        beta = self.con.beta if beta is None else beta
        key = (A.data_ptr(), B.data_ptr(), C.data_ptr(), alpha, beta)
        if key != self._key:  # (re)bind the work list for these buffers
            if self._ws is None:
                self._ws = torch.empty(max(self.workspace_bytes, 1), dtype=torch.uint8, device=C.device)
            n = self.batch
            es = lambda t: t.element_size()
            pa = (ctypes.c_void_p * n)(*[A.data_ptr() + o["A"] * es(A) for o in self.offsets])
            pb = (ctypes.c_void_p * n)(*[B.data_ptr() + o["B"] * es(B) for o in self.offsets])
            pc = (ctypes.c_void_p * n)(*[C.data_ptr() + o["C"] * es(C) for o in self.offsets])
            al = (ctypes.c_double * n)(*([alpha] * n))
            be = (ctypes.c_double * n)(*([beta] * n))
            N.check(self._lib.tccg_group_bind(self._h, pa, pb, pc, al, be,
                                              ctypes.c_void_p(self._ws.data_ptr()),
                                              ctypes.c_size_t(self._ws.numel())))
            self._key = key
            self._keep = (A, B, C)
        s = stream or torch.cuda.current_stream(C.device)
        N.check(self._lib.tccg_group_run(self._h, ctypes.c_void_p(s.cuda_stream)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.tccg_group_destroy(h)
            except Exception:  # noqa: BLE001
                pass
            self._h = None
