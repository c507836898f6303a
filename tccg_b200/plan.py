"""Host side of one contraction: the GETT descriptor and the native plan.

``gett_descriptor`` turns a (fused) ``Contraction`` into the C ABI's
``tccg_desc``: the operand holding C's stride-one index becomes the kernels'
"A" (TCCG's swap, tccg/gett.py:70-76), M and N modes keep C's order (so the
first M mode is C's stride-one index and the epilogue stores are coalesced),
and the K modes follow the operand whose stride-one index is a K index.

``Plan`` owns a native ``tccg_plan``; ``Plan.run`` takes torch tensors as
plain device buffers (torch is only the allocator and stream provider here).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Tuple

from . import _native as N
from .spec import Contraction, Tensor


@dataclass
class GettView:
    """The contraction in GETT form, as given to the kernels."""

    swap_ab: bool
    m: List[Tuple[str, int]]
    n: List[Tuple[str, int]]
    k: List[Tuple[str, int]]
    a_m: List[int]
    a_k: List[int]
    b_n: List[int]
    b_k: List[int]
    c_m: List[int]
    c_n: List[int]

    @property
    def M(self) -> int:
        return _prod(e for _, e in self.m)

    @property
    def N(self) -> int:
        return _prod(e for _, e in self.n)

    @property
    def K(self) -> int:
        return _prod(e for _, e in self.k)


def _prod(it) -> int:
    p = 1
    for v in it:
        p *= int(v)
    return p


def gett_view(con: Contraction, strides: Optional[dict] = None, n_order: int = 0,
              k_order: int = 0) -> GettView:
    """GETT view of ``con``. ``strides`` may override the dense column-major
    strides: {'A': {label: stride}, 'B': ..., 'C': ...} (elements).

    Mode orders (the autotuner searches them; 0 = the heuristics below):
    ``n_order`` 1 = N modes in C's order, 2 = GB's unit-stride N mode first;
    ``k_order`` 1 = K modes in GA's order, 2 = in GB's order."""
    con.validate()
    A, B, C = con.A, con.B, con.C
    swap = not A.has(C.indices[0].label)
    GA, GB = (B, A) if swap else (A, B)
    nameA, nameB = ("B", "A") if swap else ("A", "B")

    def st(T: Tensor, name: str, lab: str) -> int:
        if strides and name in strides and lab in strides[name]:
            return int(strides[name][lab])
        return T.stride(lab)

    m = [(i.label, i.size) for i in con.m_indices]
    n = [(i.label, i.size) for i in con.n_indices]
    kset = [i.label for i in con.k_indices]
    sizes = {i.label: i.size for i in GA.indices + GB.indices}
    # The packing pass reads an operand coalesced when its stride-one index
    # is the first mode of its row order or of the K order. M keeps C's order
    # (C's stride-one index first: coalesced epilogue stores). N is free
    # (the epilogue's lanes run along m).
    # GB's unit-stride N mode leads when GB is large next to C (K >= M/4);
    # otherwise C's order stays (its stores then sweep C's own layout)
    nb = [l for l, e in n if e > 1]
    K = _prod(i.size for i in con.k_indices)
    M = _prod(e for _, e in m)
    if nb and (n_order == 2 or (n_order == 0 and 4 * K >= M)):
        first = min(nb, key=lambda l: abs(st(GB, nameB, l)))
        if abs(st(GB, nameB, first)) == 1:
            n = [x for x in n if x[0] == first] + [x for x in n if x[0] != first]
    # K order: the operand whose stride-one index is contracted leads; when
    # both are, the larger operand.
    def lead(T: Tensor) -> Optional[str]:
        real = [i for i in T.indices if i.size > 1]
        return real[0].label if real and real[0].label in kset else None
    la, lb = lead(GA), lead(GB)
    if k_order in (1, 2):
        owner = GA if k_order == 1 else GB
    elif la and lb and la != lb:
        owner = GA if GA.num_elements() >= GB.num_elements() else GB
    elif la:
        owner = GA
    elif lb:
        owner = GB
    else:
        owner = GA
    order = [l for l in owner.labels if l in kset]
    k = [(l, sizes[l]) for l in order]
    v = GettView(
        swap_ab=swap, m=m, n=n, k=k,
        a_m=[st(GA, nameA, l) for l, _ in m], a_k=[st(GA, nameA, l) for l, _ in k],
        b_n=[st(GB, nameB, l) for l, _ in n], b_k=[st(GB, nameB, l) for l, _ in k],
        c_m=[st(C, "C", l) for l, _ in m], c_n=[st(C, "C", l) for l, _ in n])
    # a contraction without N modes (matrix-vector) or K modes (outer product)
    # gets a unit dummy mode
    if not v.n:
        v.n, v.b_n, v.c_n = [("_n", 1)], [0], [0]
    if not v.k:
        v.k, v.a_k, v.b_k = [("_k", 1)], [0], [0]
    return v


def native_desc(v: GettView) -> N.Desc:
    d = N.Desc()
    if max(len(v.m), len(v.n), len(v.k)) > N.MAX_MODES:
        raise ValueError("more than %d modes in one index class" % N.MAX_MODES)
    d.nm, d.nn, d.nk = len(v.m), len(v.n), len(v.k)
    d.swap_ab = int(v.swap_ab)
    for i, (_, e) in enumerate(v.m):
        d.m_ext[i], d.a_m_stride[i], d.c_m_stride[i] = e, v.a_m[i], v.c_m[i]
    for i, (_, e) in enumerate(v.n):
        d.n_ext[i], d.b_n_stride[i], d.c_n_stride[i] = e, v.b_n[i], v.c_n[i]
    for i, (_, e) in enumerate(v.k):
        d.k_ext[i], d.a_k_stride[i], d.b_k_stride[i] = e, v.a_k[i], v.b_k[i]
    return d


DTYPES = {"f32": N.F32, "f64": N.F64, "bf16": N.BF16}


def default_precision(float_type: str) -> str:
    """``--floatType=s`` -> fp32, ``d`` -> fp64 (tccg.py:1315-1326)."""
    return {"s": "fp32", "d": "fp64"}[float_type]


def operand_dtype(precision: str, bf16_inputs: bool = False) -> str:
    if precision == "fp64":
        return "f64"
    if precision == "bf16" and bf16_inputs:
        return "bf16"
    return "f32"


@dataclass
class Tuning:
    method: str = "gett"
    ksplit: int = 0  # 0: automatic (split K when the C tiles cannot fill the GPU)
    raster: int = 0
    max_ctas: int = 0
    variant: int = 0
    pair: int = 0
    direct: int = 0  # CUDA-core kernels: 0 auto, 1 no packing pass, -1 always pack
    shortk: int = 0  # CUDA-core kernels, K <= 32: 0 auto, 1 kernel prefetching C, -1 never
    simt_tile: int = 0  # CUDA-core tiles: 0 auto, 1 128x128, 2 128x32, 3 32x128
    tail_split: int = 0  # tcgen05: 0 auto (k slices for a short last round), -1 never
    load: int = 0  # tcgen05 BF16x3, FP32 operands: 0 auto, 1 packing pass + TMA, 2 gather
    tile_n: int = 0  # tcgen05 tile width: 0 default, 128, 192 (BF16, BF16x3) or 256 (BF16)
    skinny: int = 0  # FP32 operands, min(M, N) small: 0 auto, 1 the skinny kernel, -1 never,
    #                  2 its tensor-core form (BF16x3)
    # mode orders of the GETT view (gett_view): 0 = heuristic
    n_order: int = 0  # 1 = C's order, 2 = GB's unit-stride N mode first
    k_order: int = 0  # 1 = GA's order, 2 = GB's order

    def native(self) -> N.Tuning:
        t = N.Tuning()
        t.method = N.METHODS[self.method]
        t.ksplit = int(self.ksplit)
        t.raster = int(self.raster)
        t.max_ctas = int(self.max_ctas)
        t.variant = int(self.variant)
        t.pair = int(self.pair)
        t.direct = int(self.direct)
        t.shortk = int(self.shortk)
        t.simt_tile = int(self.simt_tile)
        t.tail_split = int(self.tail_split)
        t.load = int(self.load)
        t.tile_n = int(self.tile_n)
        t.skinny = int(self.skinny)
        return t

    def key(self) -> str:
        return "%s/k%d/r%d/c%d/v%d/p%d/d%d/s%d/t%d/l%d/g%d/n%d/o%d%d/w%d" % (
            self.method, self.ksplit, self.raster, self.max_ctas, self.variant, self.pair,
            self.direct, self.shortk, self.simt_tile, self.tail_split, self.load, self.tile_n,
            self.n_order, self.k_order, self.skinny)


class Plan:
    """A native plan: one contraction bound to kernels (the role of TCCG's
    specialised ``gett()``)."""

    def __init__(self, con: Contraction, precision: str = "fp32", dtype: Optional[str] = None,
                 tuning: Optional[Tuning] = None, strides: Optional[dict] = None,
                 view: Optional[GettView] = None):
        self.con = con
        self.precision = precision
        self.dtype = dtype or operand_dtype(precision)
        self.tuning = tuning or Tuning()
        # ``view``: a hand-made GETT view of ``con`` (mode orders of one's own)
        self.view = view if view is not None else gett_view(
            con, strides, n_order=self.tuning.n_order, k_order=self.tuning.k_order)
        self._desc = native_desc(self.view)
        self._lib = N.lib()
        h = ctypes.c_void_p()
        t = self.tuning.native()
        N.check(self._lib.tccg_plan_create(ctypes.byref(self._desc), DTYPES[self.dtype],
                                           N.PRECISIONS[precision], ctypes.byref(t),
                                           ctypes.byref(h)))
        self._h = h
        ws = ctypes.c_size_t()
        N.check(self._lib.tccg_plan_workspace(self._h, ctypes.byref(ws)))
        self.workspace_bytes = int(ws.value)

    # -- info -------------------------------------------------------------
    def describe(self) -> str:
        buf = ctypes.create_string_buffer(1024)
        N.check(self._lib.tccg_plan_describe(self._h, buf, 1024))
        return buf.value.decode()

    def flops(self, beta: float = 0.0) -> float:
        return float(self._lib.tccg_plan_flops(self._h, float(beta)))

    @property
    def c_dtype(self) -> str:
        return "f64" if self.precision == "fp64" else "f32"

    def status(self) -> int:
        """Device status word (0 = fine); synchronises the device."""
        s = ctypes.c_int32()
        N.check(self._lib.tccg_plan_status(self._h, ctypes.byref(s)))
        return int(s.value)

    # -- execution --------------------------------------------------------
    def run_ptr(self, A: int, B: int, C: int, alpha: float, beta: float, ws: int, ws_bytes: int,
                stream: int) -> None:
        N.check(self._lib.tccg_plan_run(self._h, ctypes.c_void_p(A), ctypes.c_void_p(B),
                                        ctypes.c_void_p(C), float(alpha), float(beta),
                                        ctypes.c_void_p(ws), ctypes.c_size_t(ws_bytes),
                                        ctypes.c_void_p(stream)))

    def run(self, A, B, C, alpha: Optional[float] = None, beta: Optional[float] = None,
            workspace=None, stream=None) -> None:
        """C = alpha * contract(A, B) + beta * C with torch CUDA tensors whose
        memory is the column-major tensor of the contraction (the first index
        has stride one; e.g. a contiguous tensor of the reversed shape, or a
        flat one)."""
        import torch
        alpha = self.con.alpha if alpha is None else alpha
        beta = self.con.beta if beta is None else beta
        _check_buffer(A, self.con.A0.num_elements(), self.dtype, "A")
        _check_buffer(B, self.con.B0.num_elements(), self.dtype, "B")
        _check_buffer(C, self.con.C0.num_elements(), self.c_dtype, "C")
        if workspace is None and self.workspace_bytes:
            workspace = torch.empty(self.workspace_bytes, dtype=torch.uint8, device=C.device)
        ws_ptr = workspace.data_ptr() if workspace is not None else 0
        ws_n = workspace.numel() * workspace.element_size() if workspace is not None else 0
        if stream is None:
            stream = torch.cuda.current_stream(C.device)
        self.run_ptr(A.data_ptr(), B.data_ptr(), C.data_ptr(), alpha, beta, ws_ptr, ws_n,
                     stream.cuda_stream)

    def run_timed(self, A, B, C, alpha: Optional[float] = None, beta: Optional[float] = None,
                  workspace=None, stream=None) -> Tuple[float, float, float]:
        """``run`` with CUDA-event timing of each kernel; returns milliseconds of
        (packing, GEMM kernel, reduction/transposition). Synchronises."""
        import torch
        alpha = self.con.alpha if alpha is None else alpha
        beta = self.con.beta if beta is None else beta
        if workspace is None and self.workspace_bytes:
            workspace = torch.empty(self.workspace_bytes, dtype=torch.uint8, device=C.device)
        ws_ptr = workspace.data_ptr() if workspace is not None else 0
        ws_n = workspace.numel() if workspace is not None else 0
        if stream is None:
            stream = torch.cuda.current_stream(C.device)
        ms = (ctypes.c_float * 3)()
        N.check(self._lib.tccg_plan_run_timed(
            self._h, ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(B.data_ptr()),
            ctypes.c_void_p(C.data_ptr()), float(alpha), float(beta), ctypes.c_void_p(ws_ptr),
            ctypes.c_size_t(ws_n), ctypes.c_void_p(stream.cuda_stream), ms))
        return float(ms[0]), float(ms[1]), float(ms[2])

    def run_events(self, A, B, C, events, alpha: Optional[float] = None,
                   beta: Optional[float] = None, workspace=None, stream=None) -> None:
        """``run`` that records the six ``torch.cuda.Event`` objects ``events``
        (created with enable_timing=True) around its kernels without
        synchronising: events[2i], events[2i+1] bracket packing (i = 0), the
        GEMM kernel (1) and the reduction/transposition (2)."""
        import torch
        alpha = self.con.alpha if alpha is None else alpha
        beta = self.con.beta if beta is None else beta
        if stream is None:
            stream = torch.cuda.current_stream(C.device)
        if workspace is None and self.workspace_bytes:
            workspace = torch.empty(self.workspace_bytes, dtype=torch.uint8, device=C.device)
        handles = (ctypes.c_void_p * 6)()
        for i, ev in enumerate(events):
            if not ev.cuda_event:
                ev.record(stream)  # torch creates the event on its first record
            handles[i] = ev.cuda_event
        N.check(self._lib.tccg_plan_run_events(
            self._h, ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(B.data_ptr()),
            ctypes.c_void_p(C.data_ptr()), float(alpha), float(beta),
            ctypes.c_void_p(workspace.data_ptr() if workspace is not None else 0),
            ctypes.c_size_t(workspace.numel() if workspace is not None else 0),
            ctypes.c_void_p(stream.cuda_stream), handles))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.tccg_plan_destroy(h)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self._h = None


_TORCH_DT = {"f32": "float32", "f64": "float64", "bf16": "bfloat16"}


def _check_buffer(t, numel: int, dtype: str, name: str) -> None:
    import torch
    if not isinstance(t, torch.Tensor):
        raise TypeError("%s must be a torch tensor" % name)
    if not t.is_cuda:
        raise ValueError("%s must be a CUDA tensor (there is no CPU path)" % name)
    if t.dtype != getattr(torch, _TORCH_DT[dtype]):
        raise TypeError("%s has dtype %s, expected %s" % (name, t.dtype, _TORCH_DT[dtype]))
    if t.numel() != numel:
        raise ValueError("%s has %d elements, the contraction needs %d" % (name, t.numel(), numel))
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % name)
