"""Grouped launch: many contractions of uneven extents in one persistent launch
(new in this build; TCCG has one function per contraction).

``Group([con...], precision)`` creates one native plan per contraction and a
native group. The items run in waves whose workspaces together fit a 4 GiB
region (an item above that is a wave of its own): each wave is packed and
multiplied before the next reuses the region, so the group's workspace is
that of its largest wave rather than the sum over all items.
``bind(As, Bs, Cs)`` fixes the operand pointers and the workspace (uploading
the device work lists once); after that ``run()`` issues, per wave, the
grouped packing, the grouped GETT kernels (tensor-core lanes on the given
stream, the CUDA-core skinny lanes and the CUDA-core tiles on two side
streams forked from and joined back into it) and the k-split reductions that
have work, and ``capture()`` records them into a CUDA graph (the side streams
as parallel branches) that ``replay()`` re-launches. ``run_per_item()`` is the
baseline: one tccg_plan_run per contraction.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Optional, Sequence

from . import _native as N
from .plan import Plan, Tuning
from .spec import Contraction


class Group:
    """``autotune=True`` picks each item's kernels with the autotuner: its
    tuning comes from the SQLite cache (``cache_path``, default as
    ``autotune``), and items that miss are tuned on the device (up to
    ``max_implementations`` candidates each, GETT without the tail split, as
    grouped kernels run them) and stored. ``tune_stats`` then counts cache
    hits and tuned items."""

    def __init__(self, contractions: Sequence[Contraction], precision: str = "bf16x3",
                 tunings: Optional[Sequence[Tuning]] = None, dtype: Optional[str] = None,
                 autotune: bool = False, max_implementations: int = 8,
                 cache_path: Optional[str] = None):
        self.contractions = list(contractions)
        self.precision = precision
        self.tune_stats = {}
        if autotune:
            if tunings is not None:
                raise ValueError("give tunings or autotune=True, not both")
            from .autotune import TuningDB, autotune as _autotune
            db = TuningDB(cache_path)
            tunings = [_autotune(c, precision, max_implementations, dtype=dtype, grouped=True,
                                 db=db, stats=self.tune_stats) for c in self.contractions]
        # the grouped kernels do not run the tcgen05 tail split (the other
        # items' tiles fill the persistent grid's rounds anyway): plans made
        # without it, so that grouped and per-item runs compute the same sums
        tunings = [dataclasses.replace(t or Tuning(), tail_split=-1)
                   for t in (tunings or [None] * len(self.contractions))]
        self.plans: List[Plan] = [Plan(c, precision=precision, tuning=t, dtype=dtype)
                                  for c, t in zip(self.contractions, tunings)]
        self._lib = N.lib()
        arr = (ctypes.c_void_p * len(self.plans))(*[p._h.value for p in self.plans])
        h = ctypes.c_void_p()
        N.check(self._lib.tccg_group_create(arr, len(self.plans), ctypes.byref(h)))
        self._h = h
        ws = ctypes.c_size_t()
        N.check(self._lib.tccg_group_workspace(self._h, ctypes.byref(ws)))
        self.workspace_bytes = int(ws.value)
        self._ws = None
        self._bound = None
        self._graph = None

    def flops(self) -> float:
        return sum(c.flop_count() for c in self.contractions)

    def bind(self, As, Bs, Cs, alphas=None, betas=None, workspace=None):
        import torch
        n = len(self.plans)
        if not (len(As) == len(Bs) == len(Cs) == n):
            raise ValueError("need one A, B and C per contraction")
        alphas = [c.alpha for c in self.contractions] if alphas is None else list(alphas)
        betas = [c.beta for c in self.contractions] if betas is None else list(betas)
        dev = Cs[0].device
        if workspace is None:
            workspace = torch.empty(max(self.workspace_bytes, 1), dtype=torch.uint8, device=dev)
        self._ws = workspace
        vp = ctypes.c_void_p * n
        dd = ctypes.c_double * n
        self._bound = (list(As), list(Bs), list(Cs))  # keep the buffers alive
        N.check(self._lib.tccg_group_bind(
            self._h, vp(*[a.data_ptr() for a in As]), vp(*[b.data_ptr() for b in Bs]),
            vp(*[c.data_ptr() for c in Cs]), dd(*alphas), dd(*betas),
            ctypes.c_void_p(workspace.data_ptr()), ctypes.c_size_t(workspace.numel())))
        self._alphas, self._betas = alphas, betas

    def run(self, stream=None):
        import torch
        if self._bound is None:
            raise RuntimeError("bind() first")
        s = stream or torch.cuda.current_stream(self._bound[2][0].device)
        N.check(self._lib.tccg_group_run(self._h, ctypes.c_void_p(s.cuda_stream)))

    def capture(self):
        """Record run() into a CUDA graph."""
        import torch
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self._bound[2][0].device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.run(s)  # warm-up outside capture (attributes, first-use setup)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s):
            self.run(s)
        self._graph = g
        return g

    def replay(self):
        if self._graph is None:
            self.capture()
        self._graph.replay()

    def run_per_item(self, stream=None):
        """Baseline: one plan run (pack + GETT launch) per contraction."""
        As, Bs, Cs = self._bound
        for p, a, b, c, al, be in zip(self.plans, As, Bs, Cs, self._alphas, self._betas):
            p.run(a, b, c, al, be, workspace=self._ws, stream=stream)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.tccg_group_destroy(h)
            except Exception:  # noqa: BLE001
                pass
            self._h = None
