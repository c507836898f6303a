"""Public Python API: compile a contraction once, call it many times.

``compile(spec, float_type="s", precision=None, max_implementations=16)``
mirrors the ``tccg`` command (tccg/tccg.py:1246-1424): ``spec`` is a
``.tccg`` path, ``.tccg`` text or a ``Contraction``; ``float_type`` is
TCCG's ``--floatType`` (s|d); ``max_implementations`` bounds the autotuner's
candidate count like ``--maxImplementations`` (-1 = no bound, 0 = skip the
search and take the default kernels). The result is a ``Compiled`` callable.
"""
from __future__ import annotations

import os
from typing import Optional, Union

from .plan import Plan, Tuning, default_precision
from .spec import Contraction, parse_file, parse_text


def _as_contraction(spec: Union[str, Contraction]) -> Contraction:
    if isinstance(spec, Contraction):
        return spec
    if isinstance(spec, str) and ("[" not in spec) and os.path.isfile(spec):
        return parse_file(spec)
    if isinstance(spec, str) and os.path.isfile(spec):
        return parse_file(spec)
    return parse_text(spec)


class Compiled:
    """A contraction bound to tuned kernels: ``c(A, B, C)`` computes
    ``C = alpha * A * B + beta * C`` in place (torch CUDA tensors as buffers)."""

    def __init__(self, con: Contraction, precision: str, tuning: Optional[Tuning] = None,
                 dtype: Optional[str] = None):
        self.contraction = con
        self.precision = precision
        if tuning is not None and tuning.method == "log":
            from .loops import LoG
            self.plan = _LoGAdapter(LoG(con, precision))
        else:
            self.plan = Plan(con, precision=precision, tuning=tuning, dtype=dtype)
        self._ws = None

    @property
    def alpha(self) -> float:
        return self.contraction.alpha

    @property
    def beta(self) -> float:
        return self.contraction.beta

    def workspace(self, device):
        import torch
        n = self.plan.workspace_bytes
        if n == 0:
            return None
        if self._ws is None or self._ws.device != device or self._ws.numel() < n:
            self._ws = torch.empty(n, dtype=torch.uint8, device=device)
        return self._ws

    def __call__(self, A, B, C=None, alpha: Optional[float] = None, beta: Optional[float] = None,
                 stream=None):
        import torch
        if C is None:
            dt = torch.float64 if self.plan.c_dtype == "f64" else torch.float32
            C = torch.empty(self.contraction.C0.num_elements(), dtype=dt, device=A.device)
            if beta is None and self.beta != 0:
                raise ValueError("beta != 0 needs an input C")
        self.plan.run(A, B, C, alpha, beta, workspace=self.workspace(C.device), stream=stream)
        return C

    def run_host(self, A_host, B_host, C_host, alpha=None, beta=None, device="cuda", stream=None,
                 slabs: Optional[int] = None):
        """End-to-end call on HOST buffers (torch CPU tensors, ideally pinned):
        copies A, B (and C when beta != 0) to the device, runs, copies C back.
        Returns (h2d_bytes, d2h_bytes); the work is queued on ``stream`` (the
        current one by default), which the caller synchronises.

        With ``slabs`` > 1 (default: automatic for C >= 256 MiB) C is computed
        in slabs of its last index, and the copies overlap the compute on two
        copy streams: the operand without that index goes up first, the other
        one (when that index is its last) slab by slab, and each C slab comes
        back while the next one is computed. Slab plans use the full tensors'
        strides (the multi-GPU slab machinery of ``shard``)."""
        import torch
        beta_v = self.beta if beta is None else beta
        alpha_v = self.alpha if alpha is None else alpha
        dev = torch.device(device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        s = stream or torch.cuda.current_stream(dev)
        n_slabs = self._auto_slabs(C_host) if slabs is None else max(1, int(slabs))
        bufs = self._device_buffers(A_host, B_host, C_host, dev)
        dA, dB, dC = bufs
        es = lambda t: t.numel() * t.element_size()
        h2d = es(A_host) + es(B_host) + (es(C_host) if beta_v != 0 else 0)
        d2h = es(C_host)
        if n_slabs <= 1 or not isinstance(self.plan, Plan):
            with torch.cuda.stream(s):
                dA.copy_(A_host, non_blocking=True)
                dB.copy_(B_host, non_blocking=True)
                if beta_v != 0:
                    dC.copy_(C_host, non_blocking=True)
                self.plan.run(dA, dB, dC, alpha, beta, workspace=self.workspace(dev), stream=s)
                C_host.copy_(dC, non_blocking=True)
            return h2d, d2h
        from .shard import shard
        con = self.contraction
        label = con.C0.indices[-1].label
        parts = [shard(con, r, n_slabs, label) for r in range(n_slabs)]
        plans = [self._slab_plan(sh) for sh in parts]
        ws_bytes = max(p.workspace_bytes for p in plans)
        ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev) if ws_bytes else None
        up, down = self._copy_streams(dev)
        up.wait_stream(s)    # buffers free: earlier work on the caller's stream is done
        down.wait_stream(s)
        # operands: the one carrying `label` as its last index goes slab by slab
        per_slab = {}
        for name, host, d in (("A", A_host, dA), ("B", B_host, dB)):
            t = con.A0 if name == "A" else con.B0
            if t.has(label) and t.indices[-1].label == label:
                per_slab[name] = (host, d)
            else:
                with torch.cuda.stream(up):
                    d.copy_(host, non_blocking=True)
        whole_ready = torch.cuda.Event()
        whole_ready.record(up)
        done = None
        for sh, plan in zip(parts, plans):
            n_c = sh.contraction.C0.num_elements()
            c0 = sh.offsets["C"]
            with torch.cuda.stream(up):
                for name, (host, d) in per_slab.items():
                    t = sh.contraction.A0 if name == "A" else sh.contraction.B0
                    o, n = sh.offsets[name], t.num_elements()
                    d[o:o + n].copy_(host[o:o + n], non_blocking=True)
                if beta_v != 0:
                    dC[c0:c0 + n_c].copy_(C_host[c0:c0 + n_c], non_blocking=True)
                ready = torch.cuda.Event()
                ready.record(up)
            s.wait_event(whole_ready)
            s.wait_event(ready)
            ptr = lambda t, k: t.data_ptr() + sh.offsets[k] * t.element_size()
            plan.run_ptr(ptr(dA, "A"), ptr(dB, "B"), ptr(dC, "C"), alpha_v, beta_v,
                         ws.data_ptr() if ws is not None else 0,
                         ws.numel() if ws is not None else 0, s.cuda_stream)
            computed = torch.cuda.Event()
            computed.record(s)
            down.wait_event(computed)
            with torch.cuda.stream(down):
                C_host[c0:c0 + n_c].copy_(dC[c0:c0 + n_c], non_blocking=True)
            done = torch.cuda.Event()
            done.record(down)
        s.wait_event(done)  # the caller's stream completes with the last copy
        if ws is not None:
            ws.record_stream(s)
        return h2d, d2h

    # -- helpers of run_host ------------------------------------------------
    def _auto_slabs(self, C_host) -> int:
        ext = self.contraction.C0.indices[-1].size
        big = C_host.numel() * C_host.element_size() >= (256 << 20)
        return min(16, ext) if big and ext >= 2 else 1

    def _device_buffers(self, A_host, B_host, C_host, dev):
        import torch
        key = (dev, A_host.numel(), A_host.dtype, B_host.numel(), B_host.dtype, C_host.numel(),
               C_host.dtype)
        cached = getattr(self, "_host_bufs", None)
        if cached is None or cached[0] != key:
            mk = lambda h: torch.empty(h.numel(), dtype=h.dtype, device=dev)
            cached = (key, (mk(A_host), mk(B_host), mk(C_host)))
            self._host_bufs = cached
        return cached[1]

    def _copy_streams(self, dev):
        import torch
        st = getattr(self, "_streams", None)
        if st is None or st[0] != dev:
            st = (dev, torch.cuda.Stream(dev), torch.cuda.Stream(dev))
            self._streams = st
        return st[1], st[2]

    def _slab_plan(self, sh):
        cache = self.__dict__.setdefault("_slab_plans", {})
        key = (sh.label, sh.hi - sh.lo)
        if key not in cache:
            cache[key] = Plan(sh.contraction, precision=self.precision, tuning=self.plan.tuning,
                              dtype=self.plan.dtype, strides=sh.strides)
        return cache[key]

    def describe(self) -> str:
        return self.plan.describe()

    def flops(self, beta: Optional[float] = None) -> float:
        return self.contraction.flop_count(beta)


class _LoGAdapter:
    """Gives a LoG the Plan interface used by Compiled."""

    def __init__(self, log):
        self.log = log
        self.workspace_bytes = 0
        self.c_dtype = "f64" if log.precision == "fp64" else "f32"

    def run(self, A, B, C, alpha=None, beta=None, workspace=None, stream=None):
        self.log.run(A, B, C, alpha, beta, stream=stream)

    def describe(self):
        return self.log.describe()


def compile(spec, float_type: str = "s", precision: Optional[str] = None,
            max_implementations: int = 0, method: str = "gett", tuning: Optional[Tuning] = None,
            dtype: Optional[str] = None, autotune_cache: Optional[str] = None) -> Compiled:
    """Build (and optionally autotune) a contraction; see the module docstring."""
    con = _as_contraction(spec)
    con.validate()
    if float_type not in ("s", "d"):
        raise ValueError("floatType %s is not supported yet (use 's' or 'd')" % float_type)
    precision = precision or default_precision(float_type)
    if (float_type == "d") != (precision == "fp64"):
        raise ValueError("--floatType=%s does not go with precision %s" % (float_type, precision))
    if tuning is None and max_implementations != 0:
        from .autotune import autotune
        tuning = autotune(con, precision, max_implementations=max_implementations,
                          cache_path=autotune_cache, dtype=dtype)
    if tuning is None:
        tuning = Tuning(method=method)
    return Compiled(con, precision, tuning, dtype=dtype)


def contract(spec, A, B, C=None, alpha=None, beta=None, precision: str = "fp32"):
    """One-shot convenience: compile (default kernels) and run."""
    return compile(spec, precision=precision, float_type="d" if precision == "fp64" else "s")(
        A, B, C, alpha, beta)
