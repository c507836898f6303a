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

    def run_host(self, A_host, B_host, C_host, alpha=None, beta=None, device="cuda", stream=None):
        """End-to-end call on HOST buffers (torch CPU tensors, ideally pinned):
        copies A, B (and C when beta != 0) to the device, runs, copies C back.
        Returns (h2d_bytes, d2h_bytes)."""
        import torch
        beta_v = self.beta if beta is None else beta
        dev = torch.device(device)
        s = stream or torch.cuda.current_stream(dev)
        with torch.cuda.stream(s):
            dA = A_host.to(dev, non_blocking=True)
            dB = B_host.to(dev, non_blocking=True)
            h2d = dA.numel() * dA.element_size() + dB.numel() * dB.element_size()
            if beta_v != 0:
                dC = C_host.to(dev, non_blocking=True)
                h2d += dC.numel() * dC.element_size()
            else:
                dC = torch.empty(C_host.shape, dtype=C_host.dtype, device=dev)
            self.plan.run(dA, dB, dC, alpha, beta, workspace=self.workspace(dev), stream=s)
            C_host.copy_(dC, non_blocking=True)
        return h2d, dC.numel() * dC.element_size()

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
