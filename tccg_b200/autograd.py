"""Differentiation: a torch.autograd.Function over a contraction whose
backward is itself two generated contractions (new in this build; TCCG has no
backward).

For  C = alpha * A * B (+ beta * C_in):
    dA[A's indices] = alpha * dC[C's indices] * B[B's indices]   (sum over N)
    dB[B's indices] = alpha * A[A's indices] * dC[C's indices]   (sum over M)
    dC_in = beta * dC
Each gradient contraction is parsed/fused/classified like any other and runs
through its own native plan (cached per contraction and precision).

Tensors are torch CUDA tensors whose memory is the column-major tensor of the
contraction: e.g. for A[i,m,a] a contiguous tensor of shape (a, m, i), or a
flat one. The output C has the reversed shape of C's indices.
"""
from __future__ import annotations

from collections import OrderedDict
from typing import Dict, Tuple

from .plan import Plan
from .spec import Contraction, make_contraction

# Plans shared across contraction objects with the same text, least recently
# used first; at most _MAX_PLANS are kept (each holds its device offset
# tables), the oldest is dropped past that.
_MAX_PLANS = 256
_PLANS: "OrderedDict[Tuple, Plan]" = OrderedDict()


def _sizes(con: Contraction) -> Dict[str, int]:
    return {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices}


def _labels(t):
    return [i.label for i in t.indices]


def grad_contractions(con: Contraction) -> Tuple[Contraction, Contraction]:
    """(dA = dC * B, dB = A * dC) as contractions over the original labels.
    Built once per contraction object (parsing and fusion cost ~0.4 ms of
    host time, more than the kernels of a mid-sized backward pass)."""
    cached = con.__dict__.get("_grad_contractions")
    if cached is not None:
        return cached
    s = _sizes(con)
    dA = make_contraction(_labels(con.A0), _labels(con.C0), _labels(con.B0), s, con.alpha, 0.0)
    dB = make_contraction(_labels(con.B0), _labels(con.A0), _labels(con.C0), s, con.alpha, 0.0)
    con.__dict__["_grad_contractions"] = (dA, dB)
    return dA, dB


def _plan(con: Contraction, precision: str, dtype: str, role: str) -> Plan:
    """The plan of ``con`` for (precision, dtype, role): looked up on the
    contraction object first, then by the contraction's text across objects."""
    local = con.__dict__.setdefault("_autograd_plans", {})
    p = local.get((precision, dtype, role))
    if p is not None:
        return p
    key = (str(con), tuple(sorted(_sizes(con).items())), precision, dtype, role)
    p = _PLANS.get(key)
    if p is None:
        p = Plan(con, precision=precision, dtype=dtype)
        _PLANS[key] = p
        while len(_PLANS) > _MAX_PLANS:
            _PLANS.popitem(last=False)
    else:
        _PLANS.move_to_end(key)
    local[(precision, dtype, role)] = p
    return p


def _workspace(p: Plan, device):
    """One workspace per plan, device and stream, reused across calls (uses on
    one stream are ordered; another stream gets its own)."""
    import torch
    if not p.workspace_bytes:
        return None
    key = (device, torch.cuda.current_stream(device).cuda_stream)
    cache = p.__dict__.setdefault("_autograd_ws", {})
    ws = cache.get(key)
    if ws is None:
        ws = torch.empty(p.workspace_bytes, dtype=torch.uint8, device=device)
        cache[key] = ws
    return ws


def _out_shape(t):
    return tuple(i.size for i in reversed(t.indices))


def _torch_dtype(precision: str):
    import torch
    return torch.float64 if precision == "fp64" else torch.float32


def _operand_dtype(precision: str, t) -> str:
    import torch
    if precision == "fp64":
        return "f64"
    if precision == "bf16" and t.dtype == torch.bfloat16:
        return "bf16"
    return "f32"


def _contract(con: Contraction, precision: str, A, B, role: str, C_in=None, beta: float = 0.0):
    import torch
    dt = _operand_dtype(precision, A)
    if dt == "f32" and A.dtype != torch.float32:
        A = A.float()
    if dt == "f32" and B.dtype != torch.float32:
        B = B.float()
    if dt == "bf16" and B.dtype != torch.bfloat16:
        B = B.to(torch.bfloat16)
    p = _plan(con, precision, dt, role)
    out_t = _torch_dtype(precision)
    if C_in is not None and beta != 0.0:
        C = C_in.to(out_t).contiguous().clone().reshape(_out_shape(con.C0))
    else:
        C = torch.empty(_out_shape(con.C0), dtype=out_t, device=A.device)
        beta = 0.0
    p.run(A.contiguous(), B.contiguous(), C, con.alpha, beta, workspace=_workspace(p, A.device))
    return C


class GettFunction:
    """``GettFunction.apply(A, B, con, precision="fp32", C_in=None)``.

    Implemented as a thin wrapper so that the torch import stays lazy; see
    ``_Fn`` for the autograd.Function."""

    @staticmethod
    def apply(A, B, con: Contraction, precision: str = "fp32", C_in=None):
        return _fn().apply(A, B, C_in, con, precision)


_FN = None


def _fn():
    global _FN
    if _FN is not None:
        return _FN
    import torch

    class _Fn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, A, B, C_in, con, precision):
            ctx.con, ctx.precision = con, precision
            ctx.has_c = C_in is not None
            ctx.a_dtype, ctx.b_dtype = A.dtype, B.dtype
            ctx.save_for_backward(A, B)
            return _contract(con, precision, A, B, "fwd", C_in, con.beta if C_in is not None else 0.0)

        @staticmethod
        def backward(ctx, dC):
            A, B = ctx.saved_tensors
            con, prec = ctx.con, ctx.precision
            dAc, dBc = grad_contractions(con)
            dC = dC.contiguous()
            dA = dB = dCin = None
            if ctx.needs_input_grad[0]:
                dA = _contract(dAc, prec, dC, B, "dA").reshape(A.shape).to(ctx.a_dtype)
            if ctx.needs_input_grad[1]:
                dB = _contract(dBc, prec, A, dC, "dB").reshape(B.shape).to(ctx.b_dtype)
            if ctx.has_c and ctx.needs_input_grad[2]:
                dCin = con.beta * dC
            return dA, dB, dCin, None, None

    _FN = _Fn
    return _FN
