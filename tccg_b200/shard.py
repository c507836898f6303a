"""Splitting one contraction across GPUs without communication.

C's tiles are independent, so rank r of W computes the C slab where one free
index (C's index with the largest stride whose extent is >= W) lies in
[lo_r, hi_r). The slab is itself a contraction: the same labels with that
index's extent reduced, the FULL tensors' strides, and element offsets into
the operand that carries the index and into C (the other operand is used
whole). No collective is needed on the data path.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict

from .spec import Contraction, make_contraction


@dataclass
class Shard:
    label: str                     # the split index
    lo: int
    hi: int
    contraction: Contraction       # the slab contraction (reduced extent)
    strides: Dict[str, Dict[str, int]]   # full-tensor strides, for Plan(strides=...)
    offsets: Dict[str, int]        # element offsets into A, B, C


def _dense(labels, sizes):
    st, s = {}, 1
    for l in labels:
        st[l] = s
        s *= sizes[l]
    return st


def split_index(con: Contraction, world: int) -> str:
    """C's index with the largest stride among those with extent >= world
    (the last such index of C)."""
    for idx in reversed(con.C0.indices):
        if idx.size >= world:
            return idx.label
    raise ValueError("no index of C has extent >= %d" % world)


def shard(con: Contraction, rank: int, world: int, label: str = None) -> Shard:
    if not 0 <= rank < world:
        raise ValueError("rank %d outside [0, %d)" % (rank, world))
    label = label or split_index(con, world)
    sizes = {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices}
    ext = sizes[label]
    base, rem = divmod(ext, world)
    lo = rank * base + min(rank, rem)
    hi = lo + base + (1 if rank < rem else 0)
    full = {"A": _dense(con.A0.labels, sizes), "B": _dense(con.B0.labels, sizes),
            "C": _dense(con.C0.labels, sizes)}
    sub = dict(sizes)
    sub[label] = hi - lo
    # no index fusion: the slab's strides are the full tensors', not dense ones
    sc = make_contraction(con.C0.labels, con.A0.labels, con.B0.labels, sub, con.alpha, con.beta,
                          fuse=False)
    offsets = {t: (lo * full[t][label] if label in full[t] else 0) for t in ("A", "B", "C")}
    return Shard(label, lo, hi, sc, full, offsets)


def run(plan, sh: Shard, A, B, C, workspace=None, stream=None) -> None:
    """Run the slab ``sh`` with a plan built as
    ``Plan(sh.contraction, strides=sh.strides)`` on FULL torch tensors A, B, C."""
    import torch
    if workspace is None and plan.workspace_bytes:
        workspace = torch.empty(plan.workspace_bytes, dtype=torch.uint8, device=C.device)
    s = stream or torch.cuda.current_stream(C.device)
    ptr = lambda t, k: t.data_ptr() + sh.offsets[k] * t.element_size()
    plan.run_ptr(ptr(A, "A"), ptr(B, "B"), ptr(C, "C"), sh.contraction.alpha, sh.contraction.beta,
                 workspace.data_ptr() if workspace is not None else 0,
                 workspace.numel() if workspace is not None else 0, s.cuda_stream)
