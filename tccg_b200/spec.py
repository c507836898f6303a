"""Contraction front end: the ``.tccg`` format, the tensor/index model, index
fusion and the M/N/K classification.

This module is the host-side mirror of TCCG's front end. It keeps TCCG's
surface so that a ``.tccg`` file that TCCG accepts means the same contraction
here:

* ``parse_text`` / ``parse_file`` follow ``Tccg.parseFile``
  (tccg/tccg.py:559-684): tensors are ``[A-C][...]`` with lower-case labels,
  the first distinct tensor is C, the second A, the third B (renamed with a
  warning otherwise, tccg.py:663-671), ``label = N`` lines give extents
  (tccg.py:643-647), ``#`` starts a comment, ``+=``/``-=``/``+-``/``-+`` are
  rejected (tccg.py:576-582), alpha/beta come from the numbers on the
  right-hand side with TCCG's placement rules (tccg.py:586-640).
* ``fuse_indices`` follows ``Tccg.fuseIndices`` (tccg.py:432-552).
* ``m_indices`` / ``n_indices`` / ``k_indices`` / ``loop_indices`` follow
  tccg/tccg_util.py:212-296 and 597-611.
* ``Tensor`` keeps TCCG's column-major leading dimensions
  (tccg/tensor.py:11-13): ``ld[0] = 1``, ``ld[i] = ld[i-1] * size[i-1]``.
* ``flop_count`` is ``Tccg.getFlopCount`` (tccg.py:1230-1234) for real types.

Errors are raised as ``TccgSyntaxError`` instead of ``exit(-1)``.
"""
from __future__ import annotations

import copy
import re
import warnings
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple


class TccgSyntaxError(ValueError):
    """A ``.tccg`` description that TCCG would reject."""


class TccgUnsupported(ValueError):
    """A valid contraction that this code path does not handle (e.g. batch
    indices, which TCCG's GETT rejects too, tccg/gett.py:42-45)."""


@dataclass
class Index:
    """One tensor mode: a label and an extent (tccg/Index.py:2-13). Equality
    is by label only, as in TCCG."""

    label: str
    size: int

    def __eq__(self, other):  # label equality, like index.__eq__
        return isinstance(other, Index) and self.label == other.label

    def __hash__(self):
        return hash(self.label)

    def __str__(self):
        return "(%s,%d)" % (self.label, self.size)


@dataclass
class Tensor:
    """A dense column-major tensor: the first index has stride one."""

    label: str
    indices: List[Index]
    ld: List[int] = field(default_factory=list)

    def __post_init__(self):
        self.indices = [Index(i.label, int(i.size)) for i in self.indices]
        if not self.ld:
            self.ld = self._dense_ld()

    def _dense_ld(self) -> List[int]:
        ld = [1]
        for i in range(1, len(self.indices)):
            ld.append(ld[i - 1] * self.indices[i - 1].size)
        return ld

    @property
    def labels(self) -> List[str]:
        return [i.label for i in self.indices]

    @property
    def sizes(self) -> List[int]:
        return [i.size for i in self.indices]

    def num_elements(self) -> int:
        n = 1
        for i in self.indices:
            n *= i.size
        return n

    def has(self, label: str) -> bool:
        return label in self.labels

    def pos(self, label: str) -> int:
        try:
            return self.labels.index(label)
        except ValueError:
            return -1

    def stride(self, label: str) -> int:
        p = self.pos(label)
        if p < 0:
            raise KeyError(label)
        return self.ld[p]

    def __str__(self):
        return "%s[%s]" % (self.label, ",".join(self.labels))


@dataclass
class Contraction:
    """``C = alpha * A * B + beta * C`` over column-major dense tensors.

    ``C``, ``A``, ``B`` are the tensors after index fusion; ``C0``, ``A0``,
    ``B0`` are the tensors as written in the file (the memory layout is the
    same, fusion only merges modes that are adjacent in every tensor).
    """

    C: Tensor
    A: Tensor
    B: Tensor
    alpha: float = 1.0
    beta: float = 0.0
    C0: Optional[Tensor] = None
    A0: Optional[Tensor] = None
    B0: Optional[Tensor] = None

    def __post_init__(self):
        if self.C0 is None:
            self.C0 = copy.deepcopy(self.C)
            self.A0 = copy.deepcopy(self.A)
            self.B0 = copy.deepcopy(self.B)

    # --- classification (tccg/tccg_util.py:212-296, 597-611) --------------
    @property
    def m_indices(self) -> List[Index]:
        return m_indices(self.A, self.B, self.C)

    @property
    def n_indices(self) -> List[Index]:
        return n_indices(self.A, self.B, self.C)

    @property
    def k_indices(self) -> List[Index]:
        return k_indices(self.A, self.B, self.C)

    @property
    def loop_indices(self) -> List[Index]:
        return loop_indices(self.A, self.B, self.C)

    @property
    def swapped(self) -> bool:
        """True when B holds C's stride-one index: GETT then treats B as its
        "A" operand (tccg/gett.py:70-76 swaps when A carries an N index)."""
        return not self.A.has(self.C.indices[0].label)

    @property
    def sizeM(self) -> int:
        return _prod(i.size for i in self.m_indices)

    @property
    def sizeN(self) -> int:
        return _prod(i.size for i in self.n_indices)

    @property
    def sizeK(self) -> int:
        return _prod(i.size for i in self.k_indices)

    def flop_count(self, beta: Optional[float] = None) -> float:
        """Tccg.getFlopCount (tccg.py:1230-1234), real types: 2MNK, plus 3MN
        when beta != 0."""
        b = self.beta if beta is None else beta
        f = 2.0 * self.sizeM * self.sizeN * self.sizeK
        if b != 0:
            f += 3.0 * self.sizeM * self.sizeN
        return f

    def einsum(self) -> str:
        """The contraction as an einsum string over the ORIGINAL (unfused)
        index order, with the operands in file order (A, B)."""
        letters = {}
        pool = iter("abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ")
        for t in (self.A0, self.B0, self.C0):
            for lab in t.labels:
                if lab not in letters:
                    letters[lab] = next(pool)
        s = lambda t: "".join(letters[l] for l in t.labels)
        return "%s,%s->%s" % (s(self.A0), s(self.B0), s(self.C0))

    def validate(self) -> None:
        """Reject index patterns that GETT cannot express."""
        labsA, labsB, labsC = set(self.A.labels), set(self.B.labels), set(self.C.labels)
        for t in (self.A, self.B, self.C):
            if len(set(t.labels)) != len(t.labels):
                raise TccgSyntaxError("tensor %s repeats an index" % t)
        for lab in labsC:
            if lab not in labsA and lab not in labsB:
                raise TccgSyntaxError("index '%s' of C appears in neither A nor B" % lab)
        for lab in labsA | labsB:
            inA, inB, inC = lab in labsA, lab in labsB, lab in labsC
            if not inC and not (inA and inB):
                raise TccgSyntaxError(
                    "index '%s' appears in only one input and not in C" % lab)
        sizes = {}
        for t in (self.A, self.B, self.C):
            for i in t.indices:
                if i.size < 1:
                    raise TccgSyntaxError("index '%s' has extent %d" % (i.label, i.size))
                if sizes.setdefault(i.label, i.size) != i.size:
                    raise TccgSyntaxError("index '%s' has two extents" % i.label)
        if self.loop_indices:
            raise TccgUnsupported(
                "loop indices (indices in A, B and C: %s) are not supported by GETT"
                % ",".join(i.label for i in self.loop_indices))

    def __str__(self):
        return "%s = %s * %s * %s + %s * %s" % (
            self.C, _fmt(self.alpha), self.A, self.B, _fmt(self.beta), self.C)


def _fmt(x: float) -> str:
    return "%.2f" % x


def _prod(it) -> int:
    p = 1
    for v in it:
        p *= int(v)
    return p


# --- classification helpers (tccg/tccg_util.py) ----------------------------

def loop_indices(A: Tensor, B: Tensor, C: Tensor) -> List[Index]:
    """Indices of B that are also in A and C (tccg_util.py:212-228)."""
    return [i for i in B.indices if A.has(i.label) and C.has(i.label)]


def _owner(A: Tensor, B: Tensor, C: Tensor) -> Tuple[Tensor, Tensor]:
    return (A, B) if A.has(C.indices[0].label) else (B, A)


def n_indices(A: Tensor, B: Tensor, C: Tensor) -> List[Index]:
    """C's indices that are in the operand NOT holding C's first index and not
    in the other operand, in C's order (tccg_util.py:231-252)."""
    AA, BB = _owner(A, B, C)
    return [i for i in C.indices if BB.has(i.label) and not AA.has(i.label)]


def m_indices(A: Tensor, B: Tensor, C: Tensor) -> List[Index]:
    """C's indices in the operand holding C's first index and not in the
    other, in C's order (tccg_util.py:276-296)."""
    AA, BB = _owner(A, B, C)
    return [i for i in C.indices if AA.has(i.label) and not BB.has(i.label)]


def k_indices(A: Tensor, B: Tensor, C: Tensor) -> List[Index]:
    """Indices of A (file order) that are in B and not in C
    (tccg_util.py:597-611)."""
    return [i for i in A.indices if B.has(i.label) and not C.has(i.label)]


# --- parser (tccg/tccg.py:559-684) -----------------------------------------

_TENSOR_RE = re.compile(r"[A-C]\[[a-z][a-z0-9]*(?:,[a-z][a-z0-9]*)*\]")
_NUMBER_RE = re.compile(r"[-+]?\d*\.\d+|[-+]?\d+")
_SIZE_RE = re.compile(r"[a-z][a-z0-9]*=[0-9]+")


def parse_text(text: str, fuse: bool = True, name: str = "<string>") -> Contraction:
    """Parse a ``.tccg`` description (see module docstring)."""
    tensors: List[str] = []
    alpha, beta = 0.0, 0.0
    sizes: Dict[str, int] = {}
    for line in text.splitlines():
        content = line.split("#")[0].replace(" ", "").replace("\t", "")
        if not content:
            continue
        found = _TENSOR_RE.findall(content)
        if len(found) in (3, 4):
            if "+=" in content or "-=" in content:
                raise TccgSyntaxError(
                    "+= or -= is not allowed; use C[...] = ... + beta * C[...]")
            if "+-" in content or "-+" in content:
                raise TccgSyntaxError("+- or -+ is not allowed")
            for t in found:
                if t not in tensors:
                    tensors.append(t)
            if "=" not in content:
                raise TccgSyntaxError("missing '=' in '%s'" % line.strip())
            rhs = content.split("=")[1]
            rest = rhs
            for t in tensors:
                rest = rest.replace(t, "")
            nums = _NUMBER_RE.findall(rest)
            if len(tensors) < 3:
                raise TccgSyntaxError("You must specify exactly three tensors.")
            posAB = min(_find(rhs, tensors[1]), _find(rhs, tensors[2]))
            posC = rhs.find(tensors[0])
            alpha = 1.0
            beta = 1.0 if posC != -1 else 0.0
            if len(nums) == 0:
                pass
            elif len(nums) == 1:
                posF = rhs.find(nums[0])
                if posC == -1:
                    alpha, beta = float(nums[0]), 0.0
                elif posAB < posC:
                    if posF < posAB:
                        alpha = float(nums[0])
                    else:
                        beta = float(nums[0])
            elif len(nums) == 2:
                p1, p2 = rhs.find(nums[0]), rhs.find(nums[1])
                if posAB < posC:
                    a, b = (nums[0], nums[1]) if p1 < p2 else (nums[1], nums[0])
                else:
                    b, a = (nums[0], nums[1]) if p1 < p2 else (nums[1], nums[0])
                alpha, beta = float(a), float(b)
            else:
                raise TccgSyntaxError("too many scalars specified")
        for s in _SIZE_RE.findall(content):
            lab, val = s.split("=")
            sizes[lab] = int(val)

    if len(tensors) != 3:
        raise TccgSyntaxError(
            "%s: you must specify exactly three tensors, found %d (%s)"
            % (name, len(tensors), ", ".join(tensors)))

    out = []
    for i, t in enumerate(tensors):
        label = t[0]
        want = "CAB"[i]
        if label != want:
            warnings.warn("tensor %d uses the label '%s' => renamed to %s" % (i, label, want))
            label = want
        idx = []
        for lab in t[2:-1].split(","):
            if lab not in sizes:
                raise TccgSyntaxError("You must specify the size of each index ('%s')." % lab)
            idx.append(Index(lab, sizes[lab]))
        out.append(Tensor(label, idx))
    C, A, B = out
    con = Contraction(C=C, A=A, B=B, alpha=alpha, beta=beta)
    if fuse:
        fuse_indices(con)
    return con


def _find(s: str, sub: str) -> int:
    return s.find(sub)


def parse_file(path: str, fuse: bool = True) -> Contraction:
    import os
    if not os.path.isfile(path):
        raise TccgSyntaxError("File: %s does not exist." % path)
    with open(path) as f:
        return parse_text(f.read(), fuse=fuse, name=path)


def make_contraction(c: Sequence[str], a: Sequence[str], b: Sequence[str],
                     sizes: Dict[str, int], alpha: float = 1.0, beta: float = 0.0,
                     fuse: bool = True) -> Contraction:
    """Build a contraction from index label lists, e.g.
    ``make_contraction("abij", "ima", "mjb", {...})``."""
    mk = lambda lab, labs: Tensor(lab, [Index(l, int(sizes[l])) for l in labs])
    con = Contraction(C=mk("C", list(c)), A=mk("A", list(a)), B=mk("B", list(b)),
                      alpha=float(alpha), beta=float(beta))
    if fuse:
        fuse_indices(con)
    return con


def to_tccg_text(con: Contraction, fused: bool = False) -> str:
    """Write the contraction back in ``.tccg`` syntax (original indices unless
    ``fused``)."""
    C, A, B = (con.C, con.A, con.B) if fused else (con.C0, con.A0, con.B0)
    t = lambda T: "%s[%s]" % (T.label, ",".join(T.labels))
    line = "%s = %r * %s * %s" % (t(C), float(con.alpha), t(A), t(B))
    if con.beta != 0:
        line += " + %r * %s" % (float(con.beta), t(C))
    sizes = {}
    for T in (A, B, C):
        for i in T.indices:
            sizes[i.label] = i.size
    return line + "\n" + "".join("%s = %d\n" % kv for kv in sizes.items())


# --- index fusion (tccg/tccg.py:432-552) -----------------------------------

def _pop(T: Tensor, pos: int) -> None:
    T.indices.pop(pos)
    T.ld.pop(pos)


def fuse_indices(con: Contraction) -> None:
    """Merge index runs that are adjacent, in the same order, in every tensor
    that carries them (three passes exactly as tccg.py:432-552: C-indices
    shared by A and B, then C-indices of one input, then A-indices shared with
    B). Mutates ``con.A/B/C``; the fused index keeps the first label."""
    A, B, C = con.A, con.B, con.C
    done: List[str] = []

    # pass 1: C indices that appear in both A and B (tccg.py:440-485)
    n = len(C.indices)
    for i in range(n):
        if i >= n or C.indices[i].label in done:
            break
        lab = C.indices[i].label
        search = [T for T in (A, B) if T.has(lab)]
        if len(search) == 2:
            p1, p2 = search[0].pos(lab), search[1].pos(lab)
            l, inc = 1, 1
            while (i + l < len(C.indices) and p1 + l < len(search[0].indices)
                   and p2 + l < len(search[1].indices)
                   and search[0].indices[p1 + l].label == C.indices[i + l].label
                   and search[1].indices[p2 + l].label == C.indices[i + l].label
                   and C.indices[i + l].label not in done):
                inc *= C.indices[i + l].size
                l += 1
            if l > 1:
                done.append(lab)
                C.indices[i].size *= inc
                search[0].indices[p1].size *= inc
                search[1].indices[p2].size *= inc
            while l > 1:
                n -= 1
                _pop(C, i + 1)
                _pop(search[0], p1 + 1)
                _pop(search[1], p2 + 1)
                l -= 1

    # pass 2: C indices that appear in exactly one input (tccg.py:487-519)
    n = len(C.indices)
    for i in range(n):
        if i >= n or C.indices[i].label in done:
            continue
        lab = C.indices[i].label
        search = [T for T in (A, B) if T.has(lab)]
        if len(search) == 1:
            p1 = search[0].pos(lab)
            l, inc = 1, 1
            while (i + l < len(C.indices) and p1 + l < len(search[0].indices)
                   and search[0].indices[p1 + l].label == C.indices[i + l].label
                   and C.indices[i + l].label not in done):
                inc *= C.indices[i + l].size
                l += 1
            if l > 1:
                done.append(lab)
                C.indices[i].size *= inc
                search[0].indices[p1].size *= inc
            while l > 1:
                n -= 1
                _pop(C, i + 1)
                _pop(search[0], p1 + 1)
                l -= 1

    # pass 3: indices of A that are also in B (tccg.py:521-552)
    n = len(A.indices)
    for i in range(n):
        if i >= n or A.indices[i].label in done:
            continue
        p1 = B.pos(A.indices[i].label)
        if p1 != -1:
            l, inc = 1, 1
            while (i + l < len(A.indices) and p1 + l < len(B.indices)
                   and B.indices[p1 + l].label == A.indices[i + l].label
                   and A.indices[i + l].label not in done):
                inc *= A.indices[i + l].size
                l += 1
            if l > 1:
                done.append(A.indices[i].label)
                A.indices[i].size *= inc
                B.indices[p1].size *= inc
            while l > 1:
                n -= 1
                _pop(A, i + 1)
                _pop(B, p1 + 1)
                l -= 1
