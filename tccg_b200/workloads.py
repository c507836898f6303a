"""Synthetic contraction workloads for benchmarks and tests.

``batched_workload`` draws the mixed batch of the grouped-launch benchmark:
per item a target FLOP count F ~ log-uniform[1e6, 1e10], 2..6 indices in C
(at least one in each operand), 1..3 contracted indices, a random permutation
of every tensor's indices, extents drawn from U{8..128} and rescaled (then
redrawn if needed) until 2MNK lies in [F/2, 2F]. No index is in all three
tensors, so TCCG's classification holds.
"""
from __future__ import annotations

import math
import random
from typing import List

from .spec import Contraction, make_contraction

_LABELS = "abcdefghijklmnopqrstuvwxyz"


def _flops(sizes, m, n, k):
    M = math.prod(sizes[l] for l in m)
    N = math.prod(sizes[l] for l in n)
    K = math.prod(sizes[l] for l in k)
    return 2.0 * M * N * K


def random_contraction(rng: random.Random, fmin: float = 1e6, fmax: float = 1e10,
                       emin: int = 8, emax: int = 128, max_tries: int = 200) -> Contraction:
    F = math.exp(rng.uniform(math.log(fmin), math.log(fmax)))
    for _ in range(max_tries):
        nc = rng.randint(2, 6)
        na = rng.randint(1, nc - 1)          # free indices of A
        nk = rng.randint(1, 3)
        labs = rng.sample(_LABELS, nc + nk)
        cfree, kidx = labs[:nc], labs[nc:]
        rng.shuffle(cfree)
        m, n = cfree[:na], cfree[na:]
        sizes = {l: rng.randint(emin, emax) for l in labs}
        # rescale towards F
        for _ in range(8):
            f = _flops(sizes, m, n, kidx)
            if F / 2 <= f <= 2 * F:
                break
            s = (F / f) ** (1.0 / len(labs))
            for l in labs:
                sizes[l] = max(emin, min(emax, int(round(sizes[l] * s))))
        f = _flops(sizes, m, n, kidx)
        if not (F / 2 <= f <= 2 * F):
            continue
        C = list(m) + list(n)
        rng.shuffle(C)
        A = list(m) + list(kidx)
        rng.shuffle(A)
        B = list(n) + list(kidx)
        rng.shuffle(B)
        return make_contraction(C, A, B, sizes)
    raise RuntimeError("could not draw a contraction near %.3g FLOP" % F)


def batched_workload(count: int = 256, seed: int = 0, **kw) -> List[Contraction]:
    rng = random.Random(seed)
    return [random_contraction(rng, **kw) for _ in range(count)]
