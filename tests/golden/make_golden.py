#!/usr/bin/env python
"""Regenerate the golden fixtures from the REFERENCE itself.

Needs the reference checkout (TCCG, read-only) in this container; the
fixtures it writes are committed so that the test suite needs neither the
reference nor this script:

* ``front_end.json`` -- for each ``.tccg`` text: the reference's parse, index
  fusion and M/N/K/loop classification (Tccg.parseFile, Tccg.fuseIndices,
  tccg_util.getMindices/getNindices/getContractedIndices/getLoopIndices).
* ``loopnest_<case>.npz`` -- C computed by the loop nest the reference emits
  (Tccg.getReferenceVersion, compiled with g++ -O3 -ffp-contract=off) on
  TCCG's deterministic inputs (tccg.py:957-971) and on seeded inputs
  (splitmix64 U[-1,1), tests/helpers.py). Small cases store C whole; larger
  ones store 4096 sampled entries plus float64 checksums of the whole C.

Usage:  python tests/golden/make_golden.py
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import ref_build  # noqa: E402
from helpers import splitmix_uniform  # noqa: E402
from oracle import tccg_inputs  # noqa: E402

FRONT_END_CASES = {
    "example": "C[a,b,i,j] = A[i,m,a] * B[m,j,b]\na = 24\nb = 24\ni = 24\nj = 24\nm = 24\n",
    "transc0": "C[i1,j,i2] = 2.4 * A[i1,k,i2] * B[j,k] + 1.1 * C[i1,j,i2]\nj=1152\ni1=24\ni2=48\nk=64\n",
    "transc1": ("C[i1,j1,i2,j2] = 2.4 * A[i1,k,i2] * B[j1,k,j2] + 1.1 * C[i1,j1,i2,j2]\n"
                "i1=24\ni2=48\nj1=24\nj2=48\nk=32\n"),
    "cfg1": "C[a,b,i,j] = A[i,m,a] * B[m,j,b]\na=48\nb=48\ni=48\nj=48\nm=48\n",
    "cfg2": "C[a,b,c,d] = A[a,e,b] * B[e,d,c] + C[a,b,c,d]\na=96\nb=96\nc=96\nd=96\ne=16\n",
    "cfg3": ("C[a,b,c,i,j,k] = A[a,m,b,n,c] * B[m,i,n,j,k]\n"
             "a=32\nb=32\nc=32\ni=32\nj=32\nk=32\nm=64\nn=64\n"),
    "cfg4": "C[i0,j0,j1,i1] = A[k0,i0,k1,i1] * B[k1,j1,k0,j0]\ni0=64\ni1=64\nj0=64\nj1=64\nk0=32\nk1=32\n",
    # fusion: (a,b) adjacent in C and A; (c,d) adjacent in C and B; (k1,k2) in A and B
    "fuse_all": ("C[a,b,c,d] = A[a,b,k1,k2] * B[k1,k2,c,d]\n"
                 "a=4\nb=5\nc=6\nd=7\nk1=3\nk2=2\n"),
    "fuse_partial": ("C[a,b,c,d] = A[b,a,k,x] * B[k,x,c,d]\n# a,b swapped in A: no fusion of a,b\n"
                     "a=4\nb=5\nc=3\nd=2\nk=7\nx=3\n"),
    # scalars in every position TCCG accepts
    "alpha_only": "C[a,b] = -0.5 * A[a,k] * B[k,b]\na=5\nb=6\nk=7\n",
    "beta_implicit": "C[a,b] = A[a,k] * B[k,b] + C[a,b]\na=5\nb=6\nk=7\n",
    "beta_only": "C[a,b] = A[a,k] * B[k,b] + 0.25 * C[a,b]\na=5\nb=6\nk=7\n",
    "beta_first": "C[a,b] = 1.1 * C[a,b] + 2.4 * A[a,k] * B[k,b]\na=5\nb=6\nk=7\n",
    "beta_first_one": "C[a,b] = 3.0 * C[a,b] + A[a,k] * B[k,b]\na=5\nb=6\nk=7\n",
    "integer_scalars": "C[a,b] = 2 * A[a,k] * B[k,b] + 3 * C[a,b]\na=5\nb=6\nk=7\n",
    "renamed": "X[a,b] = Y[a,k] * Z[k,b]\na=5\nb=6\nk=7\n".replace("X", "C").replace("Y", "B").replace("Z", "A"),
    "swap": "C[p,q,r] = A[q,s] * B[s,p,r]\np=37\nq=29\nr=11\ns=53\n",
    "comments": "# a comment\nC[a,b] = A[a,k] * B[k,b] # trailing\n a = 5 \nb=6\nk=7 # k\n",
    "labels_digits": "C[i0,j0] = A[i0,k0,k1] * B[k1,j0,k0]\ni0=9\nj0=10\nk0=3\nk1=4\n",
    # batch index l: no fusion applies, GETT rejects l (loop index)
    "batch": "C[a,b,l] = A[a,l,k] * B[k,l,b]\na=2\nb=3\nk=4\nl=5\n",
    # batch index l trailing b in C and B: the reference's second fusion pass
    # merges (b,l) in C and B while A keeps l
    "batch_fused": "C[a,b,l] = A[a,k,l] * B[k,b,l]\na=2\nb=3\nk=4\nl=5\n",
}

# (name, tccg text, float type, store whole C?)
LOOPNEST_CASES = [
    ("example", FRONT_END_CASES["example"], "float"),
    ("cfg1", FRONT_END_CASES["cfg1"], "float"),
    ("cfg2_small", "C[a,b,c,d] = A[a,e,b] * B[e,d,c] + C[a,b,c,d]\na=24\nb=16\nc=20\nd=12\ne=16\n", "float"),
    ("cfg3_small", ("C[a,b,c,i,j,k] = A[a,m,b,n,c] * B[m,i,n,j,k]\n"
                    "a=8\nb=4\nc=4\ni=8\nj=4\nk=4\nm=16\nn=8\n"), "float"),
    ("cfg4_small", "C[i0,j0,j1,i1] = A[k0,i0,k1,i1] * B[k1,j1,k0,j0]\ni0=16\ni1=8\nj0=8\nj1=16\nk0=8\nk1=4\n", "float"),
    ("transc0", "C[i1,j,i2] = 2.4 * A[i1,k,i2] * B[j,k] + 1.1 * C[i1,j,i2]\nj=72\ni1=24\ni2=12\nk=40\n", "float"),
    ("fuse_all", FRONT_END_CASES["fuse_all"], "float"),
    ("swap", FRONT_END_CASES["swap"], "float"),
    ("beta_first", "C[a,b] = 1.1 * C[a,b] + 2.4 * A[a,k] * B[k,b]\na=33\nb=17\nk=65\n", "float"),
    ("cfg2_small_d", "C[a,b,c,d] = A[a,e,b] * B[e,d,c] + C[a,b,c,d]\na=24\nb=16\nc=20\nd=12\ne=16\n", "double"),
    ("cfg3_small_d", ("C[a,b,c,i,j,k] = A[a,m,b,n,c] * B[m,i,n,j,k]\n"
                      "a=8\nb=4\nc=4\ni=8\nj=4\nk=4\nm=16\nn=8\n"), "double"),
]

WHOLE_LIMIT = 1 << 16


def _numel(summary, t):
    n = 1
    for _, e in summary[t]["indices"]:
        n *= e
    return n


def run_reference(name, text, ft, A, B, C, alpha, beta):
    so = ref_build.build_loop_nest(text, "golden_" + name, float_type=ft, flavor="strict")
    L = ctypes.CDLL(so)
    T = ctypes.c_float if ft == "float" else ctypes.c_double
    L.referenceVersion.argtypes = [ctypes.c_void_p] * 3 + [T, T]
    L.referenceVersion(A.ctypes.data, B.ctypes.data, C.ctypes.data, alpha, beta)
    return C


def main():
    if not ref_build.reference_present():
        sys.exit("the reference checkout is not present; fixtures cannot be regenerated here")
    fe = {}
    for name, text in FRONT_END_CASES.items():
        _, s = ref_build.reference_front_end(text)
        fe[name] = {"text": text, "reference": s}
    with open(os.path.join(HERE, "front_end.json"), "w") as f:
        json.dump(fe, f, indent=1, sort_keys=True)
    print("front_end.json: %d cases" % len(fe))

    for name, text, ft in LOOPNEST_CASES:
        _, s = ref_build.reference_front_end(text, float_type=ft)
        dt = np.float32 if ft == "float" else np.float64
        nA, nB, nC = _numel(s, "A"), _numel(s, "B"), _numel(s, "C")
        out = {"text": np.array(text), "float_type": np.array(ft),
               "summary": np.array(json.dumps(s))}
        for family in ("tccg", "seeded"):
            if family == "tccg":
                A, B, C = (tccg_inputs(nA, "A", dt), tccg_inputs(nB, "B", dt), tccg_inputs(nC, "C", dt))
            else:
                A = splitmix_uniform(nA, 11).astype(dt)
                B = splitmix_uniform(nB, 12).astype(dt)
                C = splitmix_uniform(nC, 13).astype(dt)
            R = run_reference(name, text, ft, A, B, C.copy(), s["alpha"], s["beta"])
            if nC <= WHOLE_LIMIT:
                out[family + "_C"] = R
            else:
                lins = np.linspace(0, nC - 1, 4096).astype(np.int64)
                out[family + "_lins"] = lins
                out[family + "_vals"] = R[lins]
            out[family + "_checksum"] = np.array([R.astype(np.float64).sum(),
                                                  np.abs(R.astype(np.float64)).sum(),
                                                  (R.astype(np.float64) ** 2).sum()])
        np.savez_compressed(os.path.join(HERE, "loopnest_%s.npz" % name), **out)
        print("loopnest_%s.npz: C has %d entries" % (name, nC))


if __name__ == "__main__":
    main()
