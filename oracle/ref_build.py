"""ORACLE -- test infrastructure only: builds checker programs from the
REFERENCE's own generator output.

TCCG (the reference) is a Python-2 code generator; ``ref_py3`` imports it
under Python 3. This module asks it, for a given ``.tccg`` text, for

* its parse + index fusion + M/N/K classification (``Tccg.parseFile``,
  ``Tccg.fuseIndices``, tccg_util.getMindices/getNindices/getContractedIndices),
* the loop-nest reference it emits (``Tccg.getReferenceVersion``,
  tccg/tccg.py:686-723),

and compiles that emitted C++ into a shared library exporting
``referenceVersion(A, B, C, alpha, beta)`` under oracle/_ref/ (git-ignored;
built in the container that has the reference checkout, then shipped with
the working tree). Nothing here copies reference sources into the
repository: the generator runs from the read-only checkout.

Two builds of each loop nest exist:
* ``strict``: ``g++ -O3 -ffp-contract=off`` -- IEEE single operations, used
  to pin the oracle bit for bit (tests/golden/);
* ``fast``: ``g++ -O3 -march=native -fopenmp`` (TCCG's own flags, Makefile:7-9
  with g++), used as the timed CPU reference.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile
import warnings
from typing import Dict, List, Tuple

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
DEFAULT_REF = "/root/reference"
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def reference_present(ref_root: str = DEFAULT_REF) -> bool:
    return os.path.isfile(os.path.join(ref_root, "tccg", "tccg.py"))


_mods = None


def _ref(ref_root: str = DEFAULT_REF):
    global _mods
    if _mods is None:
        if _HERE not in sys.path:
            sys.path.insert(0, _HERE)
        import ref_py3
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            _mods = ref_py3.load_reference(ref_root)
    return _mods


class _Args:
    def __init__(self, threads: int, float_type: str):
        self.numThreads = threads
        self.floatTypeA = float_type


def reference_front_end(tccg_text: str, float_type: str = "float", threads: int = 2):
    """Run the reference's parser + fusion on ``tccg_text``; returns the
    reference ``Tccg`` object (parsed, fused) and a plain-data summary."""
    T = _ref()["tccg"]
    U = _ref()["tccg_util"]
    with tempfile.NamedTemporaryFile("w", suffix=".tccg", delete=False) as f:
        f.write(tccg_text)
        path = f.name
    try:
        t = T.Tccg.__new__(T.Tccg)
        t.args = _Args(threads, float_type)
        import io
        from contextlib import redirect_stdout
        with redirect_stdout(io.StringIO()):
            C, A, B, alpha, beta = t.parseFile(path)
        t.A, t.B, t.C, t.alpha, t.beta = A, B, C, alpha, beta
        t.floatType = float_type
        t.fuseIndices()
    finally:
        os.unlink(path)
    summ = lambda X: {"label": X.label, "indices": [[i.label, int(i.size)] for i in X.indices],
                      "ld": [int(x) for x in X.ld]}
    cls = lambda L: [[i.label, int(i.size)] for i in L]
    summary = {
        "C": summ(t.C), "A": summ(t.A), "B": summ(t.B),
        "alpha": float(t.alpha), "beta": float(t.beta),
        "m": cls(U.getMindices(t.A, t.B, t.C)), "n": cls(U.getNindices(t.A, t.B, t.C)),
        "k": cls(U.getContractedIndices(t.A, t.B, t.C)),
        "loop": cls(U.getLoopIndices(t.A, t.B, t.C)),
    }
    return t, summary


def reference_loop_nest_source(tccg_text: str, float_type: str = "float", threads: int = 2) -> str:
    t, _ = reference_front_end(tccg_text, float_type, threads)
    return t.getReferenceVersion()


def build_loop_nest(tccg_text: str, name: str, float_type: str = "float", flavor: str = "strict",
                    threads: int = 2) -> str:
    """Compile the reference's emitted loop nest into oracle/_ref/<name>.so."""
    os.makedirs(REF_DIR, exist_ok=True)
    src = reference_loop_nest_source(tccg_text, float_type, threads)
    code = '#include <omp.h>\nextern "C" {\n' + src + "\n}\n"
    cpp = os.path.join(REF_DIR, name + ".cpp")
    so = os.path.join(REF_DIR, name + ".so")
    digest = hashlib.sha1((code + flavor).encode()).hexdigest()
    stamp = so + ".sha1"
    if os.path.exists(so) and os.path.exists(stamp) and open(stamp).read() == digest:
        return so
    with open(cpp, "w") as f:
        f.write(code)
    if flavor == "strict":
        flags = ["-O3", "-ffp-contract=off", "-fopenmp"]
    else:
        flags = ["-O3", "-march=native", "-fopenmp"]
    subprocess.run([CXX, *flags, "-fPIC", "-shared", "-o", so, cpp], check=True,
                   capture_output=True, text=True)
    with open(stamp, "w") as f:
        f.write(digest)
    return so


# The loop nest TCCG emits for the benchmark workload restricted to the C slab
# j = k = 0 (extents j = k = 1 give exactly that slab: both are C's and B's
# trailing indices, so no other stride changes).
CFG3_SLAB = ("C[a,b,c,i,j,k] = A[a,m,b,n,c] * B[m,i,n,j,k]\n"
             "a = 32\nb = 32\nc = 32\ni = 32\nj = 1\nk = 1\nm = 64\nn = 64\n")


def build_all(ref_root: str = DEFAULT_REF) -> List[str]:
    """Everything the GPU box needs from the reference: the timed CPU reference
    for the benchmark workload."""
    if not reference_present(ref_root):
        return []
    return [build_loop_nest(CFG3_SLAB, "cfg3_slab_reference", flavor="fast", threads=16)]
