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
from typing import List

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
# The reference checkout: $TCCG_REFERENCE_ROOT, else a directory named
# "reference" beside the repository; where neither exists the reference-built
# checkers are skipped (the committed fixtures and prebuilt files are used).
DEFAULT_REF = os.environ.get("TCCG_REFERENCE_ROOT") or os.path.join(
    os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))), "reference")
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
    for the benchmark workload, and TCCG's own generated GETT for the two
    configurations it can generate (M, N multiples of 24)."""
    if not reference_present(ref_root):
        return []
    return [build_loop_nest(CFG3_SLAB, "cfg3_slab_reference", flavor="fast", threads=16),
            build_tccg_gett(CFG1, "tccg_gett_cfg1"),
            build_tccg_gett(CFG2, "tccg_gett_cfg2")]


# ---------------------------------------------------------------------------
# TCCG's own generated GETT (AVX2) for contractions it can generate
# ---------------------------------------------------------------------------
STANDIN = os.path.join(_HERE, "hptt_standin")

CFG1 = "C[a,b,i,j] = A[i,m,a] * B[m,j,b]\na=48\nb=48\ni=48\nj=48\nm=48\n"
CFG2 = "C[a,b,c,d] = A[a,e,b] * B[e,d,c] + C[a,b,c,d]\na=96\nb=96\nc=96\nd=96\ne=16\n"


def build_tccg_gett(tccg_text: str, name: str, threads: int = 16, max_impl: int = 8) -> str:
    """Run TCCG's GETT generator (Gett.genCode, gett.py:961-1421) for an AVX2
    target with ``threads`` OpenMP threads, write TCCG's MemoryBroker
    (tccg.py:739-797), and compile every emitted candidate plus a small C glue
    into oracle/_ref/<name>.so exporting
      int tccg_gett_count(void); const char* tccg_gett_name(int);
      void tccg_gett_run(int i, float* A, float* B, float* C, float alpha, float beta);
    Flags: g++ -O3 -march=x86-64-v3 (AVX2 + FMA, what the emitted intrinsics
    need) -fopenmp, with oracle/hptt_standin/hptt.h for HPTT."""
    import io
    import shutil
    from contextlib import redirect_stdout
    os.makedirs(REF_DIR, exist_ok=True)
    so = os.path.join(REF_DIR, name + ".so")
    stamp = so + ".sha1"
    digest = hashlib.sha1((tccg_text + "%d/%d/v2" % (threads, max_impl) +
                           open(os.path.join(STANDIN, "hptt.h")).read()).encode()).hexdigest()
    if os.path.exists(so) and os.path.exists(stamp) and open(stamp).read() == digest:
        return so
    mods = _ref()
    t, _ = reference_front_end(tccg_text, "float", threads)
    work = tempfile.mkdtemp(prefix="tccg_gett_")
    cwd = os.getcwd()
    try:
        os.chdir(work)
        arch = mods["arch"].avx2("float")
        g = mods["gett"].Gett(t.A, t.B, t.C, t.alpha, t.beta, threads, arch, "float", max_impl,
                              0, 0, 1, 0, 0)
        with redirect_stdout(io.StringIO()):
            g.genCode()
            t.genMemoryBroker()
        names = [v for key in g.implementations for (v, _) in g.implementations[key]]
        if not names:
            raise RuntimeError("TCCG generated no GETT candidate for this contraction")
        # TCCG's spin barriers need every task of a team on its own thread:
        # run with exactly the generated thread count (TCCG's harness sets
        # OMP_NUM_THREADS the same way, tccg.py:285-287)
        glue = ['#include <omp.h>', '#include "memoryBroker.h"', '#include "gett.hpp"',
                "MemoryBroker memBroker;",
                "typedef void (*gett_fn)(float*, float*, float*, const float, const float);",
                "static gett_fn fns[] = {%s};" % ", ".join(names),
                "static const char* names[] = {%s};" % ", ".join('"%s"' % n for n in names),
                'extern "C" int tccg_gett_count(void) { return %d; }' % len(names),
                'extern "C" const char* tccg_gett_name(int i) { return names[i]; }',
                'extern "C" int tccg_gett_threads(void) { return %d; }' % threads,
                'extern "C" void tccg_gett_run(int i, float* A, float* B, float* C, float alpha, '
                "float beta) { omp_set_num_threads(%d); fns[i](A, B, C, alpha, beta); }" % threads]
        with open("glue.cpp", "w") as f:
            f.write("\n".join(glue) + "\n")
        srcs = sorted(x for x in os.listdir(".") if x.startswith("gett") and x.endswith(".cpp"))
        cmd = [CXX, "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++14",
               "-I" + STANDIN, "-I" + work, *srcs, "memoryBroker.cpp", "glue.cpp", "-o", so]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("g++ failed on TCCG's GETT:\n" + r.stderr[-3000:])
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)
    with open(stamp, "w") as f:
        f.write(digest)
    return so
