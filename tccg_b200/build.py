"""Build of the native library ``tccg_b200/_lib/libtccg_b200.so`` (sm_100a).

The library is built in-tree with nvcc (``-gencode arch=compute_100a,
code=sm_100a``) from ``tccg_b200/csrc/tccg_abi.cu``; the CUDA runtime is
linked shared so that it is the same runtime instance torch uses.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(_HERE, "csrc")
LIB_DIR = os.path.join(_HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libtccg_b200.so")
INCLUDE = os.path.normpath(os.path.join(_HERE, "..", "include"))
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
_lock = threading.Lock()


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the tccg_b200 CUDA library cannot be built")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                  + [os.path.join(INCLUDE, "tccg_b200.h")])


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(s) > t for s in sources())


def nvcc_command(out: str = LIB_PATH, verbose: bool = False):
    cmd = [nvcc_path(), *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-cudart", "shared", "-I" + INCLUDE,
           "-o", out, os.path.join(CSRC, "tccg_abi.cu")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    return cmd


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if a source is newer than the .so (or ``force``)."""
    with _lock:
        if not force and not needs_build():
            return LIB_PATH
        os.makedirs(LIB_DIR, exist_ok=True)
        tmp = LIB_PATH + ".tmp.%d" % os.getpid()
        env = dict(os.environ)
        env.pop("CC", None)
        env.pop("CXX", None)
        r = subprocess.run(nvcc_command(tmp, verbose), capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
        os.replace(tmp, LIB_PATH)
        if verbose:
            print(r.stdout + r.stderr)
        return LIB_PATH
