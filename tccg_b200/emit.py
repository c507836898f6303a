"""Emit the per-contraction artifact, like TCCG's tccg_implementations/gett.cpp
(tccg.py:158-186): ``gett.h``, ``gett.cu`` and ``libgett.so`` exporting TCCG's
exact entry point

    void gett(float* A, float* B, float* C, const float alpha, const float beta);

(``double`` for ``--floatType=d``; tccg/gett.py:342-344) over DEVICE pointers,
plus ``gett_stream`` (stream-ordered, caller workspace), ``gett_workspace_bytes``
and ``gett_last_status``. The contraction's descriptor and the tuned kernel
choice are baked into gett.cu as constants; the kernels live in
libtccg_b200.so, which libgett.so links (rpath).
"""
from __future__ import annotations

import os
import subprocess

from . import build as B
from .plan import Tuning, gett_view, native_desc, operand_dtype
from .spec import Contraction, to_tccg_text
from . import _native as N


def _arr(vals, n):
    vals = list(vals) + [0] * (N.MAX_MODES - len(vals))
    return "{" + ", ".join("%d" % v for v in vals[:N.MAX_MODES]) + "}"


def source(con: Contraction, precision: str, tuning: Tuning, float_type: str) -> str:
    d = native_desc(gett_view(con))
    T = "double" if float_type == "d" else "float"
    prec = {"fp32": "TCCG_PREC_FP32", "fp64": "TCCG_PREC_FP64", "bf16": "TCCG_PREC_BF16",
            "bf16x3": "TCCG_PREC_BF16X3"}[precision]
    dt = {"f32": "TCCG_F32", "f64": "TCCG_F64", "bf16": "TCCG_BF16"}[operand_dtype(precision)]
    method = {"gett": "TCCG_METHOD_GETT", "ttgt": "TCCG_METHOD_TTGT", "log": "TCCG_METHOD_LOG"}[tuning.method]
    desc = ("{%d, %d, %d, %d,\n    %s,\n    %s,\n    %s,\n    %s,\n    %s,\n    %s,\n    %s,\n"
            "    %s,\n    %s}" % (
                d.nm, d.nn, d.nk, d.swap_ab, _arr(d.m_ext, d.nm), _arr(d.n_ext, d.nn),
                _arr(d.k_ext, d.nk), _arr(d.a_m_stride, d.nm), _arr(d.a_k_stride, d.nk),
                _arr(d.b_n_stride, d.nn), _arr(d.b_k_stride, d.nk), _arr(d.c_m_stride, d.nm),
                _arr(d.c_n_stride, d.nn)))
    spec = "\n".join("// " + l for l in to_tccg_text(con).splitlines())
    return r'''// Generated by tccg_b200 for the contraction
%(spec)s
// precision %(precision)s, kernel choice: %(tkey)s
#include <cuda_runtime.h>
#include <stdio.h>
#include "tccg_b200.h"
#include "gett.h"

static const tccg_desc kDesc = %(desc)s;
static const tccg_tuning kTuning = {%(method)s, %(variant)d, %(ksplit)d, %(raster)d, %(max_ctas)d, %(pair)d, %(direct)d, %(shortk)d, %(simt_tile)d, %(tail_split)d};

static tccg_plan* g_plan = NULL;
static void* g_ws = NULL;
static size_t g_ws_bytes = 0;
static int g_status = 0;

static int ensure_plan(void) {
  if (g_plan) return TCCG_OK;
  int rc = tccg_plan_create(&kDesc, %(dt)s, %(prec)s, &kTuning, &g_plan);
  if (rc == TCCG_OK) rc = tccg_plan_workspace(g_plan, &g_ws_bytes);
  return rc;
}

size_t gett_workspace_bytes(void) {
  return ensure_plan() == TCCG_OK ? g_ws_bytes : 0;
}

int gett_stream(const %(T)s* A, const %(T)s* B, %(T)s* C, %(T)s alpha, %(T)s beta, void* ws,
                size_t ws_bytes, void* stream) {
  int rc = ensure_plan();
  if (rc != TCCG_OK) return rc;
  return tccg_plan_run(g_plan, A, B, C, (double)alpha, (double)beta, ws, ws_bytes, stream);
}

void gett(%(T)s* A, %(T)s* B, %(T)s* C, const %(T)s alpha, const %(T)s beta) {
  int rc = ensure_plan();
  if (rc == TCCG_OK && g_ws_bytes && !g_ws && cudaMalloc(&g_ws, g_ws_bytes) != cudaSuccess)
    rc = TCCG_ERR_CUDA;
  if (rc == TCCG_OK) rc = tccg_plan_run(g_plan, A, B, C, (double)alpha, (double)beta, g_ws, g_ws_bytes, NULL);
  if (rc == TCCG_OK && cudaStreamSynchronize(NULL) != cudaSuccess) rc = TCCG_ERR_CUDA;
  g_status = rc;
  if (rc != TCCG_OK) fprintf(stderr, "gett: %%s\n", tccg_last_error());
}

int gett_last_status(void) { return g_status; }
''' % dict(spec=spec, precision=precision, tkey=tuning.key(), desc=desc, method=method,
           variant=tuning.variant, ksplit=tuning.ksplit, raster=tuning.raster,
           max_ctas=tuning.max_ctas, pair=tuning.pair, direct=tuning.direct,
           shortk=tuning.shortk, simt_tile=tuning.simt_tile,
           tail_split=tuning.tail_split, dt=dt, prec=prec, T=T)


def header(float_type: str) -> str:
    T = "double" if float_type == "d" else "float"
    return r'''// TCCG-compatible entry point generated by tccg_b200 (device pointers).
#ifndef TCCG_B200_GETT_H
#define TCCG_B200_GETT_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
/* C = alpha * A * B + beta * C; synchronous on the legacy default stream. */
void gett(%(T)s* A, %(T)s* B, %(T)s* C, const %(T)s alpha, const %(T)s beta);
/* Stream-ordered variant with a caller-owned workspace of gett_workspace_bytes(). */
int gett_stream(const %(T)s* A, const %(T)s* B, %(T)s* C, %(T)s alpha, %(T)s beta, void* ws,
                size_t ws_bytes, void* stream);
size_t gett_workspace_bytes(void);
/* 0 if the last gett() succeeded, else a TCCG_ERR_* code. */
int gett_last_status(void);
#ifdef __cplusplus
}
#endif
#endif
''' % dict(T=T)


def emit(con: Contraction, precision: str, tuning: Tuning, float_type: str, outdir: str,
         compile_so: bool = True) -> dict:
    os.makedirs(outdir, exist_ok=True)
    paths = {"h": os.path.join(outdir, "gett.h"), "cu": os.path.join(outdir, "gett.cu"),
             "so": os.path.join(outdir, "libgett.so")}
    with open(paths["h"], "w") as f:
        f.write(header(float_type))
    with open(paths["cu"], "w") as f:
        f.write(source(con, precision, tuning, float_type))
    if compile_so:
        B.build()
        env = dict(os.environ)
        env.pop("CC", None)
        env.pop("CXX", None)
        cmd = [B.nvcc_path(), *B.ARCH_FLAGS, "-O2", "-shared", "-Xcompiler", "-fPIC",
               "-cudart", "shared", "-I" + B.INCLUDE, "-I" + outdir, paths["cu"],
               "-L" + B.LIB_DIR, "-ltccg_b200", "-Xlinker", "-rpath," + B.LIB_DIR,
               "-o", paths["so"]]
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError("compiling %s failed:\n%s" % (paths["cu"], r.stdout + r.stderr))
    return paths
