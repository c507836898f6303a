"""Emit the per-contraction artifact, like TCCG's tccg_implementations/gett.cpp
(tccg.py:158-186): ``gett.h``, ``gett.cu`` and ``libgett.so`` exporting TCCG's
exact entry point

    void gett(float* A, float* B, float* C, const float alpha, const float beta);

(``double`` for ``--floatType=d``; tccg/gett.py:342-344), plus ``gett_stream``
(stream-ordered, device pointers, caller workspace), ``gett_workspace_bytes``
and ``gett_last_status``. ``gett`` takes what TCCG's callers pass -- host
buffers (the reference's harness allocates A, B, C with posix_memalign,
tccg.py:910-919, and calls gett at tccg.py:1040) -- or device pointers:
with host buffers it copies the operands to the device, runs and copies C
back, in slabs of C's last index when C is large so that the copies of one
slab overlap the contraction of the next (one cudaMemcpyAsync per slab and
operand on two copy streams). The contraction's descriptor, its slab
descriptors and the tuned kernel choice are baked into gett.cu as constants;
the kernels live in libtccg_b200.so, which libgett.so links (rpath).
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


def _desc_c(d) -> str:
    return ("{%d, %d, %d, %d,\n    %s,\n    %s,\n    %s,\n    %s,\n    %s,\n    %s,\n    %s,\n"
            "    %s,\n    %s}" % (
                d.nm, d.nn, d.nk, d.swap_ab, _arr(d.m_ext, d.nm), _arr(d.n_ext, d.nn),
                _arr(d.k_ext, d.nk), _arr(d.a_m_stride, d.nm), _arr(d.a_k_stride, d.nk),
                _arr(d.b_n_stride, d.nn), _arr(d.b_k_stride, d.nk), _arr(d.c_m_stride, d.nm),
                _arr(d.c_n_stride, d.nn)))


def host_slabs(con: Contraction, elem_bytes: int, tuning: Tuning = None):
    """Slabs of C's last index for the host-buffer path: 16 (at most the
    extent) when C holds >= 256 MiB, else one. Per slab: its descriptor (the
    full tensors' strides), element offsets into A, B, C and element counts
    of the parts copied per slab; plus which operands go up slab by slab
    (those whose last index is C's last index) instead of whole."""
    from .shard import shard
    label = con.C0.indices[-1].label
    ext = con.C0.indices[-1].size
    n = min(16, ext) if con.C0.num_elements() * elem_bytes >= (256 << 20) and ext >= 2 else 1
    per = {t: (T.has(label) and T.indices[-1].label == label)
           for t, T in (("A", con.A0), ("B", con.B0))}
    out = []
    for r in range(n):
        if n == 1:
            d = native_desc(_view(con, tuning))
            out.append((d, (0, 0, 0), (con.A0.num_elements(), con.B0.num_elements(),
                                       con.C0.num_elements())))
            continue
        sh = shard(con, r, n, label)
        sc = sh.contraction
        d = native_desc(_view(sc, tuning, sh.strides))
        out.append((d, (sh.offsets["A"], sh.offsets["B"], sh.offsets["C"]),
                    (sc.A0.num_elements(), sc.B0.num_elements(), sc.C0.num_elements())))
    if n == 1:
        per = {"A": False, "B": False}
    return out, per


def _view(con: Contraction, tuning: Tuning = None, strides=None):
    """GETT view with the tuning's mode orders."""
    t = tuning or Tuning()
    return gett_view(con, strides, n_order=t.n_order, k_order=t.k_order)


def source(con: Contraction, precision: str, tuning: Tuning, float_type: str) -> str:
    d = native_desc(_view(con, tuning))
    T = "double" if float_type == "d" else "float"
    slabs, per = host_slabs(con, 8 if float_type == "d" else 4, tuning)
    slab_desc = ",\n".join(_desc_c(sd) for sd, _, _ in slabs)
    slab_off = ", ".join("{%d, %d, %d}" % o for _, o, _ in slabs)
    slab_len = ", ".join("{%d, %d, %d}" % l for _, _, l in slabs)
    prec = {"fp32": "TCCG_PREC_FP32", "fp64": "TCCG_PREC_FP64", "bf16": "TCCG_PREC_BF16",
            "bf16x3": "TCCG_PREC_BF16X3"}[precision]
    dt = {"f32": "TCCG_F32", "f64": "TCCG_F64", "bf16": "TCCG_BF16"}[operand_dtype(precision)]
    method = {"gett": "TCCG_METHOD_GETT", "ttgt": "TCCG_METHOD_TTGT", "log": "TCCG_METHOD_LOG"}[tuning.method]
    desc = _desc_c(d)
    spec = "\n".join("// " + l for l in to_tccg_text(con).splitlines())
    return r'''// Generated by tccg_b200 for the contraction
%(spec)s
// precision %(precision)s, kernel choice: %(tkey)s
#include <cuda_runtime.h>
#include <stdio.h>
#include "tccg_b200.h"
#include "gett.h"

static const tccg_desc kDesc = %(desc)s;
static const tccg_tuning kTuning = {%(method)s, %(variant)d, %(ksplit)d, %(raster)d, %(max_ctas)d, %(pair)d, %(direct)d, %(shortk)d, %(simt_tile)d, %(tail_split)d, %(load)d, %(tile_n)d};

/* host-buffer path: slabs of C's last index (full tensors' strides), element
   offsets into A, B, C and element counts of the parts copied per slab */
#define NSLAB %(nslab)d
static const tccg_desc kSlab[NSLAB] = {%(slab_desc)s};
static const long long kSlabOff[NSLAB][3] = {%(slab_off)s};
static const long long kSlabLen[NSLAB][3] = {%(slab_len)s};
static const int kPerSlab[2] = {%(per_a)d, %(per_b)d}; /* A, B copied slab by slab (else whole) */
static const long long kElems[3] = {%(na)d, %(nb)d, %(nc)d};

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

/* 1: device (or managed) memory, 0: host memory (pinned or pageable), -1: error */
static int on_device(const void* p) {
  struct cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

/* state of the host-buffer path, made on its first call and kept */
static tccg_plan* g_slab_plan[NSLAB];
static void* g_hws = NULL;
static size_t g_hws_bytes = 0;
static %(T)s *g_dA = NULL, *g_dB = NULL, *g_dC = NULL;
static cudaStream_t g_up = NULL, g_down = NULL, g_comp = NULL;
static cudaEvent_t g_ev_whole = NULL, g_ev_ready[NSLAB], g_ev_done[NSLAB];

#define TRY(x) do { if ((x) != cudaSuccess) return TCCG_ERR_CUDA; } while (0)

static int ensure_host_state(void) {
  if (g_dC) return TCCG_OK;
  for (int s = 0; s < NSLAB; ++s) {
    int rc = tccg_plan_create(&kSlab[s], %(dt)s, %(prec)s, &kTuning, &g_slab_plan[s]);
    size_t w = 0;
    if (rc == TCCG_OK) rc = tccg_plan_workspace(g_slab_plan[s], &w);
    if (rc != TCCG_OK) return rc;
    if (w > g_hws_bytes) g_hws_bytes = w;
  }
  if (g_hws_bytes) TRY(cudaMalloc(&g_hws, g_hws_bytes));
  TRY(cudaMalloc((void**)&g_dA, kElems[0] * sizeof(%(T)s)));
  TRY(cudaMalloc((void**)&g_dB, kElems[1] * sizeof(%(T)s)));
  TRY(cudaStreamCreateWithFlags(&g_up, cudaStreamNonBlocking));
  TRY(cudaStreamCreateWithFlags(&g_down, cudaStreamNonBlocking));
  TRY(cudaStreamCreateWithFlags(&g_comp, cudaStreamNonBlocking));
  TRY(cudaEventCreateWithFlags(&g_ev_whole, cudaEventDisableTiming));
  for (int s = 0; s < NSLAB; ++s) {
    TRY(cudaEventCreateWithFlags(&g_ev_ready[s], cudaEventDisableTiming));
    TRY(cudaEventCreateWithFlags(&g_ev_done[s], cudaEventDisableTiming));
  }
  TRY(cudaMalloc((void**)&g_dC, kElems[2] * sizeof(%(T)s)));
  return TCCG_OK;
}

/* Host buffers: A and B (and C when beta != 0) go up on one copy stream --
   whole, or slab by slab for an operand whose last index is C's last index
   -- each slab is contracted on a third stream once its parts are up, and its
   C comes down on a second copy stream; the copy back of slab s is issued
   after slab s + 1 is queued, so that it overlaps that slab's contraction
   also when the copy blocks the calling thread (pageable memory). */
static int gett_host(const %(T)s* A, const %(T)s* B, %(T)s* C, %(T)s alpha, %(T)s beta) {
  int rc = ensure_host_state();
  if (rc != TCCG_OK) return rc;
  const size_t es = sizeof(%(T)s);
  if (!kPerSlab[0]) TRY(cudaMemcpyAsync(g_dA, A, kElems[0] * es, cudaMemcpyHostToDevice, g_up));
  if (!kPerSlab[1]) TRY(cudaMemcpyAsync(g_dB, B, kElems[1] * es, cudaMemcpyHostToDevice, g_up));
  TRY(cudaEventRecord(g_ev_whole, g_up));
  for (int s = 0; s <= NSLAB; ++s) {
    if (s < NSLAB) {
      const long long oa = kSlabOff[s][0], ob = kSlabOff[s][1], oc = kSlabOff[s][2];
      if (kPerSlab[0])
        TRY(cudaMemcpyAsync(g_dA + oa, A + oa, kSlabLen[s][0] * es, cudaMemcpyHostToDevice, g_up));
      if (kPerSlab[1])
        TRY(cudaMemcpyAsync(g_dB + ob, B + ob, kSlabLen[s][1] * es, cudaMemcpyHostToDevice, g_up));
      if (beta != (%(T)s)0)
        TRY(cudaMemcpyAsync(g_dC + oc, C + oc, kSlabLen[s][2] * es, cudaMemcpyHostToDevice, g_up));
      TRY(cudaEventRecord(g_ev_ready[s], g_up));
      TRY(cudaStreamWaitEvent(g_comp, g_ev_whole, 0));
      TRY(cudaStreamWaitEvent(g_comp, g_ev_ready[s], 0));
      rc = tccg_plan_run(g_slab_plan[s], g_dA + oa, g_dB + ob, g_dC + oc, (double)alpha,
                         (double)beta, g_hws, g_hws_bytes, g_comp);
      if (rc != TCCG_OK) return rc;
      TRY(cudaEventRecord(g_ev_done[s], g_comp));
    }
    if (s > 0) {
      const long long oc = kSlabOff[s - 1][2];
      TRY(cudaStreamWaitEvent(g_down, g_ev_done[s - 1], 0));
      TRY(cudaMemcpyAsync(C + oc, g_dC + oc, kSlabLen[s - 1][2] * es, cudaMemcpyDeviceToHost, g_down));
    }
  }
  TRY(cudaStreamSynchronize(g_down));
  TRY(cudaStreamSynchronize(g_comp));
  TRY(cudaStreamSynchronize(g_up));
  return TCCG_OK;
}

void gett(%(T)s* A, %(T)s* B, %(T)s* C, const %(T)s alpha, const %(T)s beta) {
  int rc = ensure_plan();
  const int da = on_device(A), db = on_device(B), dc = on_device(C);
  if (rc == TCCG_OK && !da && !db && !dc) {
    rc = gett_host(A, B, C, alpha, beta);
  } else if (rc == TCCG_OK && da && db && dc) {
    if (g_ws_bytes && !g_ws && cudaMalloc(&g_ws, g_ws_bytes) != cudaSuccess) rc = TCCG_ERR_CUDA;
    if (rc == TCCG_OK) rc = tccg_plan_run(g_plan, A, B, C, (double)alpha, (double)beta, g_ws, g_ws_bytes, NULL);
    if (rc == TCCG_OK && cudaStreamSynchronize(NULL) != cudaSuccess) rc = TCCG_ERR_CUDA;
  } else if (rc == TCCG_OK) {
    rc = TCCG_ERR_INVALID; /* A, B and C must all be host buffers or all device buffers */
  }
  g_status = rc;
  if (rc != TCCG_OK) fprintf(stderr, "gett: error %%d: %%s\n", rc, tccg_last_error());
}

int gett_last_status(void) { return g_status; }
''' % dict(spec=spec, precision=precision, tkey=tuning.key(), desc=desc, method=method,
           variant=tuning.variant, ksplit=tuning.ksplit, raster=tuning.raster,
           max_ctas=tuning.max_ctas, pair=tuning.pair, direct=tuning.direct,
           shortk=tuning.shortk, simt_tile=tuning.simt_tile,
           tail_split=tuning.tail_split, load=tuning.load, tile_n=tuning.tile_n, dt=dt, prec=prec, T=T,
           nslab=len(slabs), slab_desc=slab_desc, slab_off=slab_off, slab_len=slab_len,
           per_a=int(per["A"]), per_b=int(per["B"]), na=con.A0.num_elements(),
           nb=con.B0.num_elements(), nc=con.C0.num_elements())


def header(float_type: str) -> str:
    T = "double" if float_type == "d" else "float"
    return r'''// TCCG-compatible entry point generated by tccg_b200 (host or device buffers).
#ifndef TCCG_B200_GETT_H
#define TCCG_B200_GETT_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
/* C = alpha * A * B + beta * C; synchronous. A, B, C are all host buffers
   (copied to the GPU and back, pipelined in slabs of C's last index when C
   is large) or all device buffers (run on the legacy default stream). */
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
