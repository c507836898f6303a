#!/usr/bin/env python
"""Benchmark of the GETT hot path on B200 (one JSON line on stdout).

Workload (the compute-bound 6-index contraction the headline metric is
quoted on): C[a,b,c,i,j,k] = A[a,m,b,n,c] * B[m,i,n,j,k], a=b=c=i=j=k=32,
m=n=64 (M = N = 32768, K = 4096), A and B ~ N(0,1) FP32 from a seed, beta=0.

A step is one GETT call: operand packing + the contraction kernel, inputs
resident in HBM (A, B 512 MiB each, C 4 GiB: larger than the 126 MB L2, so
no flush is needed between steps). ``value`` is split-BF16x3 TFLOP/s by
TCCG's flop count (2MNK); plain FP32 GETT on the same inputs is reported
beside it, and so are the errors of both against the FP64 path.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank computes its own C slab of
a k-sharded problem (weak scaling, no collective); time = max over ranks.
``--impl reference`` times the reference's CPU implementation of the path
(the loop nest TCCG emits, compiled from its generator when that build is
present, else the oracle's C restatement of it) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

def workload(k_extent: int = 32):
    """The .tccg text of the workload; k_extent < 32 gives the C slab k < k_extent
    (used for profiler captures of the same kernel on a smaller case)."""
    return ("C[a,b,c,i,j,k] = A[a,m,b,n,c] * B[m,i,n,j,k]\n"
            "a = 32\nb = 32\nc = 32\ni = 32\nj = 32\nk = %d\nm = 64\nn = 64\n" % k_extent)


def workload_name(k_extent: int = 32) -> str:
    return ("C[a,b,c,i,j,k] = A[a,m,b,n,c] * B[m,i,n,j,k], a=b=c=i=j=32, k=%d, m=n=64 "
            "(M=32768, N=%d, K=4096), N(0,1) FP32 inputs, alpha=1, beta=0"
            % (k_extent, 1024 * k_extent))
METRIC = "GETT TFLOP/s & %roofline: BF16x3 vs plain FP32 on 1xB200 at rel err <=1e-5"
FP32_SIMT_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # nominal FFMA peak at max clock


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    """Samples SM clock, power and clock-event reasons every 20 ms through NVML
    (falls back to ``nvidia-smi -lms 100``) while the timed region runs."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown"}

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None

    def _poll(self):
        nv = self._nvml
        h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((sm, mx, pw, rs))
            except Exception:  # noqa: BLE001
                pass
            self._stop.wait(0.02)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self._nvml = nv
            # NVML numbers devices like nvidia-smi; map the torch index through
            # CUDA_VISIBLE_DEVICES when it is set
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            if vis:
                ids = [x for x in vis.split(",") if x.strip()]
                if self.gpu < len(ids) and ids[self.gpu].strip().isdigit():
                    self.gpu = int(ids[self.gpu])
            self._thread = threading.Thread(target=self._poll, daemon=True)
            self._thread.start()
        except Exception:  # noqa: BLE001
            self._nvml = None
        time.sleep(0.05)

    def stop(self):
        self._stop.set()
        if self._thread is not None:
            self._thread.join(timeout=2)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "source": "nvml" if self._nvml else "unavailable"}
        sm = [x[0] for x in self.samples]
        reasons = sorted({name for x in self.samples for bit, name in self.REASONS.items()
                          if x[3] & bit})
        return {"sm_mhz": statistics.median(sm), "sm_min_mhz": min(sm),
                "sm_max_mhz": self.samples[0][1], "power_w_max": max(x[2] for x in self.samples),
                "reasons": reasons, "samples": len(self.samples), "source": "nvml, 20 ms"}


# --------------------------------------------------------------------------
# helpers
# --------------------------------------------------------------------------
def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def read_traffic(name: str):
    """DRAM bytes per launch of the named kernel from its committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith("dram_bytes_per_launch_full_size:"):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


def host_threads() -> int:
    """Host CPUs this process may run on (its affinity mask)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def host_operand(x):
    """The CPU baseline's copy of an operand: a fresh 64-byte aligned array
    written by this thread (as TCCG's harness allocates with posix_memalign
    and initialises serially, tccg.py:910-919, 957-971), so that both bench
    arms time the loop nest on memory placed the same way -- on the wide
    strides of this contraction the loop nest is bound by address
    translation, and pinned or torch-allocated buffers measured up to 4x
    apart on the same slab."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import aligned_copy  # noqa: E402
    return aligned_copy(x)


def thp_mode():
    try:
        with open("/sys/kernel/mm/transparent_hugepage/enabled") as f:
            return f.read().strip()
    except OSError:
        return None


def set_omp_threads(n: int) -> dict:
    """Sets the thread count of the process's OpenMP runtime (libgomp.so.1:
    torch loads its own copy under that name first, and the oracle's and the
    reference-emitted loop nests bind to whichever is loaded) for the calling
    thread, and reports what the runtime then uses. torch's first parallel CPU
    operation sets it to its own intra-op default, so it is set explicitly
    right before every timed CPU call."""
    import ctypes
    info = {"requested": int(n)}
    try:
        g = ctypes.CDLL("libgomp.so.1")
        g.omp_set_num_threads(int(n))
        g.omp_get_max_threads.restype = ctypes.c_int
        info["omp_get_max_threads"] = int(g.omp_get_max_threads())
    except OSError as e:
        info["error"] = str(e)
    for k in ("OMP_NUM_THREADS", "GOMP_CPU_AFFINITY", "OMP_PROC_BIND", "OMP_PLACES"):
        if os.environ.get(k):
            info[k] = os.environ[k]
    info["affinity_cpus"] = host_threads()
    info["transparent_hugepage"] = thp_mode()
    return info


def oracle_errors(con, A_np, B_np, lins, samples):
    """The checker: errors of sampled output entries (``samples``: name ->
    values at the column-major indices ``lins``) against the FP64 oracle, the
    C restatement of TCCG's loop-nest reference evaluated in FP64 on the same
    FP32 inputs. Four metrics per output: max abs, normwise, max relative
    error over |ref| > 1e-3 max|ref|, and TCCG's equal() criterion
    min(abs, rel) (tccg.py:843-881) with its sign blindness fixed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import LoopNest, error_metrics  # noqa: E402
    sizes = {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices}
    ln = LoopNest(con.C0.labels, con.A0.labels, con.B0.labels, sizes)
    ref = ln.sample64(A_np, B_np, None, con.alpha, 0.0, lins, host_threads())
    out = {"oracle": "FP64 loop nest (oracle/loopnest.c) on %d entries of C spread evenly over "
                     "its %d" % (len(lins), ln.size_c)}
    for name, v in samples.items():
        m = error_metrics(v, ref)
        out[name] = {"max_abs": m["max_abs"], "normwise": m["normwise"],
                     "max_rel_over_1e-3_max_ref": m["max_rel"],
                     "tccg_min_abs_rel": m["tccg_equal_worst"],
                     "max_abs_over_max_ref": m["max_abs_over_max_ref"]}
    return out


def cpu_loopnest_sample(con, A_np, B_np, seconds=10.0, threads=0, gpu_C=None):
    """Time the oracle loop nest (TCCG's referenceVersion restated) on the first
    S column-major entries of C, S sized for about `seconds`; optionally check
    the GPU result on those entries against the FP64 oracle."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    from oracle import LoopNest, error_metrics, lib  # noqa: E402
    threads = threads or host_threads()
    omp = set_omp_threads(threads)
    c, a, b = con.C0.labels, con.A0.labels, con.B0.labels
    sizes = {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices}
    ln = LoopNest(c, a, b, sizes)
    Cbuf = np.zeros(ln.size_c, dtype=np.float32)
    s, t = 8192, 0.0
    while True:  # grow the calibration sample until it runs for >= 0.5 s
        t0 = time.perf_counter()
        ln.run(A_np, B_np, Cbuf, 1.0, 0.0, 0, s, threads)
        t = max(time.perf_counter() - t0, 1e-6)
        if t >= 0.5 or s >= ln.size_c:
            break
        s = min(ln.size_c, s * 4)
    S = int(min(ln.size_c, max(s, s * seconds / t)))
    t0 = time.perf_counter()
    ln.run(A_np, B_np, Cbuf, 1.0, 0.0, 0, S, threads)
    t = time.perf_counter() - t0
    flops = 2.0 * S * ln.size_k
    out = {"value": flops / t / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "port",
           "sample": "first %d column-major entries of C (%.2e of the %d) through the oracle's C "
                     "restatement of TCCG's loop-nest reference, %d OpenMP threads, %.1f s"
                     % (S, S / ln.size_c, ln.size_c, threads, t), "openmp": omp}
    if gpu_C is not None:
        lins = np.arange(0, S, max(1, S // 4096), dtype=np.int64)
        ref = ln.sample64(A_np, B_np, None, 1.0, 0.0, lins, threads)
        m = error_metrics(gpu_C[lins], ref)
        out["check_vs_fp64_oracle"] = {"entries": int(len(lins)), "normwise": m["normwise"],
                                       "max_abs_over_max_ref": m["max_abs_over_max_ref"]}
    return out


def reference_impl_sample(con, A_np, B_np, seconds, threads):
    """The reference's own CPU code for this workload: the loop nest TCCG emits
    (tccg.py:686-723) for the C slab C[:,:,:,:,0,0], compiled from the
    generator's output into oracle/_ref/ (built in the build container).
    Returns None when that build is absent."""
    import ctypes
    import numpy as np
    so = os.path.join(ROOT, "oracle", "_ref", "cfg3_slab_reference.so")
    if not os.path.exists(so):
        return None
    L = ctypes.CDLL(so)
    L.referenceVersion.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_float, ctypes.c_float]
    # slab: all of a,b,c,i for j=k=0 -> 2^20 entries of K=4096 each
    Cs = np.zeros(32 ** 4, dtype=np.float32)
    omp = set_omp_threads(threads)
    t0 = time.perf_counter()
    L.referenceVersion(A_np.ctypes.data, B_np.ctypes.data, Cs.ctypes.data, 1.0, 0.0)
    t = time.perf_counter() - t0
    flops = 2.0 * Cs.size * 4096
    return {"value": flops / t / 1e12, "unit": "TFLOP/s", "cores": omp.get("omp_get_max_threads", threads),
            "kind": "reference",
            "sample": "slab C[:,:,:,:,0,0] (2^20 entries, 1/1024 of C) computed by the loop nest "
                      "TCCG's generator emits for this contraction, g++ -O3 -fopenmp, %d threads, "
                      "%.2f s" % (omp.get("omp_get_max_threads", threads), t), "openmp": omp}


# --------------------------------------------------------------------------
# arms
# --------------------------------------------------------------------------
def run_reference(args, world, rank):
    """CPU reference arm: rank 0 only."""
    if rank != 0:
        return 0
    import numpy as np
    import torch
    from tccg_b200 import parse_text
    con = parse_text(workload(args.k_extent))
    threads = host_threads()
    g = torch.Generator().manual_seed(0)
    A = host_operand(torch.randn(con.A0.num_elements(), generator=g).numpy())
    B = host_operand(torch.randn(con.B0.num_elements(), generator=g).numpy())
    vals = []
    info = None
    per_step = max(2.0, min(20.0, 120.0 / max(1, args.steps + args.warmup)))
    for it in range(args.warmup + args.steps):
        r = reference_impl_sample(con, A, B, per_step, threads)
        if r is None:
            r = cpu_loopnest_sample(con, A, B, seconds=per_step, threads=threads)
        if it >= args.warmup:
            vals.append(r["value"])
            info = r
    v = statistics.median(vals)
    flops_step = con.flop_count()
    line = {
        "metric": METRIC, "value": v, "unit": "TFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": flops_step / (v * 1e12) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": workload_name(args.k_extent), "precision": "fp32 (CPU loop nest)",
                   "parallelism": "host cores of rank 0"},
        "cpu_baseline": {"kind": info["kind"], "cores": info["cores"], "sample": info["sample"],
                         "value": v, "unit": "TFLOP/s", "openmp": info.get("openmp"),
                         "steps_tflops": vals},
        "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    from tccg_b200 import parse_text
    from tccg_b200.api import Compiled
    from tccg_b200.plan import Tuning

    dev = torch.device("cuda", local)
    con = parse_text(workload(args.k_extent))
    flops = con.flop_count()
    peaks, peak_src = measured_peaks()
    g = torch.Generator(device=dev).manual_seed(1000 + rank)
    nA, nB, nC = con.A0.num_elements(), con.B0.num_elements(), con.C0.num_elements()
    A = torch.randn(nA, generator=g, device=dev, dtype=torch.float32)
    B = torch.randn(nB, generator=g, device=dev, dtype=torch.float32)
    C = torch.empty(nC, device=dev, dtype=torch.float32)

    x3 = Compiled(con, "bf16x3", Tuning(raster=args.raster, max_ctas=args.max_ctas, pair=args.pair))
    ws = x3.workspace(dev)

    # ---- headline: split-BF16x3, device-resident -------------------------
    for _ in range(args.warmup):
        x3.plan.run(A, B, C, workspace=ws)
    # CUDA events around each kernel of every timed step (created and
    # recorded once here, outside the timed region)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(6)] for _ in range(args.steps)]
    for evs in ev:
        for e in evs:
            e.record()
    torch.cuda.synchronize()
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        x3.plan.run_events(A, B, C, ev[i], workspace=ws)
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    ms_total = e0.elapsed_time(e1)
    clocks = sampler.stop() if sampler else None
    ms_step = max_over_ranks(ms_total / args.steps, world)
    value = world * flops / (ms_step * 1e-3) / 1e12
    status = x3.plan.status()
    # per-kernel times of the same timed steps (pack, then the GETT kernel)
    pack_steps = [evs[0].elapsed_time(evs[1]) for evs in ev]
    gemm_steps = [evs[2].elapsed_time(evs[3]) for evs in ev]
    pack_ms = statistics.mean(pack_steps)
    gemm_ms = statistics.mean(gemm_steps)
    achieved = flops / (gemm_ms * 1e-3) / 1e12
    bf16_peak = peaks.get("bf16_tflops_sustained") or peaks.get("bf16_tflops")
    peak = bf16_peak / 3.0
    burst = peaks.get("bf16_tflops", bf16_peak) / 3.0
    traffic = read_traffic("gett_tc_bf16x3_cfg3.txt")
    # sampled output entries for the error check against the oracle
    lins = torch.from_numpy(np.unique(np.linspace(0, nC - 1, 4096).astype(np.int64))).to(dev)
    samples = {"bf16x3": C[lins].double().cpu().numpy()}

    # ---- plain FP32 GETT on the same inputs --------------------------------
    res = {}
    if not args.skip_fp32:
        f32 = Compiled(con, "fp32")
        C32 = torch.empty_like(C)
        f32.plan.run(A, B, C32, workspace=f32.workspace(dev))
        torch.cuda.synchronize()
        n32 = max(1, min(args.steps, 3))
        e0.record()
        for _ in range(n32):
            f32.plan.run(A, B, C32, workspace=f32.workspace(dev))
        e1.record()
        torch.cuda.synchronize()
        ms32 = max_over_ranks(e0.elapsed_time(e1) / n32, world)
        k32 = f32.plan.run_timed(A, B, C32, workspace=f32.workspace(dev))
        res["fp32"] = {"value": world * flops / (ms32 * 1e-3) / 1e12, "unit": "TFLOP/s",
                       "ms_per_step": ms32,
                       "kernel_frac_of_fp32_simt_peak": flops / (k32[1] * 1e-3) / 1e12 / FP32_SIMT_PEAK_TFLOPS}
        samples["fp32"] = C32[lins].double().cpu().numpy()
        f32._ws = None
    else:
        C32 = None

    # ---- errors: the FP64 oracle on sampled entries, and the FP64 path -----
    if not args.skip_errors:
        f64 = Compiled(con, "fp64")
        C64 = torch.empty(nC, device=dev, dtype=torch.float64)
        f64.plan.run(A.double(), B.double(), C64, workspace=f64.workspace(dev))
        torch.cuda.synchronize()
        samples["fp64_path"] = C64[lins].cpu().numpy()
        nrm = torch.linalg.vector_norm(C64).item()
        err = {"bf16x3_normwise_vs_fp64_path_all_entries":
               torch.linalg.vector_norm(C.double() - C64).item() / nrm}
        if C32 is not None:
            err["fp32_normwise_vs_fp64_path_all_entries"] = (
                torch.linalg.vector_norm(C32.double() - C64).item() / nrm)
        res["errors"] = err
        del C64, f64
    del C32
    torch.cuda.empty_cache()

    # ---- end to end through the public API with host buffers -------------
    if not args.skip_errors:
        res["errors"].update(oracle_errors(con, A.cpu().numpy(), B.cpu().numpy(),
                                           lins.cpu().numpy(), samples))
    if args.skip_e2e:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "TFLOP/s",
                              "ms_per_step": ms_step, "roofline_kernel_ms": gemm_ms,
                              "pack_ms": pack_ms, "partial": "--skip-e2e",
                              "errors": res.get("errors")}), flush=True)
        return 0
    Ah = A.cpu().pin_memory()
    Bh = B.cpu().pin_memory()
    Ch = torch.empty(nC, dtype=torch.float32).pin_memory()
    for _ in range(min(args.warmup, 2)):
        h2d, d2h = x3.run_host(Ah, Bh, Ch, device=dev)
    torch.cuda.synchronize()
    ne2e = max(1, min(args.steps, 5))
    barrier(world)
    e0.record()
    for _ in range(ne2e):
        h2d, d2h = x3.run_host(Ah, Bh, Ch, device=dev)
    e1.record()
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1) / ne2e, world)
    # the host link's own rates, measured on the same pinned buffers: the
    # end-to-end step cannot beat max(H2D bytes / H2D rate, D2H bytes / D2H
    # rate) when the copies run concurrently on the two copy engines
    link = {}
    for name, src, dst in (("h2d_gbs", Ah, A), ("d2h_gbs", C, Ch)):
        dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        link[name] = src.numel() * src.element_size() / (e0.elapsed_time(e1) * 1e-3) / 1e9
    e2e_bound_ms = max(h2d / (link["h2d_gbs"] * 1e9), d2h / (link["d2h_gbs"] * 1e9)) * 1e3

    # ---- CPU baseline (rank 0, single GPU only) ----------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        Cx3 = Ch.numpy()  # last e2e result = the BF16x3 output for these inputs
        # the port times the sample and checks the GPU result against FP64;
        # the reference's own emitted loop nest, where it was built, is the
        # reported baseline (the port's figure stays beside it)
        An, Bn = host_operand(Ah.numpy()), host_operand(Bh.numpy())
        cpu = cpu_loopnest_sample(con, An, Bn, seconds=args.cpu_seconds, gpu_C=Cx3)
        ref = None
        if args.k_extent == 32:
            ref = reference_impl_sample(con, An, Bn, args.cpu_seconds, host_threads())
        del An, Bn
        if ref is not None:
            ref["check_vs_fp64_oracle"] = cpu.pop("check_vs_fp64_oracle", None)
            ref["port"] = {"value": cpu["value"], "sample": cpu["sample"]}
            cpu = ref

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3", "data": "synthetic",
            "config": {"workload": workload_name(args.k_extent),
                       "precision": "split-BF16x3 (bf16 products, f32 accumulate)",
                       "M": con.sizeM, "N": con.sizeN, "K": con.sizeK, "flop_per_step": flops,
                       "l2": "inputs larger than L2 (A, B 512 MiB, C 4 GiB); no flush",
                       "parallelism": "weak: one C slab per GPU, no collective" if world > 1 else "1 GPU",
                       "plan": x3.describe()},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "gett_tc_kernel<BF16X3>",
                         "kernel_ms": gemm_ms, "pack_ms": pack_ms,
                         "kernel_ms_min_max": [min(gemm_steps), max(gemm_steps)],
                         "timing": "CUDA events around the pack and GETT kernels of every timed step "
                                   "(the same steps as ms_per_step)",
                         "frac_of_burst": achieved / burst,
                         "peak_note": "%s sustained dense BF16 %.1f TFLOP/s / 3 (three BF16 MMAs per "
                                      "algorithmic multiply-add); frac = tensor-pipe share of measured "
                                      "peak; frac_of_burst against %.1f/3"
                                      % (peak_src, bf16_peak, peaks.get("bf16_tflops", bf16_peak))},
            "e2e": {"value": world * flops / (ms_e2e * 1e-3) / 1e12, "unit": "TFLOP/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": ms_e2e,
                    "link": link,
                    "bound_ms": e2e_bound_ms,
                    "frac_of_link_bound": e2e_bound_ms / ms_e2e,
                    "path": "Compiled.run_host: pinned host A, B -> device, tccg_plan_run per slab of "
                            "C's last index (%d slabs), C -> pinned host; copies overlap the compute on "
                            "two copy streams" % x3._auto_slabs(Ch)},
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
            "device_status": status,
            "cpu_baseline": cpu,
        }
        line.update(res)
        print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# every configuration (python bench.py --suite): per-precision timings, rooflines,
# errors and the CPU baselines of configurations 1-5
# --------------------------------------------------------------------------
SUITE = {
    "cfg1": "C[a,b,i,j] = A[i,m,a] * B[m,j,b]\na=48\nb=48\ni=48\nj=48\nm=48\n",
    "cfg2": "C[a,b,c,d] = A[a,e,b] * B[e,d,c] + C[a,b,c,d]\na=96\nb=96\nc=96\nd=96\ne=16\n",
    "cfg3": workload(32),
    "cfg4": "C[i0,j0,j1,i1] = A[k0,i0,k1,i1] * B[k1,j1,k0,j0]\ni0=64\ni1=64\nj0=64\nj1=64\nk0=32\nk1=32\n",
}


def _time(fn, warm=3, reps=20, flush=None):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(reps):
        if flush is not None:
            flush.add_(1.0)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def _cpu_tccg_gett(name, A, B, C, alpha, beta, flops):
    """TCCG's generated GETT candidates (oracle/_ref/<name>.so) timed TCCG's
    way: min of 4 runs after a 2x128 MiB cache trash (tccg.py:975-1057);
    the best candidate is reported, as TCCG selects it."""
    import ctypes
    import numpy as np
    so = os.path.join(ROOT, "oracle", "_ref", name + ".so")
    if not os.path.exists(so):
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import aligned_copy
    L = ctypes.CDLL(so)
    L.tccg_gett_count.restype = ctypes.c_int
    L.tccg_gett_threads.restype = ctypes.c_int
    L.tccg_gett_name.restype = ctypes.c_char_p
    L.tccg_gett_run.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 3 + [ctypes.c_float] * 2
    A, B, C0 = aligned_copy(A), aligned_copy(B), aligned_copy(C)
    trash1 = np.ones(32 * 1024 * 1024, dtype=np.float32)
    trash2 = np.ones(32 * 1024 * 1024, dtype=np.float32)
    best = (float("inf"), None)
    for i in range(L.tccg_gett_count()):
        for _ in range(4):
            Cw = aligned_copy(C0)
            trash1 += 0.999 * trash2
            t0 = time.perf_counter()
            L.tccg_gett_run(i, A.ctypes.data, B.ctypes.data, Cw.ctypes.data, alpha, beta)
            t = time.perf_counter() - t0
            if t < best[0]:
                best = (t, L.tccg_gett_name(i).decode())
    return {"gflops": flops / best[0] / 1e9, "threads": L.tccg_gett_threads(),
            "candidates": L.tccg_gett_count(), "best": best[1][:60],
            "note": "TCCG-generated AVX2 GETT with the oracle's HPTT-API stand-in, g++ -O3 -march=x86-64-v3"}


def run_suite(args):
    import numpy as np
    import torch
    from tccg_b200 import parse_text
    from tccg_b200.api import Compiled
    from tccg_b200.autograd import GettFunction
    from tccg_b200.grouped import Group
    from tccg_b200.plan import Tuning
    from tccg_b200.workloads import batched_workload
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import LoopNest
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    flush = torch.empty(64 * 1024 * 1024, device=dev)
    peaks, _ = measured_peaks()
    out = {}

    def gen(n, seed, dist):
        g = torch.Generator(device=dev).manual_seed(seed)
        x = torch.randn(n, generator=g, device=dev)
        return x if dist == "normal" else (torch.rand(n, generator=g, device=dev) * 2 - 1)

    def errs(C, C64):
        n = torch.linalg.vector_norm(C64).item()
        return torch.linalg.vector_norm(C.double() - C64).item() / n

    def cpu_loop(con, A, B, C, alpha, beta, secs=3.0):
        c, a, b = con.C0.labels, con.A0.labels, con.B0.labels
        sizes = {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices}
        ln = LoopNest(c, a, b, sizes)
        Cb = C.copy()
        s = 8192
        while True:
            t0 = time.perf_counter()
            ln.run(A, B, Cb, alpha, beta, 0, s)
            t = time.perf_counter() - t0
            if t > 0.3 or s >= ln.size_c:
                break
            s = min(ln.size_c, s * 4)
        return 2.0 * s * ln.size_k / t / 1e9

    wanted = set(args.suite_configs.split(","))
    for name in ("cfg1", "cfg2", "cfg3"):
        if name not in wanted:
            continue
        con = parse_text(SUITE[name])
        dist = "uniform" if name == "cfg1" else "normal"
        nA, nB, nC = con.A0.num_elements(), con.B0.num_elements(), con.C0.num_elements()
        A, B, C0 = gen(nA, 1, dist), gen(nB, 2, dist), gen(nC, 3, dist)
        small = (nA + nB + nC) * 4 < 126e6
        C64 = C0.double().clone()
        Compiled(con, "fp64")(A.double(), B.double(), C64)
        flops = con.flop_count()
        byts = (nA + nB) * 4 + nC * 4 * (2 if con.beta else 1)
        res = {"flop": flops, "algorithmic_bytes_fp32": byts}
        modes = [("fp32", "gett", 0), ("bf16x3", "gett", 0), ("bf16", "gett", 0), ("fp64", "gett", 0)]
        if name == "cfg2":
            # the general CUDA-core tile kernel beside the short-K kernel the
            # library picks for K = 16
            modes += [("fp32", "gett", 0, {"shortk": -1})]
        if name in ("cfg1", "cfg2"):
            # short K: the BF16 precisions on each kernel family as well
            # (variant 0 is the library's own choice)
            modes += [("bf16x3", "gett", -1), ("bf16", "gett", -1),
                      ("bf16x3", "gett", 16), ("bf16", "gett", 1)]
        if name == "cfg2":
            modes += [("fp32", "ttgt", 0), ("bf16", "ttgt", 0), ("bf16x3", "ttgt", 0)]
        for mode in modes:
            prec, method, variant = mode[:3]
            extra = mode[3] if len(mode) > 3 else {}
            dbl = prec == "fp64"
            tune = Tuning(method=method, variant=variant, **extra)
            c = Compiled(con, prec, tune)
            Ai, Bi = (A.double(), B.double()) if dbl else (A, B)
            if prec == "bf16" and name == "cfg2":
                c = Compiled(con, prec, tune, dtype="bf16")
                Ai, Bi = A.bfloat16(), B.bfloat16()
            Cw = C0.double().clone() if dbl else C0.clone()
            ws = c.workspace(dev)
            reps = 5 if (name == "cfg3" and prec in ("fp32", "fp64")) else 20
            ms = _time(lambda: c.plan.run(Ai, Bi, Cw, workspace=ws), 2, reps, flush if small else None)
            Cw = C0.double().clone() if dbl else C0.clone()
            c.plan.run(Ai, Bi, Cw, workspace=ws)
            torch.cuda.synchronize()
            e = errs(Cw, C64) if not dbl else errs(Cw, C64)
            key = "%s_%s%s%s" % (prec, method, "_cuda_core" if variant < 0 else
                                 "_tensor_core" if variant > 0 else "",
                                 "_tile_kernel" if extra.get("shortk") == -1 else "")
            gbps = (byts * (2 if dbl else 1) if prec != "bf16" else byts - (nA + nB) * 2) / (ms * 1e-3) / 1e9
            res[key] = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12, "gbs": gbps,
                        "hbm_frac": gbps / peaks["hbm_gbs"], "normwise_vs_fp64": e,
                        "plan": c.describe()}
            del Cw, c, ws
            torch.cuda.empty_cache()
        # CPU baselines (host cores)
        An, Bn, Cn = A.cpu().numpy(), B.cpu().numpy(), C0.cpu().numpy()
        res["cpu_loop_nest_gflops"] = cpu_loop(con, An, Bn, Cn, con.alpha, con.beta)
        res["cpu_threads"] = os.cpu_count()
        if name in ("cfg1", "cfg2"):
            res["cpu_tccg_gett"] = _cpu_tccg_gett("tccg_gett_" + name, An, Bn, Cn, con.alpha,
                                                  con.beta, flops)
        out[name] = res
        print(json.dumps({name: res}), flush=True)
        del A, B, C0, C64
        torch.cuda.empty_cache()

    # configuration 4: forward + dA + dB through the autograd Function
    if "cfg4" not in wanted:
        return out if "cfg5" not in wanted else _suite_cfg5(out, gen, flush, dev)
    con = parse_text(SUITE["cfg4"])
    res = {"flop_each": con.flop_count()}
    for prec, dt in (("fp32", torch.float32), ("bf16", torch.bfloat16), ("bf16x3", torch.float32)):
        shA = tuple(i.size for i in reversed(con.A0.indices))
        shB = tuple(i.size for i in reversed(con.B0.indices))
        A = gen(con.A0.num_elements(), 4, "normal").reshape(shA).to(dt).requires_grad_()
        B = gen(con.B0.num_elements(), 5, "normal").reshape(shB).to(dt).requires_grad_()
        Cout = GettFunction.apply(A, B, con, prec)
        dC = torch.randn_like(Cout)
        fwd = _time(lambda: GettFunction.apply(A, B, con, prec), 3, 20, flush)
        both = _time(lambda: torch.autograd.grad(GettFunction.apply(A, B, con, prec), (A, B), dC),
                     3, 20, flush)
        res[prec] = {"fwd_ms": fwd, "fwd_bwd_ms": both,
                     "fwd_tflops": con.flop_count() / (fwd * 1e-3) / 1e12,
                     "fwd_bwd_tflops": 3 * con.flop_count() / (both * 1e-3) / 1e12}
    out["cfg4"] = res
    print(json.dumps({"cfg4": res}), flush=True)
    if "cfg5" in wanted:
        _suite_cfg5(out, gen, flush, dev)
    return out


def _kernel_mix(grp):
    """How many items of a group run on each kernel family / loader."""
    mix = {}
    for p in grp.plans:
        d = p.describe()
        k = ("skinny" if "skinny_gett" in d else "skinny_tc" if "skinny_tc" in d else
             "cuda_core" if "simt" in d else "tcgen05_gather" if "gather" in d else "tcgen05_packed")
        mix[k] = mix.get(k, 0) + 1
    return mix


def _tuning_mix(grp):
    mix = {}
    for p in grp.plans:
        k = p.tuning.key()
        mix[k] = mix.get(k, 0) + 1
    return dict(sorted(mix.items(), key=lambda kv: -kv[1]))


def _suite_cfg5(out, gen, flush, dev):
    """Configuration 5: 256 mixed contractions, one grouped launch in a CUDA
    graph, against one plan run (pack + GETT launch) per contraction."""
    import torch
    from tccg_b200.grouped import Group
    from tccg_b200.workloads import batched_workload
    items = batched_workload(256, seed=0)
    tot = sum(c.flop_count() for c in items)
    res = {"items": 256, "flop": tot}
    As = [gen(c.A0.num_elements(), 10 + i, "normal") for i, c in enumerate(items)]
    Bs = [gen(c.B0.num_elements(), 1000 + i, "normal") for i, c in enumerate(items)]
    Cs = [torch.empty(c.C0.num_elements(), device=dev) for c in items]
    for prec in ("bf16x3", "fp32"):
        grp = Group(items, prec)
        grp.bind(As, Bs, Cs)
        grp.capture()
        t_graph = _time(grp.replay, 3, 10, flush)
        t_items = _time(lambda: grp.run_per_item(), 2, 5, flush)
        res[prec] = {"graph_ms": t_graph, "graph_tflops": tot / (t_graph * 1e-3) / 1e12,
                     "per_item_launches_ms": t_items,
                     "per_item_tflops": tot / (t_items * 1e-3) / 1e12,
                     "workspace_gib": grp.workspace_bytes / 2 ** 30,
                     "kernels": _kernel_mix(grp)}
        del grp
        torch.cuda.empty_cache()
    if os.environ.get("TCCG_SUITE_AUTOTUNE", "1") != "0":
        # every item tuned (GETT, no tail split) from a fresh cache, then the
        # grouped run of the tuned plans
        import tempfile
        db = os.path.join(tempfile.mkdtemp(), "cfg5.db")
        t0 = time.perf_counter()
        grp = Group(items, "bf16x3", autotune=True, max_implementations=6, cache_path=db)
        t_tune = time.perf_counter() - t0
        grp.bind(As, Bs, Cs)
        grp.capture()
        t_graph = _time(grp.replay, 3, 10, flush)
        res["bf16x3_autotuned"] = {"graph_ms": t_graph, "graph_tflops": tot / (t_graph * 1e-3) / 1e12,
                                   "tuning_s": t_tune, "candidates_per_item": 6,
                                   "kernels": _kernel_mix(grp),
                                   "tunings": _tuning_mix(grp)}
        del grp
        torch.cuda.empty_cache()
    out["cfg5"] = res
    print(json.dumps({"cfg5": res}), flush=True)
    return out


CASES = {
    "cfg1": SUITE["cfg1"],
    "cfg2": SUITE["cfg2"],
    # configuration 2 with C's indices permuted against the GEMM's [M][N]
    # order: TTGT then transposes C' into C (the permute kernel)
    "cfg2t": "C[a,c,b,d] = A[a,e,b] * B[e,d,c] + C[a,c,b,d]\na=96\nb=96\nc=96\nd=96\ne=16\n",
    "cfg3k2": workload(2),
    "cfg3k4": workload(4),
    "cfg3k8": workload(8),
    "cfg4": SUITE["cfg4"],
}


def run_case(args):
    """One named workload run a few times with no timing, for profiler
    captures (ncu -k <kernel> -c <n> python bench.py --case ...):
    configurations by name (cfg3kN: configuration 3's C slab k < N),
    cfg5:N (the first N items of configuration 5 as one grouped run) or
    item:I (item I of configuration 5 alone)."""
    import torch
    from tccg_b200 import parse_text
    from tccg_b200.api import Compiled
    from tccg_b200.plan import Plan, Tuning
    from tccg_b200.workloads import batched_workload
    dev = torch.device("cuda", 0)
    tune = {}
    for kv in filter(None, args.tuning.split(",")):
        k, v = kv.split("=")
        tune[k] = v if k == "method" else int(v)
    t = Tuning(**tune)
    g = torch.Generator(device=dev).manual_seed(5)
    if args.case.startswith("cfg5:"):
        from tccg_b200.grouped import Group
        items = batched_workload(int(args.case.split(":")[1]), seed=0)
        As = [torch.randn(c.A0.num_elements(), generator=g, device=dev) for c in items]
        Bs = [torch.randn(c.B0.num_elements(), generator=g, device=dev) for c in items]
        Cs = [torch.empty(c.C0.num_elements(), device=dev) for c in items]
        grp = Group(items, args.precision, tunings=[t] * len(items) if tune else None)
        grp.bind(As, Bs, Cs)
        for _ in range(args.runs):
            grp.run()
        torch.cuda.synchronize()
        print("case %s: %d items" % (args.case, len(items)), flush=True)
        return 0
    con = (batched_workload(int(args.case.split(":")[1]) + 1, seed=0)[-1]
           if args.case.startswith("item:") else parse_text(CASES[args.case]))
    dt = "bf16" if args.precision == "bf16" else None
    c = Compiled(con, args.precision, t, dtype=dt)
    tdt = {"fp32": torch.float32, "bf16x3": torch.float32, "bf16": torch.bfloat16,
           "fp64": torch.float64}[args.precision]
    A = torch.randn(con.A0.num_elements(), generator=g, device=dev).to(tdt)
    B = torch.randn(con.B0.num_elements(), generator=g, device=dev).to(tdt)
    C = torch.randn(con.C0.num_elements(), generator=g, device=dev).to(
        torch.float64 if args.precision == "fp64" else torch.float32)
    for _ in range(args.runs):
        c(A, B, C)
    torch.cuda.synchronize()
    print("case %s %s: %s" % (args.case, args.precision, c.describe()), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--raster", type=int, default=0)
    ap.add_argument("--max-ctas", type=int, default=0)
    ap.add_argument("--pair", type=int, default=0,
                    help="1 = CTA-pair tensor-core kernel (cta_group::2, 256-row tiles)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--skip-fp32", action="store_true")
    ap.add_argument("--skip-errors", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--k-extent", type=int, default=32,
                    help="extent of C's last index (32 = the full workload)")
    ap.add_argument("--suite", action="store_true",
                    help="measure every configuration (one JSON line each) instead of the headline")
    ap.add_argument("--suite-configs", default="cfg1,cfg2,cfg3,cfg4,cfg5")
    ap.add_argument("--case", default=None,
                    help="run one named workload --runs times without timing (profiler captures): "
                         + ", ".join(sorted(CASES)) + ", cfg5:N, item:I")
    ap.add_argument("--precision", default="bf16x3", help="precision of --case")
    ap.add_argument("--runs", type=int, default=2, help="runs of --case")
    ap.add_argument("--tuning", default="", help="tuning of --case, e.g. raster=32,load=1")
    args = ap.parse_args()
    if args.case:
        return run_case(args)
    if args.suite:
        run_suite(args)
        return 0
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        return run_reference(args, world, rank)
    world, rank, local = dist_setup(args.gpus)
    try:
        return run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
