"""On-device autotuner with a persistent cache.

TCCG ranks GETT candidates with a performance model (gett.py:590-687), builds
the best ``--maxImplementations`` of them with make, times them in a
generated harness and keeps the results in SQLite keyed on the contraction,
the sizes, the CPU and the types (sql_util.py:206-306; lookup tccg.py:192-221).

Here the candidates are kernel choices of one native plan, TCCG's search
dimensions restated for the GPU:

* method: GETT or TTGT (TCCG also weighs TTGT and LoG, tccg.py:188-430);
* loop order (TCCG's two GEMM variants, panel-matrix and matrix-panel,
  gett.py:52-55): the persistent tile order, groups of tile rows (raster > 0)
  or of tile columns (raster < 0), and the group size;
* blockings (TCCG's mc/nc/kc, gett.py:1023-1062): the tcgen05 tile shape
  through the operand loader (128x192 tiles after a packing pass, or 128x128
  tiles gathered from the caller's tensors), the K-chunk of the split-BF16x3
  accumulation, k-split (CUDA cores) and the CUDA-core tile shape;
* mode orders of the GETT view (the index permutations TCCG searches with
  its index splits, gett.py:1063-1110): the N order (C's, or GB's unit-stride
  mode first) and the K order (GA's or GB's), where they change the view;
* kernel family for the BF16 precisions (tensor cores or CUDA cores).

They are ordered by a simple model (defaults first, then one dimension
varied at a time), timed on the device with CUDA events (minimum over
repetitions, L2 flushed in between like TCCG's trashCache,
tccg.py:725-737), and the winner is stored in SQLite keyed on (contraction,
extents, precision, operand type, beta != 0, GPU name, SM count, library
version). A cache hit skips the search.
"""
from __future__ import annotations

import json
import os
import sqlite3
import time
from typing import List, Optional, Tuple

from ._native import TccgError
from .plan import Plan, Tuning
from .spec import Contraction

# Part of every cache key: cached winners measured on older kernels (or
# without the tuning fields a newer build searches) are not reused.
CODE_VERSION = "tccg_b200-0.4"


def default_db_path() -> str:
    if os.environ.get("TCCG_B200_DB"):
        return os.environ["TCCG_B200_DB"]
    if os.environ.get("TCCG_ROOT"):
        return os.path.join(os.environ["TCCG_ROOT"], "tccg_b200.db")
    return os.path.join(os.path.expanduser("~"), ".cache", "tccg_b200", "tuning.db")


def contraction_key(con: Contraction) -> str:
    """Contraction string with extents, on the original (file) indices."""
    t = lambda T: "%s[%s]" % (T.label, ",".join("%s:%d" % (i.label, i.size) for i in T.indices))
    return "%s=%s*%s" % (t(con.C0), t(con.A0), t(con.B0))


class TuningDB:
    """SQLite store of measurements and of the best tuning per key."""

    def __init__(self, path: Optional[str] = None):
        self.path = path or default_db_path()
        d = os.path.dirname(self.path)
        if d:
            os.makedirs(d, exist_ok=True)
        self.conn = sqlite3.connect(self.path)
        c = self.conn.cursor()
        c.execute("CREATE TABLE IF NOT EXISTS measurements (key TEXT, tuning TEXT, ms REAL, "
                  "gflops REAL, ts REAL)")
        c.execute("CREATE TABLE IF NOT EXISTS best (key TEXT PRIMARY KEY, tuning TEXT, ms REAL, "
                  "gflops REAL, ts REAL)")
        self.conn.commit()

    def lookup(self, key: str) -> Optional[Tuple[Tuning, float]]:
        r = self.conn.execute("SELECT tuning, gflops FROM best WHERE key = ?", (key,)).fetchone()
        if r is None:
            return None
        return Tuning(**json.loads(r[0])), float(r[1])

    def record(self, key: str, tuning: Tuning, ms: float, gflops: float) -> None:
        self.conn.execute("INSERT INTO measurements VALUES (?, ?, ?, ?, ?)",
                          (key, json.dumps(tuning.__dict__), ms, gflops, time.time()))
        self.conn.commit()

    def store_best(self, key: str, tuning: Tuning, ms: float, gflops: float) -> None:
        self.conn.execute("INSERT OR REPLACE INTO best VALUES (?, ?, ?, ?, ?)",
                          (key, json.dumps(tuning.__dict__), ms, gflops, time.time()))
        self.conn.commit()

    def measurements(self, key: str):
        return self.conn.execute("SELECT tuning, ms, gflops FROM measurements WHERE key = ?",
                                 (key,)).fetchall()


def gpu_signature() -> str:
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return "%s/sm%d%d/%dSM" % (p.name, p.major, p.minor, p.multi_processor_count)


def tuning_key(con: Contraction, precision: str, dtype: str, gpu: str) -> str:
    return "|".join([contraction_key(con), precision, dtype, "beta" if con.beta != 0 else "nobeta",
                     gpu, CODE_VERSION])


def order_variants(con: Contraction):
    """(n_order, k_order) pairs whose GETT views differ, the heuristic (0, 0)
    first."""
    from .plan import gett_view
    seen, out = set(), []
    for no, ko in ((0, 0), (1, 0), (2, 0), (0, 1), (0, 2)):
        v = gett_view(con, n_order=no, k_order=ko)
        key = (tuple(v.m), tuple(v.n), tuple(v.k))
        if key not in seen:
            seen.add(key)
            out.append((no, ko))
    return out


def candidates(con: Contraction, precision: str, methods=("gett", "ttgt"), num_sms: int = 148,
               dtype: str = "f32", grouped: bool = False) -> List[Tuning]:
    """Candidate tunings, the model's favourite first: the defaults, then
    variations that matter for this shape. ``grouped``: for an item of a
    grouped launch (GETT, no tcgen05 tail split)."""
    M, N, K = con.sizeM, con.sizeN, max(1, con.sizeK)
    if grouped:
        methods = ("gett",)
    orders = order_variants(con)
    out: List[Tuning] = []
    # the skinny kernel (one small free extent) right after the model's
    # choice; held off at the end of the search
    elig = skinny_eligible(M, N, K, precision, dtype)
    skinny = [Tuning(method="gett", skinny=1)] if elig else []
    skinny_off = [Tuning(method="gett", skinny=-1)] if elig else []
    for method in methods:
        if precision in ("fp32", "fp64"):
            bm, bn = (128, 128) if precision == "fp32" else (128, 64)
            tiles = -(-M // bm) * -(-N // bn)
            splits = [1]
            # k-split only pays when there are fewer tiles than SMs can hold
            # (TCCG: only when M*N is small, gett.py:933)
            if tiles < 2 * num_sms:
                for s in (2, 4, 8, 16):
                    if K >= 64 * s:
                        splits.append(s)
            splits.sort(key=lambda s: abs(tiles * s - 2 * num_sms))
            out += [Tuning(method=method, ksplit=s) for s in splits[:1]]
            if method == "gett" and precision == "fp32":
                out += skinny
            out += [Tuning(method=method, ksplit=s) for s in splits[1:]]
            # short K: the C-prefetching kernel forced on and off
            if K <= (16 if precision == "fp64" else 32):
                out += [Tuning(method=method, ksplit=1, shortk=1),
                        Tuning(method=method, ksplit=1, shortk=-1)]
            # FP32: each CUDA-core tile shape (square, small N, small M)
            if precision == "fp32":
                out += [Tuning(method=method, simt_tile=t) for t in (1, 2, 3)]
            out += [Tuning(method=method, n_order=no, k_order=ko) for no, ko in orders[1:]]
            if method == "gett" and precision == "fp32":
                out += skinny_off
        else:
            # variant > 0 forces the tensor cores (BF16X3: k-blocks per
            # accumulation chunk), < 0 the CUDA cores; the library's own
            # choice (variant 0) goes first, then each kernel family: the
            # CUDA cores and, for BF16x3 with FP32 operands, both tcgen05
            # loaders (128x192 tiles packed, 128x128 tiles gathered); then
            # accumulation chunks, tile orders and mode orders.
            loads = [1, 2] if precision == "bf16x3" and dtype == "f32" and method == "gett" else [0]
            chunks = [16, 32, 8] if precision == "bf16x3" else [1]
            first = [Tuning(method=method)] + (skinny if method == "gett" else [])
            if len(loads) > 1:
                first += [Tuning(method=method, load=ld) for ld in loads]
            else:
                first.append(Tuning(method=method, variant=chunks[0]))  # tensor cores
            first.append(Tuning(method=method, variant=-1))
            # tcgen05 tile widths of the packed-operand loader
            tiles = [128] if precision == "bf16x3" else [192, 128]
            tl = 1 if len(loads) > 1 else 0
            more = [Tuning(method=method, load=tl, variant=chunks[0], tile_n=w) for w in tiles]
            # the tensor-core skinny kernel forced on
            if method == "gett" and skinny_tc_eligible(M, N, K, precision, dtype):
                more.insert(0, Tuning(method=method, skinny=2))
            for ld in loads:
                more += [Tuning(method=method, load=ld, raster=r) for r in (-8, 4, 16, -2)]
                more += [Tuning(method=method, load=ld, variant=c) for c in chunks[1:]]
            more += [Tuning(method=method, n_order=no, k_order=ko) for no, ko in orders[1:]]
            if K <= 32:
                more += [Tuning(method=method, variant=-1, shortk=1),
                         Tuning(method=method, variant=-1, shortk=-1)]
            if not grouped:
                # the tcgen05 tail split off (it is on where the model expects a gain)
                more.append(Tuning(method=method, tail_split=-1))
                # the CTA-pair kernel (256-row tiles, cta_group::2) where there
                # are rows for it: measured 16 % slower per GHz than the one-SM
                # kernel on configuration 3, searched so that a shape it serves
                # better can pick it (grouped launches do not run it)
                if M >= 512 and (precision != "bf16x3" or dtype == "f32"):
                    more.append(Tuning(method=method, pair=1, variant=chunks[0]))
            out += first + more + (skinny_off if method == "gett" else [])
    if grouped:
        for t in out:
            t.tail_split = -1
    # drop repeats, keeping the first of each
    seen, uniq = set(), []
    for t in out:
        if t.key() not in seen:
            seen.add(t.key())
            uniq.append(t)
    return uniq


def skinny_eligible(M: int, N: int, K: int, precision: str, dtype: str = "f32") -> bool:
    """Whether the skinny kernel can run a GETT of these extents (the C ABI's
    rule: FP32 operands, FP32 or BF16x3 precision, min(M, N) <= 256; the C ABI
    also wants tensors of fewer than 2^31 elements, and the search skips a
    candidate it refuses)."""
    return dtype == "f32" and precision in ("fp32", "bf16x3") and min(M, N) <= 256


def skinny_tc_eligible(M: int, N: int, K: int, precision: str, dtype: str = "f32") -> bool:
    """Whether the tensor-core skinny kernel (tuning.skinny = 2) can run a GETT
    of these extents: split-BF16x3 with FP32 operands, min(M, N) <= 256,
    K <= 2^29 (the C ABI's rule)."""
    return dtype == "f32" and precision == "bf16x3" and min(M, N) <= 256 and K <= (1 << 29)


def _flush_l2(buf):
    buf.add_(1.0)


def _inputs(con: Contraction, dtype: str, c_dtype: str):
    """Seeded operands of ``con`` on the current device, shared by all the
    candidates of one search."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    tdt = {"f32": torch.float32, "f64": torch.float64, "bf16": torch.bfloat16}
    g = torch.Generator(device=dev).manual_seed(0)
    A = torch.randn(con.A0.num_elements(), generator=g, device=dev).to(tdt[dtype])
    B = torch.randn(con.B0.num_elements(), generator=g, device=dev).to(tdt[dtype])
    C = torch.randn(con.C0.num_elements(), generator=g, device=dev).to(tdt[c_dtype])
    return A, B, C


_TRASH = {}


def measure(plan: Plan, reps: int = 5, inputs=None) -> float:
    """Minimum device time (ms) of one plan run over ``reps`` repetitions,
    with a 256 MB buffer written between repetitions to flush L2."""
    import torch
    con = plan.con
    dev = torch.device("cuda", torch.cuda.current_device())
    tdt = {"f32": torch.float32, "f64": torch.float64, "bf16": torch.bfloat16}
    if inputs is None:
        g = torch.Generator(device=dev).manual_seed(0)
        A = torch.randn(con.A0.num_elements(), generator=g, device=dev).to(tdt[plan.dtype])
        B = torch.randn(con.B0.num_elements(), generator=g, device=dev).to(tdt[plan.dtype])
        C = torch.randn(con.C0.num_elements(), generator=g, device=dev).to(tdt[plan.c_dtype])
    else:
        A, B, C = inputs
    ws = torch.empty(max(plan.workspace_bytes, 1), dtype=torch.uint8, device=dev)
    trash = _TRASH.get(dev)
    if trash is None:
        trash = _TRASH[dev] = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    plan.run(A, B, C, workspace=ws)  # warm-up
    torch.cuda.synchronize()
    best = float("inf")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(reps):
        _flush_l2(trash)
        e0.record()
        plan.run(A, B, C, workspace=ws)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    if plan.status() != 0:
        raise RuntimeError("device error while tuning %s" % plan.describe())
    return best


def autotune(con: Contraction, precision: str, max_implementations: int = 16,
             cache_path: Optional[str] = None, dtype: Optional[str] = None,
             ignore_cache: bool = False, methods=("gett", "ttgt"), verbose: bool = False,
             max_workspace_gb: Optional[float] = None, grouped: bool = False,
             db: Optional[TuningDB] = None, stats: Optional[dict] = None) -> Tuning:
    """Best tuning for ``con``: from the cache, else by timing up to
    ``max_implementations`` candidates (-1 = all). ``grouped``: tune an item
    of a grouped launch (GETT, no tail split; cached under its own key).
    ``stats`` (optional dict) counts cache "hits" and "tuned" contractions."""
    import torch
    from .plan import operand_dtype
    dtype = dtype or operand_dtype(precision)
    db = db or TuningDB(cache_path)
    key = tuning_key(con, precision, dtype, gpu_signature()) + ("|grouped" if grouped else "")
    if not ignore_cache:
        hit = db.lookup(key)
        if hit is not None:
            if verbose:
                print("[tccg_b200] tuning cache hit: %s (%.2f GFLOPS)" % (hit[0].key(), hit[1]))
            if stats is not None:
                stats["hits"] = stats.get("hits", 0) + 1
            return hit[0]
    if stats is not None:
        stats["tuned"] = stats.get("tuned", 0) + 1
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    cands = candidates(con, precision, methods, sms, dtype=dtype, grouped=grouped)
    if max_implementations >= 0:
        cands = cands[:max(1, max_implementations)]
    best, best_ms = None, float("inf")
    flops = con.flop_count()
    inputs = _inputs(con, dtype, "f64" if precision == "fp64" else "f32")
    for t in cands:
        try:
            p = Plan(con, precision=precision, tuning=t, dtype=dtype)
        except TccgError:  # a kernel this contraction cannot take
            continue
        if max_workspace_gb is not None and p.workspace_bytes > max_workspace_gb * 2 ** 30:
            continue
        ms = measure(p, inputs=inputs)
        gf = flops / (ms * 1e-3) / 1e9
        db.record(key, t, ms, gf)
        if verbose:
            print("[tccg_b200] %-28s %9.3f ms %10.1f GFLOPS  %s" % (t.key(), ms, gf, p.describe()))
        if ms < best_ms:
            best, best_ms = t, ms
    if best is None:
        raise RuntimeError("no candidate fits the workspace limit")
    db.store_best(key, best, best_ms, flops / (best_ms * 1e-3) / 1e9)
    return best
