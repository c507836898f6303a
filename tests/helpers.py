"""Shared helpers of the test suite: seeded inputs and running a plan on
numpy arrays (the memory of a column-major tensor is a flat numpy array)."""
import numpy as np


def splitmix_uniform(n: int, seed: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    """Deterministic U[lo, hi) float64 values from a splitmix64 stream."""
    with np.errstate(over="ignore"):
        x = np.arange(n, dtype=np.uint64) + np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    u = (x >> np.uint64(11)).astype(np.float64) / float(1 << 53)
    return lo + (hi - lo) * u


def seeded_normal(n: int, seed: int) -> np.ndarray:
    """Deterministic N(0,1) float64 values (Box-Muller on two splitmix streams)."""
    u1 = splitmix_uniform(n, 2 * seed + 1, 0.0, 1.0)
    u2 = splitmix_uniform(n, 2 * seed + 2, 0.0, 1.0)
    u1 = np.maximum(u1, 1e-300)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def run_gpu(con, precision, A, B, C, alpha=None, beta=None, tuning=None, dtype=None, view=None):
    """Run one contraction through the native plan; returns C as float64 numpy."""
    import torch
    from tccg_b200.plan import Plan
    p = Plan(con, precision=precision, tuning=tuning, dtype=dtype, view=view)
    tdt = {"f32": torch.float32, "f64": torch.float64, "bf16": torch.bfloat16}
    dA = torch.from_numpy(np.ascontiguousarray(A)).to("cuda").to(tdt[p.dtype])
    dB = torch.from_numpy(np.ascontiguousarray(B)).to("cuda").to(tdt[p.dtype])
    dC = torch.from_numpy(np.ascontiguousarray(C)).to("cuda").to(tdt[p.c_dtype])
    p.run(dA, dB, dC, alpha, beta)
    torch.cuda.synchronize()
    assert p.status() == 0
    return dC.double().cpu().numpy(), p


def labels(con):
    """Original (file) label lists of a contraction for the oracle."""
    return con.C0.labels, con.A0.labels, con.B0.labels, {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices}
