"""Multi-GPU host logic on CPU: two gloo ranks split a contraction into C
slabs (tccg_b200.shard), compute their slab from the full tensors through the
slab's offsets and strides (oracle as the computing stand-in), and the
gathered slabs equal the whole contraction."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from tccg_b200.shard import shard, split_index
from tccg_b200.spec import make_contraction

SIZES = dict(a=4, b=3, c=5, i=6, j=2, k=7, m=3, n=2)
LABELS = ("abcijk", "ambnc", "minjk")


def _slab_via_shard(sh, A, B, C):
    """Compute the slab with the oracle on strided views built ONLY from the
    shard's offsets/strides/extents (what the GPU plan receives)."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    from oracle import LoopNest
    con = sh.contraction
    sizes = {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices}

    def view(arr, t, T):
        shape = [sizes[l] for l in T.labels]
        strides = [sh.strides[t][l] * arr.itemsize for l in T.labels]
        v = np.lib.stride_tricks.as_strided(arr[sh.offsets[t]:], shape=shape, strides=strides)
        return np.asfortranarray(v).ravel(order="F")

    a, b = view(A, "A", con.A0), view(B, "B", con.B0)
    ln = LoopNest(con.C0.labels, con.A0.labels, con.B0.labels, sizes)
    out = ln.run(a.copy(), b.copy(), np.zeros(ln.size_c), 1.0, 0.0)
    return out


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    con = make_contraction(*LABELS, SIZES)
    rng = np.random.default_rng(0)
    A = rng.standard_normal(con.A0.num_elements())
    B = rng.standard_normal(con.B0.num_elements())
    sh = shard(con, rank, world)
    slab = torch.from_numpy(_slab_via_shard(sh, A, B, None))
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([slab.numel()]))
    mx = int(max(s.item() for s in sizes))
    buf = torch.zeros(mx, dtype=torch.float64)
    buf[:slab.numel()] = slab
    out = [torch.zeros(mx, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(out, buf)
    if rank == 0:
        q.put([o[:int(s.item())].numpy() for o, s in zip(out, sizes)])
    dist.barrier()
    dist.destroy_process_group()


def test_split_index_choice():
    con = make_contraction(*LABELS, SIZES)
    assert split_index(con, 2) == "k"      # C's last index
    assert split_index(con, 7) == "k"
    with pytest.raises(ValueError):
        split_index(con, 8)          # no index of C has extent >= 8


def test_shards_partition_the_index():
    con = make_contraction(*LABELS, SIZES)
    for world in (1, 2, 3, 7):
        spans = [(shard(con, r, world).lo, shard(con, r, world).hi) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == SIZES["k"]
        assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))


def test_two_gloo_ranks_reassemble_the_contraction():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    from oracle import LoopNest
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    slabs = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    con = make_contraction(*LABELS, SIZES)
    rng = np.random.default_rng(0)
    A = rng.standard_normal(con.A0.num_elements())
    B = rng.standard_normal(con.B0.num_elements())
    ln = LoopNest(*LABELS, SIZES)
    full = ln.run(A.copy(), B.copy(), np.zeros(ln.size_c), 1.0, 0.0)
    # C's last index k is split: rank slabs are contiguous pieces of C
    assert np.allclose(np.concatenate(slabs), full, rtol=1e-13, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
def test_slabs_on_one_gpu_match_the_whole(cuda, world):
    """The product path for a slab: Plan(strides=full strides) + element
    offsets into the full tensors; all slabs together equal one full run."""
    import torch
    from tccg_b200 import shard as S
    from tccg_b200.plan import Plan
    con = make_contraction(*LABELS, dict(SIZES, k=11, a=16, i=9))
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(con.A0.num_elements(), generator=g, device="cuda")
    B = torch.randn(con.B0.num_elements(), generator=g, device="cuda")
    for prec in ("fp32", "bf16x3"):
        full = torch.zeros(con.C0.num_elements(), device="cuda")
        Plan(con, precision=prec).run(A, B, full)
        parts = torch.full_like(full, float("nan"))
        for r in range(world):
            sh = S.shard(con, r, world)
            S.run(Plan(sh.contraction, precision=prec, strides=sh.strides), sh, A, B, parts)
        torch.cuda.synchronize()
        assert torch.equal(parts, full), prec
