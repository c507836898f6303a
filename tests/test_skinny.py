"""The skinny kernel (tuning.skinny = 1; tccg_b200/csrc/skinny_gett.cuh):
contractions with one small free extent, the narrow operand in shared memory
and the wide one streamed in place, FP32 FMAs.

Every case is checked against the FP64 oracle at the FP32 bound (normwise
1e-6) for both precisions that can run it (FP32, and BF16x3 -- served in
FP32, more accurate than its three-product split). The cases cover each P
load walk (along x, along y for a transposition between P and C, along k),
each C store walk (x then S, x then Y, runs of C's stride-one S mode), one
and several passes over S, k-split slices and their reduction (with beta),
the operand swap, a matrix-vector and an outer product; grouped runs equal
per-item runs bit for bit, repeated runs are deterministic, and a plan that
cannot take the kernel is refused when it is forced.
"""
import numpy as np
import pytest

from helpers import run_gpu, seeded_normal
from oracle import LoopNest, error_metrics
from tccg_b200.plan import Plan, Tuning
from tccg_b200.spec import make_contraction

pytestmark = pytest.mark.gpu

# (C, A, B, extents, alpha, beta, describe tags)
CASES = {
    # P (= B after the swap) has d at stride one, C has v: boxes of 19 x 13
    "transpose": ("vqud", "qe", "duve", dict(v=19, q=40, u=6, d=31, e=20), 0.75, 0.0,
                  ["narrow=N", "load=y", "store=xs linear"]),
    # C's stride-one index on the narrow side (runs of c), long K split over slices
    "matvec_split": ("cdn", "dnxy", "yxc", dict(c=8, d=23, n=20, x=60, y=41), 0.5, -1.5,
                     ["narrow=M", "store=sx run=8"]),
    # P's stride-one index is contracted (u): loads along k
    "kfast": ("fjr", "ufr", "ju", dict(f=10, j=28, r=46, u=8), 1.0, 0.25,
              ["narrow=N", "load=k", "store=xs"]),
    # S = 150 rows in five passes of three runs of o (C's stride-one mode,
    # directly followed by r): each run of a box row one range of 10 x 37
    "passes": ("orak", "cok", "rac", dict(o=10, r=37, a=9, k=15, c=18), -0.75, 0.0,
               ["narrow=M", "rows=5x30", "store=sx run=10 ranges"]),
    # the same with a flat box (256 x 1; the whole CTA copies each range) and
    # a ragged last box along x
    "ranges_flat": ("orak", "cok", "rac", dict(o=10, r=300, a=2, k=15, c=18), 1.0, 0.0,
                    ["rows=5x30", "box=256x1", "ranges"]),
    # runs of 8 with passes of 32 rows, K split over slices (the reduction
    # copies the ranges), beta != 0
    "ranges_split": ("orkb", "lok", "rlb", dict(o=8, r=40, k=9, b=3, l=400), 0.5, 0.5,
                     ["rows=3x32", "ranges"]),
    # C's next stride after X is a W mode: (x, y) planes; K over three chunks
    "xy": ("mpn", "pmk", "kn", dict(m=33, p=9, n=5, k=70), 1.0, 1.0,
           ["narrow=N", "load=y", "store=xy"]),
    # two passes of 32 rows over one block, K split over slices (the
    # reduction runs per block and pass)
    "passes_split": ("ab", "akl", "lkb", dict(a=56, b=93, k=60, l=50), 1.0, 0.5,
                     ["narrow=M", "rows=2x32"]),
    "matvec": ("a", "ak", "k", dict(a=300, k=77), 1.0, 0.0, ["S=1 "]),
    "outer": ("ab", "a", "b", dict(a=33, b=65), 1.5, 0.0, ["kchunks=1 "]),
}


def _data(ln, seed):
    A = seeded_normal(ln.size_a, seed).astype(np.float32)
    B = seeded_normal(ln.size_b, seed + 1).astype(np.float32)
    C = seeded_normal(ln.size_c, seed + 2).astype(np.float32)
    return A, B, C


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_skinny_matches_oracle(cuda, name, precision):
    lc, la, lb, sizes, alpha, beta, tags = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 17)
    out, p = run_gpu(con, precision, A, B, C, tuning=Tuning(skinny=1))
    d = p.describe()
    assert "kernel=skinny_gett<f32>" in d, d
    for t in tags:
        assert t in d, (t, d)
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(out, ref)["normwise"] <= 1e-6, d


@pytest.mark.parametrize("ksplit", [1, 3, 0])
def test_skinny_k_split_is_deterministic(cuda, ksplit):
    """Slices added in order by the reduction: repeated runs are bitwise
    equal, and an explicit split count is honoured."""
    lc, la, lb, sizes, alpha, beta, _ = CASES["matvec_split"]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 23)
    o1, p = run_gpu(con, "fp32", A, B, C, tuning=Tuning(skinny=1, ksplit=ksplit))
    o2, _ = run_gpu(con, "fp32", A, B, C, tuning=Tuning(skinny=1, ksplit=ksplit))
    assert np.array_equal(o1, o2)
    if ksplit:
        assert "ksplit=%d " % ksplit in p.describe(), p.describe()
    else:
        assert "ksplit=1 " not in p.describe(), p.describe()
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(o1, ref)["normwise"] <= 1e-6


@pytest.mark.parametrize("name", ["matvec_split", "matvec"])
def test_skinny_register_and_shared_paths_agree(cuda, monkeypatch, name):
    """A narrow side of at most 16 rows runs the register path (P straight
    to registers, skinny_reg_kernel); TCCG_B200_SKINNY_REG=0 keeps the
    shared-memory path. With the same k slices (given explicitly: the
    automatic count follows each path's CTAs per SM) both sum k in the same
    order: the same bits, and the oracle's values."""
    lc, la, lb, sizes, alpha, beta, _ = CASES[name]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 31)
    t = Tuning(skinny=1, ksplit=3 if name == "matvec_split" else 1)
    o_reg, p_reg = run_gpu(con, "fp32", A, B, C, tuning=t)
    monkeypatch.setenv("TCCG_B200_SKINNY_REG", "0")
    o_smem, p_smem = run_gpu(con, "fp32", A, B, C, tuning=t)
    assert "path=registers" in p_reg.describe() and "path=registers" not in p_smem.describe()
    assert np.array_equal(o_reg, o_smem)
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(o_reg, ref)["normwise"] <= 1e-6


def test_skinny_bulk_and_element_stores_agree(cuda):
    """Linear C rows with beta = 0 leave by bulk copies (alpha applied when
    staging) when C is 16-byte aligned, else by element stores: a C one
    element off a 16-byte boundary gives the same bits."""
    import torch
    lc, la, lb, sizes, alpha, beta, _ = CASES["transpose"]
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, _ = _data(ln, 29)
    p = Plan(con, "fp32", tuning=Tuning(skinny=1))
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    outs = []
    for off in (0, 1):
        buf = torch.full((ln.size_c + 4,), float("nan"), device="cuda")
        dC = buf[off:off + ln.size_c]
        p.run(dA, dB, dC, alpha, beta)
        torch.cuda.synchronize()
        assert p.status() == 0
        assert torch.isnan(buf[:off]).all() and torch.isnan(buf[off + ln.size_c:]).all()
        outs.append(dC.clone())
    assert torch.equal(outs[0], outs[1])
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), np.zeros(ln.size_c), alpha, 0.0)
    assert error_metrics(outs[0].double().cpu().numpy(), ref)["normwise"] <= 1e-6


def test_skinny_grouped_equals_per_item(cuda):
    """A grouped run with skinny items (one of them k-split) next to
    tensor-core and CUDA-core items equals the per-item runs bit for bit."""
    import torch
    from tccg_b200.grouped import Group
    names = ["transpose", "matvec_split", "kfast", "passes", "xy"]
    items = [make_contraction(*CASES[n][:4], 1.0, 0.0) for n in names]
    items.append(make_contraction("mn", "mk", "kn", dict(m=700, n=500, k=300), 1.0, 0.0))
    tunings = [Tuning(skinny=1)] * len(names) + [Tuning(variant=16)]
    g = torch.Generator(device="cuda").manual_seed(3)
    As = [torch.randn(c.A0.num_elements(), generator=g, device="cuda") for c in items]
    Bs = [torch.randn(c.B0.num_elements(), generator=g, device="cuda") for c in items]
    Cs = [torch.zeros(c.C0.num_elements(), device="cuda") for c in items]
    grp = Group(items, "bf16x3", tunings=tunings)
    assert sum("skinny_gett" in p.describe() for p in grp.plans) == len(names)
    grp.bind(As, Bs, Cs)
    grp.capture()
    grp.replay()
    torch.cuda.synchronize()
    grouped = [c.clone() for c in Cs]
    for c in Cs:
        c.zero_()
    grp.run_per_item()
    torch.cuda.synchronize()
    for a, b in zip(grouped, Cs):
        assert torch.equal(a, b)
    for con, A, B, C in zip(items[:len(names)], As, Bs, grouped):
        ln = LoopNest(con.C0.labels, con.A0.labels, con.B0.labels,
                      {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices})
        ref = ln.run(A.double().cpu().numpy(), B.double().cpu().numpy(), np.zeros(ln.size_c), 1.0, 0.0)
        assert error_metrics(C.double().cpu().numpy(), ref)["normwise"] <= 1e-6, str(con)


# the tensor-core kernel (tuning.skinny = 2): every case ("passes": S = 150 in
# passes of 64 rows)
TC_CASES = sorted(CASES)
# long K over several TMEM rounds (ksplit=1: 38 chunks = rounds of 16, 16, 6),
# a narrow side of exactly 64, and one of 200 (passes of 64, 64, 64, 8)
TC_EXTRA = {
    "rounds": ("ab", "akl", "lkb", dict(a=900, b=24, k=40, l=30), 1.0, 0.5),
    "s64": ("sw", "sk", "kw", dict(s=64, w=1000, k=300), -1.0, 0.0),
    "s200": ("ws", "kw", "sk", dict(s=200, w=700, k=100), 1.0, 0.25),
}


def _tc_case(name):
    if name in TC_EXTRA:
        return TC_EXTRA[name]
    return CASES[name][:6]


@pytest.mark.parametrize("ksplit", [0, 1])
@pytest.mark.parametrize("name", TC_CASES + sorted(TC_EXTRA))
def test_skinny_tc_matches_oracle(cuda, name, ksplit):
    """tcgen05 MMAs of the split-BF16x3 products (P converted in shared
    memory, Q packed once, FP32 sums over TMEM rounds) at the BF16x3 bound."""
    lc, la, lb, sizes, alpha, beta = _tc_case(name)
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 41)
    out, p = run_gpu(con, "bf16x3", A, B, C, tuning=Tuning(skinny=2, ksplit=ksplit))
    d = p.describe()
    assert "kernel=skinny_tc<BF16X3>" in d, d
    if ksplit == 1:
        assert "ksplit=1 " in d, d
    ref = ln.run(A.astype(np.float64), B.astype(np.float64), C.astype(np.float64), alpha, beta)
    assert error_metrics(out, ref)["normwise"] <= 1e-5, d


def test_skinny_tc_is_deterministic_and_refuses(cuda):
    """Repeated runs (k slices added in order) are bitwise equal; the kernel
    serves split-BF16x3 with a narrow side of at most 256 only."""
    from tccg_b200._native import TccgError
    lc, la, lb, sizes, alpha, beta = _tc_case("rounds")
    con = make_contraction(lc, la, lb, sizes, alpha, beta)
    ln = LoopNest(lc, la, lb, sizes)
    A, B, C = _data(ln, 43)
    o1, p = run_gpu(con, "bf16x3", A, B, C, tuning=Tuning(skinny=2))
    o2, _ = run_gpu(con, "bf16x3", A, B, C, tuning=Tuning(skinny=2))
    assert np.array_equal(o1, o2)
    assert "ksplit=1 " not in p.describe(), p.describe()
    with pytest.raises(TccgError):
        Plan(con, "fp32", tuning=Tuning(skinny=2))
    wide = make_contraction("mn", "mk", "kn", dict(m=300, n=400, k=64))
    with pytest.raises(TccgError):
        Plan(wide, "bf16x3", tuning=Tuning(skinny=2))


def test_skinny_tc_grouped_equals_per_item(cuda):
    """A grouped run with tensor-core skinny items (Q packs next to the tile
    items' packs, k-split items reduced with the CUDA-core skinny items')
    equals the per-item runs bit for bit, within the BF16x3 bound."""
    import torch
    from tccg_b200.grouped import Group
    names = ["transpose", "matvec_split", "kfast", "xy", "passes_split", "passes"]
    items = [make_contraction(*_tc_case(n)[:4], 1.0, 0.0) for n in names + sorted(TC_EXTRA)]
    items.append(make_contraction(*CASES["outer"][:4], 1.0, 0.0))  # CUDA-core skinny
    items.append(make_contraction("mn", "mk", "kn", dict(m=700, n=500, k=300), 1.0, 0.0))
    tc = len(items) - 2
    tunings = [Tuning(skinny=2)] * tc + [Tuning(skinny=1), Tuning(variant=16)]
    g = torch.Generator(device="cuda").manual_seed(7)
    As = [torch.randn(c.A0.num_elements(), generator=g, device="cuda") for c in items]
    Bs = [torch.randn(c.B0.num_elements(), generator=g, device="cuda") for c in items]
    Cs = [torch.zeros(c.C0.num_elements(), device="cuda") for c in items]
    grp = Group(items, "bf16x3", tunings=tunings)
    assert sum("skinny_tc" in p.describe() for p in grp.plans) == tc
    grp.bind(As, Bs, Cs)
    grp.capture()
    grp.replay()
    torch.cuda.synchronize()
    grouped = [c.clone() for c in Cs]
    for c in Cs:
        c.zero_()
    grp.run_per_item()
    torch.cuda.synchronize()
    for a, b in zip(grouped, Cs):
        assert torch.equal(a, b)
    for con, A, B, C in zip(items[:tc], As, Bs, grouped):
        ln = LoopNest(con.C0.labels, con.A0.labels, con.B0.labels,
                      {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices})
        ref = ln.run(A.double().cpu().numpy(), B.double().cpu().numpy(), np.zeros(ln.size_c), 1.0, 0.0)
        assert error_metrics(C.double().cpu().numpy(), ref)["normwise"] <= 1e-5, str(con)


@pytest.mark.parametrize("mix", ["both", "rows8_only", "rows16_only"])
def test_register_path_grouped_rows8_and_rows16(cuda, mix):
    """Register-path items (narrow side <= 16), k-split ones among them: a
    plan run of a narrow side of at most 8 takes the 8-row kernel, the
    grouped lane computes 16 rows for every item. Each row's sums are formed
    in the same order either way, so grouped equals the per-item runs bit for
    bit, and both match the FP64 oracle."""
    import torch
    from tccg_b200.grouped import Group
    rows8 = [("cdn", "dnxy", "yxc", dict(c=8, d=23, n=20, x=60, y=41)),       # S 8, K split
             ("ab", "ak", "kb", dict(a=5, b=700, k=90)),                      # S 5
             ("a", "ak", "k", dict(a=300, k=77))]                             # S 1
    rows16 = [("ab", "ak", "kb", dict(a=13, b=900, k=70)),                    # S 13
              ("pqn", "pqk", "kn", dict(p=40, q=30, n=16, k=45))]             # S 16
    shapes = {"both": rows8 + rows16, "rows8_only": rows8, "rows16_only": rows16}[mix]
    items = [make_contraction(lc, la, lb, sz, 0.5, 0.0) for lc, la, lb, sz in shapes]
    grp = Group(items, "fp32", tunings=[Tuning(skinny=1)] * len(items))
    for p in grp.plans:
        assert "path=registers" in p.describe(), p.describe()
    g = torch.Generator(device="cuda").manual_seed(5)
    As = [torch.randn(c.A0.num_elements(), generator=g, device="cuda") for c in items]
    Bs = [torch.randn(c.B0.num_elements(), generator=g, device="cuda") for c in items]
    Cs = [torch.zeros(c.C0.num_elements(), device="cuda") for c in items]
    grp.bind(As, Bs, Cs)
    grp.capture()
    grp.replay()
    torch.cuda.synchronize()
    grouped = [c.clone() for c in Cs]
    for c in Cs:
        c.zero_()
    grp.run_per_item()
    torch.cuda.synchronize()
    for a, b in zip(grouped, Cs):
        assert torch.equal(a, b)
    for con, A, B, C in zip(items, As, Bs, grouped):
        ln = LoopNest(con.C0.labels, con.A0.labels, con.B0.labels,
                      {i.label: i.size for t in (con.A0, con.B0, con.C0) for i in t.indices})
        ref = ln.run(A.double().cpu().numpy(), B.double().cpu().numpy(), np.zeros(ln.size_c), 0.5, 0.0)
        assert error_metrics(C.double().cpu().numpy(), ref)["normwise"] <= 1e-6, str(con)


def test_skinny_choice_and_refusal(cuda):
    from tccg_b200._native import TccgError
    # item 69 of the 256-item batched workload (N = 40, K = 20, 5.0e6 positions, P
    # transposed against C): the library takes the skinny kernel
    from tccg_b200.workloads import batched_workload
    items = batched_workload(256, seed=0)
    con = items[69]
    for precision in ("fp32", "bf16x3"):
        assert "skinny_gett" in Plan(con, precision).describe()
        assert "skinny_gett" not in Plan(con, precision, tuning=Tuning(skinny=-1)).describe()
    # split-BF16x3 with K > 32 and >= 48 blocks: 17-64 rows take the
    # tensor-core kernel (item 6: S = 18), up to 16 the register path (item
    # 46: S = 11); FP32 keeps the CUDA cores
    assert "skinny_tc" in Plan(items[6], "bf16x3").describe()
    assert "skinny_gett" in Plan(items[6], "fp32").describe()
    d = Plan(items[46], "bf16x3").describe()
    assert "skinny_gett" in d and "path=registers" in d, d
    assert "skinny_tc" not in Plan(items[6], "bf16x3", tuning=Tuning(skinny=1)).describe()
    # ... except where the wide operand's stride-one index is contracted and
    # K spans >= 8 chunks (item 48: S = 8, 32 chunks): the tensor-core kernel;
    # FP32 keeps the register path
    assert "skinny_tc" in Plan(items[48], "bf16x3").describe()
    d = Plan(items[48], "fp32").describe()
    assert "path=registers" in d and "load=k" in d, d
    # a square GEMM is not skinny; FP64 and BF16 are not served
    sq = make_contraction("mn", "mk", "kn", dict(m=512, n=512, k=512))
    assert "skinny_gett" not in Plan(sq, "fp32").describe()
    with pytest.raises(TccgError):
        Plan(sq, "fp32", tuning=Tuning(skinny=1))
    with pytest.raises(TccgError):
        Plan(con, "fp64", tuning=Tuning(skinny=1))
    with pytest.raises(TccgError):
        Plan(con, "bf16", tuning=Tuning(skinny=1))
