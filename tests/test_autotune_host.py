"""Host side of the autotuner (no GPU): the candidate lists it times and the
SQLite cache it keeps (TCCG's tuning DB, sql_util.py:206-306, looked up as in
tccg.py:192-221). Candidates must be distinct, valid for the precision and
ordered with the library's own choice (or the k-split nearest to filling the
GPU) first; a cached tuning must come back with every field; cache keys must
separate what changes the winner (extents, precision, operand type, beta,
GPU, library version)."""
import dataclasses

import pytest

from tccg_b200.autotune import CODE_VERSION, TuningDB, candidates, tuning_key
from tccg_b200.plan import Tuning
from tccg_b200.spec import make_contraction

SHAPES = {
    # configuration 1 (K = 48), configuration 2 (K = 16, beta = 1), few C
    # tiles with a long K, and a large square GEMM
    "cfg1": ("abij", "ima", "mjb", dict(a=48, b=48, i=48, j=48, m=48), 0.0),
    "cfg2": ("abcd", "aeb", "edc", dict(a=96, b=96, c=96, d=96, e=16), 1.0),
    "few_tiles": ("mn", "mk", "kn", dict(m=100, n=100, k=5000), 0.0),
    "square": ("mn", "mk", "kn", dict(m=8192, n=8192, k=1024), 0.0),
}
PRECISIONS = ["fp32", "fp64", "bf16x3", "bf16"]


def _con(name):
    lc, la, lb, sizes, beta = SHAPES[name]
    return make_contraction(lc, la, lb, sizes, 1.0, beta)


@pytest.mark.parametrize("name", sorted(SHAPES))
@pytest.mark.parametrize("precision", PRECISIONS)
def test_candidates_distinct_and_valid(name, precision):
    con = _con(name)
    cs = candidates(con, precision)
    keys = [t.key() for t in cs]
    assert len(keys) == len(set(keys)), keys
    assert {t.method for t in cs} == {"gett", "ttgt"}
    for t in cs:
        if precision in ("fp32", "fp64"):
            # the CUDA-core precisions have no tensor-core choices
            assert t.variant == 0 and t.raster == 0 and t.tail_split == 0 and t.pair == 0
            assert t.ksplit >= 0  # 0: the automatic split (the tile-shape candidates)
        if precision == "fp64":
            assert t.simt_tile == 0  # FP64 keeps its one tile shape
        if t.shortk != 0:  # short-K kernel only where it applies
            assert con.sizeK <= (16 if precision == "fp64" else 32)


@pytest.mark.parametrize("precision", ["bf16x3", "bf16"])
def test_bf16_candidates_start_with_the_library_choice(precision):
    for name in SHAPES:
        cs = candidates(_con(name), precision, methods=("gett",))
        assert cs[0] == Tuning(method="gett")
        # both kernel families and the tail split switched off are searched
        assert any(t.variant < 0 for t in cs) and any(t.variant > 0 or t.load > 0 for t in cs)
        assert any(t.tail_split == -1 for t in cs)
        # both tile orders (TCCG's two loop orders) and other tile widths
        assert any(t.raster < 0 for t in cs) and any(t.raster > 0 for t in cs)
        assert {t.tile_n for t in cs} >= ({0, 128} if precision == "bf16x3" else {0, 128, 192})


def test_split_bf16x3_searches_both_loaders_first():
    """BF16x3 with FP32 operands: right after the library's own choice (and
    the skinny kernel where it applies), the packed 128x192 tiles (load 1),
    the gathered 128x128 tiles (load 2) and the CUDA cores, so that
    --maxImplementations=5 already compares them."""
    for name in SHAPES:
        cs = candidates(_con(name), "bf16x3", methods=("gett",))
        con = _con(name)
        sk = int(min(con.sizeM, con.sizeN) <= 256)
        assert [t.skinny for t in cs[:1 + sk]] == [0] + [1] * sk
        assert [(t.load, t.variant) for t in cs[sk:4 + sk]] == [(0, 0), (1, 0), (2, 0), (0, -1)]
    # not for TTGT (its GEMM reads the transposed operands) nor BF16 operands
    cs = candidates(_con("square"), "bf16x3", methods=("ttgt",))
    assert all(t.load == 0 for t in cs)
    assert all(t.load == 0 for t in candidates(_con("square"), "bf16", dtype="bf16"))


def test_mode_order_candidates_change_the_view():
    """The N/K mode-order candidates are kept only where they give another
    GETT view (configuration 4's pattern has two K modes led by either
    operand)."""
    from tccg_b200.autotune import order_variants
    from tccg_b200.plan import gett_view
    con = make_contraction("xyzw", "pxqw", "qzpy", dict(x=64, w=64, y=64, z=64, p=32, q=32))
    orders = order_variants(con)
    assert orders[0] == (0, 0) and len(orders) >= 2
    views = {(tuple(v.m), tuple(v.n), tuple(v.k))
             for v in (gett_view(con, n_order=a, k_order=b) for a, b in orders)}
    assert len(views) == len(orders)
    cs = candidates(con, "bf16x3", methods=("gett",))
    assert {(t.n_order, t.k_order) for t in cs} >= set(orders)


def test_tensor_core_skinny_candidate():
    """The tensor-core skinny kernel (skinny = 2) is searched for split-BF16x3
    with a narrow side of at most 256, right after the kernel families
    (grouped items too); not for other precisions."""
    con = make_contraction("ab", "akl", "lkb", dict(a=900, b=24, k=40, l=30))
    cs = candidates(con, "bf16x3", methods=("gett",))
    i = [t.skinny for t in cs].index(2)
    assert [(t.load, t.variant) for t in cs[2:5]] == [(1, 0), (2, 0), (0, -1)] and i == 5
    assert any(t.skinny == 2 for t in candidates(con, "bf16x3", grouped=True))
    assert all(t.skinny != 2 for t in candidates(con, "fp32"))
    wide = make_contraction("ab", "ak", "kb", dict(a=900, b=300, k=64))
    assert all(t.skinny != 2 for t in candidates(wide, "bf16x3"))


def test_grouped_candidates():
    """Items of a grouped launch: GETT only and never the tail split."""
    for name in SHAPES:
        for prec in PRECISIONS:
            cs = candidates(_con(name), prec, grouped=True)
            assert cs and all(t.method == "gett" for t in cs)
            if prec in ("bf16", "bf16x3"):
                assert all(t.tail_split == -1 for t in cs)


def test_ksplit_candidates_follow_the_tile_count():
    # many C tiles: no explicit k-split (0 = automatic on the tile-shape
    # candidates); few tiles and a long K: the split nearest to two CTAs per
    # SM first
    assert {t.ksplit for t in candidates(_con("square"), "fp32")} == {0, 1}
    few = candidates(_con("few_tiles"), "fp32", methods=("gett",), num_sms=148)
    assert few[0].ksplit == 16 and {1, 2, 4, 8, 16} <= {t.ksplit for t in few}


def test_short_k_candidates():
    cfg2 = candidates(_con("cfg2"), "fp32", methods=("gett",))
    assert {t.shortk for t in cfg2} == {0, 1, -1}
    cfg1 = candidates(_con("cfg1"), "fp64", methods=("gett",))  # K = 48 > 16
    assert {t.shortk for t in cfg1} == {0}


def test_tuning_db_round_trip(tmp_path):
    db = TuningDB(str(tmp_path / "tuning.db"))
    con = _con("cfg2")
    key = tuning_key(con, "bf16x3", "f32", "B200/sm100/148SM")
    assert db.lookup(key) is None
    t = Tuning(method="ttgt", ksplit=3, raster=4, max_ctas=100, variant=-1, pair=1, direct=-1,
               shortk=1, simt_tile=2, tail_split=-1)
    db.record(key, t, 0.25, 1000.0)
    db.record(key, Tuning(), 0.5, 500.0)
    assert len(db.measurements(key)) == 2
    db.store_best(key, Tuning(), 0.5, 500.0)
    db.store_best(key, t, 0.25, 1000.0)  # replaces the earlier best
    got, gflops = db.lookup(key)
    assert got == t and dataclasses.asdict(got) == dataclasses.asdict(t)
    assert gflops == 1000.0
    # a second connection to the same file sees it (the cache persists)
    again = TuningDB(str(tmp_path / "tuning.db")).lookup(key)
    assert again is not None and again[0] == t


def test_tuning_keys_separate_what_changes_the_winner():
    gpu = "B200/sm100/148SM"
    base = tuning_key(_con("cfg2"), "fp32", "f32", gpu)
    assert CODE_VERSION in base
    lc, la, lb, sizes, _ = SHAPES["cfg2"]
    other = {
        "precision": tuning_key(_con("cfg2"), "bf16x3", "f32", gpu),
        "dtype": tuning_key(_con("cfg2"), "fp32", "bf16", gpu),
        "beta": tuning_key(make_contraction(lc, la, lb, sizes, 1.0, 0.0), "fp32", "f32", gpu),
        "gpu": tuning_key(_con("cfg2"), "fp32", "f32", "B200/sm100/132SM"),
        "extents": tuning_key(make_contraction(lc, la, lb, dict(sizes, e=32), 1.0, 1.0), "fp32",
                              "f32", gpu),
    }
    for what, k in other.items():
        assert k != base, what
    # alpha and the value of a nonzero beta do not change the kernels
    assert tuning_key(make_contraction(lc, la, lb, sizes, 2.0, -3.0), "fp32", "f32", gpu) == base
