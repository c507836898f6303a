"""The .tccg front end against the reference's own parser, index fusion and
classification (fixtures from tests/golden/make_golden.py), plus the syntax
errors TCCG rejects (tccg/tccg.py:559-684)."""
import json
import os
import warnings

import pytest

from tccg_b200.plan import gett_view
from tccg_b200.spec import (TccgSyntaxError, TccgUnsupported, make_contraction, parse_file,
                            parse_text, to_tccg_text)

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "front_end.json")))


def _summary(c):
    t = lambda T: [[i.label, i.size] for i in T.indices]
    return {"C": t(c.C), "A": t(c.A), "B": t(c.B), "ldC": c.C.ld, "ldA": c.A.ld, "ldB": c.B.ld,
            "alpha": c.alpha, "beta": c.beta, "m": [[i.label, i.size] for i in c.m_indices],
            "n": [[i.label, i.size] for i in c.n_indices], "k": [[i.label, i.size] for i in c.k_indices],
            "loop": [[i.label, i.size] for i in c.loop_indices]}


@pytest.mark.parametrize("name", sorted(FIX))
def test_matches_reference_front_end(name):
    r = FIX[name]["reference"]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        c = parse_text(FIX[name]["text"])
    ref = {"C": r["C"]["indices"], "A": r["A"]["indices"], "B": r["B"]["indices"],
           "ldC": r["C"]["ld"], "ldA": r["A"]["ld"], "ldB": r["B"]["ld"], "alpha": r["alpha"],
           "beta": r["beta"], "m": r["m"], "n": r["n"], "k": r["k"], "loop": r["loop"]}
    assert _summary(c) == ref


@pytest.mark.parametrize("text,err", [
    ("C[a,b] += A[a,k] * B[k,b]\na=2\nb=2\nk=2\n", TccgSyntaxError),
    ("C[a,b] -= A[a,k] * B[k,b]\na=2\nb=2\nk=2\n", TccgSyntaxError),
    ("C[a,b] = A[a,k] * B[k,b] +-C[a,b]\na=2\nb=2\nk=2\n", TccgSyntaxError),
    ("C[a,b] = A[a,k] * B[k,b]\na=2\nb=2\n", TccgSyntaxError),          # size of k missing
    ("C[a,b] = 1 * A[a,k] * B[k,b] + 2 * 3 * C[a,b]\na=2\nb=2\nk=2\n", TccgSyntaxError),
    ("a=2\nb=2\n", TccgSyntaxError),                                      # no tensors
])
def test_syntax_errors(text, err):
    with pytest.raises(err):
        parse_text(text)


def test_missing_file():
    with pytest.raises(TccgSyntaxError):
        parse_file("/nonexistent/file.tccg")


def test_renaming_warns():
    with pytest.warns(UserWarning):
        parse_text("X[a,b] = A[a,k] * B[k,b]\na=2\nb=2\nk=2\n".replace("X", "B"))


def test_loop_indices_rejected_by_gett():
    c = parse_text(FIX["batch"]["text"])
    assert [i.label for i in c.loop_indices] == ["l"]
    with pytest.raises(TccgUnsupported):
        c.validate()


def test_reference_fusion_quirk_is_rejected():
    """The reference's second fusion pass merges (b,l) in C and B but leaves l
    in A (tccg.py:487-519); the result is not a valid contraction and is
    refused instead of computed."""
    c = parse_text(FIX["batch_fused"]["text"])
    assert [i.label for i in c.B.indices] == ["k", "b"] and c.B.indices[1].size == 15
    with pytest.raises(TccgSyntaxError):
        c.validate()


def test_flop_count_tccg_formula():
    c = parse_text("C[a,b,c,d] = A[a,e,b] * B[e,d,c] + C[a,b,c,d]\na=96\nb=96\nc=96\nd=96\ne=16\n")
    M = N = 96 * 96
    assert c.flop_count() == 2.0 * M * N * 16 + 3.0 * M * N
    assert c.flop_count(beta=0.0) == 2.0 * M * N * 16


def test_round_trip_text():
    c = parse_text("C[a,b,i,j] = 2.5 * A[i,m,a] * B[m,j,b] + 0.5 * C[a,b,i,j]\na=3\nb=4\ni=5\nj=6\nm=7\n")
    c2 = parse_text(to_tccg_text(c))
    assert _summary(c) == _summary(c2)


def test_gett_view_configurations():
    v = gett_view(parse_text(FIX["cfg3"]["text"]))
    assert (v.M, v.N, v.K) == (32768, 32768, 4096)
    assert not v.swap_ab and [l for l, _ in v.m] == ["a", "b", "c"] and [l for l, _ in v.k] == ["m", "n"]
    assert v.a_m == [1, 2048, 4194304] and v.c_m == [1, 32, 1024]
    v = gett_view(parse_text(FIX["swap"]["text"]))
    assert v.swap_ab and [l for l, _ in v.m] == ["p", "r"] and [l for l, _ in v.n] == ["q"]
    # K order follows the operand whose stride-one index is contracted
    v = gett_view(parse_text(FIX["cfg4"]["text"]))
    assert [l for l, _ in v.k] == ["k0", "k1"] and v.a_k == [1, 2048]


def test_gett_view_dummy_modes():
    v = gett_view(make_contraction("a", "ak", "k", dict(a=5, k=3)))
    assert v.N == 1 and v.b_n == [0]
    v = gett_view(make_contraction("ab", "a", "b", dict(a=5, b=3)))
    assert v.K == 1 and v.a_k == [0]
