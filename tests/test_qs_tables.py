"""The QS coefficient tables restated in oracle/qs.py agree with the
reference's coefnew/qs/qs-1ch-*.dat (evaluated into tests/golden/qs_tables.json
by tests/golden/make_qs_tables.py)."""
import json
import math
import os

import pytest

import qs

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "qs_tables.json")))
T = GOLD["tables"]


def _close(a, b):
    if b is None:
        return True  # reference value not finite: row never used for that ss
    return abs(a - b) <= 1e-13 * max(1.0, abs(b))


def test_in_qn():
    assert [tuple(r["qn"]) for r in sorted(T["In2"], key=lambda r: r["i"])] == qs.IN[1]
    assert [tuple(r["qn"]) for r in sorted(T["QN"], key=lambda r: r["i"])] == qs.QN[1]


@pytest.mark.parametrize("ss", range(1, 41))
def test_offdiag(ss):
    mine = qs.offdiag_terms(1, ss)
    assert len(mine) == len(T["offdiag"])
    for (i, j, ch, f), r in zip(mine, T["offdiag"]):
        assert (i, j, ch) == (r["i"], r["j"], r["ch"])
        assert _close(f, r["factor"][str(ss)])


def test_diag():
    assert [(i, ch, float(n)) for i, ch, n in qs.diag_terms(1)] == \
        [(r["i"], r["ch"], r["number"]) for r in T["diag"]]


@pytest.mark.parametrize("ss", range(2, 41))
def test_recalc_f(ss):
    tabs = qs.recalc_f_tables(1, (0, ss))
    up, down = tabs[0][2], tabs[1][2]
    for mine, ref in ((up, T["spinupa"]), (down, T["spindowna"])):
        for (i1, ip, f), r in zip(mine, ref):
            assert (i1, ip) == (r["i1"], r["ip"])
            assert _close(f, r["factor"][str(ss)])


@pytest.mark.parametrize("ss", range(1, 41))
@pytest.mark.parametrize("kind", ["d", "t"])
def test_recalc_tables(ss, kind):
    if kind == "d":
        tabs = qs.doublet_tables(1, (0, ss))
        refs = [T["doubletp"], T["doubletm"]]
    else:
        tabs = qs.triplet_tables(1, (0, ss))
        refs = [T["triplets"], T["tripletp"], T["tripletm"]]
    for (Ip, rows), ref in zip(tabs, refs):
        assert len(rows) == len(ref)
        for (i1, ip, f), r in zip(rows, ref):
            assert (i1, ip) == (r["i1"], r["ip"])
            # the ancestor subspaces implied by In[] match the table's IN1/INp
            I1 = (0, 10)
            Ip10 = (Ip[0], Ip[1] - ss + 10)
            assert list(qs.combine(qs.IN[1][i1 - 1], I1)) == r["IN1_at_q0_ss10"]
            assert list(qs.combine(qs.IN[1][ip - 1], Ip10)) == r["INp_at_q0_ss10"]
            if not math.isnan(f):
                assert _close(f, r["factor"][str(ss)])
