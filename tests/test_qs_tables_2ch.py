"""The QS coefficient tables derived from spin coupling (oracle/qs_derive.py)
agree with the reference's coefnew/qs/qs-1ch-*.dat, qs-2ch-*.dat and
qs-3ch-*.dat (evaluated into tests/golden/qs_tables.json, qs_tables_2ch.json,
qs_tables_3ch.json by tests/golden/make_qs_tables.py; three channels for SS
up to 14).

A reference row may be missing from the derivation only where it multiplies
an empty block: its ancestor subspace does not exist (SS < 1), the site spin
cannot couple the ancestor to the subspace, or the operator's rank cannot
connect the two spins.  Every derived row must be in the reference."""
import json
import os

import pytest

import qs_derive as QD

HERE = os.path.join(os.path.dirname(__file__), "golden")
GOLD = {1: json.load(open(os.path.join(HERE, "qs_tables.json")))["tables"],
        2: json.load(open(os.path.join(HERE, "qs_tables_2ch.json")))["tables"],
        3: json.load(open(os.path.join(HERE, "qs_tables_3ch.json")))["tables"]}
# (P, ss) cases: SS 1..30 for one and two channels, 1..13 for three
CASES = [(P, ss) for P in (1, 2) for ss in range(1, 31)] + [(3, ss) for ss in range(1, 14)]
TOL = 1e-12


def _exists(T, i, I):
    """Combination i (0-based) is a non-empty block of subspace I."""
    A = T.anc(i, I)
    return A[1] >= 1 and T._state(i, (I[1] - 1) / 2.0, (I[1] - 1) / 2.0) is not None


def _compare(mine, ref, empty):
    for k, v in mine.items():
        assert k in ref and ref[k] is not None, ("derived row not in the reference", k, v)
        assert abs(v - ref[k]) <= TOL * max(1.0, abs(ref[k])), (k, v, ref[k])
    for k, v in ref.items():
        if k not in mine and v is not None and abs(v) > TOL:
            assert empty(k), ("reference row missing from the derivation", k, v)


@pytest.mark.parametrize("P", [1, 2, 3])
def test_in_qn(P):
    T = GOLD[P]
    assert [tuple(r["qn"]) for r in sorted(T["In2"], key=lambda r: r["i"])] == [c[2] for c in QD.COMBOS[P]]
    qn = [(sum(c[0]) - P, int(round(2 * c[1])) + 1) for c in QD.COMBOS[P]]
    assert [tuple(r["qn"]) for r in sorted(T["QN"], key=lambda r: r["i"])] == qn


@pytest.mark.parametrize("P", [1, 2, 3])
def test_diag(P):
    assert sorted(QD.tables(P).diag()) == sorted((r["i"], r["ch"], r["number"]) for r in GOLD[P]["diag"])


@pytest.mark.parametrize("P,ss", CASES)
def test_offdiag(P, ss):
    T = QD.tables(P)
    I = (0, ss)
    mine = {(i, j, ch): v for i, j, ch, v in QD.offdiag(P, ss)}
    ref = {(r["i"], r["j"], r["ch"]): r["factor"][str(ss)] for r in GOLD[P]["offdiag"]}
    _compare(mine, ref, lambda k: not (_exists(T, k[0] - 1, I) and _exists(T, k[1] - 1, I)))


@pytest.mark.parametrize("P,ssp", CASES)
def test_recalc_f(P, ssp):
    T = QD.tables(P)
    Ip = (0, ssp)
    got = {(I1, ch): rows for I1, ch, rows in QD.recalc_f(P, Ip)}
    names = [("spinup" + "abc"[ch], 1, ch) for ch in range(P)] + [("spindown" + "abc"[ch], -1, ch) for ch in range(P)]
    for name, dss, ch in names:
        I1 = (1, ssp + dss)
        if I1[1] < 1:
            continue
        mine = {(a, b): v for a, b, v in got.get((I1, ch), [])}
        ref = {(r["i1"], r["ip"]): r["factor"][str(ssp)] for r in GOLD[P][name]}
        _compare(mine, ref, lambda k: not (_exists(T, k[0] - 1, I1) and _exists(T, k[1] - 1, Ip)))


@pytest.mark.parametrize("P,ss1", CASES)
def test_chain_operator_tables(P, ss1):
    T = QD.tables(P)
    I1 = (0, ss1)
    d = {Ip: rows for Ip, rows in QD.doublet(P, I1)}
    t = {Ip: rows for Ip, rows in QD.triplet(P, I1)}
    for name, Ip, src, rank in (("doubletp", (-1, ss1 + 1), d, 1), ("doubletm", (-1, ss1 - 1), d, 1),
                                ("triplets", (0, ss1), t, 2), ("tripletp", (0, ss1 + 2), t, 2),
                                ("tripletm", (0, ss1 - 2), t, 2)):
        if Ip[1] < 1:
            continue
        mine = {(a, b): v for a, b, v in src.get(Ip, [])}
        ref = {(r["i1"], r["ip"]): r["factor"][str(ss1)] for r in GOLD[P][name]}
        if P == 3 and rank == 1:
            # qs-3ch-doubletp/m.dat rows between combinations 29 and 30 (the
            # site doublet whose channels 0 and 1 couple to spin 0) carry the
            # opposite sign of the same rows of every other three-electron
            # doublet (23/24, 33/34, ...), although the site part is the
            # identity and the chain operator passes three site electrons in
            # each; the derivation keeps the definition, and the three-channel
            # GPU test checks the doublet spectra against the QSZ plug-in
            ref = {k: (-v if v is not None and k[0] in (29, 30) and k[1] in (29, 30) else v)
                   for k, v in ref.items()}
        # the operator's rank cannot connect the two spins: every block is empty
        forbidden = not (abs(ss1 - Ip[1]) <= rank <= ss1 + Ip[1] - 2)
        _compare(mine, ref, lambda k: forbidden or not (_exists(T, k[0] - 1, I1) and _exists(T, k[1] - 1, Ip)))


def test_three_channel_doublet_row_sign_matters(tmp_path):
    """The sign of the reference's doublet rows between three-channel
    combinations 29 and 30 (which the derivation does not follow) is not
    immaterial: the oracle's f spectrum of a three-channel Kondo run changes
    when those rows take the reference's sign, while the derived sign
    reproduces the QSZ plug-in on the GPU (tests/test_qsz_gpu.py)."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "nrgljubljana-old_b200"))
    import inputgen
    import nrg_cases as cases
    import nrg_oracle as O
    params = {"keep": 80, "keepenergy": 2.5, "keepmin": 1, "T": 1e-2, "fdm": True, "dmnrg": False,
              "specd": "A_f0-A_f0", "bins": 20, "savebins": True, "broaden": False}
    wd = str(tmp_path / "in")
    inputgen.make_kondo(wd, [0.3, 0.2, 0.1], 3.0, 2, symtype="QS", params=params)
    spectra = []
    derived = QD.doublet
    try:
        for flip in (False, True):
            QD.doublet.cache_clear()
            if flip:
                def reference_sign(P, I1, _d=derived.__wrapped__):
                    return [(Ip, [(a, b, -v if a in (29, 30) and b in (29, 30) else v) for a, b, v in rows])
                            for Ip, rows in _d(P, I1)]
                QD.doublet = reference_sign
            od = str(tmp_path / ("out%d" % flip))
            os.makedirs(od)
            O.Oracle(wd).run(od)
            b = cases.read_bins(os.path.join(od, "spec_FDM_dens_A_f0-A_f0.bin"))
            spectra.append(dict(zip(b[:, 0], b[:, 1])))
    finally:
        QD.doublet = derived
        QD.doublet.cache_clear()
    a, b = spectra
    assert abs(sum(a.values()) - 1.0) < 1e-9 and abs(sum(b.values()) - 1.0) < 1e-9
    wmax = max(abs(v) for v in a.values())
    assert max(abs(a.get(k, 0.0) - b.get(k, 0.0)) for k in set(a) | set(b)) > 1e-2 * wmax
