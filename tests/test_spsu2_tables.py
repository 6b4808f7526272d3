"""The SPSU2 coefficient tables (spin SU(2) without charge conservation):
the oracle's derivation from the site's Fock space (oracle/spsu2_derive.py)
and the host's plug-in (host/symmetry.h, SymmetrySPSU2) against the
reference's tables (coefnew/spsu2/spsu2-1ch-*.dat, evaluated into
tests/golden/spsu2_tables.json by tests/golden/make_spsu2_tables.py):
hopping, anomalous hopping, on-site pairing, site occupancies, <f^dag>
recalculation, doublet and triplet operator tables.

Entries the reference's expressions give for subspaces an NRG run never
forms (an ancestor SS < 1, or an operator that the triangle rule forbids
between the two subspaces) are not compared: the reference's run never
evaluates them either."""
import json
import math
import os
import shutil
import subprocess

import pytest

import spsu2_derive as SD

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "spsu2_tables.json")))["tables"]
SSMAX = 20
TOL = 1e-12
IN = {1: 0, 2: 0, 3: -1, 4: 1}   # ancestor SS offset of each combination


def _su2(a, b, c):
    return abs(a - b) <= c - 1 and abs(b - c) <= a - 1 and abs(c - a) <= b - 1


def _used(ss1, ssp, i1, ip, rank_ss):
    """An entry (i1, ip) between subspaces ss1 and ssp is formed in a run."""
    a1, ap = ss1 + IN[i1], ssp + IN[ip]
    return ss1 >= 1 and ssp >= 1 and a1 >= 1 and ap >= 1 and _su2(ss1, ssp, rank_ss)


def _ref_rows(name, ss, rank_ss, dss):
    out = {}
    for r in GOLD[name]:
        v = r["factor"][str(ss)]
        if v is None:
            continue
        if _used(ss, ss + dss, r["i1"], r["ip"], rank_ss):
            out[(r["i1"], r["ip"])] = v
    return out


def _check(got, ref):
    got = {k: v for k, v in got.items() if abs(v) > 1e-13}
    ref = {k: v for k, v in ref.items() if abs(v) > 1e-13}
    assert set(got) == set(ref), sorted(set(got) ^ set(ref))
    for k in ref:
        assert abs(got[k] - ref[k]) <= TOL * max(1.0, abs(ref[k])), (k, got[k], ref[k])
    return len(ref)


def _python_tables(ss):
    T = SD.tables()
    off = {}
    for kind, fn in ((0, T.offdiag), (1, T.anomalous)):
        for i, j, ch, v in fn(ss):
            off[(i, j, kind)] = v
    for i, j, ch, v in T.isospinx():
        off[(i, j, 2)] = v
    return off


def _ref_offdiag(ss):
    out = {}
    for name, kind in (("offdiag", 0), ("anomalous", 1), ("isospinx", 2)):
        for r in GOLD[name]:
            v = r["factor"][str(ss)]
            a_i, a_j = ss + IN[r["i"]], ss + IN[r["j"]]
            if v is not None and a_i >= 1 and a_j >= 1:
                out[(r["i"], r["j"], kind)] = v
    return out


def test_derivation_matches_reference_hamiltonian_tables():
    n = 0
    for ss in range(1, SSMAX + 1):
        ref = _ref_offdiag(ss)
        got = {k: v for k, v in _python_tables(ss).items() if ss + IN[k[0]] >= 1 and ss + IN[k[1]] >= 1}
        n += _check(got, ref)
    assert n > 150
    assert sorted((r["i"], r["number"]) for r in GOLD["diag"]) == sorted((i, v) for i, ch, v in SD.tables().diag())
    assert [r["qn"][0] for r in sorted(GOLD["In2"], key=lambda r: r["i"])] == [IN[i] for i in (1, 2, 3, 4)]


def test_derivation_matches_reference_recalc_tables():
    T = SD.tables()
    n = 0
    for ss in range(1, SSMAX + 1):
        for I1, ch, rows in T.recalc_f((0, ss)):
            d = I1[1] - ss
            name = "spinupa" if d == 1 else "spindowna"
            # <f> tables are indexed by the ket subspace ssp = ss
            ref = {}
            for r in GOLD[name]:
                v = r["factor"][str(ss)]
                if v is not None and I1[1] + IN[r["i1"]] >= 1 and ss + IN[r["ip"]] >= 1:
                    ref[(r["i1"], r["ip"])] = v
            n += _check({(a, b): v for a, b, v in rows}, ref)
        for fn, rank_ss, names in ((T.doublet, 2, {1: "doubletp", -1: "doubletm"}),
                                   (T.triplet, 3, {0: "triplets", 2: "tripletp", -2: "tripletm"})):
            for Ip, rows in fn((0, ss)):
                d = Ip[1] - ss
                ref = _ref_rows(names[d], ss, rank_ss, d)
                got = {(a, b): v for a, b, v in rows if _used(ss, Ip[1], a, b, rank_ss)}
                n += _check(got, ref)
    assert n > 400


@pytest.fixture(scope="module")
def dump(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("spsu2") / "spsu2_dump")
    subprocess.run([cxx, "-O1", "-std=c++17", "-o", exe, os.path.join(ROOT, "tests", "spsu2_dump.cc"),
                    os.path.join(ROOT, "nrgljubljana-old_b200", "host", "qs_coupling.cc")], check=True)
    out = subprocess.run([exe, str(SSMAX)], check=True, capture_output=True, text=True).stdout
    return [json.loads(line) for line in out.splitlines()]


def test_plugin_matches_derivation(dump):
    T = SD.tables()
    n = 0
    for rec in dump:
        kind = rec["kind"]
        if kind == "diag":
            assert sorted(map(tuple, rec["rows"])) == sorted(T.diag())
            continue
        if kind == "offdiag":
            ss = rec["ss"]
            got = {(i, j, k): v for i, j, ch, v, k in rec["rows"] if ss + IN[i] >= 1 and ss + IN[j] >= 1}
            py = {k: v for k, v in _python_tables(ss).items() if ss + IN[k[0]] >= 1 and ss + IN[k[1]] >= 1}
            n += _check(got, py)
            continue
        ss = rec["I"][1]
        if kind == "recalc_f":
            got = {(tuple(I1), a, b): v for I1, ch, rs in rec["tables"] for a, b, v in rs
                   if I1[1] + IN[a] >= 1 and ss + IN[b] >= 1}
            py = {(tuple(I1), a, b): v for I1, ch, rs in T.recalc_f((0, ss)) for a, b, v in rs}
            n += _check(got, py)
            continue
        fn, rank_ss = (T.doublet, 2) if kind == "doublet" else (T.triplet, 3)
        got = {(tuple(Ip), a, b): v for Ip, ch, rs in rec["tables"] for a, b, v in rs
               if _used(ss, Ip[1], a, b, rank_ss)}
        py = {(tuple(Ip), a, b): v for Ip, rs in fn((0, ss)) for a, b, v in rs if _used(ss, Ip[1], a, b, rank_ss)}
        n += _check(got, py)
    assert n > 500
