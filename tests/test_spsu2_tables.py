"""The SPSU2 coefficient tables (spin SU(2) without charge conservation), 1
to 3 channels: the oracle's derivation from the site's Fock space
(oracle/spsu2_derive.py) and the host's plug-in (host/symmetry.h,
SymmetrySPSU2, with host/qs_coupling.cc for two and three channels) against the
reference's tables (coefnew/spsu2/spsu2-<P>ch-*.dat, evaluated into
tests/golden/spsu2_tables*.json by tests/golden/make_spsu2_tables.py):
hopping, anomalous hopping, on-site pairing, site occupancies, <f^dag>
recalculation, doublet and triplet operator tables.

Entries the reference's expressions give for subspaces an NRG run never
forms (an ancestor SS < 1, or an operator that the triangle rule forbids
between the two subspaces) are not compared: the reference's run never
evaluates them either.

Three channels: the doublet-operator rows between combinations 27 and 28
(the site doublet whose channels 0 and 1 couple to spin 0) carry in
spsu2-3ch-doubletp/m.dat the opposite sign of the same rows of every other
three-electron doublet, as the QS tables do for the same multiplet; the
derivation keeps the definition (see tests/test_qs_tables_2ch.py and the
three-channel GPU tests)."""
import json
import os
import shutil
import subprocess

import pytest

import spsu2_derive as SD

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SSMAX = {1: 20, 2: 12, 3: 6}
GOLDEN = {1: "spsu2_tables.json", 2: "spsu2_tables_2ch.json", 3: "spsu2_tables_3ch.json"}
TOL = 1e-12


def _gold(P):
    return json.load(open(os.path.join(ROOT, "tests", "golden", GOLDEN[P])))["tables"]


def _flip(P, name, key):
    """The reference's doublet rows of three-channel combinations 27, 28."""
    return P == 3 and name.startswith("doublet") and key[0] in (27, 28) and key[1] in (27, 28)


class _Offsets(dict):
    """Ancestor SS offset of each (1-based) combination, with the site's SS."""

    def __init__(self, P):
        super().__init__({i + 1: c[2][1] for i, c in enumerate(SD.COMBOS[P])})
        self.site = {i + 1: int(round(2 * c[1])) + 1 for i, c in enumerate(SD.COMBOS[P])}

    def formed(self, ss, i):
        """Combination i exists in subspace ss: its ancestor exists and the
        ancestor's spin and the site's couple to S."""
        a = ss + self[i]
        return ss >= 1 and a >= 1 and _su2(ss, a, self.site[i])


def _in(P):
    return _Offsets(P)


def _su2(a, b, c):
    return abs(a - b) <= c - 1 and abs(b - c) <= a - 1 and abs(c - a) <= b - 1


def _used(IN, ss1, ssp, i1, ip, rank_ss):
    """An entry (i1, ip) between subspaces ss1 and ssp is formed in a run."""
    return IN.formed(ss1, i1) and IN.formed(ssp, ip) and _su2(ss1, ssp, rank_ss)


def _check(got, ref):
    got = {k: v for k, v in got.items() if abs(v) > 1e-13}
    ref = {k: v for k, v in ref.items() if abs(v) > 1e-13}
    assert set(got) == set(ref), sorted(set(got) ^ set(ref))
    for k in ref:
        assert abs(got[k] - ref[k]) <= TOL * max(1.0, abs(ref[k])), (k, got[k], ref[k])
    return len(ref)


def _python_offdiag(P, ss):
    T = SD.tables(P)
    IN = _in(P)
    out = {}
    for kind, rows in ((0, T.offdiag(ss)), (1, T.anomalous(ss)), (2, T.isospinx())):
        for i, j, ch, v in rows:
            if IN.formed(ss, i) and IN.formed(ss, j):
                out[(i, j, ch, kind)] = v
    return out


def _ref_offdiag(P, ss):
    G, IN = _gold(P), _in(P)
    out = {}
    for name, kind in (("offdiag", 0), ("anomalous", 1), ("isospinx", 2)):
        for r in G[name]:
            v = r["factor"][str(ss)]
            if v is not None and IN.formed(ss, r["i"]) and IN.formed(ss, r["j"]):
                out[(r["i"], r["j"], r["ch"], kind)] = v
    return out


@pytest.mark.parametrize("P", [1, 2, 3])
def test_derivation_matches_reference_hamiltonian_tables(P):
    n = 0
    for ss in range(1, SSMAX[P] + 1):
        n += _check(_python_offdiag(P, ss), _ref_offdiag(P, ss))
    assert n > {1: 150, 2: 900, 3: 1500}[P]
    G = _gold(P)
    assert sorted((r["i"], r["ch"], r["number"]) for r in G["diag"]) == sorted(SD.tables(P).diag())
    assert [r["qn"][0] for r in sorted(G["In2"], key=lambda r: r["i"])] == [_in(P)[i] for i in sorted(_in(P))]


@pytest.mark.parametrize("P", [1, 2, 3])
def test_derivation_matches_reference_recalc_tables(P):
    T, G, IN = SD.tables(P), _gold(P), _in(P)
    n = 0
    for ss in range(1, SSMAX[P] + 1):
        for I1, ch, rows in T.recalc_f((0, ss)):
            d = I1[1] - ss
            name = ("spinup" if d == 1 else "spindown") + "abc"[ch]
            ref = {}
            for r in G[name]:
                v = r["factor"][str(ss)]
                if v is not None and IN.formed(I1[1], r["i1"]) and IN.formed(ss, r["ip"]):
                    ref[(r["i1"], r["ip"])] = v
            n += _check({(a, b): v for a, b, v in rows if IN.formed(I1[1], a) and IN.formed(ss, b)}, ref)
        for fn, rank_ss, names in ((T.doublet, 2, {1: "doubletp", -1: "doubletm"}),
                                   (T.triplet, 3, {0: "triplets", 2: "tripletp", -2: "tripletm"})):
            for Ip, rows in fn((0, ss)):
                d = Ip[1] - ss
                ref = {}
                for r in G[names[d]]:
                    v = r["factor"][str(ss)]
                    if v is not None and _used(IN, ss, ss + d, r["i1"], r["ip"], rank_ss):
                        k = (r["i1"], r["ip"])
                        ref[k] = -v if _flip(P, names[d], k) else v
                got = {(a, b): v for a, b, v in rows if _used(IN, ss, Ip[1], a, b, rank_ss)}
                n += _check(got, ref)
    assert n > {1: 400, 2: 1500, 3: 3000}[P]


@pytest.fixture(scope="module")
def dump(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("spsu2") / "spsu2_dump")
    subprocess.run([cxx, "-O1", "-std=c++17", "-o", exe, os.path.join(ROOT, "tests", "spsu2_dump.cc"),
                    os.path.join(ROOT, "nrgljubljana-old_b200", "host", "qs_coupling.cc")], check=True)

    def run(P):
        out = subprocess.run([exe, str(P), str(SSMAX[P])], check=True, capture_output=True, text=True).stdout
        return [json.loads(line) for line in out.splitlines()]
    return run


@pytest.mark.parametrize("P", [1, 2, 3])
def test_plugin_matches_derivation(dump, P):
    T, IN = SD.tables(P), _in(P)
    n = 0
    for rec in dump(P):
        kind = rec["kind"]
        if kind == "diag":
            assert sorted(map(tuple, rec["rows"])) == sorted(T.diag())
            continue
        if kind == "offdiag":
            ss = rec["ss"]
            got = {(i, j, ch, k): v for i, j, ch, v, k in rec["rows"] if IN.formed(ss, i) and IN.formed(ss, j)}
            n += _check(got, _python_offdiag(P, ss))
            continue
        ss = rec["I"][1]
        if kind == "recalc_f":
            got = {(tuple(I1), ch, a, b): v for I1, ch, rs in rec["tables"] for a, b, v in rs
                   if IN.formed(I1[1], a) and IN.formed(ss, b)}
            py = {(tuple(I1), ch, a, b): v for I1, ch, rs in T.recalc_f((0, ss)) for a, b, v in rs
                  if IN.formed(I1[1], a) and IN.formed(ss, b)}
            n += _check(got, py)
            continue
        fn, rank_ss = (T.doublet, 2) if kind == "doublet" else (T.triplet, 3)
        got = {(tuple(Ip), a, b): v for Ip, ch, rs in rec["tables"] for a, b, v in rs
               if _used(IN, ss, Ip[1], a, b, rank_ss)}
        py = {(tuple(Ip), a, b): v for Ip, rs in fn((0, ss)) for a, b, v in rs if _used(IN, ss, Ip[1], a, b, rank_ss)}
        n += _check(got, py)
    assert n > {1: 500, 2: 1500, 3: 3000}[P]
