"""The QSZ plug-in's tables (host/symmetry.h, SymmetryQSZ: every
combination one Fock state of the added site) against the reference's
(coefnew/qsz/qsz-<P>ch-*.dat, evaluated into tests/golden/qsz_tables.json by
tests/golden/make_qsz_tables.py), for 1 to 3 channels: the combinations'
quantum numbers, hopping, site occupancies, the <f^dag> recalculation of
both spins and channels, and the doublet recalculation.  The plug-in is
compiled with the host compiler into a small dump program (no device)."""
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "qsz_tables.json")))


@pytest.fixture(scope="module")
def dump(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("qsz") / "qsz_dump")
    subprocess.run([cxx, "-O1", "-std=c++17", "-o", exe, os.path.join(ROOT, "tests", "qsz_dump.cc"),
                    os.path.join(ROOT, "nrgljubljana-old_b200", "host", "qs_coupling.cc")], check=True)

    def run(P):
        out = subprocess.run([exe, str(P)], check=True, capture_output=True, text=True).stdout
        return {rec["kind"]: rec for rec in map(json.loads, out.splitlines())}
    return run


@pytest.mark.parametrize("P", [1, 2, 3])
def test_qsz_plugin_matches_reference_tables(dump, P):
    G, D = GOLD[str(P)], dump(P)
    assert sorted(map(tuple, D["In"]["rows"])) == sorted(map(tuple, G["In2"]))
    assert sorted(map(tuple, D["QN"]["rows"])) == sorted(map(tuple, G["QN"]))
    assert sorted(map(tuple, D["offdiag"]["rows"])) == sorted(map(tuple, G["offdiag"]))
    assert sorted(map(tuple, D["diag"]["rows"])) == sorted(map(tuple, G["diag"]))
    # <f^dag>: I1 = Ip + (1, +1) (spin up) and Ip + (1, -1) (spin down), per channel
    got = {}
    for I1, ch, rows in D["recalc_f"]["tables"]:
        name = ("spinup" if I1[1] == 1 else "spindown") + "abc"[ch]
        got[name] = sorted(map(tuple, rows))
    for name in got:
        assert got[name] == sorted(map(tuple, G[name])), name
    assert len(got) == 2 * P
    # doublets: Ip = I1 + (-1, 1) (doubletp: the ancestors of the reference's
    # rows differ by (-1, +1)) and I1 + (-1, -1) (doubletm)
    for Ip, ch, rows in D["doublet"]["tables"]:
        name = "doubletp" if Ip[1] == 1 else "doubletm"
        assert sorted(map(tuple, rows)) == sorted((r[0], r[1], r[4]) for r in G[name]), name
