"""The host's C++ derivation of the QS tables (host/qs_coupling.cc, used by
the GPU path) agrees entry by entry with the oracle's Python derivation
(oracle/qs_derive.py), which tests/test_qs_tables*.py check against the
reference's tables: diagonal and off-diagonal Hamiltonian terms, <f>
recalculation, doublet and triplet operator tables, 1, 2 and 3 channels.

tests/qs_coupling_dump.cc prints the C++ tables; it is compiled here with
the host compiler (no device needed)."""
import json
import os
import shutil
import subprocess

import pytest

import qs_derive as QD

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SSMAX = 8
TOL = 1e-12


@pytest.fixture(scope="module")
def dump(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("qsd") / "qs_coupling_dump")
    subprocess.run([cxx, "-O1", "-std=c++17", "-o", exe, os.path.join(ROOT, "tests", "qs_coupling_dump.cc"),
                    os.path.join(ROOT, "nrgljubljana-old_b200", "host", "qs_coupling.cc")], check=True)

    def run(P):
        out = subprocess.run([exe, str(P), str(SSMAX)], check=True, capture_output=True, text=True).stdout
        return [json.loads(line) for line in out.splitlines()]
    return run


def _same(cpp, py):
    """Two {key: value} maps agree: same keys (entries above 1e-13) and values."""
    a = {k: v for k, v in cpp.items() if abs(v) > 1e-13}
    b = {k: v for k, v in py.items() if abs(v) > 1e-13}
    assert set(a) == set(b), (sorted(set(a) ^ set(b)))
    for k in a:
        assert abs(a[k] - b[k]) <= TOL * max(1.0, abs(b[k])), (k, a[k], b[k])
    return len(a)


@pytest.mark.parametrize("P", [1, 2, 3])
def test_cpp_tables_match_python_derivation(dump, P):
    n = 0
    for rec in dump(P):
        kind = rec["kind"]
        if kind == "diag":
            n += _same({(i, ch): v for i, ch, v in rec["rows"]},
                       {(i, ch): v for i, ch, v in QD.tables(P).diag()})
        elif kind == "offdiag":
            n += _same({(i, j, ch): v for i, j, ch, v in rec["rows"]},
                       {(i, j, ch): v for i, j, ch, v in QD.offdiag(P, rec["ss"])})
        else:
            I = tuple(rec["I"])
            cpp = {(tuple(inv), ch, i1, ip): v for inv, ch, rows in rec["tables"] for i1, ip, v in rows}
            if kind == "recalc_f":
                py = {(tuple(I1), ch, i1, ip): v for I1, ch, rows in QD.recalc_f(P, I) for i1, ip, v in rows}
            else:
                fn = QD.doublet if kind == "doublet" else QD.triplet
                py = {(tuple(Ip), 0, i1, ip): v for Ip, rows in fn(P, I) for i1, ip, v in rows}
                cpp = {(k[0], 0, k[2], k[3]): v for k, v in cpp.items()}
            n += _same(cpp, py)
    assert n > {1: 300, 2: 3000, 3: 15000}[P]
