"""Transformation files and restart (src/dmnrg.h:183-304, src/nrg.cc:
2891-2895, 3512-3524): with removefiles=false a run writes every step's
eigen-decompositions to <workdir>/unitary<N>; with resume=true a later run
loads the steps that have a file instead of diagonalising and computes the
rest.  A run resumed from a partial set of files reproduces the original
outputs at the FP64 targets."""
import glob
import os

import pytest

import nrg_cases as cases

pytestmark = pytest.mark.gpu


def test_resume_from_transformation_files(tmp_path):
    import nrgb
    wd = cases.make_case("siam_ph", str(tmp_path / "in"))
    with open(os.path.join(wd, "param"), "a") as fh:
        fh.write("removefiles=false\n")
    out1, out2 = str(tmp_path / "first"), str(tmp_path / "resumed")
    os.makedirs(out1)
    os.makedirs(out2)
    ctx = nrgb.Context(0)
    try:
        s1 = ctx.run(wd, out1)
        files = sorted(glob.glob(os.path.join(wd, "unitary*")), key=lambda f: int(f.rsplit("unitary", 1)[1]))
        nmax = len(cases.read_table(os.path.join(out1, "td"))) - 1  # td has the calc0 row
        assert len(files) == nmax
        # the last four steps lost: they are diagonalised again
        for f in files[-4:]:
            os.remove(f)
        with open(os.path.join(wd, "param"), "a") as fh:
            fh.write("resume=true\n")
        s2 = ctx.run(wd, out2)
    finally:
        ctx.close()
    # the resumed run diagonalised only the steps without a file
    assert s2["diag_s"] < s1["diag_s"] or s2["launches"] < s1["launches"]
    cases.compare_outputs(cases.load_outputs(out2), cases.load_outputs(out1), "resumed")
