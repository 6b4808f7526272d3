"""The precision workload in split-precision form: SIAM (U = 0.5,
eps_d = -0.25, Gamma = 0.04, Lambda = 2, Nmax = 40, keep 2000, FDM A(omega)
at T = 1e-7) with the recalculation, density-matrix and spectral products as
INT8-slice tensor-core products (gemm_slices = 8), against the committed
FP64 oracle outputs of the same inputs (tests/golden/nrg/siam_c4.npz).  The
eigensolver, the Boltzmann and density-matrix weights stay FP64.  Targets:
td (chi(T), S(T)) and the spectral weights per bin within 1e-8 relative;
the largest relative errors of eigenvalues, chi(T), S(T) and A(omega) are
printed."""
import json
import os

import pytest

import nrg_cases as cases

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nrg", "siam_c4.npz")


@pytest.mark.parametrize("slices", [8, 7])
def test_split_precision_run_against_the_fp64_oracle(tmp_path, slices):
    import nrgb
    if not os.path.exists(GOLDEN):
        pytest.fail("golden output missing: " + GOLDEN)
    ref, digest = cases.load_golden(GOLDEN)
    wd = cases.make_case("siam_c4", str(tmp_path / "in"))
    assert cases.input_digest(wd) == digest
    with open(os.path.join(wd, "param"), "a") as fh:
        fh.write("gemm_slices=%d\n" % slices)
    out = str(tmp_path / "split")
    os.makedirs(out)
    ctx = nrgb.Context(0)
    try:
        ctx.run(wd, out)
    finally:
        ctx.close()
    got = cases.load_outputs(out)
    rep = cases.error_report(got, ref)
    print("split precision, %d slices, max rel err vs FP64 oracle: %s" % (slices, json.dumps(rep)))
    assert rep["chi_T"] <= 1e-8 and rep["S_T"] <= 1e-8
    assert rep["spectra_per_bin"] <= 1e-8
    assert rep["energies"] <= 1e-8
