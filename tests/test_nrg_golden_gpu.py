"""Parity of the GPU NRG run with committed oracle outputs at full size: runs
of the served stream at Nkeep 500, 1000 and 2000 (T = 1e-6, Nmax = 40) and
the two-channel Kondo model at Nmax = 40 with keep 3000 (blocks up to about
8000, three FDM spectra).  The oracle needs minutes to hours per run on host
cores, so tests/golden/make_nrg_goldens.py ran it once and stored its outputs
(tests/golden/nrg/<case>.npz) with the sha256 of the inputs it read; here the
same inputs are generated again, their digest is checked, and the GPU's
outputs are compared at the FP64 targets of nrg_cases.compare_outputs."""
import os

import pytest

import nrg_cases as cases

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nrg")


@pytest.fixture(scope="module")
def ctx():
    import nrgb
    c = nrgb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(cases.GOLDEN_CASES))
def test_nrg_run_matches_oracle_golden(ctx, tmp_path, name):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.fail("golden output missing: " + path)
    ref, digest = cases.load_golden(path)
    wd = cases.make_case(name, str(tmp_path / "in"))
    assert cases.input_digest(wd) == digest, "generated inputs differ from the ones the golden was made from"
    out_g = str(tmp_path / "gpu")
    os.makedirs(out_g)
    ctx.run(wd, out_g)
    cases.compare_outputs(cases.load_outputs(out_g), ref, name, wabs=cases.GOLDEN_CASES[name].get("wabs"))
