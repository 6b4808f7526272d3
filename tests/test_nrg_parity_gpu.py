"""End-to-end parity of the GPU NRG run (nrgb_run through the C ABI) with the
CPU oracle on the same generated inputs.

The targets are those of the plain FP64 path (nrg_cases.compare_outputs):
td (chi(T) = <Sz^2>, S(T), ...) and the singlet expectation values within
1e-8 relative, energies of the energy flow (annotated.dat) within 1e-10
relative, spectral weights within 1e-8 relative per bin (bins above 1e-6 of
the largest) and within 1e-8 of the largest bin everywhere.  Every case
prints its outputs with 16 significant digits."""
import os

import pytest

import nrg_cases as cases
import nrg_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import nrgb
    c = nrgb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_nrg_run_matches_oracle(ctx, tmp_path, name):
    wd = cases.make_case(name, str(tmp_path / "in"))
    out_o = str(tmp_path / "oracle")
    out_g = str(tmp_path / "gpu")
    os.makedirs(out_g)
    o = O.Oracle(wd)
    o.run(out_o)
    stats = ctx.run(wd, out_g)
    assert stats["launches"] > 0
    cases.compare_outputs(cases.load_outputs(out_g), cases.load_outputs(out_o), name)
