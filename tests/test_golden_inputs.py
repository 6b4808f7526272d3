"""The committed oracle outputs under tests/golden/nrg were made from inputs
that inputgen.py generates again at test time.  Regenerate every case's
inputs here (no GPU) and check the sha256 stored with the outputs, and that
each file holds the outputs the GPU comparison reads."""
import os

import pytest

import nrg_cases as cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nrg")


@pytest.mark.parametrize("name", sorted(cases.GOLDEN_CASES))
def test_golden_inputs_regenerate(tmp_path, name):
    path = os.path.join(GOLDEN, name + ".npz")
    assert os.path.exists(path), "golden output missing: " + path
    ref, digest = cases.load_golden(path)
    wd = cases.make_case(name, str(tmp_path / "in"))
    assert cases.input_digest(wd) == digest
    assert "td" in ref and len(ref["td"]) > 0
    assert len(ref["bins"]) > 0 and len(ref["annotated"]) > 0
