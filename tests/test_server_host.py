"""Host side of the run server (no device needed): the memory projection
used for admission, and the refusals of the C ABI without a GPU."""
import os

import pytest

import inputgen


def _run(root, keep, Nmax, fdm=True, z=1.0):
    wd = os.path.join(root, "k%d_n%d_%d" % (keep, Nmax, fdm))
    inputgen.make_siam(wd, 0.2, -0.1, 0.02, 2.0, Nmax, z=z,
                       params={"keep": keep, "fdm": fdm, "dmnrg": not fdm, "T": 1e-5, "specd": "A_d-A_d"})
    return wd


def test_projection_grows_with_keep_and_chain_length(tmp_path):
    import nrgb
    p = {k: nrgb.project_bytes(_run(str(tmp_path), k, 20)) for k in (100, 200, 400)}
    assert p[100] < p[200] < p[400]
    # eigenvectors of every step are held: each step adds D^2 + D doubles
    # (D = 4 (keep + safeguardmax) bounds the block dimensions) and two
    # K'^2 density matrices with FDM
    p40 = nrgb.project_bytes(_run(str(tmp_path), 200, 40))
    kp = 200 + 200
    dim = 4 * kp
    assert p40 - p[200] == pytest.approx(8.0 * 20 * (dim * dim + dim + 2 * kp * kp), rel=1e-12)
    assert p[200] >= 8.0 * 20 * dim * dim


def test_projection_of_two_channel_runs(tmp_path):
    """Two channels: 16 combinations per subspace, so the block dimension bound
    is D = 16 (keep + safeguardmax); each extra step adds D^2 + D doubles of
    eigenvectors and, with FDM, two K'^2 density matrices."""
    import nrgb
    p = {}
    for nmax in (8, 12):
        wd = os.path.join(str(tmp_path), "kondo2_%d" % nmax)
        inputgen.make_kondo(wd, [0.2, 0.2], 3.0, nmax, params={"keep": 300, "fdm": True, "T": 1e-3})
        p[nmax] = nrgb.project_bytes(wd)
    kp = 300 + 200
    dim = 16 * kp
    assert p[12] - p[8] == pytest.approx(8.0 * 4 * (dim * dim + dim + 2 * kp * kp), rel=1e-12)
    # one channel with the same keep and chain length needs far less
    one = nrgb.project_bytes(_run(str(tmp_path), 300, 12))
    assert p[12] > 10 * one


def test_projection_rejects_missing_input(tmp_path):
    import nrgb
    with pytest.raises(RuntimeError):
        nrgb.project_bytes(str(tmp_path / "nothing"))


@pytest.mark.parametrize("damage", ["half", "five_lines", "empty", "garbage_line"])
def test_damaged_data_is_refused(tmp_path, damage):
    """A truncated or corrupted data file is refused with an error status
    (the host reader checks every read), never a crash or a partial result."""
    import nrgb
    wd = _run(str(tmp_path), 100, 10)
    lines = open(os.path.join(wd, "data")).read().splitlines(True)
    txt = {"half": "".join(lines[:len(lines) // 2]), "five_lines": "".join(lines[:5]), "empty": "",
           "garbage_line": "".join(lines[:3]) + "xyz abc\n" + "".join(lines[4:])}[damage]
    open(os.path.join(wd, "data"), "w").write(txt)
    with pytest.raises(RuntimeError, match="status 2"):
        nrgb.project_bytes(wd)


def test_damaged_param_is_refused(tmp_path):
    import nrgb
    wd = _run(str(tmp_path), 100, 10)
    txt = open(os.path.join(wd, "param")).read()
    assert "keep=100" in txt
    open(os.path.join(wd, "param"), "w").write(txt.replace("keep=100", "keep=abc"))
    with pytest.raises(RuntimeError, match="status 2"):
        nrgb.project_bytes(wd)


def test_server_needs_a_device():
    import torch

    import nrgb
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(RuntimeError, match="status 3"):
        nrgb.Server(0)
