"""The SPSU2 input generator and data-file layout (no device): subspaces
labelled by SS alone, the Z block with the on-site pairing and anomalous
hopping tables, and, without pairing, the same cluster levels as QS; the
three-channel data files of the QS, QSZ and SPSU2 writers."""
import numpy as np

import inputgen


def _read(path):
    with open(path) as fh:
        return [l.rstrip("\n") for l in fh]


def test_spsu2_data_layout(tmp_path):
    info = inputgen.make_siam(str(tmp_path), 0.3, -0.1, 0.05, 2.0, 6, symtype="SPSU2", gap=0.02)
    lines = _read(str(tmp_path / "data"))
    assert "# symtype SPSU2" in lines
    ch, nmax, nsub = (int(x) for x in lines[4].split())
    assert (ch, nmax, nsub) == (1, 6, 3)
    # subspaces: one integer each (SS = 1, 2, 3), with 5, 4 and 1 states
    assert [lines[7], lines[8], lines[10], lines[11], lines[13], lines[14]] == ["1", "5", "2", "4", "3", "1"]
    assert lines.index("Z") > lines.index("z")
    z = lines.index("Z")
    assert lines[z + 1] == "6" and all(float(x) == 0.02 for x in lines[z + 2:z + 9])
    assert lines[z + 9] == "6" and all(float(x) == 0.0 for x in lines[z + 10:z + 17])
    assert np.all(info["delta"] == 0.02) and np.all(info["kappa"] == 0.0)


def test_spsu2_cluster_levels_equal_qs_without_pairing():
    m = inputgen.siam_cluster(0.3, -0.1, 0.2)
    qs = inputgen.decompose(m)
    sp = inputgen.decompose_spsu2(m)
    for ss in (1, 2, 3):
        a = np.sort(np.concatenate([s.energies for s in qs if s.SS == ss]))
        b = np.sort(np.concatenate([s.energies for s in sp if s.SS == ss]))
        assert np.allclose(a, b, atol=1e-13)


def test_pairing_mixes_charges():
    m = inputgen.siam_cluster(0.3, -0.1, 0.2, delta0=0.05)
    ev_full = np.sort(np.linalg.eigvalsh(m.H))
    sp = inputgen.decompose_spsu2(m)
    ev = np.sort(np.concatenate([np.repeat(s.energies, s.SS) for s in sp]))
    assert np.allclose(ev, ev_full, atol=1e-12)


def test_three_channel_kondo_cluster_levels_agree_across_symmetries():
    """The three-channel Kondo cluster (impurity spin and f_0 of each channel,
    128 states) decomposed by the QS, QSZ and SPSU2 writers: every state of
    the cluster appears once, with the same energy, in each; QS multiplets
    count SS states, QSZ sectors one state each, SPSU2 multiplets SS states."""
    m = inputgen.kondo_cluster([0.3, 0.2, 0.1])
    ev_full = np.sort(np.linalg.eigvalsh(m.H[np.ix_(m.basis_mask, m.basis_mask)]))
    assert ev_full.shape == (128,)
    qs = np.sort(np.concatenate([np.repeat(s.energies, s.SS) for s in inputgen.decompose(m)]))
    qsz = np.sort(np.concatenate([s.energies for s in inputgen.decompose_qsz(m)]))
    sp = np.sort(np.concatenate([np.repeat(s.energies, s.SS) for s in inputgen.decompose_spsu2(m)]))
    for ev in (qs, qsz, sp):
        assert ev.shape == ev_full.shape
        assert np.allclose(ev, ev_full, atol=1e-12)


def test_three_channel_data_files(tmp_path):
    """The three writers take three channels: the header's channel count, an
    f block per channel and a chain table per channel."""
    for sym in ("QS", "QSZ", "SPSU2"):
        wd = tmp_path / sym
        inputgen.make_kondo(str(wd), [0.3, 0.2, 0.1], 3.0, 4, symtype=sym)
        lines = _read(str(wd / "data"))
        assert "# symtype " + sym in lines
        assert int(lines[4].split()[0]) == 3
        assert sum(1 for l in lines if l.startswith("f ")) == 3
        z = lines.index("z")
        # xi then zeta, one table of Nmax + 1 = 5 values per channel each
        assert [lines[z + 1 + 6 * k] for k in range(6)] == ["4"] * 6
