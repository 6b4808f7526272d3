"""QSZ input of the single-impurity Anderson model (inputgen.write_data_qsz):
the sector energies are the QS multiplet energies repeated over their spin
projections, and the f list carries both spin components, each block
connecting I2 to I2 + (1, +-1)."""
import numpy as np

import inputgen
import nrg_oracle as O


def test_qsz_sectors_expand_the_qs_multiplets(tmp_path):
    inputgen.make_siam(str(tmp_path / "qs"), 0.2, -0.07, 0.02, 2.0, 6, params={"keep": 50})
    inputgen.make_siam(str(tmp_path / "qsz"), 0.2, -0.07, 0.02, 2.0, 6, params={"keep": 50}, symtype="QSZ")
    dq = O.read_data(str(tmp_path / "qs" / "data"))
    dz = O.read_data(str(tmp_path / "qsz" / "data"))
    assert dz.symtype == "QSZ"
    eq = np.sort(np.concatenate([np.repeat(v, I[1]) for I, v in dq.energies.items()]))
    ez = np.sort(np.concatenate(list(dz.energies.values())))
    assert np.max(np.abs(eq - ez)) < 1e-12
    for (I1, I2), M in dz.opch[0].items():
        assert I1[0] == I2[0] + 1 and abs(I1[1] - I2[1]) == 1
        assert M.shape == (len(dz.energies[I1]), len(dz.energies[I2]))
    # sum rule: sum over all blocks of |<I1|f^dag|I2>|^2 = number of states
    # times <n_f0 empty> ... per spin: Tr(f f^dag) over the sector basis
    tot = sum(float(np.sum(M * M)) for M in dz.opch[0].values())
    # Tr f_s f_s^dag = half of the 16-state Fock space for each spin
    assert abs(tot - 16.0) < 1e-12
