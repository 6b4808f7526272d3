"""The QSZ symmetry plug-in (charge U(1) x spin-projection U(1), one and
two channels) against the QS plug-in on the same model: a single-impurity
Anderson model truncated by an energy cutoff (keepenergy, with the safeguard
completing split multiplets) keeps the same states in both, so every
thermodynamic column they share (<Sz^2>, <Q>, <Q^2>, <E>, <E^2>, C, F, S)
must agree, <Sz> must vanish, the singlet expectation values must agree,
the QSZ energy flow must be the QS one with each level repeated over its
spin projections, and each spin component of the QSZ spectral function
(spec_*_dens_A_d-A_d-u / -d, DM-NRG and FDM) must equal the QS one."""
import collections
import os

import numpy as np
import pytest

import inputgen
import nrg_cases as cases

pytestmark = pytest.mark.gpu

PARAMS = {"keep": 100000, "keepenergy": 6.0, "keepmin": 1, "T": 1e-4, "dumpannotated": 1, "dumpgroups": False,
          "prec_td": 16, "prec_custom": 16, "dumpprecision": 16, "fdm": True, "dmnrg": True,
          "specd": "A_d-A_d", "bins": 40, "savebins": True, "broaden": False}


@pytest.mark.parametrize("U,eps", [(0.1, -0.05), (0.3, -0.05)])
def test_qsz_matches_qs(tmp_path, U, eps):
    import nrgb
    out = {}
    ctx = nrgb.Context(0)
    try:
        for sym in ("QS", "QSZ"):
            wd = str(tmp_path / ("in" + sym))
            inputgen.make_siam(wd, U, eps, 0.02, 2.0, 14, symtype=sym, params=dict(PARAMS))
            od = str(tmp_path / ("out" + sym))
            os.makedirs(od)
            ctx.run(wd, od)
            out[sym] = od
    finally:
        ctx.close()
    tq = cases.read_table(os.path.join(out["QS"], "td"))
    tz = cases.read_table(os.path.join(out["QSZ"], "td"))
    # QS columns: T <Sz^2> <Q> <Q^2> <E> <E^2> C F S;  QSZ: T <Sz^2> <Sz> <Q> <Q^2> <E> <E^2> C F S
    assert tq.shape[0] == tz.shape[0]
    shared_z = tz[:, [0, 1, 3, 4, 5, 6, 7, 8, 9]]
    assert np.all(np.abs(shared_z - tq) <= 1e-8 * np.abs(tq) + 1e-11), float(np.max(np.abs(shared_z - tq)))
    assert np.max(np.abs(tz[:, 2])) < 1e-11
    cq = cases.read_table(os.path.join(out["QS"], "custom"))
    cz = cases.read_table(os.path.join(out["QSZ"], "custom"))
    assert np.all(np.abs(cq - cz) <= 1e-8 * np.abs(cq) + 1e-11)
    # energy flow: every QS multiplet (Q, SS) at energy E appears SS times in QSZ
    aq = cases.read_annotated(os.path.join(out["QS"], "annotated.dat"))
    az = cases.read_annotated(os.path.join(out["QSZ"], "annotated.dat"))
    assert len(aq) == len(az)
    for sq, sz in zip(aq, az):
        eq = np.sort(np.concatenate([[e] * int(lab[0].split()[1]) for e, lab, _ in sq]))
        ez = np.sort(np.array([e for e, _, _ in sz]))
        assert eq.shape == ez.shape
        assert np.max(np.abs(eq - ez)) <= 1e-9 * max(1.0, np.max(np.abs(eq)))
        # the charges of the levels agree as a multiset
        qq = collections.Counter()
        for e, lab, _ in sq:
            q, ss = (int(x) for x in lab[0].split())
            qq[q] += ss
        qz = collections.Counter(int(lab[0].split()[0]) for _, lab, _ in sz)
        assert qq == qz

    for typ in ("DMNRG", "FDM"):
        q = cases.read_bins(os.path.join(out["QS"], "spec_%s_dens_A_d-A_d.bin" % typ))
        dq = dict(zip(q[:, 0], q[:, 1]))
        wmax = max(abs(v) for v in dq.values())
        for spin in ("u", "d"):
            z = cases.read_bins(os.path.join(out["QSZ"], "spec_%s_dens_A_d-A_d-%s.bin" % (typ, spin)))
            dz = dict(zip(z[:, 0], z[:, 1]))
            keys = set(dq) | set(dz)
            err = max(abs(dq.get(k, 0.0) - dz.get(k, 0.0)) for k in keys)
            assert err <= 1e-8 * wmax, (typ, spin, err / wmax)


def test_qsz_two_channels_matches_qs(tmp_path):
    """Two-channel Kondo model in QSZ and in QS: under an energy cutoff both
    keep the same states, so the shared thermodynamic columns agree, every
    QS multiplet appears with its SS spin projections in QSZ, and each spin
    component of the QSZ spectral function of the channel-0 f operator
    equals the QS one."""
    import nrgb
    params = {"keep": 100000, "keepenergy": 5.0, "keepmin": 1, "T": 1e-3, "fdm": True, "dmnrg": True,
              "specd": "A_f0-A_f0", "bins": 30, "savebins": True, "broaden": False, "dumpannotated": 100000,
              "dumpgroups": False, "prec_td": 16, "dumpprecision": 16}
    out = {}
    ctx = nrgb.Context(0)
    try:
        for sym in ("QS", "QSZ"):
            wd = str(tmp_path / ("in" + sym))
            inputgen.make_kondo(wd, [0.2, 0.2], 3.0, 8, symtype=sym, params=dict(params))
            od = str(tmp_path / ("out" + sym))
            os.makedirs(od)
            ctx.run(wd, od)
            out[sym] = od
    finally:
        ctx.close()
    tq = cases.read_table(os.path.join(out["QS"], "td"))
    tz = cases.read_table(os.path.join(out["QSZ"], "td"))
    assert tq.shape[0] == tz.shape[0]
    shared_z = tz[:, [0, 1, 3, 4, 5, 6, 7, 8, 9]]
    assert np.all(np.abs(shared_z - tq) <= 1e-8 * np.abs(tq) + 1e-11), float(np.max(np.abs(shared_z - tq)))
    assert np.max(np.abs(tz[:, 2])) < 1e-11
    aq = cases.read_annotated(os.path.join(out["QS"], "annotated.dat"))
    az = cases.read_annotated(os.path.join(out["QSZ"], "annotated.dat"))
    assert len(aq) == len(az)
    for sq, sz in zip(aq, az):
        eq = np.sort(np.concatenate([[e] * int(lab[0].split()[1]) for e, lab, _ in sq]))
        ez = np.sort(np.array([e for e, _, _ in sz]))
        assert eq.shape == ez.shape
        assert np.max(np.abs(eq - ez)) <= 1e-9 * max(1.0, np.max(np.abs(eq)))
    for typ in ("DMNRG", "FDM"):
        q = cases.read_bins(os.path.join(out["QS"], "spec_%s_dens_A_f0-A_f0.bin" % typ))
        dq = dict(zip(q[:, 0], q[:, 1]))
        wmax = max(abs(v) for v in dq.values())
        for spin in ("u", "d"):
            z = cases.read_bins(os.path.join(out["QSZ"], "spec_%s_dens_A_f0-A_f0-%s.bin" % (typ, spin)))
            dz = dict(zip(z[:, 0], z[:, 1]))
            err = max(abs(dq.get(k, 0.0) - dz.get(k, 0.0)) for k in set(dq) | set(dz))
            assert err <= 1e-8 * wmax, (typ, spin, err / wmax)
