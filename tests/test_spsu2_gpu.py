"""The SPSU2 symmetry plug-in (spin SU(2), charge not conserved, one and
two channels) on the GPU.

* Normal band (no pairing): the single-impurity Anderson model in SPSU2 and
  in QS keeps the same states under an energy cutoff, so the thermodynamic
  columns they share (<Sz^2>, <E>, <E^2>, C, F, S), the singlet expectation
  values, the energy flow (every SPSU2 level is a QS level, with the same
  spin degeneracy) and the spectral function A_d (DM-NRG and FDM) agree.
* Superconducting band and anomalous hopping: with every state kept, the
  levels of the first steps equal the exact diagonalisation of the chain
  (impurity, sites f_0 .. f_N+1) with on-site pairing delta_n and anomalous
  hopping kappa_n, which tests the pairing and anomalous tables and the Z
  block of the data file.
* Two channels: the two-channel Kondo model in SPSU2 and in QS agree the
  same way, spin (triplet) spectrum included."""
import os

import numpy as np
import pytest

import inputgen
import nrg_cases as cases

pytestmark = pytest.mark.gpu

PARAMS = {"keep": 100000, "keepenergy": 6.0, "keepmin": 1, "T": 1e-4, "dumpannotated": 100000,
          "prec_td": 16, "prec_custom": 16, "dumpprecision": 16, "fdm": True, "dmnrg": True,
          "specd": "A_d-A_d", "bins": 40, "savebins": True, "broaden": False}


def _td(path):
    with open(path) as fh:
        names = fh.readline().lstrip("#").split()
    return names, cases.read_table(path)


def _levels(step):
    """Energies of one step of annotated.dat, each repeated by its degeneracy."""
    return np.sort(np.concatenate([[e] * deg for e, _, deg in step]))


@pytest.mark.parametrize("U,eps", [(0.1, -0.05), (0.3, -0.05)])
def test_spsu2_matches_qs_without_pairing(tmp_path, U, eps):
    import nrgb
    out = {}
    ctx = nrgb.Context(0)
    try:
        for sym in ("QS", "SPSU2"):
            wd = str(tmp_path / ("in" + sym))
            inputgen.make_siam(wd, U, eps, 0.02, 2.0, 14, symtype=sym, params=dict(PARAMS))
            od = str(tmp_path / ("out" + sym))
            os.makedirs(od)
            ctx.run(wd, od)
            out[sym] = od
    finally:
        ctx.close()
    nq, tq = _td(os.path.join(out["QS"], "td"))
    ns, ts = _td(os.path.join(out["SPSU2"], "td"))
    assert tq.shape[0] == ts.shape[0]
    for name in ("T", "<Sz^2>", "<E>", "<E^2>", "C", "F", "S"):
        a, b = tq[:, nq.index(name)], ts[:, ns.index(name)]
        assert np.all(np.abs(a - b) <= 1e-8 * np.abs(a) + 1e-11), (name, float(np.max(np.abs(a - b))))
    cq = cases.read_table(os.path.join(out["QS"], "custom"))
    cs = cases.read_table(os.path.join(out["SPSU2"], "custom"))
    assert np.all(np.abs(cq - cs) <= 1e-8 * np.abs(cq) + 1e-11)
    aq = cases.read_annotated(os.path.join(out["QS"], "annotated.dat"))
    as_ = cases.read_annotated(os.path.join(out["SPSU2"], "annotated.dat"))
    assert len(aq) == len(as_)
    for sq, ss in zip(aq, as_):
        lq, ls = _levels(sq), _levels(ss)
        assert lq.shape == ls.shape
        assert np.max(np.abs(lq - ls)) <= 1e-9 * max(1.0, np.max(np.abs(lq)))
    for typ in ("DMNRG", "FDM"):
        q = cases.read_bins(os.path.join(out["QS"], "spec_%s_dens_A_d-A_d.bin" % typ))
        s = cases.read_bins(os.path.join(out["SPSU2"], "spec_%s_dens_A_d-A_d.bin" % typ))
        dq, ds = dict(zip(q[:, 0], q[:, 1])), dict(zip(s[:, 0], s[:, 1]))
        wmax = max(abs(v) for v in dq.values())
        err = max(abs(dq.get(k, 0.0) - ds.get(k, 0.0)) for k in set(dq) | set(ds))
        assert err <= 1e-8 * wmax, (typ, err / wmax)


def _ed_levels(U, eps, V, xi, zeta, delta, kappa, N):
    """All eigenvalues of the impurity + f_0 .. f_{N+1} chain with pairing."""
    F = inputgen.Fock(N + 3)   # orbital 0 = d, orbital 1 + n = f_n
    H = eps * F.n(0) + U * F.n(0, 0) @ F.n(0, 1)
    for s in (0, 1):
        h = F.cd(0, s) @ F.c(1, s)
        H = H + V * (h + h.T)
    one = np.eye(F.dim)
    for n in range(N + 2):
        pair = F.cd(1 + n, 0) @ F.cd(1 + n, 1)
        H = H + zeta[n] * (F.n(1 + n) - one) + delta[n] * (pair + pair.T)
    for n in range(N + 1):
        for s in (0, 1):
            h = F.cd(1 + n, s) @ F.c(2 + n, s)
            H = H + xi[n] * (h + h.T)
        a = F.cd(1 + n, 0) @ F.cd(2 + n, 1) - F.cd(1 + n, 1) @ F.cd(2 + n, 0)
        H = H + kappa[n] * (a + a.T)
    return np.linalg.eigvalsh(H)


@pytest.mark.parametrize("gap,kap", [(0.03, 0.0), (0.02, 0.015)])
def test_spsu2_pairing_matches_exact_diagonalisation(tmp_path, gap, kap):
    import nrgb
    U, eps, Gamma, Lam, Nmax = 0.3, -0.1, 0.05, 2.0, 3
    wd = str(tmp_path / "in")
    # levels one per line (dumpgroups off): grouping would print levels closer
    # than the group tolerance under one energy
    info = inputgen.make_siam(wd, U, eps, Gamma, Lam, Nmax, symtype="SPSU2", gap=gap,
                              params={"keep": 100000, "dumpannotated": 100000, "dumpprecision": 16,
                                      "dumpgroups": False})
    xi, zeta, delta = info["xi"], info["zeta"], info["delta"]
    kappa = np.full(Nmax + 1, kap)
    if kap:
        # the same model with an anomalous hopping on every bond
        m = inputgen.siam_cluster(U, eps, info["V"], zeta0=zeta[0], delta0=gap)
        inputgen.write_data_spsu2(os.path.join(wd, "data"), m, Lam, 1.0, Nmax, xi, zeta, delta, kappa)
    od = str(tmp_path / "out")
    os.makedirs(od)
    ctx = nrgb.Context(0)
    try:
        ctx.run(wd, od)
    finally:
        ctx.close()
    steps = [s for s in cases.read_annotated(os.path.join(od, "annotated.dat")) if s]
    assert len(steps) == Nmax + 1     # the initial cluster and steps 0 .. Nmax-1
    # the initial cluster (impurity + f_0) is step -1
    for k, step in enumerate(steps):
        N = k - 1
        sc = inputgen.scale_factor(N + 1, Lam, 1.0)
        if N < 0:
            m = inputgen.siam_cluster(U, eps, info["V"], zeta0=zeta[0], delta0=gap)
            ev = np.linalg.eigvalsh(m.H)
        else:
            ev = _ed_levels(U, eps, info["V"], xi, zeta, delta, kappa, N)
        ev = np.sort(ev / sc)
        ev -= ev[0]
        # one line per multiplet: energy and SS, the multiplet's 2S+1 states
        got = np.sort(np.concatenate([[e] * int(lab[0]) for e, lab, _ in step]))
        assert got.shape == ev.shape, (N, got.shape, ev.shape)
        assert np.max(np.abs(got - ev)) < 1e-10, (N, float(np.max(np.abs(got - ev))))


def test_spsu2_two_channels_matches_qs(tmp_path):
    """Two-channel Kondo model (no pairing) in SPSU2 and in QS: the tables
    of both are derived for 16 combinations (QSCoupling in its two modes);
    thermodynamics, energy flow and the f and spin spectra (doublet and
    triplet operators) agree."""
    import nrgb
    params = {"keep": 100000, "keepenergy": 5.0, "keepmin": 1, "T": 1e-3, "fdm": True, "dmnrg": True,
              "spect": "SZd-SZd", "specd": "A_f0-A_f0", "bins": 30, "savebins": True, "broaden": False,
              "dumpannotated": 100000, "prec_td": 16, "dumpprecision": 16}
    out = {}
    ctx = nrgb.Context(0)
    try:
        for sym in ("QS", "SPSU2"):
            wd = str(tmp_path / ("in" + sym))
            inputgen.make_kondo(wd, [0.2, 0.2], 3.0, 8, symtype=sym, params=dict(params))
            od = str(tmp_path / ("out" + sym))
            os.makedirs(od)
            ctx.run(wd, od)
            out[sym] = od
    finally:
        ctx.close()
    nq, tq = _td(os.path.join(out["QS"], "td"))
    ns, ts = _td(os.path.join(out["SPSU2"], "td"))
    assert tq.shape[0] == ts.shape[0]
    for name in ("T", "<Sz^2>", "<E>", "<E^2>", "C", "F", "S"):
        a, b = tq[:, nq.index(name)], ts[:, ns.index(name)]
        assert np.all(np.abs(a - b) <= 1e-8 * np.abs(a) + 1e-11), (name, float(np.max(np.abs(a - b))))
    aq = cases.read_annotated(os.path.join(out["QS"], "annotated.dat"))
    as_ = cases.read_annotated(os.path.join(out["SPSU2"], "annotated.dat"))
    assert len(aq) == len(as_)
    for sq, ss in zip(aq, as_):
        lq, ls = _levels(sq), _levels(ss)
        assert lq.shape == ls.shape
        assert np.max(np.abs(lq - ls)) <= 1e-9 * max(1.0, np.max(np.abs(lq)))
    for fname in ("spec_FDM_dens_A_f0-A_f0.bin", "spin_FDM_dens_SZd-SZd.bin", "spec_DMNRG_dens_A_f0-A_f0.bin"):
        q = cases.read_bins(os.path.join(out["QS"], fname))
        s = cases.read_bins(os.path.join(out["SPSU2"], fname))
        dq, ds = dict(zip(q[:, 0], q[:, 1])), dict(zip(s[:, 0], s[:, 1]))
        wmax = max(abs(v) for v in dq.values())
        err = max(abs(dq.get(k, 0.0) - ds.get(k, 0.0)) for k in set(dq) | set(ds))
        assert err <= 1e-8 * wmax, (fname, err / wmax)


def test_spsu2_three_channels_matches_qs(tmp_path):
    """Three-channel Kondo model with unequal couplings (no pairing) in SPSU2
    and in QS, both with tables derived for 64 combinations: thermodynamics,
    energy flow and the f spectral function of every channel (doublet
    operators) agree."""
    import nrgb
    params = {"keep": 100000, "keepenergy": 3.0, "keepmin": 1, "T": 1e-3, "fdm": True, "dmnrg": True,
              "specd": "A_f0-A_f0 A_f1-A_f1 A_f2-A_f2", "bins": 30, "savebins": True, "broaden": False,
              "dumpannotated": 100000, "prec_td": 16, "dumpprecision": 16}
    out = {}
    ctx = nrgb.Context(0)
    try:
        for sym in ("QS", "SPSU2"):
            wd = str(tmp_path / ("in" + sym))
            inputgen.make_kondo(wd, [0.3, 0.2, 0.1], 3.0, 5, symtype=sym, params=dict(params))
            od = str(tmp_path / ("out" + sym))
            os.makedirs(od)
            ctx.run(wd, od)
            out[sym] = od
    finally:
        ctx.close()
    nq, tq = _td(os.path.join(out["QS"], "td"))
    ns, ts = _td(os.path.join(out["SPSU2"], "td"))
    assert tq.shape[0] == ts.shape[0]
    for name in ("T", "<Sz^2>", "<E>", "<E^2>", "C", "F", "S"):
        a, b = tq[:, nq.index(name)], ts[:, ns.index(name)]
        assert np.all(np.abs(a - b) <= 1e-8 * np.abs(a) + 1e-11), (name, float(np.max(np.abs(a - b))))
    aq = cases.read_annotated(os.path.join(out["QS"], "annotated.dat"))
    as_ = cases.read_annotated(os.path.join(out["SPSU2"], "annotated.dat"))
    assert len(aq) == len(as_)
    for sq, ss in zip(aq, as_):
        lq, ls = _levels(sq), _levels(ss)
        assert lq.shape == ls.shape
        assert np.max(np.abs(lq - ls)) <= 1e-9 * max(1.0, np.max(np.abs(lq)))
    for ch in range(3):
        for typ in ("FDM", "DMNRG"):
            fname = "spec_%s_dens_A_f%d-A_f%d.bin" % (typ, ch, ch)
            q = cases.read_bins(os.path.join(out["QS"], fname))
            s = cases.read_bins(os.path.join(out["SPSU2"], fname))
            dq, ds = dict(zip(q[:, 0], q[:, 1])), dict(zip(s[:, 0], s[:, 1]))
            wmax = max(abs(v) for v in dq.values())
            assert wmax > 0
            err = max(abs(dq.get(k, 0.0) - ds.get(k, 0.0)) for k in set(dq) | set(ds))
            assert err <= 1e-8 * wmax, (fname, err / wmax)
