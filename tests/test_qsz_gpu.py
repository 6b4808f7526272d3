"""The QSZ symmetry plug-in (charge U(1) x spin-projection U(1), one to
three channels) against the QS plug-in on the same model: a single-impurity
Anderson model truncated by an energy cutoff (keepenergy, with the safeguard
completing split multiplets) keeps the same states in both, so every
thermodynamic column they share (<Sz^2>, <Q>, <Q^2>, <E>, <E^2>, C, F, S)
must agree, <Sz> must vanish, the singlet expectation values must agree,
the QSZ energy flow must be the QS one with each level repeated over its
spin projections, and each spin component of the QSZ spectral function
(spec_*_dens_A_d-A_d-u / -d, DM-NRG and FDM) must equal the QS one.

Three channels: with every state kept, the levels and (Q, SSZ) labels of
the initial cluster and of step 0 equal the exact diagonalisation of the
impurity spin and two sites of each channel; under truncation, the
channel-symmetric model gives the same spectral function for the f operator
of every channel and both spins, and the model with unequal couplings agrees
with the three-channel QS run."""
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


def _kondo_ed_levels(J, xi0):
    """(Q, SSZ, E) of every eigenstate of the Kondo impurity spin coupled to
    f_0 of each channel, with hopping xi0 from f_0 to f_1 in every channel.
    Fock states are bit masks over the modes 2*o + spin (orbital 0 = d,
    orbital 1 + n*P + ch = f_n of channel ch), the impurity singly occupied;
    each (Q, SSZ) sector is diagonalised on its own."""
    P = len(J)
    nmode = 2 * (1 + 2 * P)
    orb = lambda n, ch: 1 + n * P + ch

    def apply(ops, x):
        # ops: [(mode, dagger)], rightmost first
        sign = 1
        for m, dag in reversed(ops):
            occ = (x >> m) & 1
            if occ == dag:
                return 0, None
            if bin(x & ((1 << m) - 1)).count("1") & 1:
                sign = -sign
            x ^= 1 << m
        return sign, x

    states = [x for x in range(1 << nmode) if (x & 1) + ((x >> 1) & 1) == 1]
    def qn(x):
        q = sum((x >> (2 * o + s)) & 1 for n in range(2) for ch in range(P)
                for o in (orb(n, ch),) for s in (0, 1)) - 2 * P
        up = sum((x >> (2 * o)) & 1 for o in range(1 + 2 * P))
        dn = sum((x >> (2 * o + 1)) & 1 for o in range(1 + 2 * P))
        return q, up - dn
    sectors = collections.defaultdict(list)
    for x in states:
        sectors[qn(x)].append(x)
    terms = []      # (coefficient, operator string)
    for ch in range(P):
        a, b = orb(0, ch), orb(1, ch)
        for s in (0, 1):
            terms.append((xi0, [(2 * a + s, 1), (2 * b + s, 0)]))
            terms.append((xi0, [(2 * b + s, 1), (2 * a + s, 0)]))
        # J S_d . s_f = J (Sz_d sz_f + (S+_d s-_f + S-_d s+_f) / 2)
        for sd in (0, 1):
            for sf in (0, 1):
                c = 0.25 * J[ch] * (1 if sd == sf else -1)
                terms.append((c, [(2 * 0 + sd, 1), (2 * 0 + sd, 0), (2 * a + sf, 1), (2 * a + sf, 0)]))
        terms.append((0.5 * J[ch], [(0, 1), (1, 0), (2 * a + 1, 1), (2 * a, 0)]))
        terms.append((0.5 * J[ch], [(1, 1), (0, 0), (2 * a, 1), (2 * a + 1, 0)]))
    out = []
    for key, basis in sectors.items():
        index = {x: i for i, x in enumerate(basis)}
        H = np.zeros((len(basis), len(basis)))
        for x in basis:
            for c, ops in terms:
                sg, y = apply(ops, x)
                if sg:
                    H[index[y], index[x]] += c * sg
        out.extend((key[0], key[1], e) for e in np.linalg.eigvalsh(H))
    return out


def test_qsz_three_channels_matches_exact_diagonalisation(tmp_path):
    """Three-channel Kondo model, every state kept: the initial cluster (128
    states) and step 0 (8192 states) against exact diagonalisation, level by
    level within each (Q, SSZ) sector."""
    import nrgb
    J, Lam = [0.3, 0.2, 0.1], 3.0
    wd = str(tmp_path / "in")
    info = inputgen.make_kondo(wd, J, Lam, 1, symtype="QSZ",
                               params={"keep": 100000, "dumpannotated": 100000, "dumpgroups": False,
                                       "dumpprecision": 16})
    assert np.all(info["zeta"] == 0)
    od = str(tmp_path / "out")
    os.makedirs(od)
    ctx = nrgb.Context(0)
    try:
        ctx.run(wd, od)
    finally:
        ctx.close()
    steps = [s for s in cases.read_annotated(os.path.join(od, "annotated.dat")) if s]
    assert len(steps) == 2
    # the initial cluster: the impurity and f_0 of each channel
    m = inputgen.kondo_cluster(J)
    sub = inputgen.decompose_qsz(m)
    ref = {-1: [(s.Q, s.SS, e) for s in sub for e in s.energies],
           0: _kondo_ed_levels(J, info["xi"][0])}
    for N, step in zip((-1, 0), steps):
        sc = inputgen.scale_factor(N + 1, Lam, 1.0)
        gs = min(e for _, _, e in ref[N])
        want = collections.defaultdict(list)
        for q, z, e in ref[N]:
            want[(q, z)].append((e - gs) / sc)
        got = collections.defaultdict(list)
        for e, lab, _ in step:
            q, z = (int(x) for x in lab[0].split())
            got[(q, z)].append(e)
        assert sorted(got) == sorted(want), N
        for key in want:
            a, b = np.sort(got[key]), np.sort(want[key])
            assert a.shape == b.shape, (N, key)
            assert np.max(np.abs(a - b)) < 1e-10, (N, key, float(np.max(np.abs(a - b))))


def test_qsz_three_channels_symmetric_spectra(tmp_path):
    """Channel-symmetric three-channel Kondo model under an energy cutoff:
    <Sz> vanishes and the f spectral function (DM-NRG and FDM) is the same
    for every channel and both spins."""
    import nrgb
    params = {"keep": 600, "keepenergy": 4.0, "keepmin": 1, "T": 1e-3, "fdm": True, "dmnrg": True,
              "specd": "A_f0-A_f0 A_f1-A_f1 A_f2-A_f2", "bins": 30, "savebins": True, "broaden": False,
              "prec_td": 16}
    wd = str(tmp_path / "in")
    inputgen.make_kondo(wd, [0.2, 0.2, 0.2], 3.0, 6, symtype="QSZ", params=params)
    od = str(tmp_path / "out")
    os.makedirs(od)
    ctx = nrgb.Context(0)
    try:
        ctx.run(wd, od)
    finally:
        ctx.close()
    tz = cases.read_table(os.path.join(od, "td"))
    assert np.max(np.abs(tz[:, 2])) < 1e-11
    for typ in ("DMNRG", "FDM"):
        ref = cases.read_bins(os.path.join(od, "spec_%s_dens_A_f0-A_f0-u.bin" % typ))
        dr = dict(zip(ref[:, 0], ref[:, 1]))
        wmax = max(abs(v) for v in dr.values())
        assert wmax > 0
        for ch in range(3):
            for spin in ("u", "d"):
                z = cases.read_bins(os.path.join(od, "spec_%s_dens_A_f%d-A_f%d-%s.bin" % (typ, ch, ch, spin)))
                dz = dict(zip(z[:, 0], z[:, 1]))
                err = max(abs(dr.get(k, 0.0) - dz.get(k, 0.0)) for k in set(dr) | set(dz))
                assert err <= 1e-8 * wmax, (typ, ch, spin, err / wmax)


def test_qs_three_channels_matches_qsz(tmp_path):
    """Three-channel Kondo model with unequal couplings in QS (tables derived
    by spin coupling, host/qs_coupling.cc) and in QSZ (Fock-state
    combinations, pinned above to exact diagonalisation): under an energy
    cutoff both keep the same states, so the shared thermodynamic columns
    agree, every QS multiplet appears with its SS spin projections in QSZ,
    and the f spectral function of every channel (a doublet operator, whose
    recalculation runs through the doublet tables) equals each QSZ spin
    component."""
    import nrgb
    params = {"keep": 100000, "keepenergy": 3.0, "keepmin": 1, "T": 1e-3, "fdm": True, "dmnrg": True,
              "specd": "A_f0-A_f0 A_f1-A_f1 A_f2-A_f2", "bins": 30, "savebins": True, "broaden": False,
              "dumpannotated": 100000, "dumpgroups": False, "prec_td": 16, "dumpprecision": 16}
    out = {}
    ctx = nrgb.Context(0)
    try:
        for sym in ("QS", "QSZ"):
            wd = str(tmp_path / ("in" + sym))
            inputgen.make_kondo(wd, [0.3, 0.2, 0.1], 3.0, 5, symtype=sym, params=dict(params))
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
    aq = cases.read_annotated(os.path.join(out["QS"], "annotated.dat"))
    az = cases.read_annotated(os.path.join(out["QSZ"], "annotated.dat"))
    assert len(aq) == len(az)
    for sq, sz in zip(aq, az):
        eq = np.sort(np.concatenate([[e] * int(lab[0].split()[1]) for e, lab, _ in sq]))
        ez = np.sort(np.array([e for e, _, _ in sz]))
        assert eq.shape == ez.shape
        assert np.max(np.abs(eq - ez)) <= 1e-9 * max(1.0, np.max(np.abs(eq)))
    for ch in range(3):
        for typ in ("DMNRG", "FDM"):
            q = cases.read_bins(os.path.join(out["QS"], "spec_%s_dens_A_f%d-A_f%d.bin" % (typ, ch, ch)))
            dq = dict(zip(q[:, 0], q[:, 1]))
            wmax = max(abs(v) for v in dq.values())
            assert wmax > 0
            for spin in ("u", "d"):
                z = cases.read_bins(os.path.join(out["QSZ"], "spec_%s_dens_A_f%d-A_f%d-%s.bin" % (typ, ch, ch, spin)))
                dz = dict(zip(z[:, 0], z[:, 1]))
                err = max(abs(dq.get(k, 0.0) - dz.get(k, 0.0)) for k in set(dq) | set(dz))
                assert err <= 1e-8 * wmax, (ch, typ, spin, err / wmax)
