"""Known-answer tests that pin the oracle (and the input generator) where the
reference has no regression tests for the NRG step: Wilson's closed-form
chain, exact diagonalisation of short chains, the FDM sum rule and the
density-matrix trace invariants of src/nrg.cc:1176-1181, src/dmnrg.h:588-592."""
import math

import numpy as np
import pytest

import inputgen as g
import nrg_oracle as O


def test_wilson_chain_closed_form():
    xi, zeta = g.wilson_chain_flat(2.0, 1.0, 30)
    ref = g.wilson_closed_form(2.0, 30)
    assert np.max(np.abs(xi / ref - 1)) < 1e-14
    assert np.max(np.abs(zeta)) < 1e-15
    xi3, _ = g.wilson_chain_flat(3.0, 1.0, 20)
    assert np.max(np.abs(xi3 / g.wilson_closed_form(3.0, 20) - 1)) < 1e-14


def test_wilson_chain_precision_converged():
    a, _ = g.wilson_chain_flat(2.0, 0.625, 40, dps=150)
    b, _ = g.wilson_chain_flat(2.0, 0.625, 40, dps=300)
    assert np.max(np.abs(a / b - 1)) < 1e-15


def _chain_H(F, xi, N, first_site=1):
    H = np.zeros((F.dim, F.dim))
    for n in range(0, N + 1):
        for s in (0, 1):
            h = F.cd(first_site + n, s) @ F.c(first_site + n + 1, s)
            H += xi[n] * (h + h.T)
    return H


def _nrg_levels(rec):
    return np.sort(np.concatenate([np.repeat(e.value, I[1]) for I, e in rec.eig.items()]))


@pytest.mark.parametrize("U,eps", [(0.3, -0.1), (0.1, -0.05), (0.0, 0.02)])
def test_siam_energies_match_exact_diagonalisation(tmp_path, U, eps):
    info = g.make_siam(str(tmp_path), U, eps, 0.05, 2.0, Nmax=3, params={"keep": 100000})
    o = O.Oracle(str(tmp_path))
    o.setup()
    o.sweep1()
    for N in range(3):
        F = g.Fock(N + 3)
        H = eps * F.n(0) + U * F.n(0, 0) @ F.n(0, 1)
        for s in (0, 1):
            h = F.cd(0, s) @ F.c(1, s)
            H += info["V"] * (h + h.T)
        H += _chain_H(F, info["xi"], N)
        ev = np.linalg.eigvalsh(H) / O.SCALE(o.P, N + 1)
        ev -= ev.min()
        assert np.max(np.abs(np.sort(ev) - _nrg_levels(o.steps[N]))) < 1e-12


def test_kondo_energies_match_exact_diagonalisation(tmp_path):
    J = 0.4
    info = g.make_kondo(str(tmp_path), [J], 2.5, Nmax=3, params={"keep": 100000})
    o = O.Oracle(str(tmp_path))
    o.setup()
    o.sweep1()
    for N in range(2):
        F = g.Fock(N + 3)
        spd, smd, szd = F.spin_ops(0)
        sp, sm, sz = F.spin_ops(1)
        H = J * (szd @ sz + 0.5 * (spd @ sm + smd @ sp)) + _chain_H(F, info["xi"], N)
        mask = (F.occ[:, 0] + F.occ[:, 1]) == 1
        ev = np.linalg.eigvalsh(H[np.ix_(mask, mask)]) / O.SCALE(o.P, N + 1)
        ev -= ev.min()
        assert np.max(np.abs(np.sort(ev) - _nrg_levels(o.steps[N]))) < 1e-12


def _sparse_fock(nmodes):
    """Sparse Jordan-Wigner creation operators of `nmodes` modes and the
    occupation table (rows: basis states)."""
    import scipy.sparse as sp
    dim = 1 << nmodes
    states = np.arange(dim)
    occ = (states[:, None] >> np.arange(nmodes)[None, :]) & 1
    cd = []
    for k in range(nmodes):
        src = states[occ[:, k] == 0]
        sign = (-1.0) ** occ[src, :k].sum(1)
        cd.append(sp.csr_matrix((sign, (src | (1 << k), src)), shape=(dim, dim)))
    return cd, occ


def _sector_eigs(H, occ, keep):
    """All eigenvalues of H on the basis states `keep`, by blocks of fixed
    particle number and S_z (H conserves both)."""
    n = occ.sum(1)
    sz = occ[:, 0::2].sum(1) - occ[:, 1::2].sum(1)
    out = []
    for a in set(n[keep]):
        for b in set(sz[keep]):
            idx = np.where(keep & (n == a) & (sz == b))[0]
            if len(idx):
                out.append(np.linalg.eigvalsh(H[idx][:, idx].toarray()))
    return np.sort(np.concatenate(out))


def test_two_channel_kondo_energies_match_exact_diagonalisation(tmp_path):
    """Two-channel QS tables (derived from spin coupling): NRG levels of the
    first two steps equal the exact spectrum of the two-channel Kondo chain."""
    J = [0.4, 0.25]
    info = g.make_kondo(str(tmp_path), J, 2.5, Nmax=2, params={"keep": 100000})
    o = O.Oracle(str(tmp_path))
    o.setup()
    o.sweep1()
    for N in range(2):
        L = N + 2                      # chain sites per channel
        norb = 1 + 2 * L               # orbital 0: impurity; (ch, n) -> 1 + 2n + ch
        cd, occ = _sparse_fock(2 * norb)
        c = [x.T.tocsr() for x in cd]

        def spin(o):
            up, dn = 2 * o, 2 * o + 1
            return cd[up] @ c[dn], cd[dn] @ c[up], 0.5 * (cd[up] @ c[up] - cd[dn] @ c[dn])
        spd, smd, szd = spin(0)
        H = 0 * cd[0]
        for ch in range(2):
            sp_, sm_, sz_ = spin(1 + ch)
            H = H + J[ch] * (szd @ sz_ + 0.5 * (spd @ sm_ + smd @ sp_))
            for n in range(L - 1):
                for s_ in (0, 1):
                    h = cd[2 * (1 + 2 * n + ch) + s_] @ c[2 * (1 + 2 * (n + 1) + ch) + s_]
                    H = H + info["xi"][n] * (h + h.T)
        mask = (occ[:, 0] + occ[:, 1]) == 1
        ev = _sector_eigs(H.tocsr(), occ, mask) / O.SCALE(o.P, N + 1)
        ev -= ev.min()
        assert np.max(np.abs(ev - _nrg_levels(o.steps[N]))) < 1e-12


def test_doublet_recalculation_matches_exact_diagonalisation(tmp_path):
    U, eps, Gam = 0.3, -0.1, 0.05
    info = g.make_siam(str(tmp_path), U, eps, Gam, 2.0, Nmax=3,
                       params={"keep": 100000, "specd": "A_d-A_d"})
    o = O.Oracle(str(tmp_path))
    o.setup()
    o.sweep1()
    N = 2
    F = g.Fock(N + 3)
    H = eps * F.n(0) + U * F.n(0, 0) @ F.n(0, 1)
    for s in (0, 1):
        h = F.cd(0, s) @ F.c(1, s)
        H += info["V"] * (h + h.T)
    H += _chain_H(F, info["xi"], N)
    m = g.ClusterModel(F, H, charge_orbitals=list(range(N + 3)), f_orbitals=[N + 2],
                       spin_orbitals=list(range(N + 3)), basis_mask=np.ones(F.dim, bool))
    subs = g.decompose(m)
    red = g.reduced_doublet(m, subs, 0)
    sc = O.SCALE(o.P, N + 1)
    E = {(s.Q, s.SS): s.energies / sc for s in subs}
    gs = min(v.min() for v in E.values())
    E = {k: v - gs for k, v in E.items()}

    def moments(blocks, En):
        out = []
        for a in (0.0, 0.5, 2.0):
            for k in (0, 1, 2):
                t = 0.0
                for (I1, I2), M in blocks.items():
                    e1 = En[I1][:M.shape[0]]
                    e2 = En[I2][:M.shape[1]]
                    t += np.sum(M ** 2 * np.exp(-a * (e1[:, None] + e2[None, :]))
                                * (e1[:, None] - e2[None, :]) ** k)
                out.append(t)
        return np.array(out)

    ref = moments(red, E)
    got = moments(o.final_ops["d"]["A_d"], {I: e.value for I, e in o.steps[N].eig.items()})
    assert np.max(np.abs(ref - got) / np.abs(ref)) < 1e-12


def test_fdm_sum_rule_with_truncation(tmp_path):
    g.make_siam(str(tmp_path), 0.2, -0.1, 0.04, 2.0, Nmax=10,
                params={"keep": 60, "specd": "A_d-A_d", "fdm": True, "T": 1e-3, "bins": 20,
                        "broaden": False})
    o = O.Oracle(str(tmp_path))
    o.run()
    sp = o.spectra[0]
    assert abs(sp.pos.w.sum() + sp.neg.w.sum() - 1.0) < 1e-10
    assert abs(o.wn.sum() - 1.0) < 1e-12


def test_dmnrg_density_matrix_traces_and_fdm_agreement(tmp_path):
    g.make_siam(str(tmp_path), 0.2, -0.1, 0.04, 2.0, Nmax=22,
                params={"keep": 300, "specd": "A_d-A_d", "dmnrg": True, "fdm": True,
                        "T": 1e-6, "bins": 10, "broaden": False})
    o = O.Oracle(str(tmp_path))
    o.run()
    for N, rho in o.rho.items():
        assert abs(o.trace(rho) - 1.0) < 1e-12
    dm, fdm = o.spectra
    assert dm.spectype == "DMNRG" and fdm.spectype == "FDM"
    # FDM satisfies the sum rule exactly; DM-NRG with N/N+2 patching only
    # approximately, and the two agree decade by decade above the last window.
    assert abs(fdm.pos.w.sum() + fdm.neg.w.sum() - 1.0) < 1e-10
    assert abs(dm.pos.w.sum() + dm.neg.w.sum() - 1.0) < 0.08
    wd = dm.pos.w + dm.neg.w
    wf = fdm.pos.w + fdm.neg.w
    for i in range(40, len(wd), 10):
        assert abs(wd[i:i + 10].sum() - wf[i:i + 10].sum()) < 0.03


def test_broadening_kernel_weight_and_log_shift():
    """BR_NEW broadening of one peak well above omega0 is the log-Gaussian
    kernel of src/spectral.h:70-102: it carries the peak's whole weight onto
    the positive mesh, none onto the negative one, and shifts the mean of
    ln E by alpha * gamma = alpha^2 / 4 (substitute x = ln(E/E0) / alpha)."""
    P = {"alpha": 0.3, "omega0": 1e-6, "omega0_ratio": 1.0, "T": 1e-6, "Nmax": 30, "discretization": "Y",
         "Lambda": 2.0, "z": 1.0, "bandrescale": 1.0, "broaden_min": 1e-5, "broaden_min_ratio": 3.0,
         "broaden_max": 2.5, "broaden_ratio": 1.01}
    E0, wt = 1e-2, 0.7
    out = O.broaden(P, np.array([E0]), np.array([wt]), np.array([]), np.array([]))
    E = np.array([e for e, _ in out])
    A = np.array([a for _, a in out])
    pos = E > 0
    Ep, Ap = E[pos], A[pos]
    assert np.all(A[~pos] == 0.0)
    # integrate on the log mesh: dE = E d(ln E)
    lnE = np.log(Ep)
    f = Ap * Ep
    total = np.trapezoid(f, lnE)
    assert total == pytest.approx(wt, rel=1e-6)
    mean = np.trapezoid(f * lnE, lnE) / total
    assert mean == pytest.approx(math.log(E0) + P["alpha"] ** 2 / 4.0, abs=1e-6)


def test_log_bins_split_rules():
    """Bins::add (src/bins.h): a peak between bin energies e_i and e_i+1 is
    split linearly in log10 E, which keeps its weight and its mean bin
    position; peaks below the grid go to the first bin and above it to the
    last; weights below discard_immediately * E are dropped."""
    P = {"bins": 10, "emax": 10.0, "emin": 1e-5, "discard_immediately": 1e-16}
    b = O.Bins(P, 10)
    assert b.n == (1 - (-5)) * 10 + 1 and b.e[0] == pytest.approx(1e-5) and b.e[-1] == pytest.approx(10.0)
    rng = np.random.default_rng(3)
    E = 10.0 ** rng.uniform(-4.9, 0.9, 500)
    W = rng.uniform(0.1, 1.0, 500)
    b.add_many(E, W)
    pos = (np.log10(E) + 5) * 10
    assert b.w.sum() == pytest.approx(W.sum(), rel=1e-14)
    assert np.dot(b.w, np.arange(b.n)) == pytest.approx(np.dot(W, pos), rel=1e-12)
    # a peak on a bin energy lands whole in that bin
    c = O.Bins(P, 10)
    c.add_many([c.e[17]], [2.0])
    assert c.w[17] == pytest.approx(2.0, rel=1e-12) and abs(c.w.sum() - 2.0) < 1e-14
    # under- and overflow, and the discard rule
    d = O.Bins(P, 10)
    d.add_many([1e-9, 1e3, 1e-2], [0.5, 0.25, 1e-20])
    assert d.w[0] == 0.5 and d.w[-1] == 0.25 and d.w.sum() == 0.75


def test_free_moment_plateaus(tmp_path):
    """A decoupled level (V = 0) with U = 0.2, eps_d = -U/2 is a free spin
    1/2 at T << U/2: against a run whose level is pushed far above the band,
    the td columns differ by T chi = <Sz^2> = 1/4 and S = ln 2 (columns of
    src/nrg.cc:454-461, src/sym-QS.cc:12-14).  The residue is truncation: with
    the impurity doublet each band multiplet splits in two, so the same keep
    holds fewer band states (at keep 200 the entropy gap is 0.670)."""
    import nrg_cases as cases
    td = {}
    for name, U, eps in (("moment", 0.2, -0.1), ("empty", 0.0, 10.0)):
        wd = str(tmp_path / name)
        g.make_siam(wd, U, eps, 0.02, 2.0, 20, V=0.0, params={"keep": 700, "T": 1e-5})
        O.Oracle(wd).run(wd + "/out")
        td[name] = cases.read_table(wd + "/out/td")
    low = td["moment"][:, 0] < 0.01  # T << U/2
    assert low.sum() >= 6
    d_tchi = td["moment"][low, 1] - td["empty"][low, 1]
    d_s = td["moment"][low, 8] - td["empty"][low, 8]
    assert np.all(np.abs(d_tchi - 0.25) < 2e-4)
    assert np.all(np.abs(d_s - math.log(2.0)) < 3e-3)


@pytest.mark.parametrize("nntanh", [0.0, 3.0])
def test_dmnrg_shell_windows_partition_unity(nntanh):
    """N/N+2 merge of DM-NRG spectra (src/spectrumrealfreq.cc:109-185): shell
    N covers (E_min, E_max) = goodE s (1, Lambda^2) with the crossover at
    goodE s Lambda, and shell N+2 has s / Lambda, so on their overlap the
    falling window of N+2 and the rising window of N sum to one, for the
    linear ramp and for the tanh profile; the first shell keeps full weight
    above its crossover and the last below it."""
    P = {"NNtanh": nntanh}
    lam, good, s = 2.0, 2.0, 1e-3

    def shell(scale, first=False, last=False):
        lo, x, hi = good * scale, good * scale * lam, good * scale * lam ** 2
        return lambda e: O._window(P, e, lo, x, hi, first, last)

    e = np.geomspace(good * s * 1.0001, good * s * lam * 0.9999, 200)
    total = shell(s)(e) + shell(s / lam)(e)
    assert np.max(np.abs(total - 1.0)) < 1e-12
    # three shells: every energy strictly inside the covered range sums to 1
    e3 = np.geomspace(good * s / lam ** 2 * 1.0001, good * s * lam ** 2 * 0.9999, 400)
    e3 = e3[np.abs(np.log(e3 / (good * s)) / np.log(lam) - np.round(np.log(e3 / (good * s)) / np.log(lam))) > 1e-6]
    t3 = shell(s, first=True)(e3) + shell(s / lam)(e3) + shell(s / lam ** 2, last=True)(e3)
    assert np.max(np.abs(t3 - 1.0)) < 1e-12


def test_fixeps_cluster_snapping_quirks():
    """find_clusters / fix_splittings (src/splitting.cc:5-77): sorted energies
    closer than fixeps to the first of their cluster are mapped onto it; the
    last cluster of the list is not processed; the map persists across steps
    and keeps its first entry for a value; fix_splittings rewrites only mapped
    values."""
    class Host:
        P = {"fixeps": 1e-15}
        cluster_map = {}

    h = Host()
    h.cluster_map = {}
    one_b = 1.0 + 4.0 * np.finfo(float).eps
    two_b = 2.0 + 4.0 * np.finfo(float).eps
    E = np.array([0.0, 1e-16, 5e-16, 1.0, one_b, 1.5, 2.0, two_b])
    O.Oracle.find_clusters(h, E)
    assert h.cluster_map == {1e-16: 0.0, 5e-16: 0.0, one_b: 1.0}
    # a later step: 1e-16 heads a new cluster, but its old entry stays
    O.Oracle.find_clusters(h, np.array([1e-16, 3e-16, 7.0, 8.0]))
    assert h.cluster_map[1e-16] == 0.0 and h.cluster_map[3e-16] == 1e-16
    diag = {"I": O.Eig(value=np.array([5e-16, 0.7, one_b]), vec=np.eye(3), kept=3)}
    assert O.Oracle.fix_splittings(h, diag)
    assert list(diag["I"].value) == [0.0, 0.7, 1.0]


def test_noninteracting_level_lowest_excitation_is_single_particle(tmp_path):
    """U = 0: every many-body level is a sum of single-particle levels of the
    tridiagonal chain Hamiltonian (impurity, hybridisation V, Wilson chain
    zeta_n, xi_n), so at step N the lowest excitation, times SCALE(N+1), is
    the smallest |eps_k| of the impurity plus N+2 chain sites: exactly while
    nothing is truncated, and to the truncation error after."""
    info = g.make_siam(str(tmp_path), 0.0, 0.0, 0.02, 2.0, 20, params={"keep": 400, "T": 1e-3})
    o = O.Oracle(str(tmp_path))
    o.run(str(tmp_path / "out"))
    xi, zeta, V = info["xi"], info["zeta"], info["V"]
    for k, rec in enumerate(o.steps):
        N = o.Ninit + k
        L = N + 2
        H = np.zeros((L + 1, L + 1))
        H[0, 1] = H[1, 0] = V
        for i in range(L):
            H[1 + i, 1 + i] = zeta[i]
            if i + 1 < L:
                H[1 + i, 2 + i] = H[2 + i, 1 + i] = xi[i]
        eps = np.abs(np.linalg.eigvalsh(H))
        lowest_sp = np.min(eps[eps > 1e-12])
        vals = np.concatenate([e.value for e in rec.eig.values()])
        lowest_mb = np.min(vals[vals > 1e-9]) * O.SCALE(o.P, N + 1)
        truncated = any(o.steps[j].kept[I] < o.steps[j].total[I] for j in range(k) for I in o.steps[j].kept)
        tol = 2e-5 if truncated else 1e-12
        assert lowest_mb == pytest.approx(lowest_sp, rel=tol), (N, truncated)
