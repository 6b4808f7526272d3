"""The step-level C ABI (nrgb_step, nrgb_recalc, nrgb_dm_backward,
nrgb_spectrum_fdm, nrgb_spectrum_dmnrg): the caller keeps the NRG
driver and the symmetry plug-in, as the reference's nrg_iterate
(src/nrg.cc:3043-3051) and Symmetry classes would, and hands the device one
step at a time as flat task lists.  Here the caller is this test, playing the
reference's host side for the QS symmetry with the restated QS tables
(oracle/qs.py, the checker's copy of coefnew/qs): per step it lists the
diagonal terms (sqrt(Lambda) E_prev and the zeta shifts), the off-diagonal
<f> terms of offdiag_build and, after the step, the recalc_f terms of the new
<f> blocks.  The device's kept counts must equal the oracle's sweep step by
step, the ground-state energies agree to 1e-12 relative, and the
thermodynamics built from the device's Boltzmann sums agree with the
oracle's td at the FP64 targets."""
import math
import os

import numpy as np
import pytest

import nrg_cases as cases
import nrg_oracle as O
import qs

pytestmark = pytest.mark.gpu


def _td_row(T, blocks, zs, betabar):
    Z = E = E2 = trSZ = trQ = trQ2 = 0.0
    for (I, _), (z, e, e2) in zip(blocks, zs):
        m = qs.mult(I)
        Z += m * z
        E += m * e
        E2 += m * e2
        trSZ += m * z * (I[1] ** 2 - 1) / 12.0
        trQ += m * z * I[0]
        trQ2 += m * z * I[0] ** 2
    E /= Z
    E2 /= Z
    C = E2 - E * E
    F = -math.log(Z)
    return [T, trSZ / Z, trQ / Z, trQ2 / Z, E, E2, C, F, E - F]


@pytest.mark.parametrize("name", ["siam_ph", "kondo2ch"])
def test_step_plan_reproduces_the_oracle_sweep(tmp_path, name):
    import nrgb
    wd = cases.make_case(name, str(tmp_path / "in"))
    o = O.Oracle(wd)
    o.run(None)
    P, D = o.P, o.D
    nch = D.channels
    ctx = nrgb.Context(0)
    try:
        ctx.run_begin()
        prev = {I: (ctx.mat_upload(np.asarray(v, dtype=float).reshape(-1, 1)), len(v)) for I, v in D.energies.items()}
        opch = [{k: ctx.mat_upload(np.asarray(M, dtype=float)) for k, M in b.items()} for b in D.opch]
        rules = {"fixeps": P["fixeps"], "keepenergy": P["keepenergy"], "keep": P["keep"], "keepmin": P["keepmin"],
                 "safeguard": P["safeguard"], "safeguardmax": P["safeguardmax"], "betabar": P["betabar"]}
        td = []
        for N in range(o.Ninit, o.Nmax):
            last = N + 1 == o.Nmax
            scale1 = O.SCALE(P, N + 1)
            subs = o.subspaces({I: O.Eig(value=None, vec=None, kept=k) for I, (_, k) in prev.items()})
            blocks = []
            for I in subs:
                r = [prev[a][1] if (qs.triangle(I, a, o.QN[i]) and a in prev) else 0
                     for i, a in enumerate(o.ancestors(I))]
                if sum(r):
                    blocks.append((I, r))
            dims = [sum(r) for _, r in blocks]
            dterms, oterms = [], []
            for b, (I, r) in enumerate(blocks):
                anc = o.ancestors(I)
                off = np.concatenate([[0], np.cumsum(r)]).astype(int)
                for i in range(o.combs):
                    if not r[i]:
                        continue
                    shift = sum(o.zeta(N + 1, ch) * (number - 1.0) / scale1
                                for (ii, ch, number) in qs.diag_terms(nch) if ii - 1 == i)
                    dterms.append(nrgb.DiagTerm(b, int(off[i]), r[i], prev[anc[i]][0], math.sqrt(P["Lambda"]), shift))
                for (i, j, ch, factor) in qs.offdiag_terms(nch, I[1]):
                    i0, j0 = i - 1, j - 1
                    if not (r[i0] and r[j0]):
                        continue
                    fs = factor * o.xi(N, ch) / scale1
                    if abs(fs) < 1e-8:
                        continue
                    src = opch[ch][(anc[i0], anc[j0])]
                    oterms.append(nrgb.OffdiagTerm(b, int(off[i0]), int(off[j0]), r[i0], r[j0], src, fs))
            rules["keep_all"] = 1 if (last and (P["fdm"] or P["cfs"]) and not P["lastalloverride"]) else 0
            zh, wh, kept, egs, zs = ctx.step(dims, dterms, oterms, rules)
            rec = o.steps[N - o.Ninit]
            assert [rec.kept[I] for I, _ in blocks] == kept, ("kept", N)
            assert abs(egs - rec.Egs) <= 1e-12 * max(1.0, abs(rec.Egs)), ("Egs", N, egs, rec.Egs)
            td.append(_td_row(scale1 / P["betabar"], blocks, zs, P["betabar"]))
            if last:
                break
            # <f> of the new site: recalc_f tables, identity terms
            idx = {I: b for b, (I, _) in enumerate(blocks)}
            offs = {I: np.concatenate([[0], np.cumsum(r)]).astype(int) for I, r in blocks}
            outs, terms, keys = [], [], []
            for Ip, rp in blocks:
                for (I1, ch, rows) in qs.recalc_f_tables(nch, Ip):
                    if I1 not in idx:
                        continue
                    k1, kp = kept[idx[I1]], kept[idx[Ip]]
                    if k1 == 0 or kp == 0:
                        continue
                    t0 = len(terms)
                    r1s = dict(blocks)[I1]
                    for (i1, ip, factor) in rows:
                        a, c = r1s[i1 - 1], rp[ip - 1]
                        if a and c:
                            terms.append(nrgb.RecalcTerm(zh[idx[I1]], int(offs[I1][i1 - 1]), a,
                                                         zh[idx[Ip]], int(offs[Ip][ip - 1]), c, -1, factor))
                    outs.append(nrgb.RecalcOut(k1, kp, t0, len(terms) - t0))
                    keys.append((ch, I1, Ip))
            hs = ctx.recalc(outs, terms)
            opch = [dict() for _ in range(nch)]
            for (ch, I1, Ip), h in zip(keys, hs):
                opch[ch][(I1, Ip)] = h
            prev = {I: (wh[b], kept[b]) for b, (I, _) in enumerate(blocks)}
        ref = np.array(o.td_rows[1:] if P["calc0"] else o.td_rows)
        got = np.array(td)
        assert got.shape == ref.shape
        assert np.all(np.abs(got - ref) <= cases.RTOL_TD * np.abs(ref) + cases.ATOL_TD), \
            float(np.max(np.abs(got - ref)))
    finally:
        ctx.close()


def test_dm_backward_matches_numpy():
    """nrgb_dm_backward: each output r1 x rp is the sum over its terms of
    factor * Z1[off1:off1+r1, :k1] @ rho[:k1, :kp] @ Zp[offp:offp+rp, :kp]^T
    (the density-matrix step from step N+1 back to step N), with empty
    outputs and terms of zero kept states."""
    import nrgb
    rng = np.random.default_rng(3)
    ctx = nrgb.Context(0)
    try:
        Z = {n: rng.standard_normal((n, n)) for n in (12, 10, 7)}
        R = {k: rng.standard_normal((k, k)) for k in (5, 4, 3)}
        hz = {n: ctx.mat_upload(M) for n, M in Z.items()}
        hr = {k: ctx.mat_upload(M) for k, M in R.items()}
        terms = [nrgb.DmTerm(hz[12], 2, 5, hz[10], 1, 4, hr[5], 0.7),
                 nrgb.DmTerm(hz[7], 0, 3, hz[7], 4, 3, hr[3], -1.3),
                 nrgb.DmTerm(hz[12], 0, 4, hz[12], 6, 4, hr[4], 2.0),
                 nrgb.DmTerm(hz[10], 0, 0, hz[10], 0, 4, hr[4], 1.0)]   # no kept states: no term
        outs = [nrgb.DmOut(3, 6, 0, 1), nrgb.DmOut(3, 3, 1, 1), nrgb.DmOut(5, 4, 2, 2), nrgb.DmOut(0, 4, 0, 0)]
        got = [ctx.mat_download(h) for h in ctx.dm_backward(outs, terms)]
    finally:
        ctx.close()

    def ref(t, r1, rp):
        Z1 = {hz[n]: Z[n] for n in Z}[t.z1]
        Zp = {hz[n]: Z[n] for n in Z}[t.zp]
        rho = {hr[k]: R[k] for k in R}[t.rho]
        if t.k1 == 0 or t.kp == 0:
            return np.zeros((r1, rp))
        return t.factor * Z1[t.off1:t.off1 + r1, :t.k1] @ rho[:t.k1, :t.kp] @ Zp[t.offp:t.offp + rp, :t.kp].T
    for o, G in zip(outs, got):
        assert G.shape == (o.r1, o.rp)
        want = sum((ref(terms[t], o.r1, o.rp) for t in range(o.term0, o.term0 + o.nterms)), np.zeros((o.r1, o.rp)))
        assert np.max(np.abs(G - want), initial=0.0) <= 1e-13 * max(1.0, np.max(np.abs(want), initial=0.0))


@pytest.mark.parametrize("fermionic", [1, 0])
def test_spectrum_fdm_matches_oracle_binning(fermionic):
    """nrgb_spectrum_fdm: the FDM greater and lesser sums of random block
    pairs with kept and discarded states (src/spec_FDM.cc:41-119, as the
    oracle states them) binned by the oracle's logarithmic bins
    (src/bins.h:22-131), against the device's, per bin at 1e-12 of the
    largest bin; a last-step pair (no kept states) included."""
    import nrgb
    rng = np.random.default_rng(9)
    T, wn, bpd, emin, emax = 0.05, 0.37, 10, 1e-4, 10.0
    blocks = {0: (7, 3), 1: (5, 2), 2: (6, 0)}   # dim, kept
    E = {b: np.sort(rng.uniform(0.0, 2.0, d)) for b, (d, _) in blocks.items()}
    rho = {b: (lambda M: M @ M.T)(rng.standard_normal((k, k))) for b, (_, k) in blocks.items()}
    pairs_np = [(0, 1, 0.8), (1, 0, 1.5), (2, 2, 1.0), (1, 2, 0.6)]
    ops = {}
    for i, j, _ in pairs_np:
        ops[(i, j)] = (rng.standard_normal((blocks[j][0], blocks[i][0])), rng.standard_normal((blocks[j][0], blocks[i][0])))
    ctx = nrgb.Context(0)
    try:
        h = {}
        for b in blocks:
            h[("e", b)] = ctx.mat_upload(E[b][None, :])
            h[("r", b)] = ctx.mat_upload(rho[b]) if blocks[b][1] else -1
        pairs = []
        for i, j, sf in pairs_np:
            A, B = ops[(i, j)]
            pairs.append(nrgb.FdmPair(ctx.mat_upload(A), ctx.mat_upload(B), h[("r", i)], h[("r", j)], h[("e", i)],
                                      h[("e", j)], blocks[i][1], blocks[j][1], sf))
        pos, neg = ctx.spectrum_fdm(pairs, T, wn, fermionic, bpd, emin, emax)
    finally:
        ctx.close()
    P = {"bins": bpd, "emin": emin, "emax": emax, "discard_immediately": 1e-16}
    cs = O.ChainSpectrum(P, 10)
    sign = -1.0 if fermionic else 1.0
    for i, j, sf in pairs_np:
        A, B = ops[(i, j)]
        Ei, Ej = E[i], E[j]
        reti, retj = blocks[i][1], blocks[j][1]
        ri, rj = rho[i], rho[j]
        alli, allj = len(Ei), len(Ej)
        dE = Ej[:, None] - Ei[None, :]
        AB = A * B
        gt = sf * AB * wn * np.exp(-Ei / T)[None, :]
        m = np.zeros_like(AB, dtype=bool)
        m[:, reti:] = True
        cs.add(dE[m], gt[m])
        if reti > 0:
            cs.add(dE[retj:, :reti], sf * A[retj:, :reti] * (B[:allj, :reti] @ ri)[retj:, :])
        ls = sf * AB * (-sign) * wn * np.exp(-Ej / T)[:, None]
        m = np.zeros_like(AB, dtype=bool)
        m[retj:, reti:] = True
        cs.add(dE[m], ls[m])
        if retj > 0:
            cs.add(dE[:retj, reti:], sf * A[:retj, reti:] * (rj @ B[:retj, :alli])[:, reti:] * (-sign))
        m = np.zeros_like(AB, dtype=bool)
        m[retj:, :reti] = True
        cs.add(dE[m], ls[m])
    assert pos.shape == cs.pos.w.shape and neg.shape == cs.neg.w.shape
    wmax = max(np.max(np.abs(cs.pos.w)), np.max(np.abs(cs.neg.w)))
    assert wmax > 0
    assert np.max(np.abs(pos - cs.pos.w)) <= 1e-12 * wmax
    assert np.max(np.abs(neg - cs.neg.w)) <= 1e-12 * wmax


@pytest.mark.parametrize("fermionic", [1, 0])
def test_spectrum_dmnrg_matches_oracle_binning(fermionic):
    """nrgb_spectrum_dmnrg: the DM-NRG weights of random block pairs over
    their kept states (src/spec_DMNRG.cc:13-52, as the oracle states them),
    windowed and binned by the oracle's logarithmic bins, against the
    device's, per bin at 1e-12 of the largest bin."""
    import nrgb
    rng = np.random.default_rng(13)
    scale, wmin, wmax, bpd, emin, emax = 0.3, 0.2, 1.6, 10, 1e-4, 10.0
    blocks = {0: 6, 1: 4, 2: 5}   # kept states
    E = {b: np.sort(rng.uniform(0.0, 3.0, k + 2)) for b, k in blocks.items()}
    rho = {b: (lambda M: M @ M.T)(rng.standard_normal((k, k))) for b, k in blocks.items()}
    pairs_np = [(0, 1, 0.8), (1, 0, 1.5), (2, 2, 1.0), (1, 2, 0.6)]   # (p, 1, factor)
    ops = {(p, b1): (rng.standard_normal((blocks[b1] + 1, blocks[p] + 2)),
                     rng.standard_normal((blocks[b1] + 1, blocks[p] + 2))) for p, b1, _ in pairs_np}
    ctx = nrgb.Context(0)
    try:
        he = {b: ctx.mat_upload(E[b][None, :]) for b in blocks}
        hr = {b: ctx.mat_upload(rho[b]) for b in blocks}
        pairs = [nrgb.DmnrgPair(ctx.mat_upload(ops[(p, b1)][0]), ctx.mat_upload(ops[(p, b1)][1]), hr[b1], hr[p],
                                he[b1], he[p], sf) for p, b1, sf in pairs_np]
        pos, neg = ctx.spectrum_dmnrg(pairs, scale, wmin, wmax, fermionic, bpd, emin, emax)
    finally:
        ctx.close()
    cs = O.ChainSpectrum({"bins": bpd, "emin": emin, "emax": emax, "discard_immediately": 1e-16}, 10)
    sign = -1.0 if fermionic else 1.0
    for p, b1, sf in pairs_np:
        dimp, dim1 = blocks[p], blocks[b1]
        A_ = ops[(p, b1)][0][:dim1, :dimp]
        B_ = ops[(p, b1)][1][:dim1, :dimp]
        sumA = B_ @ rho[p].T
        sumB = rho[b1] @ A_
        w = sf * (sumA * A_ + (-sign) * sumB * B_)
        dE = E[b1][:dim1, None] - E[p][None, :dimp]
        ok = (np.abs(dE) >= wmin) & (np.abs(dE) <= wmax)
        cs.add(scale * dE[ok], w[ok])
    wmx = max(np.max(np.abs(cs.pos.w)), np.max(np.abs(cs.neg.w)))
    assert wmx > 0
    assert np.max(np.abs(pos - cs.pos.w)) <= 1e-12 * wmx
    assert np.max(np.abs(neg - cs.neg.w)) <= 1e-12 * wmx
