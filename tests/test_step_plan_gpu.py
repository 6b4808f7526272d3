"""The step-level C ABI (nrgb_step, nrgb_recalc): the caller keeps the NRG
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
