"""QS coefficient tables derived from spin coupling (the oracle's restatement
of coefnew/qs/qs-<P>ch-*.dat for P = 1, 2, 3 channels).

Test infrastructure: part of the CPU checker for the CUDA path, imported only
by tests, smoke() and the bench's CPU baseline.

The reference ships the tables as Mathematica output (coefnew/qs/*.dat,
included by src/sym-QS.cc:38-68 and src/nrg-recalc-QS.cc).  Here they are
computed from their definition instead:

* a new subspace I = (Q, SS) of step N+1 is spanned, for each combination i,
  by the states  sum_{m_a, m_s} <S_a m_a; s_i m_s | S M> |site_i m_s> |anc_i m_a>
  where anc_i = I + In[i] is a subspace of step N (spin S_a) and site_i a spin
  multiplet of the added site (spin s_i, fixed electron number per channel);
* fermion operators of the added site stand to the left of those of the
  chain, so an odd operator of the chain acting through the site picks up
  (-1)^(electrons on the site);
* operators of the chain enter through reduced matrix elements in the
  Wigner-Eckart normalisation  <S1 M1|T^k_q|S2 M2> = <S2 M2; k q|S1 M1> <S1||T||S2>.

Each table entry is then a matrix element computed numerically in the
64-, 16- or 4-state Fock space of the site (three, two or one channels),
divided by the Clebsch-Gordan coefficient of the Wigner-Eckart theorem.  The
phases of the site multiplets are conventions; SITE_SIGNS fixes them to the
reference's.  tests/test_qs_tables.py checks every entry against the
reference's tables (tests/golden/).
"""
from __future__ import annotations

import functools
import math

import numpy as np

# Combinations of a new subspace (1-based index = position + 1):
# (electrons per channel on the site, site spin, In = ancestor - subspace[,
# label]).  With three channels the site has two spin-1/2 multiplets with one
# electron in each channel: label 0 couples channels 0 and 1 to spin 0, label
# 1 to spin 1, and either with channel 2 to spin 1/2 (the reference's basis;
# its tables of coefnew/qs/qs-3ch-*.dat fix it).
COMBOS = {
    1: [((0,), 0.0, (1, 0)), ((1,), 0.5, (0, -1)), ((1,), 0.5, (0, 1)), ((2,), 0.0, (-1, 0))],
    2: [((0, 0), 0.0, (2, 0)), ((0, 1), 0.5, (1, -1)), ((0, 1), 0.5, (1, 1)), ((1, 0), 0.5, (1, -1)),
        ((1, 0), 0.5, (1, 1)), ((0, 2), 0.0, (0, 0)), ((1, 1), 0.0, (0, 0)), ((2, 0), 0.0, (0, 0)),
        ((1, 1), 1.0, (0, -2)), ((1, 1), 1.0, (0, 0)), ((1, 1), 1.0, (0, 2)), ((1, 2), 0.5, (-1, -1)),
        ((1, 2), 0.5, (-1, 1)), ((2, 1), 0.5, (-1, -1)), ((2, 1), 0.5, (-1, 1)), ((2, 2), 0.0, (-2, 0))],
    3: [
        ((0, 0, 0), 0.0, (3, 0)), ((0, 0, 1), 0.5, (2, -1)), ((0, 0, 1), 0.5, (2, 1)),
        ((0, 1, 0), 0.5, (2, -1)), ((0, 1, 0), 0.5, (2, 1)), ((1, 0, 0), 0.5, (2, -1)),
        ((1, 0, 0), 0.5, (2, 1)), ((0, 0, 2), 0.0, (1, 0)), ((0, 1, 1), 0.0, (1, 0)),
        ((1, 0, 1), 0.0, (1, 0)), ((0, 2, 0), 0.0, (1, 0)), ((1, 1, 0), 0.0, (1, 0)),
        ((2, 0, 0), 0.0, (1, 0)), ((0, 1, 1), 1.0, (1, -2)), ((0, 1, 1), 1.0, (1, 0)),
        ((0, 1, 1), 1.0, (1, 2)), ((1, 0, 1), 1.0, (1, -2)), ((1, 0, 1), 1.0, (1, 0)),
        ((1, 0, 1), 1.0, (1, 2)), ((1, 1, 0), 1.0, (1, -2)), ((1, 1, 0), 1.0, (1, 0)),
        ((1, 1, 0), 1.0, (1, 2)), ((0, 1, 2), 0.5, (0, -1)), ((0, 1, 2), 0.5, (0, 1)),
        ((1, 0, 2), 0.5, (0, -1)), ((1, 0, 2), 0.5, (0, 1)), ((0, 2, 1), 0.5, (0, -1)),
        ((0, 2, 1), 0.5, (0, 1)), ((1, 1, 1), 0.5, (0, -1)), ((1, 1, 1), 0.5, (0, 1)),
        ((2, 0, 1), 0.5, (0, -1)), ((2, 0, 1), 0.5, (0, 1)), ((1, 1, 1), 0.5, (0, -1), 1),
        ((1, 1, 1), 0.5, (0, 1), 1), ((1, 2, 0), 0.5, (0, -1)), ((1, 2, 0), 0.5, (0, 1)),
        ((2, 1, 0), 0.5, (0, -1)), ((2, 1, 0), 0.5, (0, 1)), ((1, 1, 1), 1.5, (0, -3)),
        ((1, 1, 1), 1.5, (0, -1)), ((1, 1, 1), 1.5, (0, 1)), ((1, 1, 1), 1.5, (0, 3)),
        ((0, 2, 2), 0.0, (-1, 0)), ((1, 1, 2), 0.0, (-1, 0)), ((2, 0, 2), 0.0, (-1, 0)),
        ((1, 2, 1), 0.0, (-1, 0)), ((2, 1, 1), 0.0, (-1, 0)), ((2, 2, 0), 0.0, (-1, 0)),
        ((1, 1, 2), 1.0, (-1, -2)), ((1, 1, 2), 1.0, (-1, 0)), ((1, 1, 2), 1.0, (-1, 2)),
        ((1, 2, 1), 1.0, (-1, -2)), ((1, 2, 1), 1.0, (-1, 0)), ((1, 2, 1), 1.0, (-1, 2)),
        ((2, 1, 1), 1.0, (-1, -2)), ((2, 1, 1), 1.0, (-1, 0)), ((2, 1, 1), 1.0, (-1, 2)),
        ((1, 2, 2), 0.5, (-2, -1)), ((1, 2, 2), 0.5, (-2, 1)), ((2, 1, 2), 0.5, (-2, -1)),
        ((2, 1, 2), 0.5, (-2, 1)), ((2, 2, 1), 0.5, (-2, -1)), ((2, 2, 1), 0.5, (-2, 1)),
        ((2, 2, 2), 0.0, (-3, 0)),
    ],
}

# Sign of each site multiplet relative to the highest-weight state whose first
# nonzero amplitude (occupation bit order: channel-major, spin up first) is
# positive, with c^dag operators applied in increasing mode order; for the two
# coupled doublets of three channels, relative to the coupled state
# sum <S01 m01; 1/2 mc|1/2 1/2> c^dag_{2,mc} |S01 m01> with
# |S01 m01> = sum <1/2 ma; 1/2 mb|S01 m01> c^dag_{0,ma} c^dag_{1,mb} |0>.
# Three-channel keys carry the label.
SITE_SIGNS = {
    1: {((2,), 0.0): -1.0},
    2: {((2, 0), 0.0): -1.0, ((0, 2), 0.0): -1.0, ((1, 1), 1.0): -1.0, ((1, 2), 0.5): -1.0,
        ((2, 1), 0.5): -1.0},
    3: {
        ((0, 0, 2), 0.0, 0): -1.0, ((0, 1, 1), 1.0, 0): -1.0,
        ((0, 1, 2), 0.5, 0): -1.0, ((0, 2, 0), 0.0, 0): -1.0,
        ((0, 2, 1), 0.5, 0): -1.0, ((1, 0, 1), 1.0, 0): -1.0,
        ((1, 0, 2), 0.5, 0): -1.0, ((1, 1, 0), 1.0, 0): -1.0,
        ((1, 1, 1), 0.5, 0): -1.0, ((1, 1, 1), 0.5, 1): -1.0,
        ((1, 1, 1), 1.5, 0): -1.0, ((1, 1, 2), 0.0, 0): -1.0,
        ((1, 2, 0), 0.5, 0): -1.0, ((1, 2, 1), 0.0, 0): -1.0,
        ((2, 0, 0), 0.0, 0): -1.0, ((2, 0, 1), 0.5, 0): -1.0,
        ((2, 1, 0), 0.5, 0): -1.0, ((2, 1, 1), 0.0, 0): -1.0,
        ((2, 2, 2), 0.0, 0): -1.0,
    },
}


def cg(j1, m1, j2, m2, J, M):
    """Clebsch-Gordan coefficient <j1 m1; j2 m2 | J M> (Racah's formula)."""
    if abs(m1 + m2 - M) > 1e-9 or not (abs(j1 - j2) - 1e-9 <= J <= j1 + j2 + 1e-9):
        return 0.0
    if abs(m1) > j1 + 1e-9 or abs(m2) > j2 + 1e-9 or abs(M) > J + 1e-9:
        return 0.0

    def lf(x):
        return math.lgamma(round(x) + 1)

    pre = 0.5 * (math.log(2 * J + 1) + lf(J + j1 - j2) + lf(J - j1 + j2) + lf(j1 + j2 - J) - lf(j1 + j2 + J + 1)
                 + lf(J + M) + lf(J - M) + lf(j1 - m1) + lf(j1 + m1) + lf(j2 - m2) + lf(j2 + m2))
    s = 0.0
    kmax = int(round(min(j1 + j2 - J, j1 - m1, j2 + m2)))
    kmin = int(round(max(0.0, j2 - J - m1, j1 - J + m2)))
    for k in range(kmin, kmax + 1):
        den = lf(k) + lf(j1 + j2 - J - k) + lf(j1 - m1 - k) + lf(j2 + m2 - k) + lf(J - j2 + m1 + k) + lf(J - j1 - m2 + k)
        s += (-1) ** k * math.exp(pre - den)
    return s


class _Site:
    """Fock space of one added site: 2P modes, mode 2*ch + (0 up, 1 down)."""

    def __init__(self, P):
        self.P = P
        self.nm = 2 * P
        self.dim = 1 << self.nm
        self.cd = [self._cdag(k) for k in range(self.nm)]
        self.c = [x.T for x in self.cd]
        self.Sp = sum(self.cd[2 * ch] @ self.c[2 * ch + 1] for ch in range(P))
        self.Sz = np.diag([sum(0.5 * (((b >> (2 * ch)) & 1) - ((b >> (2 * ch + 1)) & 1)) for ch in range(P))
                           for b in range(self.dim)])

    def _cdag(self, k):
        M = np.zeros((self.dim, self.dim))
        for b in range(self.dim):
            if not (b >> k) & 1:
                M[b | (1 << k), b] = (-1) ** bin(b & ((1 << k) - 1)).count("1")
        return M

    def multiplet(self, occ, s, sign):
        """{M: state vector} of the spin-s multiplet with occupations occ."""
        idx = [b for b in range(self.dim)
               if all(bin((b >> (2 * ch)) & 3).count("1") == occ[ch] for ch in range(self.P))
               and abs(self.Sz[b, b] - s) < 1e-9]
        sub = np.zeros((self.dim, len(idx)))
        for t, b in enumerate(idx):
            sub[b, t] = 1.0
        _, sv, vt = np.linalg.svd(self.Sp @ sub)
        null = vt[int(np.sum(sv > 1e-9)):].T
        if null.shape[1] != 1:
            raise ValueError("site multiplet (%s, %s) is not unique" % (occ, s))
        hw = sub @ null[:, 0]
        hw = hw * np.sign(hw[np.argmax(np.abs(hw) > 1e-9)]) * sign
        out = {s: hw}
        m, v = s, hw
        while m > -s + 1e-9:
            v = self.Sp.T @ v / math.sqrt((s + m) * (s - m + 1))
            m -= 1
            out[m] = v
        return out

    def coupled_doublet(self, s01, sign):
        """{M: state} of the three-channel spin-1/2 multiplet with one electron
        per channel whose channels 0 and 1 couple to spin s01."""
        vac = np.zeros(self.dim)
        vac[0] = 1.0

        def cdag(ch, m):
            return self.cd[2 * ch + (0 if m > 0 else 1)]
        hw = np.zeros(self.dim)
        for m01 in np.arange(-s01, s01 + 0.5, 1.0):
            pair = np.zeros(self.dim)
            for ma in (0.5, -0.5):
                c = cg(0.5, ma, 0.5, m01 - ma, s01, m01)
                if c:
                    pair += c * (cdag(0, ma) @ cdag(1, m01 - ma) @ vac)
            g = cg(s01, m01, 0.5, 0.5 - m01, 0.5, 0.5)
            if g:
                hw += g * (cdag(2, 0.5 - m01) @ pair)
        hw = hw / np.linalg.norm(hw) * sign
        return {0.5: hw, -0.5: self.Sp.T @ hw}


def _key(c):
    """Site multiplet of a combination: (occupations, spin, label)."""
    return (c[0], c[1], c[3] if len(c) > 3 else 0)


class Tables:
    """All QS tables for P channels."""

    def __init__(self, P):
        if P not in COMBOS:
            raise NotImplementedError("QS tables are derived for 1, 2 and 3 channels")
        self.P = P
        self.combos = COMBOS[P]
        self.site = _Site(P)
        self.mult = {}
        for c in self.combos:
            k = _key(c)
            if k in self.mult:
                continue
            sign = SITE_SIGNS[P].get(k if P == 3 else k[:2], 1.0)
            if P == 3 and c[0] == (1, 1, 1) and c[1] == 0.5:
                self.mult[k] = self.site.coupled_doublet(float(k[2]), sign)
            else:
                self.mult[k] = self.site.multiplet(c[0], c[1], sign)

    # ---- helpers ----
    def anc(self, i, I):
        In = self.combos[i][2]
        return (I[0] + In[0], I[1] + In[1])

    def nsite(self, i):
        return sum(self.combos[i][0])

    def _state(self, i, S, M):
        s, In = self.combos[i][1], self.combos[i][2]
        Sa = S + In[1] / 2.0
        if Sa < -1e-9 or not (abs(Sa - s) - 1e-9 <= S <= Sa + s + 1e-9):
            return None
        out = {}
        for ms, vec in self.mult[_key(self.combos[i])].items():
            ma = M - ms
            if abs(ma) > Sa + 1e-9:
                continue
            c = cg(Sa, ma, s, ms, S, M)
            if c != 0.0:
                key = int(round(2 * ma))
                out[key] = out.get(key, 0.0) + c * vec
        return out, Sa

    def _elem(self, i, S1, M1, j, S2, M2, rank, q, site_op, odd):
        """<i;S1 M1| site_op T^rank_q(chain) |j;S2 M2>, chain reduced element 1."""
        a, b = self._state(i, S1, M1), self._state(j, S2, M2)
        if a is None or b is None:
            return 0.0
        (sa, Sa1), (sb, Sa2) = a, b
        tot = 0.0
        for ma1, v1 in sa.items():
            for ma2, v2 in sb.items():
                if rank is None:
                    if ma1 != ma2 or abs(Sa1 - Sa2) > 1e-9:
                        continue
                    ae = 1.0
                else:
                    ae = cg(Sa2, ma2 / 2.0, rank, q, Sa1, ma1 / 2.0)
                    if ae == 0.0:
                        continue
                w = v2 if site_op is None else site_op @ v2
                sgn = (-1.0) ** self.nsite(i) if odd else 1.0
                tot += ae * float(v1 @ w) * sgn
        return tot

    def _reduced(self, I1, Ip, rank, comp):
        S1, Sp = (I1[1] - 1) / 2.0, (Ip[1] - 1) / 2.0
        for q2 in range(int(-2 * rank), int(2 * rank) + 1, 2):
            q = q2 / 2.0
            M2 = S1 - q
            if abs(M2) > Sp + 1e-9:
                continue
            c = cg(Sp, M2, rank, q, S1, S1)
            if abs(c) > 1e-12:
                return comp(q, S1, Sp, M2) / c
        return 0.0

    # ---- tables (same shapes as the closed forms of qs.py) ----
    def offdiag(self, ss):
        S = (ss - 1) / 2.0
        out = []
        n = len(self.combos)
        for i in range(n):
            for j in range(i + 1, n):
                for ch in range(self.P):
                    v = sum(self._elem(i, S, S, j, S, S, 0.5, q, self.site.c[2 * ch + sig], True)
                            for sig, q in ((0, 0.5), (1, -0.5)))
                    if abs(v) > 1e-13:
                        out.append((i + 1, j + 1, ch, v))
        return out

    def diag(self):
        return [(i + 1, ch, float(c[0][ch])) for ch in range(self.P) for i, c in enumerate(self.combos)]

    def recalc_f(self, Ip):
        out = []
        for dss in (1, -1):
            I1 = (Ip[0] + 1, Ip[1] + dss)
            if I1[1] < 1:
                continue
            for ch in range(self.P):
                rows = []
                for i1 in range(len(self.combos)):
                    for ip in range(len(self.combos)):
                        A = self.anc(i1, I1)
                        if A != self.anc(ip, Ip) or A[1] < 1:
                            continue

                        def comp(q, S1, Sp, M2, i1=i1, ip=ip, ch=ch):
                            op = self.site.cd[2 * ch + (0 if q > 0 else 1)]
                            return self._elem(i1, S1, S1, ip, Sp, M2, None, 0.0, op, False)
                        v = self._reduced(I1, Ip, 0.5, comp)
                        if abs(v) > 1e-13:
                            rows.append((i1 + 1, ip + 1, v))
                out.append((I1, ch, rows))
        return out

    def _chain_op(self, I1, Ip, rank, odd):
        rows = []
        for i1 in range(len(self.combos)):
            for ip in range(len(self.combos)):
                if _key(self.combos[i1]) != _key(self.combos[ip]):
                    continue
                if self.anc(i1, I1)[1] < 1 or self.anc(ip, Ip)[1] < 1:
                    continue

                def comp(q, S1, Sp, M2, i1=i1, ip=ip):
                    return self._elem(i1, S1, S1, ip, Sp, M2, rank, q, None, odd)
                v = self._reduced(I1, Ip, rank, comp)
                if abs(v) > 1e-13:
                    rows.append((i1 + 1, ip + 1, v))
        return rows

    def doublet(self, I1):
        q1, ss1 = I1
        out = [((q1 - 1, ss1 + 1), self._chain_op(I1, (q1 - 1, ss1 + 1), 0.5, True))]
        if ss1 > 1:
            out.append(((q1 - 1, ss1 - 1), self._chain_op(I1, (q1 - 1, ss1 - 1), 0.5, True)))
        return out

    def triplet(self, I1):
        q1, ss1 = I1
        out = [((q1, ss1), self._chain_op(I1, (q1, ss1), 1.0, False)),
               ((q1, ss1 + 2), self._chain_op(I1, (q1, ss1 + 2), 1.0, False))]
        if ss1 > 2:
            out.append(((q1, ss1 - 2), self._chain_op(I1, (q1, ss1 - 2), 1.0, False)))
        return out


@functools.lru_cache(maxsize=None)
def tables(P):
    return Tables(P)


@functools.lru_cache(maxsize=4096)
def offdiag(P, ss):
    return tables(P).offdiag(ss)


@functools.lru_cache(maxsize=4096)
def recalc_f(P, Ip):
    return tables(P).recalc_f(Ip)


@functools.lru_cache(maxsize=4096)
def doublet(P, I1):
    return tables(P).doublet(I1)


@functools.lru_cache(maxsize=4096)
def triplet(P, I1):
    return tables(P).triplet(I1)
