"""SPSU2 coefficient tables (spin SU(2), charge not conserved) derived from
spin coupling: the oracle's restatement of coefnew/spsu2/spsu2-<P>ch-*.dat
for P = 1, 2, 3 channels (src/sym-SPSU2.cc, src/nrg-recalc-SPSU2.cc).

Test infrastructure: part of the CPU checker for the CUDA path, imported only
by tests.

Same construction as qs_derive.py, with the charge dropped from the
invariants (subspaces are labelled by SS = 2S+1 alone, written (0, SS)).  A
new subspace SS of step N+1 combines an ancestor subspace SS + dSS of step N
with a spin multiplet of the added site (electrons per channel, spin s); for
one channel:

  1: site empty        (s = 0),   ancestor SS
  2: site doubly occ.  (s = 0),   ancestor SS
  3: site singly occ.  (s = 1/2), ancestor SS - 1
  4: site singly occ.  (s = 1/2), ancestor SS + 1

for two channels the five singlets, the four doublets (two ancestors each)
and the triplet (three ancestors) of the 16-state site, and for three
channels the 64 combinations of the 64-state site, in the reference's order
(COMBOS; the two spin-1/2 multiplets with one electron per channel are those
of qs_derive.py, told apart by a label).  Because the charge is not conserved, three kinds
of coupling between the chain's last site N and the added site N+1 enter
the Hamiltonian, per channel:

  hopping   xi_N     sum_s (f^dag_{N,s} f_{N+1,s} + h.c.)      (OFFDIAG)
  pairing   kappa_N  (f^dag_{N,up} f^dag_{N+1,dn}
                      - f^dag_{N,dn} f^dag_{N+1,up} + h.c.)    (ANOMALOUS)
  on-site   delta_{N+1} (f^dag_{N+1,up} f^dag_{N+1,dn} + h.c.)  (ISOSPINX)

The reference's input generator writes the on-site pairing of the odd
channels with the opposite sign along the chain (initial.m, the "sign for
isospin is inverted for f_1" of its bcsgap section), and its ISOSPINX tables
for those channels carry the opposite sign to match (channels 1 of two, and
1 but not 2 of three); the tables here follow that convention.

Each table entry is a matrix element in the site's Fock space times a
Clebsch-Gordan recoupling, divided by the coefficient of the Wigner-Eckart
theorem for the chain's reduced element <anc_i||f^dag||anc_j> that the
assembly multiplies it with.  tests/test_spsu2_tables.py checks every entry
against the reference's tables (tests/golden/spsu2_tables*.json).
"""
from __future__ import annotations

import functools

import qs_derive as qd

# (electrons per channel on the site, site spin, ancestor offset (0, dSS))
COMBOS = {
    1: [((0,), 0.0, (0, 0)), ((2,), 0.0, (0, 0)), ((1,), 0.5, (0, -1)), ((1,), 0.5, (0, 1))],
    2: [((0, 0), 0.0, (0, 0)), ((0, 2), 0.0, (0, 0)), ((1, 1), 0.0, (0, 0)), ((2, 0), 0.0, (0, 0)),
        ((2, 2), 0.0, (0, 0)), ((0, 1), 0.5, (0, -1)), ((0, 1), 0.5, (0, 1)), ((1, 0), 0.5, (0, -1)),
        ((1, 0), 0.5, (0, 1)), ((1, 2), 0.5, (0, -1)), ((1, 2), 0.5, (0, 1)), ((2, 1), 0.5, (0, -1)),
        ((2, 1), 0.5, (0, 1)), ((1, 1), 1.0, (0, -2)), ((1, 1), 1.0, (0, 0)), ((1, 1), 1.0, (0, 2))],
    3: [
        ((0, 0, 0), 0.0, (0, 0)), ((0, 0, 2), 0.0, (0, 0)), ((0, 1, 1), 0.0, (0, 0)),
        ((1, 0, 1), 0.0, (0, 0)), ((0, 2, 0), 0.0, (0, 0)), ((1, 1, 0), 0.0, (0, 0)),
        ((2, 0, 0), 0.0, (0, 0)), ((0, 2, 2), 0.0, (0, 0)), ((1, 1, 2), 0.0, (0, 0)),
        ((2, 0, 2), 0.0, (0, 0)), ((1, 2, 1), 0.0, (0, 0)), ((2, 1, 1), 0.0, (0, 0)),
        ((2, 2, 0), 0.0, (0, 0)), ((2, 2, 2), 0.0, (0, 0)), ((0, 0, 1), 0.5, (0, -1)),
        ((0, 0, 1), 0.5, (0, 1)), ((0, 1, 0), 0.5, (0, -1)), ((0, 1, 0), 0.5, (0, 1)),
        ((1, 0, 0), 0.5, (0, -1)), ((1, 0, 0), 0.5, (0, 1)), ((0, 1, 2), 0.5, (0, -1)),
        ((0, 1, 2), 0.5, (0, 1)), ((1, 0, 2), 0.5, (0, -1)), ((1, 0, 2), 0.5, (0, 1)),
        ((0, 2, 1), 0.5, (0, -1)), ((0, 2, 1), 0.5, (0, 1)), ((1, 1, 1), 0.5, (0, -1)),
        ((1, 1, 1), 0.5, (0, 1)), ((2, 0, 1), 0.5, (0, -1)), ((2, 0, 1), 0.5, (0, 1)),
        ((1, 1, 1), 0.5, (0, -1), 1), ((1, 1, 1), 0.5, (0, 1), 1), ((1, 2, 0), 0.5, (0, -1)),
        ((1, 2, 0), 0.5, (0, 1)), ((2, 1, 0), 0.5, (0, -1)), ((2, 1, 0), 0.5, (0, 1)),
        ((1, 2, 2), 0.5, (0, -1)), ((1, 2, 2), 0.5, (0, 1)), ((2, 1, 2), 0.5, (0, -1)),
        ((2, 1, 2), 0.5, (0, 1)), ((2, 2, 1), 0.5, (0, -1)), ((2, 2, 1), 0.5, (0, 1)),
        ((0, 1, 1), 1.0, (0, -2)), ((0, 1, 1), 1.0, (0, 0)), ((0, 1, 1), 1.0, (0, 2)),
        ((1, 0, 1), 1.0, (0, -2)), ((1, 0, 1), 1.0, (0, 0)), ((1, 0, 1), 1.0, (0, 2)),
        ((1, 1, 0), 1.0, (0, -2)), ((1, 1, 0), 1.0, (0, 0)), ((1, 1, 0), 1.0, (0, 2)),
        ((1, 1, 2), 1.0, (0, -2)), ((1, 1, 2), 1.0, (0, 0)), ((1, 1, 2), 1.0, (0, 2)),
        ((1, 2, 1), 1.0, (0, -2)), ((1, 2, 1), 1.0, (0, 0)), ((1, 2, 1), 1.0, (0, 2)),
        ((2, 1, 1), 1.0, (0, -2)), ((2, 1, 1), 1.0, (0, 0)), ((2, 1, 1), 1.0, (0, 2)),
        ((1, 1, 1), 1.5, (0, -3)), ((1, 1, 1), 1.5, (0, -1)), ((1, 1, 1), 1.5, (0, 1)),
        ((1, 1, 1), 1.5, (0, 3)),
    ],
}
# phases of the site multiplets (those of QS: qs_derive.SITE_SIGNS)
SITE_SIGNS = qd.SITE_SIGNS


def iso_sign(ch):
    """The reference's sign of the on-site pairing table of channel ch."""
    return 1.0 if ch % 2 == 0 else -1.0


class Tables(qd.Tables):
    def __init__(self, P=1):
        if P not in COMBOS:
            raise NotImplementedError("SPSU2 tables are derived for 1, 2 and 3 channels")
        self.P = P
        self.combos = COMBOS[P]
        self.site = qd._Site(P)
        self.mult = {}
        for c in self.combos:
            k = qd._key(c)
            if k in self.mult:
                continue
            sign = SITE_SIGNS[P].get(k if P == 3 else k[:2], 1.0)
            if P == 3 and c[0] == (1, 1, 1) and c[1] == 0.5:
                self.mult[k] = self.site.coupled_doublet(float(k[2]), sign)
            else:
                self.mult[k] = self.site.multiplet(c[0], c[1], sign)

    def _pairs(self, ss, site_ops):
        """Ordered pairs (i, j) and channels with sum over (c, op, q) of
        c <i; S S| op T^1/2_q |j; S S> (site_ops(ch) gives the list)."""
        S = (ss - 1) / 2.0
        out = []
        n = len(self.combos)
        for i in range(n):
            for j in range(n):
                if i == j:
                    continue
                for ch in range(self.P):
                    v = sum(c * self._elem(i, S, S, j, S, S, 0.5, q, op, True) for c, op, q in site_ops(ch))
                    if abs(v) > 1e-13:
                        out.append((i + 1, j + 1, ch, v))
        return out

    def offdiag(self, ss):
        # f^dag_{N,s} f_{N+1,s}: the chain creates, the site annihilates
        c = self.site.c
        return self._pairs(ss, lambda ch: [(1.0, c[2 * ch], 0.5), (1.0, c[2 * ch + 1], -0.5)])

    def anomalous(self, ss):
        # f^dag_{N,up} f^dag_{N+1,dn} - f^dag_{N,dn} f^dag_{N+1,up}
        cd = self.site.cd
        return self._pairs(ss, lambda ch: [(1.0, cd[2 * ch + 1], 0.5), (-1.0, cd[2 * ch], -0.5)])

    def isospinx(self):
        # the site's pairing operator between combinations of one ancestor,
        # in units of 2 delta (the assembly's factor); the value does not
        # depend on the subspace, so it is taken at SS = 5
        out = []
        n = len(self.combos)
        for ch in range(self.P):
            op = self.site.cd[2 * ch] @ self.site.cd[2 * ch + 1]
            op = op + op.T
            for i in range(n):
                for j in range(i + 1, n):
                    if self.combos[i][2] != self.combos[j][2]:
                        continue
                    v = self._elem(i, 2.0, 2.0, j, 2.0, 2.0, None, 0.0, op, False)
                    if abs(v) > 1e-13:
                        out.append((i + 1, j + 1, ch, iso_sign(ch) * v / 2.0))
        return out

    def diag(self):
        return [(i + 1, ch, float(c[0][ch])) for ch in range(self.P) for i, c in enumerate(self.combos)]

    def recalc_f(self, Ip):
        out = []
        for dss in (1, -1):
            I1 = (0, Ip[1] + dss)
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

    def doublet(self, I1):
        ss1 = I1[1]
        out = [((0, ss1 + 1), self._chain_op(I1, (0, ss1 + 1), 0.5, True))]
        if ss1 > 1:
            out.append(((0, ss1 - 1), self._chain_op(I1, (0, ss1 - 1), 0.5, True)))
        return out

    def triplet(self, I1):
        ss1 = I1[1]
        out = [((0, ss1), self._chain_op(I1, (0, ss1), 1.0, False)),
               ((0, ss1 + 2), self._chain_op(I1, (0, ss1 + 2), 1.0, False))]
        if ss1 > 2:
            out.append(((0, ss1 - 2), self._chain_op(I1, (0, ss1 - 2), 1.0, False)))
        return out


@functools.lru_cache(maxsize=None)
def tables(P=1):
    return Tables(P)
