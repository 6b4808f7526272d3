"""SPSU2 coefficient tables (spin SU(2), charge not conserved) derived from
spin coupling: the oracle's restatement of coefnew/spsu2/spsu2-1ch-*.dat
(src/sym-SPSU2.cc, src/nrg-recalc-SPSU2.cc).

Test infrastructure: part of the CPU checker for the CUDA path, imported only
by tests.

Same construction as qs_derive.py, with the charge dropped from the
invariants (subspaces are labelled by SS = 2S+1 alone, written (0, SS)):
a new subspace SS of step N+1 is spanned by four combinations of an ancestor
subspace of step N with a spin multiplet of the added site,

  1: site empty        (s = 0),   ancestor SS
  2: site doubly occ.  (s = 0),   ancestor SS
  3: site singly occ.  (s = 1/2), ancestor SS - 1
  4: site singly occ.  (s = 1/2), ancestor SS + 1

and, because the charge is not conserved, three kinds of coupling between
the chain's last site N and the added site N+1 enter the Hamiltonian:

  hopping   xi_N     sum_s (f^dag_{N,s} f_{N+1,s} + h.c.)      (OFFDIAG)
  pairing   kappa_N  (f^dag_{N,up} f^dag_{N+1,dn}
                      - f^dag_{N,dn} f^dag_{N+1,up} + h.c.)    (ANOMALOUS)
  on-site   delta_{N+1} (f^dag_{N+1,up} f^dag_{N+1,dn} + h.c.)  (ISOSPINX)

Each table entry is a matrix element in the site's Fock space times a
Clebsch-Gordan recoupling, divided by the coefficient of the Wigner-Eckart
theorem for the chain's reduced element <anc_i||f^dag||anc_j> that the
assembly multiplies it with.  tests/test_spsu2_tables.py checks every entry
against the reference's tables (tests/golden/spsu2_tables.json).
"""
from __future__ import annotations

import functools

import qs_derive as qd

# (electrons on the site, site spin, ancestor offset (0, dSS))
COMBOS = [((0,), 0.0, (0, 0)), ((2,), 0.0, (0, 0)), ((1,), 0.5, (0, -1)), ((1,), 0.5, (0, 1))]
# phase of the doubly occupied site state relative to c^dag_up c^dag_dn |0>
SITE_SIGNS = {((2,), 0.0): -1.0}


class Tables(qd.Tables):
    def __init__(self):
        self.P = 1
        self.combos = COMBOS
        self.site = qd._Site(1)
        self.mult = {}
        for occ, s, _ in self.combos:
            if (occ, s) not in self.mult:
                self.mult[(occ, s)] = self.site.multiplet(occ, s, SITE_SIGNS.get((occ, s), 1.0))

    def _pairs(self, ss, site_ops):
        """Ordered pairs (i, j) with sum over (op, q) of <i; S S| op T^1/2_q |j; S S>."""
        S = (ss - 1) / 2.0
        out = []
        n = len(self.combos)
        for i in range(n):
            for j in range(n):
                if i == j:
                    continue
                v = sum(c * self._elem(i, S, S, j, S, S, 0.5, q, op, True) for c, op, q in site_ops)
                if abs(v) > 1e-13:
                    out.append((i + 1, j + 1, 0, v))
        return out

    def offdiag(self, ss):
        # f^dag_{N,s} f_{N+1,s}: the chain creates, the site annihilates
        return self._pairs(ss, [(1.0, self.site.c[0], 0.5), (1.0, self.site.c[1], -0.5)])

    def anomalous(self, ss):
        # f^dag_{N,up} f^dag_{N+1,dn} - f^dag_{N,dn} f^dag_{N+1,up}
        return self._pairs(ss, [(1.0, self.site.cd[1], 0.5), (-1.0, self.site.cd[0], -0.5)])

    def isospinx(self):
        # the site's pairing operator between the empty and the doubly
        # occupied combination, in units of 2 delta (the assembly's factor)
        op = self.site.cd[0] @ self.site.cd[1]
        op = op + op.T
        v = self._elem(0, 0.0, 0.0, 1, 0.0, 0.0, None, 0.0, op, False)
        return [(1, 2, 0, v / 2.0)]

    def diag(self):
        return [(i + 1, 0, float(c[0][0])) for i, c in enumerate(self.combos)]

    def recalc_f(self, Ip):
        out = []
        for dss in (1, -1):
            I1 = (0, Ip[1] + dss)
            if I1[1] < 1:
                continue
            rows = []
            for i1 in range(len(self.combos)):
                for ip in range(len(self.combos)):
                    A = self.anc(i1, I1)
                    if A != self.anc(ip, Ip) or A[1] < 1:
                        continue

                    def comp(q, S1, Sp, M2, i1=i1, ip=ip):
                        op = self.site.cd[0 if q > 0 else 1]
                        return self._elem(i1, S1, S1, ip, Sp, M2, None, 0.0, op, False)
                    v = self._reduced(I1, Ip, 0.5, comp)
                    if abs(v) > 1e-13:
                        rows.append((i1 + 1, ip + 1, v))
            out.append((I1, 0, rows))
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
def tables():
    return Tables()
