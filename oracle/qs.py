"""QS symmetry plug-in (charge U(1) x spin SU(2)) restated for the oracle.

Test infrastructure: this module is part of the CPU checker for the CUDA
path and is imported only by tests, smoke() and the bench's CPU baseline.

Invariant subspaces are tuples (Q, SS) with SS = 2S+1 (src/sym-QS.cc:11-22).
The coefficient tables restate coefnew/qs/qs-1ch-*.dat (included by
src/sym-QS.cc:38-68, 134-209 and src/nrg-recalc-QS.cc) with each
Clebsch-Gordan expression simplified to a closed form in the multiplicity
SS; every entry is checked numerically against the reference tables by
tests/test_qs_tables.py.  Indices i, j are the 1-based combination numbers of
the reference ("|r,i>" blocks of a new subspace).
"""
from __future__ import annotations

import math

import qs_derive

COMBS = {1: 4, 2: 16, 3: 64}

# In[i]: quantum-number difference between a subspace and its i-th ancestor
# (ancestor = I + In[i]); QN[i]: quantum numbers of the states added on the
# new site (coefnew/qs/qs-1ch-In2.dat, qs-1ch-QN.dat; for two and three
# channels the combinations of qs_derive.COMBOS, which follow
# qs-<P>ch-In2.dat, qs-<P>ch-QN.dat).
IN = {1: [(1, 0), (0, -1), (0, 1), (-1, 0)]}
QN = {1: [(-1, 1), (0, 2), (0, 2), (1, 1)]}
for _P in (2, 3):
    IN[_P] = [c[2] for c in qs_derive.COMBOS[_P]]
    QN[_P] = [(sum(c[0]) - _P, int(round(2 * c[1])) + 1) for c in qs_derive.COMBOS[_P]]

SINGLET = (0, 1)   # InvarSinglet
DOUBLET = (1, 2)   # Invar_f: quantum numbers of f^dag
TRIPLET = (0, 3)


def mult(I):
    return I[1]


def allowed(I):
    return I[1] > 0


def su2_triangle(a, b, c):
    return abs(a - b) <= c - 1 and abs(b - c) <= a - 1 and abs(c - a) <= b - 1


def triangle(I1, I2, I3):
    """src/sym-QS.cc:27-31: U(1) charge balance and SU(2) triangle."""
    return I1[0] == I2[0] + I3[0] and su2_triangle(I1[1], I2[1], I3[1])


def combine(A, B):
    return (A[0] + B[0], A[1] + B[1])


def inverse(A):
    return (-A[0], -A[1])


def offdiag_terms(nch, ss):
    """Hopping blocks of H_{N+1} in subspace with multiplicity ss:
    (i, j, ch, factor) adds factor*xi_N/SCALE(N+1) * <In[i]||f^dag_ch||In[j]>
    to block (i, j) (qs-1ch-offdiag.dat; two and three channels: derived,
    qs_derive)."""
    if nch in (2, 3):
        return qs_derive.offdiag(nch, ss)
    if nch != 1:
        raise NotImplementedError("QS tables for 1 to 3 channels")
    return [(1, 2, 0, 1.0),
            (1, 3, 0, 1.0),
            (2, 4, 0, -math.sqrt((ss - 1) / ss)),
            (3, 4, 0, math.sqrt((ss + 1) / ss))]


def diag_terms(nch):
    """(i, ch, number): electrons added in channel ch by combination i
    (qs-1ch-diag.dat)."""
    if nch in (2, 3):
        return qs_derive.tables(nch).diag()
    if nch != 1:
        raise NotImplementedError
    return [(1, 0, 0), (2, 0, 1), (3, 0, 1), (4, 0, 2)]


def recalc_f_tables(nch, Ip):
    """<I1||f^dag_ch||Ip> of the new site: list of (I1, ch, [(i1, ip, factor)])
    (qs-1ch-spinupa.dat, qs-1ch-spindowna.dat; src/nrg-recalc-QS.cc:210-458)."""
    if nch in (2, 3):
        return qs_derive.recalc_f(nch, tuple(Ip))
    if nch != 1:
        raise NotImplementedError
    qp, ssp = Ip
    out = []
    out.append(((qp + 1, ssp + 1), 0, [(2, 1, 1.0), (4, 3, -math.sqrt(ssp / (ssp + 1)))]))
    if ssp > 1:
        out.append(((qp + 1, ssp - 1), 0, [(3, 1, 1.0), (4, 2, math.sqrt(ssp / (ssp - 1)))]))
    else:
        out.append(((qp + 1, ssp - 1), 0, [(3, 1, 1.0), (4, 2, math.inf)]))
    return out


def doublet_tables(nch, I1):
    """Recalculation of a doublet operator: list of (Ip, [(i1, ip, factor)])
    (qs-1ch-doubletp.dat, qs-1ch-doubletm.dat; src/nrg-recalc-QS.cc:34-203)."""
    if nch in (2, 3):
        return qs_derive.doublet(nch, tuple(I1))
    if nch != 1:
        raise NotImplementedError
    q1, ss1 = I1
    c = math.sqrt((ss1 - 1) * (ss1 + 1)) / ss1
    plus = ((q1 - 1, ss1 + 1), [(1, 1, 1.0), (2, 2, -c), (3, 2, 1.0 / ss1),
                                (3, 3, -1.0), (4, 4, 1.0)])
    minus = ((q1 - 1, ss1 - 1), [(1, 1, 1.0), (2, 2, -1.0), (2, 3, -1.0 / ss1),
                                 (3, 3, -c), (4, 4, 1.0)])
    return [plus, minus]


def triplet_tables(nch, I1):
    """Recalculation of a triplet (spin) operator: list of (Ip, rows)
    (qs-1ch-triplets.dat, tripletp.dat, tripletm.dat; src/nrg-recalc-QS.cc:497-697)."""
    if nch in (2, 3):
        return qs_derive.triplet(nch, tuple(I1))
    if nch != 1:
        raise NotImplementedError
    q1, ss1 = I1
    S = (ss1 - 1) / 2.0
    # Ip = (q1, ss1): the spin-conserving table
    if S > 0:
        t22 = math.sqrt(1 - 1 / S + 2 / (1 + 2 * S))
        t23 = 1 / math.sqrt((1 + S) * (1 + 2 * S))
        t32 = -1 / math.sqrt(S * (1 + 2 * S))
        t33 = (math.sqrt(S * (1 + 2 * S) / ((1 + S) ** 3 * (3 + 2 * S))) * (1 + S)
               + 2 * math.sqrt(S / (3 + 11 * S + 12 * S * S + 4 * S ** 3)))
    else:
        t22 = t23 = t32 = t33 = math.nan
    same = ((q1, ss1), [(1, 1, 1.0), (2, 2, t22), (2, 3, t23), (3, 2, t32), (3, 3, t33), (4, 4, 1.0)])
    plus = ((q1, ss1 + 2), [(1, 1, 1.0),
                            (2, 2, math.sqrt(1 + 1 / (1 + S) - 2 / (1 + 2 * S))),
                            (3, 2, -1 / math.sqrt((1 + S) * (1 + 2 * S))),
                            (3, 3, 1.0), (4, 4, 1.0)])
    if S > 0.5:
        m33 = (math.sqrt((-1 + 4 * S * S) / (S + S * S))
               + math.sqrt((-1 + 2 * S) / (S + 3 * S * S + 2 * S ** 3))) / 2
        m23 = 1 / math.sqrt(S * (1 + 2 * S))
    else:
        m33 = m23 = math.nan
    minus = ((q1, ss1 - 2), [(1, 1, 1.0), (2, 2, 1.0), (2, 3, m23), (3, 3, m33), (4, 4, 1.0)])
    return [same, plus, minus]


def specdens_factor(Ip, I1):
    """src/sym-QS.cc:95-104."""
    ssp, ss1 = Ip[1], I1[1]
    Sp = (ssp - 1) / 2.0
    return Sp + 1.0 if ss1 == ssp + 1 else Sp


def dynamicsusceptibility_factor(Ip, I1):
    """src/sym-QS.cc:70-93 (switch3)."""
    ssp, ss1 = Ip[1], I1[1]
    if ss1 == ssp + 2:
        return 1.0 + (ssp - 1) / 3.0
    if ss1 == ssp:
        return ssp / 3.0
    if ss1 == ssp - 2:
        return (-2.0 + ssp) / 3.0
    raise ValueError("not a triplet pair")


def td_fields(blocks, factor):
    """QS part of calculate_TD (src/sym-QS.cc:106-123): returns
    (Tr[S_z^2], Tr[Q], Tr[Q^2]) weighted by Boltzmann factors (not divided by Z).
    `blocks` maps I -> eigenvalue array."""
    import numpy as np
    trSZ = trQ = trQ2 = 0.0
    for I, vals in blocks.items():
        q, ss = I
        sumZ = float(np.sum(np.exp(-factor * vals))) * mult(I)
        trQ += sumZ * q
        trQ2 += sumZ * q * q
        trSZ += sumZ * (ss * ss - 1) / 12.0
    return trSZ, trQ, trQ2
