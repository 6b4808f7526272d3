"""Input generator for the NRG step: writes the `param` and `data` (version 9)
files that the reference's C++ back end reads.

The reference produces `data` with its Mathematica front end (initial.m,
maketable at initial.m:4309-4392), which is not available here.  This module
restates the parts of that front end that the QS (charge U(1) x spin SU(2))
workloads need:

* the Wilson chain of a flat band in the Yoshida-Whitaker-Oliveira (Y),
  Campo-Oliveira (C) or Zitko-Pruschke (Z) discretization, by Lanczos
  tridiagonalisation of the star Hamiltonian in arbitrary precision
  (initial.m:2902-2908 band, 3538-3598 representative energies, 3055-3164
  Lanczos recursion, 4040-4044 table output);
* the Wilson chain of a tabulated hybridisation function on the adaptive
  logarithmic mesh (the tools/adapt nrgchain program), checked against the
  reference's own fixtures;
* the initial cluster (impurity + site f_0 of every channel): Fock-space
  Hamiltonian, its eigenstates per invariant subspace (Q, SS) with the
  representative member at S_z = S (initial.m:1664-1668), energies shifted by
  the ground state and divided by SCALE(0) (initial.m:4104-4124);
* irreducible matrix elements in the Wigner-Eckart normalisation of
  initial.m:2089-2104:  <I1||O||I2> = <I1,S1|O_sigma|I2,S2> / CG(S2 S2; 1/2 sigma | S1 S1);
* the data-file layout of initial.m:4094-4101 (header), 4309-4392 (blocks)
  and the reader at src/nrg.cc:3323-3401, src/read-input.cc:98-143.

Models: single-impurity Anderson (models.m SIAM variant) and the 1- or
2-channel Kondo model (models.m:366-377).  Hybridisation and exchange are
taken literally as given by the caller (V, J); the A_Lambda correction of
initial.m:1023 is not applied unless the caller folds it into V or J.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np

try:
    import mpmath
except ImportError:  # pragma: no cover - mpmath ships with the image
    mpmath = None


# ---------------------------------------------------------------------------
# Wilson chain
# ---------------------------------------------------------------------------

def scale_factor(N: int, Lambda: float, z: float = 1.0, discretization: str = "Y",
                 bandrescale: float = 1.0) -> float:
    """SCALE(N) of src/nrg.cc:491-506 (no substeps)."""
    if discretization == "Y":
        s = 0.5 * (1.0 + 1.0 / Lambda)
    elif discretization in ("C", "Z"):
        s = (1.0 - 1.0 / Lambda) / math.log(Lambda)
    else:
        raise ValueError("unknown discretization " + discretization)
    return s * Lambda ** (-(N - 1) / 2.0 + 1.0 - z) * bandrescale


def _lanczos_star(de_pos, de_neg, u_pos, u_neg, Nmax):
    """Tridiagonalise the star Hamiltonian diag(+de_pos, -de_neg) from the
    start vector (u_pos, u_neg) (normalised here) at the current mpmath
    precision; returns the raw chain coefficients xi[0..Nmax], zeta[0..Nmax]
    as mpf (initial.m:3055-3164; tools/adapt/nrgchain.cc tridiag)."""
    diagA = list(de_pos) + [-x for x in de_neg]
    u = list(u_pos) + list(u_neg)
    norm = mpmath.fsum(x * x for x in u)
    u = [x / mpmath.sqrt(norm) for x in u]  # rescale exactly to one
    xi, zeta = [], []
    uprev = [mpmath.mpf(0)] * len(u)
    xiprev = mpmath.mpf(0)
    for n in range(Nmax + 1):
        Au = [a * x for a, x in zip(diagA, u)]
        zn = mpmath.fsum(a * x for a, x in zip(Au, u))
        r = [a - zn * x - xiprev * p for a, x, p in zip(Au, u, uprev)]
        # at this precision no reorthogonalisation is needed; renormalise
        # as initial.m:3450-3458
        xn = mpmath.sqrt(mpmath.fsum(x * x for x in r))
        zeta.append(zn)
        xi.append(xn)
        uprev, u = u, [x / xn for x in r]
        xiprev = xn
    return xi, zeta


def wilson_chain_flat(Lambda: float, z: float, Nmax: int, mMAX: int | None = None,
                      dps: int = 200, discretization: str = "Y") -> Tuple[np.ndarray, np.ndarray]:
    """Chain coefficients xi[0..Nmax], zeta[0..Nmax] of a flat band (D=1).

    Star levels (initial.m:2902-2908): interval edges eps_0 = 1,
    eps_m = Lambda^(1-z-m); hybridisation weights df_m = eps_m - eps_{m+1}
    (theta = 2, symmetric).  Representative energies by discretization
    scheme:
      Y (Yoshida-Whitaker-Oliveira, initial.m:3538-3545):
          de_0 = (1+Lambda^-z)/2,  de_m = (1+1/Lambda)/2 * Lambda^(1-z-m);
      C (Campo-Oliveira, initial.m:3568-3572):
          de_m = (eps_m - eps_{m+1}) / ln(eps_m / eps_{m+1});
      Z (Zitko-Pruschke, initial.m:3592-3598):
          de_0 = (1 - Lambda^-z + ln Lambda - z ln Lambda) / ln Lambda,
          de_m as for C (m >= 1).
    mMAX defaults to max(80, 2*Nmax) as in initial.m:2877.  The Lanczos
    recursion runs at `dps` decimal digits, since double precision loses
    orthogonality along the chain (the reference uses 1000 digits,
    initial.m:2790-2793).
    """
    if mpmath is None:
        raise RuntimeError("mpmath is required for the Wilson chain")
    if discretization not in ("Y", "C", "Z"):
        raise ValueError("unknown discretization " + discretization)
    if mMAX is None:
        mMAX = max(80, 2 * Nmax)
    mp = mpmath.mp
    old = mp.dps
    mp.dps = dps
    try:
        L = mpmath.mpf(Lambda)
        Z = mpmath.mpf(z)
        lnL = mpmath.log(L)
        eps = [mpmath.mpf(1)] + [L ** (1 - Z - m) for m in range(1, mMAX + 2)]
        df = [eps[m] - eps[m + 1] for m in range(mMAX + 1)]
        if discretization == "Y":
            de = [(1 + L ** (-Z)) / 2] + [(1 + 1 / L) / 2 * L ** (1 - Z - m) for m in range(1, mMAX + 1)]
        else:
            de = [(eps[m] - eps[m + 1]) / mpmath.log(eps[m] / eps[m + 1]) for m in range(mMAX + 1)]
            if discretization == "Z":
                de[0] = (1 - L ** (-Z) + lnL - Z * lnL) / lnL
        theta = mpmath.mpf(2)
        u = [mpmath.sqrt(x / theta) for x in df]
        xi, zeta = _lanczos_star(de, de, u, u, Nmax)
        return (np.array([float(x) for x in xi]), np.array([float(x) for x in zeta]))
    finally:
        mp.dps = old


# ---------------------------------------------------------------------------
# Wilson chain of a tabulated density of states with the adaptive mesh
# ---------------------------------------------------------------------------

class _LinInt:
    """Linear interpolation of a table, constant beyond its ends (the
    tabulated functions of tools/adapt: linint.h LinInt)."""

    def __init__(self, xy):
        xy = sorted(xy)
        self.x = np.array([p[0] for p in xy])
        self.y = np.array([p[1] for p in xy])

    def __call__(self, x):
        if x <= self.x[0]:
            return float(self.y[0])
        if x >= self.x[-1]:
            return float(self.y[-1])
        i = int(np.searchsorted(self.x, x, side="right")) - 1
        x0, x1, f0, f1 = self.x[i], self.x[i + 1], self.y[i], self.y[i + 1]
        return float(f0 + (f1 - f0) / (x1 - x0) * (x - x0))


class _IntLinInt(_LinInt):
    """Running integral of the linearly interpolated table from its first
    point: trapezoid sums at the nodes, exact quadratic inside an interval,
    linear continuation beyond the ends (linint.h IntLinInt, calc.h
    integrate)."""

    def __init__(self, xy):
        super().__init__(xy)
        dx = np.diff(self.x)
        self.I = np.concatenate([[0.0], np.cumsum(dx * (self.y[1:] + self.y[:-1]) / 2.0)])

    def __call__(self, x):
        if x <= self.x[0]:
            return float(self.I[0] + self.y[0] * (x - self.x[0]))
        if x >= self.x[-1]:
            return float(self.I[-1] + self.y[-1] * (x - self.x[-1]))
        i = int(np.searchsorted(self.x, x, side="right")) - 1
        x0, x1, f0, f1 = self.x[i], self.x[i + 1], self.y[i], self.y[i + 1]
        d = x - x0
        return float(self.I[i] + d * f0 + d * d * ((f1 - f0) / (x1 - x0)) / 2.0)


def _trapezoid_to(xy, b):
    """Integral of the table from its first point up to b (calc.h integrate_ab)."""
    xy = sorted(xy)
    s = 0.0
    for (x0, y0), (x1, y1) in zip(xy[:-1], xy[1:]):
        if x0 < b and x1 <= b:
            dx = x1 - x0
        elif x0 < b < x1:
            dx = b - x0
        else:
            dx = 0.0
        s += dx * (y0 + y1) / 2.0
    return s


def read_two_columns(path):
    out = []
    with open(path) as fh:
        for line in fh:
            t = line.split()
            if not t or t[0].startswith("#"):
                continue
            out.append((float(t[0]), float(t[1])))
    return out


def wilson_chain_tabulated(dos, g_pos, g_neg, f_pos, f_neg, Lambda: float, z: float, Nmax: int,
                           mMAX: int | None = None, adapt: bool = True, bandrescale: float = 1.0,
                           dps: int = 600) -> Tuple[np.ndarray, np.ndarray, float]:
    """Wilson chain of a tabulated hybridisation function with the adaptive
    logarithmic mesh (Zitko, Comput. Phys. Commun. 180, 1271 (2009)): the
    restatement of tools/adapt/nrgchain.cc (tables, tridiag).

    dos: (omega, rho) pairs on both sides of zero; g_*/f_*: (x, g(x)) and
    (x, f(x)) tables of the mesh ODE solutions (GSOL*.dat, FSOL*.dat).
    Mesh eps(x) = g(x) Lambda^(2-x) for x > 2 (1 below), representative
    energies E(x) = f(x) Lambda^(2-x); interval m (x = z+m+1) carries weight
    int_{eps(x+1)}^{eps(x)} rho and energy E(x), m = 0..mMAX.  Returns the raw
    xi[0..Nmax] (divide by SCALE(n+1) of the Z scheme for nrgchain's xi.dat)
    and zeta[0..Nmax], and theta (total weight up to |omega| = 1)."""
    if mMAX is None:
        mMAX = 2 * Nmax
    pos = [(abs(x), y * bandrescale) for x, y in dos if x > 0]
    neg = [(abs(x), y * bandrescale) for x, y in dos if x < 0]
    pos = [(x / bandrescale, y) for x, y in pos]
    neg = [(x / bandrescale, y) for x, y in neg]
    ip, ineg = _IntLinInt(pos), _IntLinInt(neg)
    gp, gn, fp, fn = _LinInt(g_pos), _LinInt(g_neg), _LinInt(f_pos), _LinInt(f_neg)

    def eps(g, x):
        return 1.0 if x <= 2.0 else (g(x) if adapt else 1.0) * Lambda ** (2.0 - x)

    theta = _trapezoid_to(pos, 1.0) + _trapezoid_to(neg, 1.0)
    du_p, du_n, de_p, de_n = [], [], [], []
    for m in range(mMAX + 1):
        x1, x2 = z + m + 1, z + m + 2
        du_p.append(math.sqrt(ip(eps(gp, x1)) - ip(eps(gp, x2))) / math.sqrt(theta))
        du_n.append(math.sqrt(ineg(eps(gn, x1)) - ineg(eps(gn, x2))) / math.sqrt(theta))
        de_p.append(fp(x1) * Lambda ** (2.0 - x1))
        de_n.append(fn(x1) * Lambda ** (2.0 - x1))
    check = sum(a * a for a in du_p) + sum(a * a for a in du_n)
    if abs(1.0 - check) > 1e-10:
        raise ValueError("weights of the discretization do not sum to theta (1 - sum = %g)" % (1.0 - check))
    du_p = [a / math.sqrt(check) for a in du_p]
    du_n = [a / math.sqrt(check) for a in du_n]
    mp = mpmath.mp
    old = mp.dps
    mp.dps = dps
    try:
        M = mpmath.mpf
        xi, zeta = _lanczos_star([M(x) for x in de_p], [M(x) for x in de_n], [M(x) for x in du_p],
                                 [M(x) for x in du_n], Nmax)
        return np.array([float(x) for x in xi]), np.array([float(x) for x in zeta]), theta
    finally:
        mp.dps = old


def wilson_closed_form(Lambda: float, Nmax: int) -> np.ndarray:
    """Wilson's closed form for xi_n (flat band, z=1, infinite star), used as
    a cross-check of the Lanczos result."""
    n = np.arange(Nmax + 1, dtype=float)
    L = Lambda
    return ((1 + 1 / L) / 2 * (1 - L ** (-n - 1))
            / np.sqrt((1 - L ** (-2 * n - 1)) * (1 - L ** (-2 * n - 3))) * L ** (-n / 2))


# ---------------------------------------------------------------------------
# Fock space of the initial cluster
# ---------------------------------------------------------------------------

class Fock:
    """Dense Fock space of `nmodes` fermionic modes, Jordan-Wigner ordered.

    Mode k is (orbital, spin) with spin 0 = up, 1 = down.  cdag[k] is the
    creation-operator matrix (2^n x 2^n)."""

    def __init__(self, norb: int):
        self.norb = norb
        self.nmodes = 2 * norb
        dim = 1 << self.nmodes
        self.dim = dim
        self.cdag = []
        states = np.arange(dim)
        for k in range(self.nmodes):
            M = np.zeros((dim, dim))
            for s in states:
                if not (s >> k) & 1:
                    t = s | (1 << k)
                    # sign: number of occupied modes below k
                    sign = -1.0 if bin(s & ((1 << k) - 1)).count("1") % 2 else 1.0
                    M[t, s] = sign
            self.cdag.append(M)
        self.occ = np.array([[(s >> k) & 1 for k in range(self.nmodes)] for s in states])

    def mode(self, orb: int, spin: int) -> int:
        return 2 * orb + spin

    def c(self, orb, spin):
        return self.cdag[self.mode(orb, spin)].T

    def cd(self, orb, spin):
        return self.cdag[self.mode(orb, spin)]

    def n(self, orb, spin=None):
        if spin is None:
            return self.n(orb, 0) + self.n(orb, 1)
        m = self.cdag[self.mode(orb, spin)]
        return m @ m.T

    def spin_ops(self, orb):
        sp = self.cd(orb, 0) @ self.c(orb, 1)
        sz = 0.5 * (self.n(orb, 0) - self.n(orb, 1))
        return sp, sp.T, sz


@dataclass
class Subspace:
    Q: int
    SS: int
    energies: np.ndarray            # ascending, absolute units
    vectors: np.ndarray             # (fock_dim, nstates), representative S_z = S


@dataclass
class ClusterModel:
    """Initial cluster: Hamiltonian, operators and the site-0 f operators."""
    fock: Fock
    H: np.ndarray
    charge_orbitals: List[int]      # orbitals whose occupancy defines Q
    f_orbitals: List[int]           # orbital of f_0 for each channel
    spin_orbitals: List[int]        # orbitals that carry spin
    basis_mask: np.ndarray          # Fock states that are allowed
    doublet_ops: Dict[str, int] = field(default_factory=dict)   # name -> orbital (creation op)
    singlet_ops: Dict[str, np.ndarray] = field(default_factory=dict)
    triplet_ops: Dict[str, int] = field(default_factory=dict)   # name -> orbital (spin op)


def siam_cluster(U: float, eps_d: float, V: float, zeta0: float = 0.0, delta0: float = 0.0) -> ClusterModel:
    """Single-impurity Anderson model, impurity d + first chain site f_0:
    H = eps_d n_d + U n_up n_dn + V sum_s (d^dag_s f_0s + h.c.) + zeta0 (n_f0 - 1)
        + delta0 (f^dag_0up f^dag_0dn + h.c.)   (pairing: superconducting bath)."""
    F = Fock(2)  # orbital 0 = d, orbital 1 = f0
    H = eps_d * F.n(0) + U * F.n(0, 0) @ F.n(0, 1)
    for s in (0, 1):
        hop = F.cd(0, s) @ F.c(1, s)
        H = H + V * (hop + hop.T)
    H = H + zeta0 * (F.n(1) - np.eye(F.dim))
    if delta0:
        pair = F.cd(1, 0) @ F.cd(1, 1)
        H = H + delta0 * (pair + pair.T)
    m = ClusterModel(F, H, charge_orbitals=[0, 1], f_orbitals=[1], spin_orbitals=[0, 1],
                     basis_mask=np.ones(F.dim, dtype=bool))
    m.doublet_ops["A_d"] = 0
    m.singlet_ops["n_d"] = F.n(0)
    m.singlet_ops["n_d^2"] = F.n(0) @ F.n(0)
    m.triplet_ops["SZd"] = 0
    return m


def kondo_cluster(J: List[float]) -> ClusterModel:
    """Kondo model with len(J) channels: impurity spin (orbital 0, singly
    occupied) coupled to f_0 of each channel, H = sum_ch J_ch S_d . s_ch
    (models.m:366-377 for two channels)."""
    nch = len(J)
    F = Fock(1 + nch)
    H = np.zeros((F.dim, F.dim))
    spd, smd, szd = F.spin_ops(0)
    for ch in range(nch):
        sp, sm, sz = F.spin_ops(1 + ch)
        H = H + J[ch] * (szd @ sz + 0.5 * (spd @ sm + smd @ sp))
    mask = F.occ[:, 0] + F.occ[:, 1] == 1
    m = ClusterModel(F, H, charge_orbitals=list(range(1, 1 + nch)),
                     f_orbitals=list(range(1, 1 + nch)),
                     spin_orbitals=list(range(1 + nch)), basis_mask=mask)
    for ch in range(nch):
        m.doublet_ops["A_f%d" % ch] = 1 + ch
    m.triplet_ops["SZd"] = 0
    return m


def _total_spin_ops(m: ClusterModel):
    F = m.fock
    Sp = np.zeros((F.dim, F.dim))
    Sz = np.zeros((F.dim, F.dim))
    for o in m.spin_orbitals:
        sp, sm, sz = F.spin_ops(o)
        Sp = Sp + sp
        Sz = Sz + sz
    return Sp, Sz


def cg_half(S2: float, S1: float) -> float:
    """Clebsch-Gordan <S2 S2; 1/2 (S1-S2) | S1 S1> (Condon-Shortley)."""
    if abs(S1 - (S2 + 0.5)) < 1e-12:
        return 1.0
    if abs(S1 - (S2 - 0.5)) < 1e-12:
        return math.sqrt(2 * S2 / (2 * S2 + 1))
    raise ValueError("not a doublet coupling")


def cg_one(S2: float, S1: float) -> float:
    """<S2 S2; 1 (S1-S2) | S1 S1> for a rank-1 (triplet) operator."""
    q = S1 - S2
    if abs(q - 1) < 1e-12:
        return 1.0
    if abs(q) < 1e-12:
        return math.sqrt(S2 / (S2 + 1)) if S2 > 0 else 0.0
    if abs(q + 1) < 1e-12:
        return math.sqrt(S2 * (2 * S2 - 1) / ((S2 + 1) * (2 * S2 + 1))) if S2 > 0.5 else 0.0
    raise ValueError("not a triplet coupling")


def decompose(m: ClusterModel, tol: float = 1e-9) -> List[Subspace]:
    """Eigenstates per invariant subspace (Q, SS); representative S_z = S."""
    F = m.fock
    Sp, Sz = _total_spin_ops(m)
    ncharge = F.occ[:, [2 * o for o in m.charge_orbitals]].sum(1) + \
        F.occ[:, [2 * o + 1 for o in m.charge_orbitals]].sum(1)
    Q = ncharge - len(m.charge_orbitals)
    sz = np.round(np.diag(Sz) * 2).astype(int)  # 2*S_z
    subs = []
    for q in sorted(set(Q[m.basis_mask])):
        for two_s in sorted(set(sz[(Q == q) & m.basis_mask])):
            if two_s < 0:
                continue
            idx = np.where((Q == q) & (sz == two_s) & m.basis_mask)[0]
            idx_up = np.where((Q == q) & (sz == two_s + 2) & m.basis_mask)[0]
            if len(idx_up):
                A = Sp[np.ix_(idx_up, idx)]
                # null space of S+ within this sector: highest-weight states
                u, s, vt = np.linalg.svd(A)
                rank = int((s > tol).sum())
                B = vt[rank:].T
            else:
                B = np.eye(len(idx))
            if B.shape[1] == 0:
                continue
            Hs = B.T @ m.H[np.ix_(idx, idx)] @ B
            Hs = 0.5 * (Hs + Hs.T)
            e, w = np.linalg.eigh(Hs)
            vec = np.zeros((F.dim, B.shape[1]))
            vec[idx] = B @ w
            subs.append(Subspace(int(q), int(two_s + 1), e, vec))
    return subs


def _sub_map(subs):
    return {(s.Q, s.SS): s for s in subs}


def reduced_doublet(m: ClusterModel, subs, orb: int):
    """<I1||a^dag||I2> for pairs with Q1 = Q2+1, |SS1-SS2| = 1 (ireducMatrixSpeedy, QS)."""
    F = m.fock
    smap = _sub_map(subs)
    out = {}
    for (q2, ss2), s2 in smap.items():
        for ss1 in (ss2 + 1, ss2 - 1):
            key1 = (q2 + 1, ss1)
            if ss1 < 1 or key1 not in smap:
                continue
            s1 = smap[key1]
            S1, S2 = (ss1 - 1) / 2, (ss2 - 1) / 2
            spin = 0 if S1 > S2 else 1  # sigma = S1 - S2
            op = F.cd(orb, spin)
            M = s1.vectors.T @ op @ s2.vectors / cg_half(S2, S1)
            out[(key1, (q2, ss2))] = M
    return out


def reduced_singlet(m: ClusterModel, subs, op: np.ndarray):
    smap = _sub_map(subs)
    out = {}
    for key, s in smap.items():
        out[(key, key)] = s.vectors.T @ op @ s.vectors
    return out


def reduced_triplet(m: ClusterModel, subs, orb: int):
    """<I1||S||I2> for a spin-1 operator, pairs with equal Q and
    SS1 - SS2 in {0, +-2}; spherical components S_{+1} = -S+/sqrt2, S_0 = Sz,
    S_{-1} = S-/sqrt2 (initial.m:2549-2570)."""
    F = m.fock
    sp, sm, sz = F.spin_ops(orb)
    smap = _sub_map(subs)
    out = {}
    for (q2, ss2), s2 in smap.items():
        for ss1 in (ss2 + 2, ss2, ss2 - 2):
            key1 = (q2, ss1)
            if ss1 < 1 or key1 not in smap:
                continue
            S1, S2 = (ss1 - 1) / 2, (ss2 - 1) / 2
            q = S1 - S2
            op = {1: -sp / math.sqrt(2), 0: sz, -1: sm / math.sqrt(2)}[int(round(q))]
            cg = cg_one(S2, S1)
            if cg == 0.0:
                continue
            out[(key1, (q2, ss2))] = smap[key1].vectors.T @ op @ s2.vectors / cg
    return out


# ---------------------------------------------------------------------------
# data / param writers
# ---------------------------------------------------------------------------

def _fmt(x: float) -> str:
    return repr(float(x))


def _write_matrix(lines, M):
    for row in np.atleast_2d(M):
        lines.append(" ".join(_fmt(v) for v in row))


def write_data(path: str, m: ClusterModel, Lambda: float, z: float, Nmax: int,
               xi: np.ndarray, zeta: np.ndarray, nchannels: int,
               discretization: str = "Y") -> dict:
    """Write a version-9 `data` file; returns a summary dict."""
    subs = decompose(m)
    gs = min(s.energies[0] for s in subs)
    sc0 = scale_factor(0, Lambda, z, discretization)
    lines = ["# Input file for NRG Ljubljana (generated by inputgen.py)",
             "# symtype QS",
             "#!9",
             "# Number of channels, chain sites, subspaces: ",
             "%d %d %d" % (nchannels, Nmax, len(subs)),
             "# SCALE " + _fmt(sc0),
             "# Energies (GS energy subtracted, multiplied by 1/SCALE):"]
    for s in subs:
        lines.append("%d %d" % (s.Q, s.SS))
        lines.append("%d" % len(s.energies))
        lines.append(" ".join(_fmt((e - gs) / sc0) for e in s.energies))
    lines.append("# Irreducible matrix elements for Wilson chains:")
    for ch in range(nchannels):
        f = reduced_doublet(m, subs, m.f_orbitals[ch])
        lines.append("f %d 0" % ch)
        lines.append("%d" % len(f))
        for (k1, k2), M in f.items():
            lines.append("%d %d %d %d" % (k1[0], k1[1], k2[0], k2[1]))
            _write_matrix(lines, M)
    lines.append("# GS energy in absolute units:")
    lines.append("e")
    lines.append(_fmt(gs))
    lines.append("# Irreducible matrix elements for other operators:")
    for name, op in m.singlet_ops.items():
        blocks = reduced_singlet(m, subs, op)
        lines.append("s" + name)
        lines.append("%d" % len(blocks))
        for (k1, k2), M in blocks.items():
            lines.append("%d %d %d %d" % (k1[0], k1[1], k2[0], k2[1]))
            _write_matrix(lines, M)
    for name, orb in m.doublet_ops.items():
        blocks = reduced_doublet(m, subs, orb)
        lines.append("d" + name)
        lines.append("%d" % len(blocks))
        for (k1, k2), M in blocks.items():
            lines.append("%d %d %d %d" % (k1[0], k1[1], k2[0], k2[1]))
            _write_matrix(lines, M)
    for name, orb in m.triplet_ops.items():
        blocks = reduced_triplet(m, subs, orb)
        lines.append("t" + name)
        lines.append("%d" % len(blocks))
        for (k1, k2), M in blocks.items():
            lines.append("%d %d %d %d" % (k1[0], k1[1], k2[0], k2[1]))
            _write_matrix(lines, M)
    lines.append("# Discretization tables:")
    lines.append("z")
    for ch in range(nchannels):
        lines.append("%d" % (len(xi) - 1))
        lines.extend(_fmt(x) for x in xi)
    for ch in range(nchannels):
        lines.append("%d" % (len(zeta) - 1))
        lines.extend(_fmt(x) for x in zeta)
    lines.append("")
    with open(path, "w") as fh:
        fh.write("\n".join(lines))
    return {"subspaces": len(subs), "gs_energy": gs, "scale0": sc0}


def decompose_qsz(m: ClusterModel) -> List[Subspace]:
    """Eigenstates per invariant subspace (Q, SSZ = 2 S_z) of the QSZ symmetry
    (charge U(1) x spin-projection U(1), src/sym-QSZ.cc): every state of a
    sector, no spin multiplets.  The Subspace field SS holds SSZ here."""
    F = m.fock
    _, Sz = _total_spin_ops(m)
    ncharge = F.occ[:, [2 * o for o in m.charge_orbitals]].sum(1) + \
        F.occ[:, [2 * o + 1 for o in m.charge_orbitals]].sum(1)
    Q = ncharge - len(m.charge_orbitals)
    ssz = np.round(np.diag(Sz) * 2).astype(int)
    subs = []
    for q in sorted(set(Q[m.basis_mask])):
        for z2 in sorted(set(ssz[(Q == q) & m.basis_mask])):
            idx = np.where((Q == q) & (ssz == z2) & m.basis_mask)[0]
            Hs = m.H[np.ix_(idx, idx)]
            Hs = 0.5 * (Hs + Hs.T)
            e, w = np.linalg.eigh(Hs)
            vec = np.zeros((F.dim, len(idx)))
            vec[idx] = w
            subs.append(Subspace(int(q), int(z2), e, vec))
    return subs


def write_data_qsz(path: str, m: ClusterModel, Lambda: float, z: float, Nmax: int,
                   xi: np.ndarray, zeta: np.ndarray, discretization: str = "Y") -> dict:
    """Write a version-9 `data` file of the QSZ symmetry (one to three
    channels): the sector energies, the matrix elements <I1|f^dag_sigma|I2>
    of the first chain site of each channel for both spins in one list
    (I1 = I2 + (1, +-1); the reference keeps one f list per channel for QSZ,
    src/read-input.cc:67-74, 131-145), the singlet operators and the doublet
    operators (both spins in one list, like f).  Triplet operators are not
    written."""
    nch = len(m.f_orbitals)
    if nch not in (1, 2, 3):
        raise ValueError("QSZ data: one to three channels")
    F = m.fock
    subs = decompose_qsz(m)
    smap = {(s.Q, s.SS): s for s in subs}
    gs = min(s.energies[0] for s in subs)
    sc0 = scale_factor(0, Lambda, z, discretization)
    lines = ["# Input file for NRG Ljubljana (generated by inputgen.py)",
             "# symtype QSZ",
             "#!9",
             "# Number of channels, chain sites, subspaces: ",
             "%d %d %d" % (nch, Nmax, len(subs)),
             "# SCALE " + _fmt(sc0),
             "# Energies (GS energy subtracted, multiplied by 1/SCALE):"]
    for s in subs:
        lines.append("%d %d" % (s.Q, s.SS))
        lines.append("%d" % len(s.energies))
        lines.append(" ".join(_fmt((e - gs) / sc0) for e in s.energies))
    lines.append("# Irreducible matrix elements for Wilson chains:")
    for ch in range(nch):
        orb = m.f_orbitals[ch]
        f = {}
        for (q2, z2), s2 in smap.items():
            for spin, dz in ((0, +1), (1, -1)):
                key1 = (q2 + 1, z2 + dz)
                if key1 in smap:
                    f[(key1, (q2, z2))] = smap[key1].vectors.T @ F.cd(orb, spin) @ s2.vectors
        lines.append("f %d 0" % ch)
        lines.append("%d" % len(f))
        for (k1, k2), M in f.items():
            lines.append("%d %d %d %d" % (k1[0], k1[1], k2[0], k2[1]))
            _write_matrix(lines, M)
    lines.append("# GS energy in absolute units:")
    lines.append("e")
    lines.append(_fmt(gs))
    lines.append("# Irreducible matrix elements for other operators:")
    for name, op in m.singlet_ops.items():
        lines.append("s" + name)
        lines.append("%d" % len(smap))
        for key, sub in smap.items():
            lines.append("%d %d %d %d" % (key[0], key[1], key[0], key[1]))
            _write_matrix(lines, sub.vectors.T @ op @ sub.vectors)
    # doublet operators: <I1|a^dag_s|I2> for both spins in one list, as f
    for name, orb2 in m.doublet_ops.items():
        blocks = {}
        for (q2, z2), s2 in smap.items():
            for spin, dz in ((0, +1), (1, -1)):
                key1 = (q2 + 1, z2 + dz)
                if key1 in smap:
                    blocks[(key1, (q2, z2))] = smap[key1].vectors.T @ F.cd(orb2, spin) @ s2.vectors
        lines.append("d" + name)
        lines.append("%d" % len(blocks))
        for (k1, k2), M in blocks.items():
            lines.append("%d %d %d %d" % (k1[0], k1[1], k2[0], k2[1]))
            _write_matrix(lines, M)
    lines.append("# Discretization tables:")
    lines.append("z")
    for t in (xi, zeta):
        for ch in range(nch):
            lines.append("%d" % (len(t) - 1))
            lines.extend(_fmt(x) for x in t)
    lines.append("")
    with open(path, "w") as fh:
        fh.write("\n".join(lines))
    return {"subspaces": len(subs), "gs_energy": gs, "scale0": sc0}


def decompose_spsu2(m: ClusterModel, tol: float = 1e-9) -> List[Subspace]:
    """Eigenstates per spin subspace SS of the SPSU2 symmetry (spin SU(2),
    charge not conserved, src/sym-SPSU2.cc): the highest-weight states of
    every S_z = S sector over all charges; representative S_z = S.  The
    Subspace field Q is 0."""
    F = m.fock
    Sp, Sz = _total_spin_ops(m)
    sz = np.round(np.diag(Sz) * 2).astype(int)
    subs = []
    for two_s in sorted(set(sz[m.basis_mask])):
        if two_s < 0:
            continue
        idx = np.where((sz == two_s) & m.basis_mask)[0]
        idx_up = np.where((sz == two_s + 2) & m.basis_mask)[0]
        if len(idx_up):
            _, sv, vt = np.linalg.svd(Sp[np.ix_(idx_up, idx)])
            B = vt[int((sv > tol).sum()):].T
        else:
            B = np.eye(len(idx))
        if B.shape[1] == 0:
            continue
        Hs = B.T @ m.H[np.ix_(idx, idx)] @ B
        e, w = np.linalg.eigh(0.5 * (Hs + Hs.T))
        vec = np.zeros((F.dim, B.shape[1]))
        vec[idx] = B @ w
        subs.append(Subspace(0, int(two_s + 1), e, vec))
    return subs


def write_data_spsu2(path: str, m: ClusterModel, Lambda: float, z: float, Nmax: int,
                     xi: np.ndarray, zeta: np.ndarray, delta: np.ndarray, kappa: np.ndarray,
                     discretization: str = "Y") -> dict:
    """Write a version-9 `data` file of the SPSU2 symmetry (one to three
    channels): subspaces labelled by SS alone, reduced matrix elements
    <SS1||a^dag||SS2> of f_0 of each channel and of the doublet operators for
    |SS1 - SS2| = 1 in the Wigner-Eckart normalisation of QS
    (ireducMatrixSpeedy, initial.m:2089), singlet and triplet operators, the
    chain tables z (xi, zeta) and Z (delta: on-site pairing, kappa: anomalous
    hopping; src/nrg.cc:3383-3386), each the same for every channel or given
    per channel (one row per channel)."""
    nch = len(m.f_orbitals)
    if nch not in (1, 2, 3):
        raise ValueError("SPSU2 data: one to three channels")
    F = m.fock
    subs = decompose_spsu2(m)
    smap = {s.SS: s for s in subs}
    gs = min(s.energies[0] for s in subs)
    sc0 = scale_factor(0, Lambda, z, discretization)

    def doublet(orb):
        out = {}
        for ss2, s2 in smap.items():
            for ss1 in (ss2 + 1, ss2 - 1):
                if ss1 in smap:
                    S1, S2 = (ss1 - 1) / 2, (ss2 - 1) / 2
                    op = F.cd(orb, 0 if S1 > S2 else 1)
                    out[(ss1, ss2)] = smap[ss1].vectors.T @ op @ s2.vectors / cg_half(S2, S1)
        return out

    def triplet(orb):
        sp, sm, szo = F.spin_ops(orb)
        out = {}
        for ss2, s2 in smap.items():
            for ss1 in (ss2 + 2, ss2, ss2 - 2):
                if ss1 not in smap:
                    continue
                S1, S2 = (ss1 - 1) / 2, (ss2 - 1) / 2
                q = int(round(S1 - S2))
                op = {1: -sp / math.sqrt(2), 0: szo, -1: sm / math.sqrt(2)}[q]
                c = cg_one(S2, S1)
                if c != 0.0:
                    out[(ss1, ss2)] = smap[ss1].vectors.T @ op @ s2.vectors / c
        return out

    lines = ["# Input file for NRG Ljubljana (generated by inputgen.py)",
             "# symtype SPSU2",
             "#!9",
             "# Number of channels, chain sites, subspaces: ",
             "%d %d %d" % (nch, Nmax, len(subs)),
             "# SCALE " + _fmt(sc0),
             "# Energies (GS energy subtracted, multiplied by 1/SCALE):"]
    for s in subs:
        lines.append("%d" % s.SS)
        lines.append("%d" % len(s.energies))
        lines.append(" ".join(_fmt((e - gs) / sc0) for e in s.energies))

    def blocks(kind_name, bl):
        lines.append(kind_name)
        lines.append("%d" % len(bl))
        for (k1, k2), M in bl.items():
            lines.append("%d %d" % (k1, k2))
            _write_matrix(lines, M)

    lines.append("# Irreducible matrix elements for Wilson chains:")
    for ch in range(nch):
        blocks("f %d 0" % ch, doublet(m.f_orbitals[ch]))
    lines.append("# GS energy in absolute units:")
    lines.append("e")
    lines.append(_fmt(gs))
    lines.append("# Irreducible matrix elements for other operators:")
    for name, op in m.singlet_ops.items():
        blocks("s" + name, {(k, k): s.vectors.T @ op @ s.vectors for k, s in smap.items()})
    for name, orb in m.doublet_ops.items():
        blocks("d" + name, doublet(orb))
    for name, orb in m.triplet_ops.items():
        blocks("t" + name, triplet(orb))
    lines.append("# Discretization tables:")
    for tag, tabs in (("z", (xi, zeta)), ("Z", (delta, kappa))):
        lines.append(tag)
        for t in tabs:
            rows = np.atleast_2d(np.asarray(t, dtype=float))
            for ch in range(nch):
                r = rows[min(ch, rows.shape[0] - 1)]
                lines.append("%d" % (len(r) - 1))
                lines.extend(_fmt(x) for x in r)
    lines.append("")
    with open(path, "w") as fh:
        fh.write("\n".join(lines))
    return {"subspaces": len(subs), "gs_energy": gs, "scale0": sc0}


def write_param(path: str, params: Dict[str, object]) -> None:
    with open(path, "w") as fh:
        fh.write("[param]\n")
        for k, v in params.items():
            if isinstance(v, bool):
                v = "true" if v else "false"
            fh.write("%s=%s\n" % (k, v))


def make_siam(dirpath: str, U: float, eps_d: float, Gamma: float, Lambda: float,
              Nmax: int, z: float = 1.0, params: Dict[str, object] | None = None,
              V: float | None = None, dps: int = 200, discretization: str = "Y",
              symtype: str = "QS", gap: float = 0.0) -> dict:
    """Generate `data` and `param` for a single-impurity Anderson model on a
    flat band (D=1) in directory `dirpath`, symmetry QS, QSZ or SPSU2.  V
    defaults to sqrt(2 Gamma/pi); discretization Y, C or Z
    (wilson_chain_flat).  SPSU2 only: `gap` is the BCS gap of the band; the
    pairing Delta sum_k (c^dag_k,up c^dag_k,dn + h.c.) is the identity in
    the band's modes, so every chain site carries the same on-site pairing
    delta_n = gap, and the anomalous hopping kappa_n vanishes."""
    os.makedirs(dirpath, exist_ok=True)
    if V is None:
        V = math.sqrt(2.0 * Gamma / math.pi)
    xi, zeta = wilson_chain_flat(Lambda, z, Nmax, dps=dps, discretization=discretization)
    if gap and symtype != "SPSU2":
        raise ValueError("a superconducting band needs symtype SPSU2")
    m = siam_cluster(U, eps_d, V, zeta0=zeta[0], delta0=gap)
    delta = np.full(Nmax + 1, float(gap))
    kappa = np.zeros(Nmax + 1)
    if symtype == "SPSU2":
        info = write_data_spsu2(os.path.join(dirpath, "data"), m, Lambda, z, Nmax, xi, zeta, delta, kappa,
                                discretization)
        info.update({"delta": delta, "kappa": kappa})
    elif symtype == "QSZ":
        info = write_data_qsz(os.path.join(dirpath, "data"), m, Lambda, z, Nmax, xi, zeta, discretization)
    elif symtype == "QS":
        info = write_data(os.path.join(dirpath, "data"), m, Lambda, z, Nmax, xi, zeta, 1, discretization)
    else:
        raise ValueError("symtype QS, QSZ or SPSU2")
    p = {"Lambda": Lambda, "z": z, "discretization": discretization}
    if params:
        p.update(params)
    write_param(os.path.join(dirpath, "param"), p)
    info.update({"V": V, "xi": xi, "zeta": zeta})
    return info


def make_kondo(dirpath: str, J: List[float], Lambda: float, Nmax: int, z: float = 1.0,
               params: Dict[str, object] | None = None, dps: int = 200, discretization: str = "Y",
               symtype: str = "QS") -> dict:
    """Generate `data` and `param` for the Kondo model with len(J) channels on
    a flat band, symmetry QS, QSZ or SPSU2 (SPSU2: a normal band, the
    pairing and anomalous-hopping tables zero)."""
    os.makedirs(dirpath, exist_ok=True)
    xi, zeta = wilson_chain_flat(Lambda, z, Nmax, dps=dps, discretization=discretization)
    m = kondo_cluster(J)
    if symtype == "SPSU2":
        zero = np.zeros(Nmax + 1)
        info = write_data_spsu2(os.path.join(dirpath, "data"), m, Lambda, z, Nmax, xi, zeta, zero, zero,
                                discretization)
    elif symtype == "QSZ":
        info = write_data_qsz(os.path.join(dirpath, "data"), m, Lambda, z, Nmax, xi, zeta, discretization)
    elif symtype == "QS":
        info = write_data(os.path.join(dirpath, "data"), m, Lambda, z, Nmax, xi, zeta, len(J), discretization)
    else:
        raise ValueError("symtype QS, QSZ or SPSU2")
    p = {"Lambda": Lambda, "z": z, "discretization": discretization}
    if params:
        p.update(params)
    write_param(os.path.join(dirpath, "param"), p)
    info.update({"xi": xi, "zeta": zeta})
    return info
