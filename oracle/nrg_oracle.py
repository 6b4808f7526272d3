"""CPU oracle for the NRG iteration hot path (FP64, LAPACK/BLAS via scipy).

Test infrastructure only: the checker that the CUDA path is compared with.
Imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline; it
is never part of the product path.

It restates, for the QS symmetry, the reference's two-sweep NRG run:

* src/nrg.cc:3429-3469  start_calculation (sweep 1, DM, sweep 2)
* src/nrg.cc:2415-2478  subspace list, ancestors, Hamiltonian assembly
  (src/matrix.cc:86-192 offdiag_build / diag_function)
* src/diag.h:54-89      dsyev: ascending eigenvalues, eigenvectors
* src/nrg.cc:1420-1455, 1919-2048, src/splitting.cc  ground state, fixeps
  clusters, truncation
* src/nrg.cc:2333-2369  thermodynamics (td)
* src/recalc.cc:12-97, 164-281, src/nrg.cc:2112-2142  recalc_f,
  recalc_general, recalc_singlet
* src/dmnrg.h:327-596, src/nrg.cc:1877-1913, 2002-2041  DM-NRG and FDM
  density matrices, Z_n^D, w_n
* src/spec.cc:26-62, src/spec_DMNRG.cc:13-52, src/spec_FDM.cc:41-119
  spectral weights; src/bins.h and src/spectrumrealfreq.cc binning, merging,
  trimming, .bin output and broadening (src/spectral.h:70-102).

One deliberate difference: at the last DM-NRG step the reference evaluates
the spectrum with the density matrix still in memory from step Nmax-2
(src/nrg.cc:2386 loads rho only when !LAST_ITERATION).  This restatement
uses the last-shell density matrix rho_{Nmax-1} (init_rho), which is the
DM-NRG definition; the CUDA path does the same.
"""
from __future__ import annotations

import math
import os
import sys
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np
import scipy.linalg as sla

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import qs  # noqa: E402

# ---------------------------------------------------------------------------
# parameters (src/param.cc defaults for the keys this path uses)
# ---------------------------------------------------------------------------

DEFAULTS = {
    "Lambda": 1.0, "z": 1.0, "discretization": "Y", "bandrescale": 1.0,
    "Ninit": 0, "Nmax": 0, "keep": 100, "keepenergy": -1.0, "keepmin": 0,
    "safeguard": 1e-5, "safeguardmax": 200, "fixeps": 1e-15,
    "betabar": 1.0, "T": -999.0, "strategy": "kept",
    "lastall": False, "lastalloverride": False,
    "dmnrg": False, "fdm": False, "cfs": False, "dm": False,
    "specs": "", "specd": "", "spect": "",
    "bins": 100, "emin": -1.0, "emax": -1.0, "goodE": 2.0,
    "NN1": False, "NN2even": True, "NN2avg": False, "NNtanh": 0.0,
    "discard_trim": 1e-16, "discard_immediately": 1e-16,
    "savebins": False, "broaden": True, "broaden_max": 2.5, "broaden_min": -99.0,
    "broaden_min_ratio": 3.0, "broaden_ratio": 1.05, "alpha": 0.3,
    "omega0": -1.0, "omega0_ratio": 1.0,
    "dumpannotated": 0, "dumpscaled": True, "dumpabs": False, "dumpprecision": 8,
    "dumpgroups": True, "grouptol": 1e-6,
    "width_td": 16, "prec_td": 10, "width_custom": 16, "prec_custom": 10,
    "prec_xy": 10, "diagth": 1, "calc0": True, "diag": "default", "dsyevrlimit": 100,
}


def _convert(default, s):
    if isinstance(default, bool):
        return s.strip().lower() in ("true", "1", "yes")
    if isinstance(default, int):
        return int(float(s))
    if isinstance(default, float):
        return float(s)
    return s


def read_params(path):
    """[param] block, key=value (src/misc.h:71-124)."""
    P = dict(DEFAULTS)
    inblock = False
    with open(path) as fh:
        for line in fh:
            line = line.rstrip("\n")
            if line.strip() == "[param]":
                inblock = True
                continue
            if not inblock:
                continue
            if line.startswith("["):
                break
            if "=" not in line or line.lstrip().startswith("#"):
                continue
            k, v = line.split("=", 1)
            v = v.rstrip()
            P[k] = _convert(DEFAULTS[k], v) if k in DEFAULTS else v
    # validateparameters (src/read-input.cc:6-36)
    if P["dmnrg"] or P["fdm"] or P["cfs"]:
        P["dm"] = True
    if (P["fdm"] or P["cfs"]) and not P["lastalloverride"]:
        P["lastall"] = True
    P["discretization"] = P["discretization"][:1]
    return P


# ---------------------------------------------------------------------------
# data file (src/nrg.cc:3293-3401, src/read-input.cc)
# ---------------------------------------------------------------------------

@dataclass
class Data:
    symtype: str = ""
    channels: int = 1
    Nmax: int = 0
    energies: Dict[tuple, np.ndarray] = field(default_factory=dict)
    opch: List[dict] = field(default_factory=list)
    gs_energy: float = 0.0
    ops: Dict[str, Dict[str, dict]] = field(default_factory=dict)  # kind -> name -> blocks
    xi: List[np.ndarray] = field(default_factory=list)
    zeta: List[np.ndarray] = field(default_factory=list)


def read_data(path) -> Data:
    D = Data()
    with open(path) as fh:
        lines = fh.read().split("\n")
    pos = 0
    version = None
    while pos < len(lines) and lines[pos].startswith("#"):
        l = lines[pos]
        if l.startswith("#!"):
            version = int(l[2:].split()[0])
        elif "symtype" in l:
            D.symtype = l.split()[-1]
        pos += 1
    if version != 9:
        raise ValueError("data file version %r, expected 9" % version)

    toks: List[str] = []

    def fill():
        nonlocal pos
        while not toks:
            if pos >= len(lines):
                raise EOFError
            l = lines[pos]
            pos += 1
            if l.strip().startswith("#"):
                continue
            toks.extend(l.split())

    def tok():
        fill()
        return toks.pop(0)

    D.channels = int(tok())
    D.Nmax = int(tok())
    nsubs = int(tok())
    order = []
    for _ in range(nsubs):
        I = (int(tok()), int(tok()))
        n = int(tok())
        D.energies[I] = np.array([float(tok()) for _ in range(n)])
        order.append(I)

    def read_blocks():
        nf = int(tok())
        blocks = {}
        for _ in range(nf):
            I1 = (int(tok()), int(tok()))
            I2 = (int(tok()), int(tok()))
            n1 = len(D.energies.get(I1, []))
            n2 = len(D.energies.get(I2, []))
            M = np.array([float(tok()) for _ in range(n1 * n2)]).reshape(n1, n2)
            blocks[(I1, I2)] = M
        return blocks

    for ch in range(D.channels):
        hdr = [tok(), tok(), tok()]
        if hdr[0] != "f" or int(hdr[1]) != ch or int(hdr[2]) != 0:
            raise ValueError("bad f block header %r" % hdr)
        D.opch.append(read_blocks())
    assert not toks
    while pos < len(lines):
        l = lines[pos].strip()
        pos += 1
        if not l or l.startswith("#"):
            continue
        kind, name = l[0], l[1:].strip()
        if kind == "e":
            D.gs_energy = float(tok())
        elif kind in "sdtpgoq":
            D.ops.setdefault(kind, {})[name] = read_blocks()
        elif kind == "z":
            for ch in range(D.channels):
                n = int(tok())
                D.xi.append(np.array([float(tok()) for _ in range(n + 1)]))
            for ch in range(D.channels):
                n = int(tok())
                D.zeta.append(np.array([float(tok()) for _ in range(n + 1)]))
        else:
            raise ValueError("unknown block %r" % kind)
        assert not toks
    return D


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def SCALE(P, N):
    if P["discretization"] == "Y":
        s = 0.5 * (1.0 + 1.0 / P["Lambda"])
    else:
        s = (1.0 - 1.0 / P["Lambda"]) / math.log(P["Lambda"])
    return s * P["Lambda"] ** (-(N - 1) / 2.0 + 1.0 - P["z"]) * P["bandrescale"]


class Bins:
    """Logarithmic bins, src/bins.h:22-131 (accumulation=0)."""

    def __init__(self, P, Nmax):
        self.bpd = P["bins"]
        emax = P["emax"] if P["emax"] > 0 else SCALE(P, 0) * 10 ** 2.0
        emin = P["emin"] if P["emin"] > 0 else SCALE(P, Nmax) / 10 ** 2.0
        self.l0 = math.floor(math.log10(emin))
        self.l1 = math.ceil(math.log10(emax))
        self.n = int((self.l1 - self.l0) * self.bpd + 1.0)
        self.e = np.array([10.0 ** (self.l0 + i / self.bpd) for i in range(self.n)])
        self.w = np.zeros(self.n)
        self.discard = P["discard_immediately"]

    def add_many(self, energy, weight):
        """Bins::add for arrays of positive energies."""
        energy = np.asarray(energy, dtype=float)
        weight = np.asarray(weight, dtype=float)
        keep = ~(np.abs(weight) < self.discard * energy)
        energy, weight = energy[keep], weight[keep]
        if energy.size == 0:
            return
        with np.errstate(divide="ignore"):
            pos = (np.log10(energy) - self.l0) * self.bpd
        idx = np.where(np.isfinite(pos), np.trunc(pos), -1).astype(np.int64)
        lo = idx < 0
        hi = idx >= self.n - 1
        np.add.at(self.w, np.zeros(int(lo.sum()), dtype=np.int64), weight[lo])
        np.add.at(self.w, np.full(int(hi.sum()), self.n - 1, dtype=np.int64), weight[hi])
        mid = ~(lo | hi)
        rem = pos[mid] - idx[mid]
        np.add.at(self.w, idx[mid], (1.0 - rem) * weight[mid])
        np.add.at(self.w, idx[mid] + 1, rem * weight[mid])


class ChainSpectrum:
    def __init__(self, P, Nmax):
        self.pos = Bins(P, Nmax)
        self.neg = Bins(P, Nmax)

    def add(self, energy, weight):
        energy = np.asarray(energy, dtype=float).ravel()
        weight = np.asarray(weight, dtype=float).ravel()
        p = energy >= 0.0
        self.pos.add_many(energy[p], weight[p])
        self.neg.add_many(-energy[~p], weight[~p])


def _window(P, E, Emin, Ex, Emax, first, last):
    """src/spectrumrealfreq.cc:109-127 (vectorised)."""
    def fnc(x):
        if P["NNtanh"] > 0.0:
            f = lambda y: np.tanh(P["NNtanh"] * (y - 0.5))
            return (f(x) - f(0.0)) / (f(1.0) - f(0.0))
        return x
    out = np.zeros_like(E)
    a = (Emin < E) & (E <= Ex)
    b = (Ex < E) & (E < Emax)
    out[a] = fnc((E[a] - Emin) / (Ex - Emin))
    out[b] = 1.0 - fnc((E[b] - Ex) / (Emax - Ex))
    out[(E <= Emin) | (E >= Emax)] = 0.0
    if first:
        out[E >= Ex] = 1.0
    if last:
        out[E <= Ex] = 1.0
    return out


class Spectrum:
    """SpectrumRealFreq: merged spectrum of one operator pair."""

    def __init__(self, P, Nmax, name, kind, spectype):
        self.P = P
        self.name = name
        self.kind = kind          # "spec" (doublet) or "spin" (triplet) ...
        self.spectype = spectype  # "DMNRG" or "FDM"
        self.pos = Bins(P, Nmax)
        self.neg = Bins(P, Nmax)

    def merge(self, cs: ChainSpectrum, N, scale, Nmax, Ninit):
        P = self.P
        if self.spectype == "FDM":
            self.pos.w += cs.pos.w
            self.neg.w += cs.neg.w
            return
        # N/N+2 merge (mergeNN2, src/spectrumrealfreq.cc:139-185)
        if not (P["NN1"] or P["NN2avg"] or ((N % 2 == 0) if P["NN2even"] else (N % 2 == 1))):
            return
        factor = P["Lambda"] if (P["channels"] == 1 and not P["NN1"]) else math.sqrt(P["Lambda"])
        Emin = scale * P["goodE"]
        Ex = scale * P["goodE"] * factor
        Emax = scale * P["goodE"] * factor ** 2
        for full, part in ((self.pos, cs.pos), (self.neg, cs.neg)):
            e = part.e
            w = part.w
            sel = (Emin < e) & (e < Emax) & (w != 0.0)
            f = 0.5 if P["NN2avg"] else 1.0
            win = _window(P, e[sel], Emin, Ex, Emax, N == Ninit, N + 1 == Nmax)
            full.w[sel] += f * w[sel] * win

    def trimmed(self, b: Bins):
        """Bins::trim (src/bins.h:163-190)."""
        e, w = b.e, b.w
        keep = []
        for i in range(len(e) - 1):
            if not (abs(w[i]) < self.P["discard_trim"] * (e[i + 1] - e[i])):
                keep.append(i)
        keep.append(len(e) - 1)
        return e[keep], w[keep]

    def output(self, outdir):
        ep, wp = self.trimmed(self.pos)
        en, wn = self.trimmed(self.neg)
        fn = os.path.join(outdir, "%s_%s_dens_%s" % (self.kind, self.spectype, self.name))
        if self.P["savebins"]:
            arr = np.concatenate([np.stack([ep, wp], 1), np.stack([-en, wn], 1)])
            arr.astype("<f8").tofile(fn + ".bin")
        if self.P["broaden"]:
            dens = broaden(self.P, ep, wp, en, wn)
            with open(fn + ".dat", "w") as fh:
                for E, v in dens:
                    fh.write("%s %s\n" % (_g(E, self.P["prec_xy"]), _g(v, self.P["prec_xy"])))
        return {"pos_e": ep, "pos_w": wp, "neg_e": en, "neg_w": wn}


def _g(x, prec):
    return "%.*g" % (prec, x)


def _cpp_g(x, prec):
    """An ostream's default float format at setprecision(prec), i.e. %g."""
    return "%.*g" % (prec, x)


def my_fcmp(x, y, eps):
    """my_fcmp (src/numerics.h:37-53): 0 when x and y agree to the relative
    tolerance eps (absolute when both are below eps), else the sign of x-y."""
    if x == 0.0 and y == 0.0:
        return 0
    if abs(x) < eps and abs(y) < eps:
        return 0
    if abs(x - y) / (abs(x) + abs(y)) < eps:
        return 0
    return 1 if x > y else -1


def broaden(P, ep, wp, en, wn):
    """SpectrumRealFreq::continuous with BR_NEW (src/spectrumrealfreq.cc:271-306,
    src/spectral.h:70-102); returns [(E, value)] sorted by E."""
    alpha = P["alpha"]
    omega0 = P["omega0_ratio"] * P["T"] if P["omega0"] < 0 else P["omega0"]
    gamma = alpha / 4.0
    last_scale = SCALE(P, P["Nmax"])
    bmin = P["broaden_min_ratio"] * last_scale if P["broaden_min"] <= 0 else P["broaden_min"]
    mesh = []
    E = P["broaden_max"]
    while E > bmin:
        mesh.append(E)
        E /= P["broaden_ratio"]

    def br_l(e, ept):
        same = ((e > 0) & (ept > 0)) | ((e < 0) & (ept < 0))
        with np.errstate(divide="ignore", invalid="ignore"):
            v = np.exp(-(np.log(e / ept) / alpha - gamma) ** 2) / (alpha * abs(e) * math.sqrt(math.pi))
        return np.where(same & (ept != 0), v, 0.0)

    def br_new(e, ept):
        pl = br_l(e, ept)
        if abs(e) > omega0:
            return pl
        brh = math.exp(-(math.log(abs(e) / omega0) / alpha) ** 2)
        brg = np.exp(-((e - ept) / omega0) ** 2) / (omega0 * math.sqrt(math.pi))
        return pl * brh + brg * (1 - brh)

    pos, neg = [], []
    for E in mesh:
        vp = np.sum(wp * br_new(E, ep)) + np.sum(wn * br_new(E, -en))
        vn = np.sum(wp * br_new(-E, ep)) + np.sum(wn * br_new(-E, -en))
        pos.append((E, vp))
        neg.append((-E, vn))
    return sorted(neg) + sorted(pos)


# ---------------------------------------------------------------------------
# the NRG run
# ---------------------------------------------------------------------------

@dataclass
class Eig:
    value: np.ndarray          # eigenvalues (ascending; GS-subtracted after step)
    vec: np.ndarray            # columns are eigenvectors (dim x nr)
    shift: float = 0.0
    absenergy: np.ndarray = None
    kept: int = 0


@dataclass
class StepRecord:
    """What the reference stores per step (dm[N] and unitary<N>)."""
    eig: Dict[tuple, Eig]
    rmax: Dict[tuple, List[int]]
    kept: Dict[tuple, int]
    total: Dict[tuple, int]
    Egs: float


class Oracle:
    def __init__(self, workdir, threads=1, eigh_driver=None, spill_dir=None, progress=False):
        """threads: blocks diagonalised concurrently (OpenMP over blocks,
        src/nrg.cc:2484-2507), each with one BLAS thread; 1 leaves BLAS its
        own threads.  eigh_driver: "ev" (dsyev), "evd" or "evr" for every
        block; None follows the `diag` parameter as the reference does
        (src/read-input.cc:16-33, src/diag.h:297-311): dsyev by default,
        dsyevr for blocks of at least `dsyevrlimit` with diag=dsyevr."""
        self.dir = workdir
        self.P = read_params(os.path.join(workdir, "param"))
        self.threads = max(1, int(threads))
        self.eigh_driver = eigh_driver
        # spill_dir: keep each step's eigenvectors in .npy files there,
        # memory-mapped (the reference's unitary<N> files, src/dmnrg.h:183-304),
        # for runs whose eigenvectors exceed the host memory
        self.spill_dir = spill_dir
        self.progress = progress
        if self.P["diag"] not in ("default", "dsyev", "dsyevr"):
            raise ValueError("Unknown diagonalization routine: %s" % self.P["diag"])
        self.timing = {}

    # -- time bookkeeping (Timing sections of src/nrg.h:135-213) --
    def _tadd(self, name, t):
        self.timing[name] = self.timing.get(name, 0.0) + t

    def setup(self):
        P = self.P
        self.D = read_data(os.path.join(self.dir, "data"))
        D = self.D
        if D.symtype != "QS":
            raise NotImplementedError("oracle supports symtype QS")
        P["channels"] = D.channels
        if P["Nmax"] == 0:
            P["Nmax"] = D.Nmax
        assert len(D.xi[0]) - 1 == P["Nmax"]
        self.nch = D.channels
        self.combs = 4 ** D.channels
        self.In = qs.IN[D.channels]
        self.QN = qs.QN[D.channels]
        self.Nmax = P["Nmax"]
        self.Ninit = P["Ninit"]
        self.specd = [s for s in P["specd"].split() if s]
        self.spect = [s for s in P["spect"].split() if s]

    def xi(self, N, ch):
        return self.D.xi[ch][N]

    def zeta(self, N, ch):
        return self.D.zeta[ch][N]

    # ---- sweep 1 pieces ----
    def subspaces(self, prev):
        out = set()
        for I, e in prev.items():
            if e.kept > 0:
                for d in self.In:
                    J = qs.combine(qs.inverse(d), I)
                    if qs.allowed(J):
                        out.add(J)
        return sorted(out)

    def ancestors(self, I):
        return [qs.combine(d, I) for d in self.In]

    def rmax_of(self, I, prev):
        r = []
        for i, anc in enumerate(self.ancestors(I)):
            if qs.triangle(I, anc, self.QN[i]) and anc in prev:
                r.append(prev[anc].kept)
            else:
                r.append(0)
        return r

    def assemble(self, N, I, prev, rmax, opch):
        """nrg_prepare_task_for_diag + makematrix (upper triangle, then
        symmetrised like dsyev reading one triangle)."""
        P = self.P
        anc = self.ancestors(I)
        off = np.concatenate([[0], np.cumsum(rmax)])
        n = int(off[-1])
        h = np.zeros((n, n))
        sl = math.sqrt(P["Lambda"])
        for i in range(self.combs):
            if rmax[i]:
                a, b = off[i], off[i + 1]
                h[np.arange(a, b), np.arange(a, b)] = sl * prev[anc[i]].value[:rmax[i]]
        scale1 = SCALE(P, N + 1)
        ss = I[1]
        for (i, j, ch, factor) in qs.offdiag_terms(self.nch, ss):
            i0, j0 = i - 1, j - 1
            if not (rmax[i0] > 0 and rmax[j0] > 0):
                continue
            fs = factor * self.xi(N, ch) / scale1
            if not math.isfinite(fs):
                raise RuntimeError("offdiag factor not finite")
            if abs(fs) < 1e-8:
                continue
            key = (anc[i0], anc[j0])
            if key not in opch[ch]:
                raise RuntimeError("<||f||> subspace does not exist: %r" % (key,))
            M = opch[ch][key]
            h[off[i0]:off[i0 + 1], off[j0]:off[j0 + 1]] += fs * M
        for (i, ch, number) in qs.diag_terms(self.nch):
            i0 = i - 1
            shift = self.zeta(N + 1, ch) * (number - 1.0) / scale1
            h[np.arange(off[i0], off[i0 + 1]), np.arange(off[i0], off[i0 + 1])] += shift
        # dsyev with UPLO='L' on the row-major upper triangle
        h = np.triu(h) + np.triu(h, 1).T
        return h

    def diagonalise(self, h):
        if h.shape[0] == 0:
            return np.zeros(0), np.zeros((0, 0))
        drv = self.eigh_driver
        if drv is None:
            drv = "evr" if (self.P["diag"] == "dsyevr" and h.shape[0] >= self.P["dsyevrlimit"]) else "ev"
        w, v = sla.eigh(h, driver=drv, check_finite=False)
        return w, v

    def find_clusters(self, energies):
        """src/splitting.cc:45-77, reproduced with its quirks (the last
        cluster is not processed; the map persists across steps)."""
        eps = self.P["fixeps"]
        e0 = energies[0]
        i0 = 0
        csize = 1
        for i in range(len(energies)):
            if energies[i] - e0 < eps:
                csize += 1
            else:
                i1 = i
                if csize > 1:
                    seg = energies[i0:i1]
                    if np.any(seg != seg[0]):
                        rep = energies[i0]
                        for k in range(i0 + 1, i1):
                            if energies[k] != energies[i0]:
                                self.cluster_map.setdefault(float(energies[k]), float(rep))
                e0 = energies[i]
                i0 = i
                csize = 1

    def fix_splittings(self, diag):
        changed = False
        if not self.cluster_map:
            return False
        for I, e in diag.items():
            for r in range(len(e.value)):
                x = float(e.value[r])
                if x in self.cluster_map:
                    e.value[r] = self.cluster_map[x]
                    changed = True
        return changed

    def highest_retained_energy(self, energies):
        P = self.P
        assert energies[0] == 0.0
        total = len(energies)
        if P["keepenergy"] <= 0.0:
            nrkeep = P["keep"]
        else:
            nrkeep = 1 + int(np.count_nonzero(energies <= P["keepenergy"]))
            nrkeep = min(max(nrkeep, P["keepmin"]), P["keep"])
        if P["safeguard"] > 0.0:
            extra = 0
            while (nrkeep < total and energies[nrkeep] - energies[nrkeep - 1] <= P["safeguard"]
                   and extra < P["safeguardmax"]):
                nrkeep += 1
                extra += 1
        nrkeep = min(max(nrkeep, 1), total)
        return energies[nrkeep - 1]

    def truncate_prepare(self, diag, N, dmnrg_run):
        energies = np.sort(np.concatenate([e.value for e in diag.values()]))
        Emax = self.highest_retained_energy(energies)
        last = (N + 1 == self.Nmax)
        for I, e in diag.items():
            cnt = int(np.count_nonzero(e.value <= Emax))
            if (self.P["cfs"] or self.P["fdm"]) and last and not self.P["lastalloverride"]:
                cnt = len(e.value)
            if dmnrg_run and last and self.P["lastall"]:
                cnt = len(e.value)
            e.kept = cnt

    def td(self, diag, N):
        """nrg_calculate_TD (src/nrg.cc:2333-2369)."""
        P = self.P
        f = P["betabar"]
        Z = E = E2 = 0.0
        for I, e in diag.items():
            bE = f * e.value
            ex = np.exp(-bE)
            m = qs.mult(I)
            Z += m * ex.sum()
            E += m * (bE * ex).sum()
            E2 += m * (bE * bE * ex).sum()
        E /= Z
        E2 /= Z
        C = E2 - E * E
        F = -math.log(Z)
        S = E - F
        trSZ, trQ, trQ2 = qs.td_fields({I: e.value for I, e in diag.items()}, f)
        T = SCALE(P, N + 1) / P["betabar"]
        return [T, trSZ / Z, trQ / Z, trQ2 / Z, E, E2, C, F, S]

    @staticmethod
    def block(e: Eig, off, r, k):
        """U block of split_in_blocks: rows = first k eigenvectors, columns =
        the r components of combination block at `off` -> returns (k x r)."""
        return e.vec[off:off + r, :k].T

    def recalc_f(self, diag, rmax):
        """recalc_irreduc + recalc_f: new <I1||f^dag||Ip> blocks."""
        offs = {I: np.concatenate([[0], np.cumsum(rmax[I])]) for I in diag}
        opch = [dict() for _ in range(self.nch)]
        for Ip, ep in diag.items():
            for (I1, ch, rows) in qs.recalc_f_tables(self.nch, Ip):
                if I1 not in diag:
                    continue
                e1 = diag[I1]
                k1, kp = e1.kept, ep.kept
                if k1 == 0 or kp == 0:
                    continue
                f = np.zeros((k1, kp))
                for (i1, ip, factor) in rows:
                    r1 = rmax[I1][i1 - 1]
                    rp = rmax[Ip][ip - 1]
                    if not (r1 > 0 and rp > 0):
                        continue
                    assert r1 == rp
                    U1 = self.block(e1, offs[I1][i1 - 1], r1, k1)
                    Up = self.block(ep, offs[Ip][ip - 1], rp, kp)
                    f += factor * (U1 @ Up.T)
                opch[ch][(I1, Ip)] = f
        return opch

    def recalc_general(self, diag, rmax, cold, I1, Ip, rows, Iop, nstates):
        if not qs.triangle(I1, Ip, Iop):
            return None
        e1, ep = diag[I1], diag[Ip]
        k1, kp = nstates(e1), nstates(ep)
        cn = np.zeros((k1, kp))
        if k1 == 0 or kp == 0:
            return cn
        off1 = np.concatenate([[0], np.cumsum(rmax[I1])])
        offp = np.concatenate([[0], np.cumsum(rmax[Ip])])
        for (i1, ip, factor) in rows:
            IN1 = qs.combine(self.In[i1 - 1], I1)
            INp = qs.combine(self.In[ip - 1], Ip)
            if not (qs.allowed(IN1) and qs.allowed(INp)):
                continue
            r1 = rmax[I1][i1 - 1]
            rp = rmax[Ip][ip - 1]
            if r1 == 0 or rp == 0:
                continue
            key = (IN1, INp)
            cnt = key in cold
            if not qs.triangle(IN1, Iop, INp) and not cnt:
                continue
            if not cnt:
                raise RuntimeError("cold.count(ININ) != 1 for %r" % (key,))
            m = cold[key]
            m = m[:r1, :rp]
            U1 = self.block(e1, off1[i1 - 1], r1, k1)
            Up = self.block(ep, offp[ip - 1], rp, kp)
            temp = m @ Up.T
            cn += factor * (U1 @ temp)
        return cn

    def recalc_op(self, kind, diag, rmax, cold, nstates):
        cnew = {}
        if kind == "s":
            rows = [(i, i, 1.0) for i in range(1, self.combs + 1)]
            for I1 in diag:
                c = self.recalc_general(diag, rmax, cold, I1, I1, rows, qs.SINGLET, nstates)
                if c is not None:
                    cnew[(I1, I1)] = c
        elif kind == "d":
            for I1 in diag:
                for (Ip, rows) in qs.doublet_tables(self.nch, I1):
                    if Ip in diag:
                        c = self.recalc_general(diag, rmax, cold, I1, Ip, rows, qs.DOUBLET, nstates)
                        if c is not None:
                            cnew[(I1, Ip)] = c
        elif kind == "t":
            for I1 in diag:
                for (Ip, rows) in qs.triplet_tables(self.nch, I1):
                    if Ip in diag:
                        c = self.recalc_general(diag, rmax, cold, I1, Ip, rows, qs.TRIPLET, nstates)
                        if c is not None:
                            cnew[(I1, Ip)] = c
        return cnew

    # ---------------------------------------------------------------
    def _diag_all(self, tasks):
        if self.threads > 1 and len(tasks) > 1:
            from threadpoolctl import threadpool_limits
            with threadpool_limits(limits=1, user_api="blas"):
                with ThreadPoolExecutor(self.threads) as ex:
                    return list(ex.map(self.diagonalise, tasks))
        return [self.diagonalise(h) for h in tasks]

    def sweep1(self):
        import time
        P, D = self.P, self.D
        prev = {I: Eig(value=v.copy(), vec=np.eye(len(v)), kept=len(v)) for I, v in D.energies.items()}
        opch = [dict(b) for b in D.opch]
        ops = {k: {n: dict(b) for n, b in v.items()} for k, v in D.ops.items()}
        self.cluster_map = {}
        totalenergy = D.gs_energy
        self.steps: List[StepRecord] = []
        self.td_rows = []
        self.annotated = []
        self.expv_rows = []
        self.stats = []
        if P["calc0"]:
            self.calc0(ops)
        for N in range(self.Ninit, self.Nmax):
            scale = SCALE(P, N + 1)
            subs = self.subspaces(prev)
            rmax = {}
            tasks = []
            order = []
            for I in subs:
                r = self.rmax_of(I, prev)
                if sum(r) == 0:
                    continue
                rmax[I] = r
                order.append(I)
            t0 = time.perf_counter()
            hs = [self.assemble(N, I, prev, rmax[I], opch) for I in order]
            t1 = time.perf_counter()
            res = self._diag_all(hs)
            t2 = time.perf_counter()
            self._tadd("assemble", t1 - t0)
            self._tadd("diag", t2 - t1)
            diag = {I: Eig(value=w.copy(), vec=v) for I, (w, v) in zip(order, res)}
            Egs = min(e.value[0] + e.shift for e in diag.values())
            for e in diag.values():
                e.value -= Egs
                e.shift = Egs
            energies = np.sort(np.concatenate([e.value for e in diag.values()]))
            self.find_clusters(energies)
            if self.fix_splittings(diag):
                energies = np.sort(np.concatenate([e.value for e in diag.values()]))
                self.find_clusters(energies)
            self.truncate_prepare(diag, N, dmnrg_run=False)
            totalenergy += Egs * scale
            for e in diag.values():
                e.absenergy = totalenergy + e.value * scale
            self.td_rows.append(self.td(diag, N))
            if P["dumpannotated"]:
                self.annotated.append((scale, totalenergy,
                                       sorted((float(x), I) for I, e in diag.items() for x in e.value)))
            if self.spill_dir:
                for I, e in diag.items():
                    fn = os.path.join(self.spill_dir, "u%d_%d_%d.npy" % (N, I[0], I[1]))
                    np.save(fn, e.vec)
                    e.vec = np.load(fn, mmap_mode="r")
            if self.progress:
                print("oracle step %d: %d blocks, kept %d of %d" % (N, len(diag), sum(e.kept for e in diag.values()),
                                                                   sum(len(e.value) for e in diag.values())),
                      flush=True)
            rec = StepRecord(eig={I: Eig(value=e.value.copy(), vec=e.vec, shift=e.shift,
                                         absenergy=e.absenergy.copy(), kept=e.kept)
                                  for I, e in diag.items()},
                             rmax=rmax, kept={I: e.kept for I, e in diag.items()},
                             total={I: len(e.value) for I, e in diag.items()}, Egs=Egs)
            self.steps.append(rec)
            self.stats.append((len(order), min(sum(r) for r in rmax.values()),
                               max(sum(r) for r in rmax.values()),
                               sum(e.kept for e in diag.values()), sum(len(e.value) for e in diag.values())))
            last = (N + 1 == self.Nmax)
            t0 = time.perf_counter()
            if not last:
                opch = self.recalc_f(diag, rmax)
            t1 = time.perf_counter()
            self._tadd("recalc f", t1 - t0)
            kept_n = lambda e: e.kept
            newops = {}
            for kind, named in ops.items():
                newops[kind] = {}
                for name, blocks in named.items():
                    need = (kind == "s") or (kind == "d" and self._needed_d(name)) or \
                           (kind == "t" and self._needed_t(name))
                    if need:
                        newops[kind][name] = self.recalc_op(kind, diag, rmax, blocks, kept_n)
                    else:
                        newops[kind][name] = {}
            ops = newops
            self._tadd("recalc ops", time.perf_counter() - t1)
            # expectation values of singlet operators (nrg_measure_singlet)
            Zs = sum(qs.mult(I) * np.exp(-P["betabar"] * e.value[:e.kept]).sum() for I, e in diag.items())
            row = {}
            for name, blocks in ops.get("s", {}).items():
                tr = 0.0
                for I, e in diag.items():
                    nI = blocks[(I, I)]
                    tr += qs.mult(I) * np.sum(np.exp(-P["betabar"] * e.value[:e.kept]) * np.diag(nI))
                row[name] = tr / Zs
            self.expv_rows.append((scale / P["betabar"], row))
            # truncate and move on
            prev = {}
            for I, e in diag.items():
                prev[I] = Eig(value=e.value[:e.kept].copy(), vec=None, kept=e.kept)
        self.totalenergy = totalenergy
        self.GSenergy = totalenergy
        self.last_prev = prev
        self.final_ops = ops

    def calc0(self, ops):
        """docalc0 (src/nrg.cc:3063-3070, called from start_run at 3183-3186
        when calc0 is set, the default of src/param.cc:490): thermodynamics,
        the annotated energies and the singlet expectation values of the
        initial cluster read from `data`, at N = Ninit - 1, i.e. at the
        temperature SCALE(Ninit)/betabar (STAT::set_N, src/nrg.cc:545-553).
        All states of the cluster count (calc_Z, src/nrg.cc:1460-1467)."""
        P, D = self.P, self.D
        diag0 = {I: Eig(value=np.asarray(v, dtype=float).copy(), vec=None, kept=len(v))
                 for I, v in D.energies.items()}
        self.td_rows.append(self.td(diag0, self.Ninit - 1))
        if P["dumpannotated"]:
            self.annotated.append((SCALE(P, self.Ninit), D.gs_energy,
                                   sorted((float(x), I) for I, e in diag0.items() for x in e.value)))
        Zs = sum(qs.mult(I) * np.exp(-P["betabar"] * e.value).sum() for I, e in diag0.items())
        row = {}
        for name, blocks in ops.get("s", {}).items():
            tr = 0.0
            for I, e in diag0.items():
                nI = np.asarray(blocks[(I, I)])
                tr += qs.mult(I) * np.sum(np.exp(-P["betabar"] * e.value) * np.diag(nI))
            row[name] = tr / Zs
        self.expv_rows.append((SCALE(P, self.Ninit) / P["betabar"], row))

    def _needed_d(self, name):
        return any(name in pair.split("-") for pair in self.specd)

    def _needed_t(self, name):
        return any(name in pair.split("-") for pair in self.spect)

    # ---- density matrices ----
    def init_rho(self):
        P = self.P
        scale = SCALE(P, self.Nmax)
        last = self.steps[-1]
        ZZ = 0.0
        for I, e in last.eig.items():
            ZZ += qs.mult(I) * np.exp(-e.value[:e.kept] * scale / P["T"]).sum()
        rho = {}
        for I, e in last.eig.items():
            rho[I] = np.diag(np.exp(-e.value[:e.kept] * scale / P["T"]) / ZZ)
        return rho

    def trace(self, rho):
        return sum(qs.mult(I) * np.trace(m) for I, m in rho.items())

    def cdm_step(self, N, rho_by_child, accumulate_into, kept_prev):
        """calc_densitymatrix_iterN: rho_{N-1}[I] += sum_i coef U_i^T rho_N U_i."""
        rec = self.steps[N - self.Ninit]
        for I, dim in kept_prev.items():
            out = accumulate_into.setdefault(I, np.zeros((dim, dim)))
            if dim == 0:
                continue
            for i in range(self.combs):
                child = qs.combine(qs.inverse(self.In[i]), I)
                coef = qs.mult(child) / qs.mult(I)
                if child not in rho_by_child or child not in rec.eig:
                    continue
                r = rho_by_child[child]
                nomega = r.shape[0]
                if nomega == 0:
                    continue
                rm = rec.rmax[child][i]
                if rm == 0:
                    continue
                assert rm == dim
                off = int(sum(rec.rmax[child][:i]))
                Z = rec.eig[child].vec[off:off + dim, :nomega]      # = U^T
                out += coef * (Z @ r @ Z.T)

    def calc_densitymatrix(self):
        rho = self.init_rho()
        assert abs(self.trace(rho) - 1.0) < 1e-8
        self.rho = {self.Nmax - 1: rho}
        for N in range(self.Nmax - 1, self.Ninit, -1):
            kept_prev = self.steps[N - 1 - self.Ninit].kept
            rp = {}
            self.cdm_step(N, self.rho[N], rp, kept_prev)
            tr = self.trace(rp)
            if abs(tr - 1.0) > 1e-10 * max(1.0, abs(tr)) * 100:
                raise RuntimeError("check_trace_rho failed: %r" % tr)
            self.rho[N - 1] = rp

    def calc_ZnD(self):
        P = self.P
        Nlen = self.Nmax
        self.ZnD = np.zeros(Nlen)
        for N in range(self.Ninit, Nlen):
            rec = self.steps[N - self.Ninit]
            last = (N + 1 == self.Nmax)
            Z = 0.0
            for I, e in rec.eig.items():
                lo = 0 if last else rec.kept[I]
                Eabs = e.absenergy[lo:] - self.GSenergy
                assert np.all(Eabs >= -1e-14)
                Z += qs.mult(I) * np.exp(np.longdouble(-Eabs / P["T"])).sum()
            self.ZnD[N] = Z
        Ztot = 0.0
        for N in range(self.Ninit, Nlen):
            Ztot += float(self.combs) ** (Nlen - N - 1) * self.ZnD[N]
        self.ZZ = Ztot
        self.wn = np.array([float(self.combs) ** (Nlen - N - 1) * self.ZnD[N] / Ztot
                            for N in range(Nlen)])
        assert abs(self.wn.sum() - 1.0) < 1e-12 * 10
        with np.errstate(invalid="ignore", divide="ignore"):
            w = self.wn / self.ZnD
        self.wnfactor = np.where(np.isnan(w), 0.0, w)

    def init_rho_fdm(self, N):
        P = self.P
        rec = self.steps[N - self.Ninit]
        last = (N + 1 == self.Nmax)
        out = {}
        for I, e in rec.eig.items():
            tot = rec.total[I]
            lo = 0 if last else rec.kept[I]
            d = np.zeros(tot)
            Eabs = e.absenergy[lo:] - self.GSenergy
            with np.errstate(invalid="ignore", divide="ignore"):
                val = np.exp(-Eabs / P["T"]) * (self.wn[N] / self.ZnD[N])
            d[lo:] = np.where(np.isfinite(val), val, 0.0)
            out[I] = np.diag(d)
        return out

    def calc_fulldensitymatrix(self):
        rho = self.init_rho_fdm(self.Nmax - 1)
        self.rhofdm = {self.Nmax - 1: rho}
        for N in range(self.Nmax - 1, self.Ninit, -1):
            kept_prev = self.steps[N - 1 - self.Ninit].kept
            rp = {}
            self.cdm_step(N, self.rhofdm[N], rp, kept_prev)
            if N + 1 != self.Nmax:
                self.cdm_step(N, self.init_rho_fdm(N), rp, kept_prev)
            tr = self.trace(rp)
            expected = self.wn[N:].sum()
            if abs((tr - expected) / expected) > 1e-10:
                raise RuntimeError("FDM trace %r vs %r" % (tr, expected))
            self.rhofdm[N - 1] = rp

    # ---- sweep 2: spectra ----
    def sweep2(self):
        import time
        P, D = self.P, self.D
        ops = {k: {n: dict(b) for n, b in v.items()} for k, v in D.ops.items()}
        totalenergy = D.gs_energy
        spectra = []
        for pair in self.specd:
            a, b = pair.split("-")
            if P["dmnrg"]:
                spectra.append((Spectrum(P, self.Nmax, pair, "spec", "DMNRG"), "d", a, b))
            if P["fdm"]:
                spectra.append((Spectrum(P, self.Nmax, pair, "spec", "FDM"), "d", a, b))
        for pair in self.spect:
            a, b = pair.split("-")
            if P["dmnrg"]:
                spectra.append((Spectrum(P, self.Nmax, pair, "spin", "DMNRG"), "t", a, b))
            if P["fdm"]:
                spectra.append((Spectrum(P, self.Nmax, pair, "spin", "FDM"), "t", a, b))
        recalc_all = P["fdm"] or P["cfs"]
        for N in range(self.Ninit, self.Nmax):
            scale = SCALE(P, N + 1)
            rec = self.steps[N - self.Ninit]
            diag = {I: Eig(value=e.value.copy(), vec=e.vec, shift=e.shift,
                           absenergy=e.absenergy - self.GSenergy) for I, e in rec.eig.items()}
            Egs = min(e.value[0] + e.shift for e in diag.values())
            energies = np.sort(np.concatenate([e.value for e in diag.values()]))
            self.find_clusters(energies)
            if self.fix_splittings(diag):
                energies = np.sort(np.concatenate([e.value for e in diag.values()]))
                self.find_clusters(energies)
            self.truncate_prepare(diag, N, dmnrg_run=True)
            totalenergy += Egs * scale
            last = (N + 1 == self.Nmax)
            t0 = time.perf_counter()
            nst = (lambda e: len(e.value)) if recalc_all else (lambda e: e.kept)
            newops = {}
            for kind, named in ops.items():
                newops[kind] = {}
                for name, blocks in named.items():
                    need = (kind == "d" and self._needed_d(name)) or (kind == "t" and self._needed_t(name))
                    newops[kind][name] = self.recalc_op(kind, diag, rec.rmax, blocks, nst) if need else {}
            ops = newops
            t1 = time.perf_counter()
            self._tadd("recalc ops (2)", t1 - t0)
            for (sp, kind, a, b) in spectra:
                cs = ChainSpectrum(P, self.Nmax)
                op1, op2 = ops[kind][a], ops[kind][b]
                if sp.spectype == "DMNRG":
                    rho = self.rho[N]
                    self.spec_dmnrg(diag, op1, op2, rho, cs, scale, kind)
                else:
                    rho = self.rhofdm[N]
                    self.spec_fdm(diag, op1, op2, rho, cs, N, last, kind)
                sp.merge(cs, N, scale, self.Nmax, self.Ninit)
            self._tadd("spec", time.perf_counter() - t1)
            # trim operators to the kept states for the next step
            for kind in ops:
                for name in ops[kind]:
                    ops[kind][name] = {k: m[:diag[k[0]].kept, :diag[k[1]].kept]
                                       for k, m in ops[kind][name].items()}
        if abs(totalenergy - self.GSenergy) > 1e-12 * max(1.0, abs(totalenergy)):
            raise RuntimeError("GSenergy != totalenergy")
        self.spectra = [s[0] for s in spectra]

    def _pairs(self, diag, op1, op2):
        for Ii in diag:
            for Ij in diag:
                II = (Ij, Ii)
                if II in op1 and II in op2:
                    yield Ij, Ii, op1[II], op2[II]

    def _factor(self, kind, Ii, Ij):
        if kind == "d":
            return qs.specdens_factor(Ii, Ij)
        return qs.dynamicsusceptibility_factor(Ii, Ij)

    def spec_dmnrg(self, diag, op1, op2, rho, cs, scale, kind):
        """SPEC_DMNRG::calc over subspace pairs (calc_generic order)."""
        P = self.P
        sign = -1.0 if kind == "d" else 1.0
        fac = P["Lambda"] if (self.nch == 1 and not P["NN1"]) else math.sqrt(P["Lambda"])
        Emin = P["goodE"]
        Emax = P["goodE"] * fac * fac
        for Ij, Ii, A, B in self._pairs(diag, op1, op2):
            sf = self._factor(kind, Ii, Ij)
            rp = rho.get(Ii, np.zeros((0, 0)))
            r1 = rho.get(Ij, np.zeros((0, 0)))
            dimp, dim1 = rp.shape[0], r1.shape[0]
            if dimp == 0 or dim1 == 0:
                continue
            Em = diag[Ii].value[:dimp]
            Ej = diag[Ij].value[:dim1]
            A_ = A[:dim1, :dimp]
            B_ = B[:dim1, :dimp]
            sumA = B_ @ rp.T                # (dim1 x dimp): sum_ri op2(rj,ri) rho_p(rm,ri)
            sumB = r1 @ A_                  # sum_ri rho_1(rj,ri) op1(ri,rm)
            w = sf * (sumA * A_ + (-sign) * sumB * B_)
            dE = Ej[:, None] - Em[None, :]
            ok = (np.abs(dE) >= Emin) & (np.abs(dE) <= Emax)
            cs.add(scale * dE[ok], w[ok])

    def spec_fdm(self, diag, op1, op2, rho, cs, N, last, kind):
        """SPEC_FDMgt + SPEC_FDMls (src/spec_FDM.cc:41-119)."""
        P = self.P
        sign = -1.0 if kind == "d" else 1.0
        wnf = self.wnfactor[N]
        T = P["T"]
        for Ij, Ii, A, B in self._pairs(diag, op1, op2):
            sf = self._factor(kind, Ii, Ij)
            ri = rho.get(Ii, np.zeros((0, 0)))
            rj = rho.get(Ij, np.zeros((0, 0)))
            reti = 0 if last else ri.shape[0]
            retj = 0 if last else rj.shape[0]
            alli = len(diag[Ii].value)
            allj = len(diag[Ij].value)
            Ei = diag[Ii].absenergy
            Ej = diag[Ij].absenergy
            dE = Ej[:, None] - Ei[None, :]          # (allj x alli)
            AB = A * B                              # op1(j,i) op2(j,i)
            # greater: A3 (D,D) + A2 (i in D, j in K): exp(-Ei/T)
            bi = np.exp(-Ei / T)
            bj = np.exp(-Ej / T)
            gt = sf * AB * wnf * bi[None, :]
            m = np.zeros_like(AB, dtype=bool)
            m[:, reti:] = True                      # i discarded, any j
            cs.add(dE[m], gt[m])
            if allj > 0 and reti > 0:
                op2rho = B[:allj, :reti] @ ri
                w = sf * A[retj:, :reti] * op2rho[retj:, :]
                cs.add(dE[retj:, :reti], w)
            # lesser: B3 (D,D), B2 (i D, j K) via rho, B1 (i K, j D)
            ls = sf * AB * (-sign) * wnf * bj[:, None]
            m = np.zeros_like(AB, dtype=bool)
            m[retj:, reti:] = True
            cs.add(dE[m], ls[m])
            if retj > 0 and alli > 0:
                rhoop2 = rj @ B[:retj, :alli]
                w = sf * A[:retj, reti:] * rhoop2[:, reti:] * (-sign)
                cs.add(dE[:retj, reti:], w)
            m = np.zeros_like(AB, dtype=bool)
            m[retj:, :reti] = True
            cs.add(dE[m], ls[m])

    # ---- outputs ----
    def write_outputs(self, outdir):
        P = self.P
        os.makedirs(outdir, exist_ok=True)
        names = ["T", "<Sz^2>", "<Q>", "<Q^2>", "<E>", "<E^2>", "C", "F", "S"]
        w, pr = P["width_td"], P["prec_td"]
        with open(os.path.join(outdir, "td"), "w") as fh:
            fh.write("#" + "".join("%*s " % (w, n) for n in names) + "\n")
            for row in self.td_rows:
                fh.write(" " + "".join("%*s " % (w, _g(v, pr)) for v in row) + "\n")
        if self.expv_rows and self.expv_rows[0][1]:
            wc, pc = P["width_custom"], P["prec_custom"]
            names = sorted(self.expv_rows[0][1])
            with open(os.path.join(outdir, "custom"), "w") as fh:
                fh.write("#" + "".join("%*s " % (wc, str(i + 1)) for i in range(len(names) + 1)) + "\n")
                fh.write("#" + "".join("%*s " % (wc, n) for n in ["T"] + names) + "\n")
                for T, row in self.expv_rows:
                    fh.write(" " + "".join("%*s " % (wc, _g(v, pc)) for v in [T] + [row[n] for n in names]) + "\n")
        if P["dumpannotated"]:
            self.write_annotated(os.path.join(outdir, "annotated.dat"))
        res = {}
        for sp in getattr(self, "spectra", []):
            res[(sp.kind, sp.spectype, sp.name)] = sp.output(outdir)
        return res

    def write_annotated(self, path):
        """dump_annotated (src/nrg.cc:2062-2107): per step the lowest
        `dumpannotated` levels (extended through a cluster within grouptol),
        grouped by degeneracy with their quantum numbers and total
        multiplicity, or every level with its quantum numbers when dumpgroups
        is off; energies in units of omega_N (dumpscaled) and relative to the
        ground state unless dumpabs (scaled_energy, src/nrg.cc:2052-2056).
        Steps are separated by an empty line."""
        P = self.P
        prec = P["dumpprecision"]
        gt = P["grouptol"]

        def en(e, scale, total):
            return e * (1.0 if P["dumpscaled"] else scale) + (total if P["dumpabs"] else 0.0)

        with open(path, "w") as fh:
            for scale, total, lst in self.annotated:
                ln = min(len(lst), int(P["dumpannotated"]))
                i = ln
                while i < len(lst) - 1 and i > 0:
                    if my_fcmp(lst[i][0], lst[i - 1][0], gt) == 0:
                        ln += 1
                        i += 1
                    else:
                        break
                if P["dumpgroups"]:
                    i = 0
                    while i < ln:
                        i0 = i
                        qn = []
                        deg = 0
                        while i < ln and my_fcmp(lst[i][0], lst[i0][0], gt) == 0:
                            qn.append("%d %d" % lst[i][1])
                            deg += qs.mult(lst[i][1])
                            i += 1
                        qn.sort()
                        fh.write(_cpp_g(en(lst[i0][0], scale, total), prec)
                                 + "".join(" (%s)" % q for q in qn) + " [%d]\n" % deg)
                else:
                    for e, I in lst:
                        fh.write("%s %d %d\n" % (_cpp_g(en(e, scale, total), prec), I[0], I[1]))
                fh.write("\n")

    def run(self, outdir=None):
        import time
        t0 = time.perf_counter()
        self.setup()
        self.sweep1()
        self._tadd("sweep1", time.perf_counter() - t0)
        if self.P["dm"]:
            t1 = time.perf_counter()
            if self.P["dmnrg"]:
                self.calc_densitymatrix()
            if self.P["fdm"]:
                self.calc_ZnD()
                self.calc_fulldensitymatrix()
            self._tadd("DM", time.perf_counter() - t1)
            t2 = time.perf_counter()
            self.sweep2()
            self._tadd("sweep2", time.perf_counter() - t2)
        if outdir:
            return self.write_outputs(outdir)
        return None


def run(workdir, outdir=None, threads=1):
    o = Oracle(workdir, threads=threads)
    o.run(outdir)
    return o
