"""NRG workloads shared by the parity tests and smoke(): generated
`param`/`data` pairs (inputgen), readers of the output files, and the
comparison of two runs' outputs at the FP64 path's accuracy targets.

Output precision: every case prints td/custom with 16 significant digits
(prec_td, prec_custom) and the energy flow with 16 (dumpprecision), so the
files carry the digits that the 1e-8 (td, spectra) and 1e-10 (energies)
comparisons need."""
import collections
import glob
import hashlib
import os

import numpy as np

import inputgen

# printed precision of every case (the reference's defaults are 10 and 8)
PRECISION = {"prec_td": 16, "prec_custom": 16, "dumpprecision": 16}

CASES = {
    # SIAM at the particle-hole symmetric point, DM-NRG and FDM spectra
    "siam_ph": dict(model="siam", U=0.1, eps_d=-0.05, Gamma=0.01, Lambda=2.0, Nmax=16,
                    params={"keep": 120, "keepenergy": 10.0, "dmnrg": True, "fdm": True, "T": 1e-4,
                            "specd": "A_d-A_d", "bins": 50, "savebins": True, "broaden": True,
                            "dumpannotated": 20}),
    # asymmetric SIAM, larger Lambda, fixed-number truncation, FDM only
    "siam_asym": dict(model="siam", U=0.3, eps_d=-0.05, Gamma=0.03, Lambda=3.0, Nmax=12,
                      params={"keep": 200, "fdm": True, "T": 1e-3, "specd": "A_d-A_d", "bins": 40,
                              "savebins": True, "broaden": False, "dumpannotated": 1, "dumpgroups": False}),
    # single-channel Kondo model: spin (triplet) spectral function, DM-NRG
    "kondo1": dict(model="kondo", J=[0.3], Lambda=2.0, Nmax=14,
                   params={"keep": 150, "dmnrg": True, "fdm": True, "T": 1e-4, "spect": "SZd-SZd",
                           "bins": 30, "savebins": True, "broaden": False, "dumpannotated": 30}),
    # the plain-method SIAM workload at full size: Nmax=30, keep 500 or
    # 10 omega_N, DM-NRG A(omega) at T=1e-8, 50 bins per decade
    "siam_nmax30": dict(model="siam", U=0.1, eps_d=-0.05, Gamma=0.01, Lambda=2.0, Nmax=30,
                        params={"keep": 500, "keepenergy": 10.0, "dmnrg": True, "T": 1e-8,
                                "specd": "A_d-A_d", "bins": 50, "savebins": True, "broaden": True,
                                "dumpannotated": 20}),
    # two-channel Kondo model (QS tables derived from spin coupling): spin and
    # channel-0 f spectra, DM-NRG and FDM
    "kondo2ch": dict(model="kondo", J=[0.2, 0.2], Lambda=3.0, Nmax=10,
                     params={"keep": 300, "dmnrg": True, "fdm": True, "T": 1e-3, "spect": "SZd-SZd",
                             "specd": "A_f0-A_f0", "bins": 30, "savebins": True, "broaden": False,
                             "dumpannotated": 1, "dumpgroups": False}),
    # three-channel Kondo model with unequal couplings (QS tables derived for
    # 64 combinations, the oracle's and the host's derivations): spin and f
    # spectra of channels 0 and 2, DM-NRG and FDM
    "kondo3ch": dict(model="kondo", J=[0.3, 0.2, 0.1], Lambda=3.0, Nmax=3,
                     params={"keep": 150, "keepenergy": 2.5, "dmnrg": True, "fdm": True, "T": 1e-2,
                             "spect": "SZd-SZd", "specd": "A_f0-A_f0 A_f2-A_f2", "bins": 20, "savebins": True,
                             "broaden": False, "dumpannotated": 1, "dumpgroups": False}),
    # one run of the served z-averaging workload (z = 5/8, Nmax = 40, T = 1e-6),
    # at its smallest Nkeep: FDM A(omega)
    "siam_zshift": dict(model="siam", U=0.2, eps_d=-0.1, Gamma=0.02, Lambda=2.0, Nmax=40, z=0.625,
                        params={"keep": 200, "fdm": True, "T": 1e-6, "specd": "A_d-A_d", "bins": 50,
                                "savebins": True, "broaden": False, "dumpannotated": 40}),
}


# Full-size workloads whose oracle runs take minutes to hours on the host: the
# GPU tests compare with committed oracle outputs (tests/golden/nrg/*.npz,
# made by tests/golden/make_nrg_goldens.py).
GOLDEN_CASES = {
    # runs of the served z-averaging stream at its bench temperature T = 1e-6,
    # one per Nkeep class above the smallest (z = 5/8, eps_d = -0.1, Nmax = 40)
    **{"served_k%d" % k: dict(model="siam", U=0.2, eps_d=-0.1, Gamma=0.02, Lambda=2.0, Nmax=40, z=0.625,
                              params={"keep": k, "fdm": True, "T": 1e-6, "specd": "A_d-A_d", "bins": 50,
                                      "savebins": True, "broaden": False, "dumpannotated": 40})
       for k in (500, 1000, 2000)},
    # the precision workload: SIAM U = 0.5, eps_d = -0.25, Gamma = 0.04,
    # Lambda = 2, Nmax = 40, keep 2000, FDM A(omega) at T = 1e-7; the GPU runs
    # it in FP64 and with split-precision products (gemm_slices)
    "siam_c4": dict(model="siam", U=0.5, eps_d=-0.25, Gamma=0.04, Lambda=2.0, Nmax=40,
                    params={"keep": 2000, "fdm": True, "T": 1e-7, "specd": "A_d-A_d", "bins": 50,
                            "savebins": True, "broaden": False, "dumpannotated": 40}),
    # two-channel Kondo model at full size: J = 0.2 per channel, Lambda = 3,
    # Nmax = 40, keep 3000 (blocks up to ~8000), FDM spectra of three operator
    # pairs at T = 1e-6, 50 bins per decade
    # The per-bin absolute floor of this case is n_max eps = 2e-12 of the
    # largest bin instead of 1e-13: a bin's weight is a sum of products of
    # eigenvector components of blocks up to ~8000 carried through 40
    # recalculations, and two summation orders of n terms differ by up to
    # about n eps of the sum of magnitudes.  Two FP64 GPU builds that differ
    # only in the tridiagonalisation kernel differ by 1.7e-8 relative on a
    # bin of 3e-5 of the largest (5e-13 of it).
    "kondo2ch_full": dict(model="kondo", J=[0.2, 0.2], Lambda=3.0, Nmax=40, wabs=2e-12,
                          params={"keep": 3000, "fdm": True, "T": 1e-6, "spect": "SZd-SZd",
                                  "specd": "A_f0-A_f0 A_f1-A_f1", "bins": 50, "savebins": True,
                                  "broaden": False, "dumpannotated": 40}),
}


def make_case(name, path):
    c = CASES[name] if name in CASES else GOLDEN_CASES[name]
    os.makedirs(path, exist_ok=True)
    params = dict(PRECISION)
    params.update(c["params"])
    if c["model"] == "siam":
        inputgen.make_siam(path, c["U"], c["eps_d"], c["Gamma"], c["Lambda"], c["Nmax"], z=c.get("z", 1.0),
                           params=params)
    else:
        inputgen.make_kondo(path, c["J"], c["Lambda"], c["Nmax"], params=params)
    return path


def input_digest(path):
    """sha256 of the case's `param` and `data` files (pins a golden to its inputs)."""
    h = hashlib.sha256()
    for f in ("param", "data"):
        with open(os.path.join(path, f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def read_table(path):
    rows = []
    with open(path) as fh:
        for line in fh:
            if line.startswith("#") or not line.strip():
                continue
            rows.append([float(x) for x in line.split()])
    return np.array(rows)


def read_bins(path):
    a = np.fromfile(path, dtype="<f8")
    return a.reshape(-1, 2)


def read_annotated(path):
    """annotated.dat (src/nrg.cc:2062-2107) as a list of steps; each step is a
    list of (energy, labels, degeneracy) with labels the sorted '(Q SS)'
    strings of a group (dumpgroups) or the one label of a level."""
    steps, cur = [], []
    with open(path) as fh:
        for line in fh:
            line = line.strip()
            if not line:
                steps.append(cur)
                cur = []
                continue
            if "[" in line:
                e, rest = line.split(" ", 1)
                labels = tuple(x.strip(" ()") for x in rest.split("[")[0].split(")") if x.strip(" ("))
                deg = int(rest.split("[")[1].rstrip("]"))
                cur.append((float(e), labels, deg))
            else:
                f = line.split()
                cur.append((float(f[0]), (" ".join(f[1:]),), 0))
    if cur:
        steps.append(cur)
    return steps


def load_outputs(outdir):
    """Every output file of a run that the parity tests compare."""
    out = {"td": read_table(os.path.join(outdir, "td")), "bins": {}, "dat": {}}
    if os.path.exists(os.path.join(outdir, "custom")):
        out["custom"] = read_table(os.path.join(outdir, "custom"))
    if os.path.exists(os.path.join(outdir, "annotated.dat")):
        with open(os.path.join(outdir, "annotated.dat")) as fh:
            out["annotated"] = fh.read()
    for f in sorted(glob.glob(os.path.join(outdir, "*.bin"))):
        out["bins"][os.path.basename(f)] = read_bins(f)
    for f in sorted(glob.glob(os.path.join(outdir, "*_dens_*.dat"))):
        out["dat"][os.path.basename(f)] = read_table(f)
    return out


def _parse_annotated_text(text):
    import tempfile
    with tempfile.NamedTemporaryFile("w", suffix=".dat", delete=False) as fh:
        fh.write(text)
        name = fh.name
    try:
        return read_annotated(name)
    finally:
        os.unlink(name)


# Accuracy targets of the plain FP64 path against the oracle.
RTOL_TD = 1e-8      # td (chi(T) = <Sz^2>, S(T), ...) and custom, relative, ...
ATOL_TD = 1e-12     # ... plus 1e-12 absolute: every column is a ratio of sums of O(1) terms, and a
                    # column that vanishes by symmetry (<Q> at particle-hole symmetry) keeps
                    # their FP64 cancellation noise (up to ~2e-13 here), which differs run to run
RTOL_E = 1e-10      # energy flow (annotated.dat), relative
ATOL_E = 1e-12      # floor for levels at or near the ground state (E = 0)
RTOL_W = 1e-8       # spectral weight per bin, relative, where |w| >= WFLOOR max|w|, ...
WFLOOR = 1e-6
WABS = 1e-13        # ... plus the FP64 rounding floor of the sums that make a bin (1e-13 max|w|)
RTOL_WMAX = 1e-8    # every bin (the tail included), relative to the largest bin


def compare_outputs(got, ref, what="", wabs=None):
    """Assert that run `got` reproduces run `ref` (dicts of load_outputs) at
    the FP64 targets: td and custom within 1e-8 relative (columns that vanish
    by symmetry against 1e-13 of the column scale), energies of the energy
    flow within 1e-10 relative (1e-12 absolute at E ~ 0) with identical
    quantum numbers and degeneracies (td/custom also 1e-12 absolute, the
    cancellation noise of columns that vanish by symmetry), spectral bins
    within 1e-8 relative per
    bin wherever |w| >= 1e-6 of the largest bin and within 1e-8 of the largest
    bin everywhere (the per-bin check allows an absolute 1e-13 of the
    largest bin, the FP64 rounding level of the sums behind a small bin),
    broadened spectra within 1e-8 of their maximum.  `wabs` replaces the
    per-bin absolute floor (a fraction of the largest bin) for runs whose
    blocks are large enough to need a higher one."""
    wabs = WABS if wabs is None else wabs
    to, tg = ref["td"], got["td"]
    assert to.shape == tg.shape, (what, to.shape, tg.shape)
    tol = RTOL_TD * np.abs(to) + ATOL_TD
    assert np.all(np.abs(tg - to) <= tol), (what, "td", float(np.max((np.abs(tg - to) - tol) / (np.abs(to) + 1e-300))))
    if "custom" in ref:
        co, cg = ref["custom"], got["custom"]
        assert co.shape == cg.shape, (what, "custom shape")
        assert np.all(np.abs(cg - co) <= RTOL_TD * np.abs(co) + ATOL_TD), (what, "custom")
    if "annotated" in ref:
        assert "annotated" in got, (what, "annotated.dat missing")
        ao, ag = _parse_annotated_text(ref["annotated"]), _parse_annotated_text(got["annotated"])
        assert len(ao) == len(ag), (what, "annotated steps", len(ao), len(ag))
        for n, (so, sg) in enumerate(zip(ao, ag)):
            assert len(so) == len(sg), (what, "annotated step", n, len(so), len(sg))
            eo = np.array([x[0] for x in so])
            eg = np.array([x[0] for x in sg])
            assert np.all(np.abs(eg - eo) <= RTOL_E * np.abs(eo) + ATOL_E), \
                (what, "energy flow", n, float(np.max(np.abs(eg - eo))))
            if so and so[0][2]:  # grouped: labels and degeneracies per group
                assert [x[1:] for x in so] == [x[1:] for x in sg], (what, "annotated groups", n)
            else:
                assert collections.Counter(x[1] for x in so) == collections.Counter(x[1] for x in sg)
    assert sorted(ref["bins"]) == sorted(got["bins"]), (what, sorted(ref["bins"]), sorted(got["bins"]))
    assert ref["bins"], what
    for name in ref["bins"]:
        a, b = ref["bins"][name], got["bins"][name]
        # trimming may keep or drop bins at the 1e-16 level: compare on the union grid
        da = dict(zip(a[:, 0], a[:, 1]))
        db = dict(zip(b[:, 0], b[:, 1]))
        keys = sorted(set(da) | set(db))
        wo = np.array([da.get(k, 0.0) for k in keys])
        wg = np.array([db.get(k, 0.0) for k in keys])
        wmax = np.max(np.abs(wo))
        err = np.abs(wg - wo)
        assert np.max(err) <= RTOL_WMAX * wmax, (what, name, "max-normalised", float(np.max(err) / wmax))
        big = np.abs(wo) >= WFLOOR * wmax
        assert np.all(err[big] <= RTOL_W * np.abs(wo[big]) + wabs * wmax), \
            (what, name, "per bin", float(np.max(err[big] / np.abs(wo[big]))))
    assert sorted(ref["dat"]) == sorted(got["dat"]), what
    for name in ref["dat"]:
        a, b = ref["dat"][name], got["dat"][name]
        assert a.shape == b.shape and np.allclose(a[:, 0], b[:, 0], rtol=1e-9, atol=0), (what, name)
        amax = np.max(np.abs(a[:, 1]))
        assert np.all(np.abs(a[:, 1] - b[:, 1]) <= RTOL_TD * amax + 1e-9 * np.abs(a[:, 1])), (what, name)


def save_golden(path, outputs, digest, meta):
    """Write a run's outputs as a compressed .npz fixture."""
    arrays = {"td": outputs["td"], "digest": np.array(digest), "meta": np.array(repr(meta))}
    if "custom" in outputs:
        arrays["custom"] = outputs["custom"]
    if "annotated" in outputs:
        arrays["annotated"] = np.array(outputs["annotated"])
    for k, v in outputs["bins"].items():
        arrays["bin:" + k] = v
    for k, v in outputs["dat"].items():
        arrays["dat:" + k] = v
    np.savez_compressed(path, **arrays)


def load_golden(path):
    z = np.load(path, allow_pickle=False)
    out = {"td": z["td"], "bins": {}, "dat": {}}
    if "custom" in z:
        out["custom"] = z["custom"]
    if "annotated" in z:
        out["annotated"] = str(z["annotated"])
    for k in z.files:
        if k.startswith("bin:"):
            out["bins"][k[4:]] = z[k]
        elif k.startswith("dat:"):
            out["dat"][k[4:]] = z[k]
    return out, str(z["digest"])


def error_report(got, ref):
    """Largest relative errors of run `got` against `ref` (load_outputs
    dicts): energies of the energy flow, chi(T) (T<Sz^2>) and S(T) of td, and
    the spectral weights per bin (bins above 1e-6 of the largest)."""
    out = {}
    ao, ag = _parse_annotated_text(ref["annotated"]), _parse_annotated_text(got["annotated"])
    e, ea = 0.0, 0.0
    for so, sg in zip(ao, ag):
        for x, y in zip(so, sg):
            ea = max(ea, abs(y[0] - x[0]))
            if abs(x[0]) >= 1e-2:  # relative error of levels above 1e-2 omega_N
                e = max(e, abs(y[0] - x[0]) / abs(x[0]))
    out["energies"] = e
    out["energies_abs"] = ea
    to, tg = ref["td"], got["td"]
    out["chi_T"] = float(np.max(np.abs(tg[:, 1] - to[:, 1]) / np.abs(to[:, 1])))
    out["S_T"] = float(np.max(np.abs(tg[:, 8] - to[:, 8]) / np.maximum(np.abs(to[:, 8]), 1e-300)))
    w = 0.0
    for name in ref["bins"]:
        a, b = ref["bins"][name], got["bins"][name]
        da, db = dict(zip(a[:, 0], a[:, 1])), dict(zip(b[:, 0], b[:, 1]))
        wmax = max(abs(v) for v in da.values())
        for k, v in da.items():
            if abs(v) >= WFLOOR * wmax:
                w = max(w, abs(db.get(k, 0.0) - v) / abs(v))
    out["spectra_per_bin"] = w
    return out
