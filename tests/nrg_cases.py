"""Small NRG workloads shared by the parity tests and smoke(): generated
`param`/`data` pairs (inputgen) with their oracle results."""
import os

import numpy as np

import inputgen

CASES = {
    # SIAM at the particle-hole symmetric point, DM-NRG and FDM spectra
    "siam_ph": dict(model="siam", U=0.1, eps_d=-0.05, Gamma=0.01, Lambda=2.0, Nmax=16,
                    params={"keep": 120, "keepenergy": 10.0, "dmnrg": True, "fdm": True, "T": 1e-4,
                            "specd": "A_d-A_d", "bins": 50, "savebins": True, "broaden": True,
                            "dumpannotated": 20}),
    # asymmetric SIAM, larger Lambda, fixed-number truncation, FDM only
    "siam_asym": dict(model="siam", U=0.3, eps_d=-0.05, Gamma=0.03, Lambda=3.0, Nmax=12,
                      params={"keep": 200, "fdm": True, "T": 1e-3, "specd": "A_d-A_d", "bins": 40,
                              "savebins": True, "broaden": False}),
    # single-channel Kondo model: spin (triplet) spectral function, DM-NRG
    "kondo1": dict(model="kondo", J=[0.3], Lambda=2.0, Nmax=14,
                   params={"keep": 150, "dmnrg": True, "fdm": True, "T": 1e-4, "spect": "SZd-SZd",
                           "bins": 30, "savebins": True, "broaden": False}),
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
                             "specd": "A_f0-A_f0", "bins": 30, "savebins": True, "broaden": False}),
    # one run of the served z-averaging workload (z = 5/8, Nmax = 40), at its
    # smallest Nkeep: FDM A(omega)
    "siam_zshift": dict(model="siam", U=0.2, eps_d=-0.1, Gamma=0.02, Lambda=2.0, Nmax=40, z=0.625,
                        params={"keep": 200, "fdm": True, "T": 1e-5, "specd": "A_d-A_d", "bins": 50,
                                "savebins": True, "broaden": False}),
}


def make_case(name, path):
    c = CASES[name]
    os.makedirs(path, exist_ok=True)
    if c["model"] == "siam":
        inputgen.make_siam(path, c["U"], c["eps_d"], c["Gamma"], c["Lambda"], c["Nmax"], z=c.get("z", 1.0),
                           params=c["params"])
    else:
        inputgen.make_kondo(path, c["J"], c["Lambda"], c["Nmax"], params=c["params"])
    return path


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
