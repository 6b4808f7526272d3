"""Copy the reference's own fixtures of the Wilson-chain generator for a
tabulated density of states (tools/adapt: the hybridisation function
Delta.dat, the mesh ODE solutions GSOL/FSOL for positive and negative
energies, and the chain coefficients xi.dat/zeta.dat that its nrgchain
program computes from them with the sample `param`: Lambda = 2, z = 0.5,
mMAX = 50, Nmax = 30, adapt = true) into tests/golden/adapt/, so that the
generator's test runs where the reference is absent.  Run in a container
that has the reference checkout:

    python tests/golden/make_adapt_fixtures.py /root/reference
"""
import os
import shutil
import sys

FILES = {"Delta.dat": "Delta.dat", "GSOL.dat.ref": "GSOL.dat", "GSOLNEG.dat.ref": "GSOLNEG.dat",
         "FSOL.dat.ref": "FSOL.dat", "FSOLNEG.dat.ref": "FSOLNEG.dat", "xi.dat.ref": "xi.dat",
         "zeta.dat.ref": "zeta.dat"}


def main(ref):
    src = os.path.join(ref, "tools", "adapt")
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "adapt")
    os.makedirs(dst, exist_ok=True)
    for a, b in FILES.items():
        shutil.copyfile(os.path.join(src, a), os.path.join(dst, b))
        print(a, "->", os.path.join(dst, b))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
