"""The Wilson-chain generator against reference-held golden data: the
restatement of tools/adapt/nrgchain.cc (inputgen.wilson_chain_tabulated)
applied to the reference's own fixtures (tools/adapt/Delta.dat and the mesh
ODE solutions GSOL/FSOL, copied to tests/golden/adapt/ by
tests/golden/make_adapt_fixtures.py) reproduces the reference's xi.dat and
zeta.dat (Lambda = 2, z = 0.5, mMAX = 50, Nmax = 30, adapt = true, the
sample `param` of tools/adapt).  Also: the three flat-band discretizations
(Y, C, Z) agree where they must."""
import os

import numpy as np
import pytest

import inputgen as g

D = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "adapt")


def test_tabulated_chain_reproduces_the_reference_fixture():
    R = g.read_two_columns
    xi, zeta, theta = g.wilson_chain_tabulated(R(D + "/Delta.dat"), R(D + "/GSOL.dat"), R(D + "/GSOLNEG.dat"),
                                               R(D + "/FSOL.dat"), R(D + "/FSOLNEG.dat"), 2.0, 0.5, 30, mMAX=50)
    # nrgchain writes xi / SCALE(n+1) (Z-scheme SCALE) and zeta unscaled
    sc = np.array([g.scale_factor(n + 1, 2.0, 0.5, "Z") for n in range(31)])
    xr = np.loadtxt(D + "/xi.dat")
    zr = np.loadtxt(D + "/zeta.dat")
    assert len(xr) == 31 and len(zr) == 31
    assert np.max(np.abs(xi / sc - xr) / np.abs(xr)) < 1e-14
    # the symmetric hybridisation gives zeta = 0 up to the rounding of the
    # tabulated inputs, which the restatement reproduces
    assert np.max(np.abs(zeta - zr)) < 1e-20
    assert abs(theta - 1.0) < 1e-8


def test_flat_band_discretizations_agree_at_z1():
    """At z = 1 the Y, C and Z star levels differ by one overall factor,
    which SCALE removes: the scaled chains coincide."""
    ref = None
    for d in "YCZ":
        xi, zeta = g.wilson_chain_flat(2.0, 1.0, 12, discretization=d)
        s = xi / np.array([g.scale_factor(n + 1, 2.0, 1.0, d) for n in range(13)])
        assert np.max(np.abs(zeta)) < 1e-14
        if ref is None:
            ref = s
        assert np.max(np.abs(s - ref) / ref) < 1e-13


@pytest.mark.parametrize("d", ["C", "Z"])
def test_flat_band_discretization_twisted(d):
    """z != 1: the scaled C/Z chains tend to 1 along the chain (the point of
    these schemes: no Lambda-dependent rescaling of the hopping) and the
    chain is particle-hole symmetric."""
    xi, zeta = g.wilson_chain_flat(2.0, 0.5, 30, discretization=d)
    s = xi / np.array([g.scale_factor(n + 1, 2.0, 0.5, d) for n in range(31)])
    assert np.max(np.abs(zeta)) < 1e-14
    assert abs(s[-1] - 1.0) < 1e-3
