"""Pins against the reference's own committed output (tests/golden/).

The reference ships no test vectors for the hot path; its default run left
2D planes of the wall-label mask and of the time-averaged potential and
E-field (DATA/DATA_2D).  They pin two restatements:
  * the mask generator (Src/generate_boundary.f90) -- bit-exact labels;
  * the E-field stencil (Src/Efield.f90) -- the averaged E equals
    calc_Efield of the averaged phi (E is linear in phi), compared to the
    6 printed digits.
"""
import os

import numpy as np
import pytest

from essaitemporaire_lepic_module_b200.geometry import generate_boundary

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_default_planes.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


@pytest.fixture(scope="module")
def geom(gold):
    n = tuple(int(v) for v in gold["n"])
    segs = [list(r[:6]) + [int(r[6])] for r in gold["segments"]]
    return generate_boundary(n, list(gold["box_cm"]), segs, list(gold["V"]))


def test_geometry_planes_match_reference(gold, geom):
    n1, n2, n3 = geom.n
    b = geom.bcnd
    xy = b[n3 // 2 + 1, 1:n2 + 2, 1:n1 + 2]
    xz = b[1:n3 + 2, n2 // 2 + 1, 1:n1 + 2]
    yz = b[1:n3 + 2, 1:n2 + 2, n1 // 2 + 1]
    np.testing.assert_array_equal(xy, gold["bcnd_xy"])
    np.testing.assert_array_equal(xz, gold["bcnd_xz"])
    np.testing.assert_array_equal(yz, gold["bcnd_yz"])
    assert geom.flag_pbc == 1 and geom.flag_nmn == 0


def _extruded_phi(geom, plane, axis):
    """3D potential whose plane `axis` equals the printed plane everywhere
    (ghost nodes keep the wall potential 0 of this case)."""
    n1, n2, n3 = geom.n
    phi = np.zeros(geom.bcnd.shape)
    if axis == "z":
        phi[:, 1:n2 + 2, 1:n1 + 2] = plane[None, :, :]
    else:
        phi[1:n3 + 2, 1:n2 + 2, :] = plane[:, :, None]
    return phi


def _bound(phi_nb_abs, h, e_abs):
    # each value printed as 0.dddddd E+xx carries <= 5e-6 relative rounding;
    # a central difference mixes two phi values, a wall extrapolation three
    # differences
    return 3.0 * (5e-6 * phi_nb_abs / h) + 5e-6 * e_abs + 1e-9


def _check(E_calc, E_ref, phi_plane, h, what):
    # neighbourhood magnitude of phi entering each difference
    pa = np.abs(phi_plane)
    nb = pa.copy()
    for ax in (0, 1):
        for s in (1, 2):
            nb = np.maximum(nb, np.roll(pa, s, ax))
            nb = np.maximum(nb, np.roll(pa, -s, ax))
    tol = _bound(2 * nb, h, np.abs(E_ref))
    err = np.abs(E_calc - E_ref)
    bad = err > tol
    assert not bad.any(), f"{what}: {bad.sum()} nodes off, worst {np.max(err - tol):.3g}"


def test_efield_xy_plane_oracle(gold, geom, oracle_lib):
    from types import SimpleNamespace
    n1, n2, n3 = geom.n
    st = SimpleNamespace(n=geom.n, h=geom.h, geom=geom)
    phi = _extruded_phi(geom, gold["phi_xy"], "z")
    E = oracle_lib.calc_efield(st, phi)
    iz = n3 // 2 + 1
    _check(E[iz, 1:n2 + 2, 1:n1 + 2, 0], gold["Ex_xy"], gold["phi_xy"], geom.h[0], "Ex_xy")
    _check(E[iz, 1:n2 + 2, 1:n1 + 2, 1], gold["Ey_xy"], gold["phi_xy"], geom.h[1], "Ey_xy")


def test_efield_yz_plane_oracle(gold, geom, oracle_lib):
    from types import SimpleNamespace
    n1, n2, n3 = geom.n
    st = SimpleNamespace(n=geom.n, h=geom.h, geom=geom)
    phi = _extruded_phi(geom, gold["phi_yz"], "x")
    E = oracle_lib.calc_efield(st, phi)
    ix = n1 // 2 + 1
    _check(E[1:n3 + 2, 1:n2 + 2, ix, 1], gold["Ey_yz"], gold["phi_yz"], geom.h[1], "Ey_yz")
    _check(E[1:n3 + 2, 1:n2 + 2, ix, 2], gold["Ez_yz"], gold["phi_yz"], geom.h[2], "Ez_yz")


@pytest.mark.gpu
def test_efield_xy_plane_gpu(gold, geom):
    from types import SimpleNamespace
    from essaitemporaire_lepic_module_b200 import dropin
    n1, n2, n3 = geom.n
    st = SimpleNamespace(n=geom.n, h=geom.h, geom=geom)
    phi = _extruded_phi(geom, gold["phi_xy"], "z")
    E = dropin.calc_efield(st, phi)
    iz = n3 // 2 + 1
    _check(E[iz, 1:n2 + 2, 1:n1 + 2, 0], gold["Ex_xy"], gold["phi_xy"], geom.h[0], "Ex_xy")
    _check(E[iz, 1:n2 + 2, 1:n1 + 2, 1], gold["Ey_xy"], gold["phi_xy"], geom.h[1], "Ey_xy")
    phi = _extruded_phi(geom, gold["phi_yz"], "x")
    E = dropin.calc_efield(st, phi)
    ix = n1 // 2 + 1
    _check(E[1:n3 + 2, 1:n2 + 2, ix, 1], gold["Ey_yz"], gold["phi_yz"], geom.h[1], "Ey_yz")
    _check(E[1:n3 + 2, 1:n2 + 2, ix, 2], gold["Ez_yz"], gold["phi_yz"], geom.h[2], "Ez_yz")
