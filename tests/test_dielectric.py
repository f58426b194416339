"""Dielectric wall charging in the mover (Src/part_expmover.f90:302-348) on
the CPU oracle: the labels of generate_boundary (Src/generate_boundary.f90:
yr < 0 a Y = const dielectric, xr < 0 an X = const one), a hand-computed
known answer for one electron on each plane, and charge conservation --
each lost particle puts exactly Nm q on its plane; the potential update of
the walls from the sums (Src/main.f90:859-949)."""
import numpy as np
import pytest

import oracle
from essaitemporaire_lepic_module_b200 import config


def _sums(st):
    n1, n2, n3 = st.n
    return np.zeros((st.ntype, n3 + 3, n1 + 3)), np.zeros((st.ntype, n3 + 3, n2 + 3, 2))


def test_die16_labels():
    st = config.build("die16")
    g = st.geom
    assert g.flag_die == 1 and g.ngrid == 3
    np.testing.assert_array_equal(g.dtype_array(), [0, 1, 2, 3])
    n1, n2, n3 = st.n
    assert g.bcnd[5, n2 + 1, 5] == 2 and g.bcnd[5, 5, n1 + 1] == 3 and g.bcnd[5, 5, 1] == 1


def test_dielectric_known_answer():
    st = config.build("die16")
    h = st.h
    L = st.geom.box
    S = oracle.State(st, 8)
    # electron 0 crosses y = ymax, electron 1 crosses x = xmax
    S.vxp[0, 0] = [5.3 * h[0], L[1] - 0.1 * h[1], 7.6 * h[2], 0.0, 0.5 * h[1] / st.dt, 0.0]
    S.vxp[0, 1] = [L[0] - 0.1 * h[0], 5.3 * h[1], 7.6 * h[2], 0.5 * h[0] / st.dt, 0.0, 0.0]
    S.np_tot[0] = 2
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    qxz, qyz = _sums(st)
    pm = np.zeros((st.geom.ngrid + 1, 2, st.ntype))
    oracle.part_mover(st, Ei, S, pm, np.zeros((st.ntype, 4)), 1, sum_q=(qxz, qyz))
    assert S.np_tot[0] == 0
    assert pm[2, 0, 0] == 1 and pm[3, 0, 0] == 1
    k3 = st.Nm[0] * st.charge[0]
    want = np.zeros_like(qxz[0])
    px, pz = 6 - 5.3, 8 - 7.6
    want[8, 6] = k3 * px * pz
    want[8, 7] = k3 * (1 - px) * pz
    want[9, 7] = k3 * (1 - px) * (1 - pz)
    want[9, 6] = k3 * px * (1 - pz)
    np.testing.assert_allclose(qxz[0], want, rtol=1e-12, atol=0)
    # the same weights with y in place of x (n1 = n2)
    np.testing.assert_allclose(qyz[0, :, :, 0], want, rtol=1e-12, atol=0)
    assert not qyz[0, :, :, 1].any()
    assert not qxz[1:].any() and not qyz[1:].any()


def test_dielectric_charge_conservation():
    oracle.set_threads(1)
    st = config.build("die16")
    S = oracle.load_part(st, nmax=st.n_particles() + 16)
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    qxz, qyz = _sums(st)
    pm = np.zeros((st.geom.ngrid + 1, 2, st.ntype))
    pl = np.zeros((st.ntype, 4))
    for _ in range(6):
        for p in range(1, st.ntype + 1):
            oracle.part_mover(st, Ei, S, pm, pl, p, sum_q=(qxz, qyz))
    for p in range(st.ntype):
        k3 = st.Nm[p] * st.charge[p]
        n2, n3 = pm[2, 0, p], pm[3, 0, p]
        if p == 0:
            assert n2 > 50 and n3 > 50, (n2, n3)
        assert abs(qxz[p].sum() - k3 * n2) <= 1e-12 * abs(k3) * max(n2, 1)
        assert abs(qyz[p, ..., 0].sum() - k3 * n3) <= 1e-12 * abs(k3) * max(n3, 1)
        assert not qyz[p, ..., 1].any()


def test_step_loop_dielectric_guards():
    """the walls need a capacitance"""
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("die16")
    assert abs(st.Ca - 2e-8 * st.h[0] * st.h[2]) <= 1e-30
    st.Ca = 0.0
    with pytest.raises(ValueError):
        Simulation(st, cap=1000, device="cpu")


def _random_sums(st, seed):
    rng = np.random.default_rng(seed)
    qxz, qyz = _sums(st)
    qxz[...] = rng.normal(0.0, 1e-17, qxz.shape)
    qyz[...] = rng.normal(0.0, 1e-17, qyz.shape)
    return qxz, qyz


@pytest.mark.parametrize("pbc", [0, 1])
def test_dielectric_phi_known_answer(pbc):
    """Src/main.f90:859-949: Q/(2 Ca) per species on the Y plane's nodes,
    Q/Ca on the X plane's, the periodic-z doubling of rows 1, n3+1 and the
    copies into rows 0 and n3+2, nothing elsewhere, the sums cleared."""
    st = config.build("die16")
    st.geom.flag_pbc = pbc
    n1, n2, n3 = st.n
    qxz, qyz = _random_sums(st, 3)
    rxz, ryz = qxz.copy(), qyz.copy()
    phi = st.geom.phi.copy()
    oracle.dielectric_phi(st, phi, (qxz, qyz))
    assert not qxz.any() and not qyz.any()
    Ca = st.Ca

    def row(iz):
        if not pbc:
            return iz, 1.0
        if iz == 0:
            return n3, 2.0
        if iz == n3 + 2:
            return 2, 2.0
        return iz, 2.0 if iz in (1, n3 + 1) else 1.0

    for iz in (0, 1, 2, 7, n3, n3 + 1, n3 + 2):
        jz, f = row(iz)
        # a Y-plane node (label 2) and an X-plane node (label 3)
        want = st.geom.phi[iz, n2 + 1, 5]
        for p in range(st.ntype):
            want = want + (f * rxz[p, jz, 5]) / (2.0 * Ca)
        assert phi[iz, n2 + 1, 5] == want
        want = st.geom.phi[iz, 6, n1 + 1]
        for p in range(st.ntype):
            want = want + (f * ryz[p, jz, 6, 0]) / Ca
        assert phi[iz, 6, n1 + 1] == want
    other = st.geom.bcnd != 2
    other &= st.geom.bcnd != 3
    np.testing.assert_array_equal(phi[other], st.geom.phi[other])


def _corner_electron(st):
    """an electron that leaves through the y = ymax dielectric and z = zmax
    at once (the corner cell carries label 2)"""
    h, L = st.h, st.geom.box
    S = oracle.State(st, 4)
    S.vxp[0, 0] = [5.3 * h[0], L[1] - 0.1 * h[1], L[2] - 0.2 * h[2], 0.0, 0.5 * h[1] / st.dt,
                   0.5 * h[2] / st.dt]
    S.np_tot[0] = 1
    return S


def test_dielectric_periodic_z_wrap():
    """Src/part_expmover.f90:306-316: with periodic z planes the position of
    a particle lost on a dielectric wraps before the weights (z - zmax, row
    floor(z/h)+1)."""
    st = config.build("die16")
    st.geom.flag_pbc = 1
    S = _corner_electron(st)
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    qxz, qyz = _sums(st)
    pm = np.zeros((st.geom.ngrid + 1, 2, st.ntype))
    oracle.part_mover(st, Ei, S, pm, np.zeros((st.ntype, 4)), 1, sum_q=(qxz, qyz))
    assert S.np_tot[0] == 0 and pm[2, 0, 0] == 1
    k3 = st.Nm[0] * st.charge[0]
    zq = (st.geom.box[2] - 0.2 * st.h[2] + 0.5 * st.h[2]) - st.geom.box[2]
    iq = int(np.floor(zq / st.h[2])) + 1
    assert iq == 1
    px, pz = 6 - 5.3, (iq * st.h[2] - zq) / st.h[2]
    want = np.zeros_like(qxz[0])
    want[1, 6] = k3 * px * pz
    want[1, 7] = k3 * (1 - px) * pz
    want[2, 7] = k3 * (1 - px) * (1 - pz)
    want[2, 6] = k3 * px * (1 - pz)
    np.testing.assert_allclose(qxz[0], want, rtol=1e-9, atol=0)
