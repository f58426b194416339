"""B-field maps on the CPU: the map builders (Src/Bfield.f90, Src/main.f90:
361-431) and known answers of the oracle's map push
(Src/part_expmover.f90:148-203).

Known answers:
  * a map holding one uniform field, on the node grid or on its own grid,
    moves particles like the uniform field Bi(1:3,1,1,1) (to rounding: the
    interpolation weights sum to one to within an ulp);
  * a map below the 1e-5 T gate everywhere moves particles exactly like no
    field (leapfrog), bit for bit;
  * the gate looks at the left map node only: a particle whose left node is
    below the gate takes the leapfrog step even when its other nodes are
    above it;
  * with flag_B_pos = 1 positive ions ignore the map.
"""
import numpy as np
import pytest

import oracle
from essaitemporaire_lepic_module_b200 import bfield, config


def _grid_particles(st, n=64, seed=5):
    rng = np.random.default_rng(seed)
    S = oracle.State(st, n)
    L = np.array(st.geom.box)
    h = np.array(st.h)
    for p in range(st.ntype):
        S.vxp[p, :n, 0:3] = h + rng.uniform(0, 1, (n, 3)) * (L - 2 * h)
        S.vxp[p, :n, 3:6] = rng.normal(0, st.vt0[p] + 1e5, (n, 3))
        S.np_tot[p] = n
    return S


def _push(st, S, Ei, steps=1):
    ng1 = st.geom.ngrid + 1
    for _ in range(steps):
        for p in range(1, st.ntype + 1):
            oracle.part_mover(st, Ei, S, np.zeros((ng1, 2, st.ntype)), np.zeros((st.ntype, 4)), p)
    return S


def _uniform_setup(B):
    st = config.build("box16")
    st.flag_B = 1
    st.Bconst = np.array(B, dtype=np.float64)
    return st


def _fields(st, seed=2):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 2e4, tuple(st.geom.bcnd.shape) + (3,))


@pytest.mark.parametrize("own", [False, True])
def test_uniform_map_matches_uniform_field(own):
    B = (0.004, -0.007, 0.05)
    st_u = _uniform_setup(B)
    st_m = config.build("box16")
    bf = bfield.new_map(st_m, n_B=(8, 4, 8) if own else None)
    bf.Bi[..., 0:3] = B
    bfield.attach(st_m, bfield.finish(bf))
    assert abs(bf.Bmax - np.linalg.norm(B)) <= 1e-15
    E = _fields(st_u)
    Su = _push(st_u, _grid_particles(st_u), E, steps=20)
    Sm = _push(st_m, _grid_particles(st_m), E, steps=20)
    np.testing.assert_array_equal(Sm.np_tot, Su.np_tot)
    for p in range(st_u.ntype):
        n = Su.np_tot[p]
        a, b = Sm.vxp[p, :n], Su.vxp[p, :n]
        assert np.abs(a - b).max(axis=0).max() <= 1e-11 * np.abs(b).max()
    # and differs from no field at all (the map is used)
    st_0 = config.build("box16")
    S0 = _push(st_0, _grid_particles(st_0), E, steps=20)
    assert np.abs(S0.vxp[0, :64, 3:6] - Su.vxp[0, :64, 3:6]).max() > 1e-3 * np.abs(Su.vxp[0, :64, 3:6]).max()


def test_map_below_gate_is_leapfrog_bit_for_bit():
    st_m = config.build("box16")
    bf = bfield.new_map(st_m)
    bf.Bi[..., 2] = 0.9e-5
    bfield.attach(st_m, bfield.finish(bf))
    st_0 = config.build("box16")
    E = _fields(st_0)
    Sm = _push(st_m, _grid_particles(st_m), E, steps=5)
    S0 = _push(st_0, _grid_particles(st_0), E, steps=5)
    np.testing.assert_array_equal(Sm.vxp, S0.vxp)


def test_gate_reads_the_left_node_only():
    """|B| above the gate only on the node planes ix >= 9: a particle in a
    cell with left plane 8 (x in [7h, 8h)) is not magnetised although its
    right nodes carry the field; one in a cell with left plane 9 is."""
    st = config.build("box16")
    bf = bfield.new_map(st)
    bf.Bi[:, :, 9:, 2] = 0.05
    bfield.attach(st, bfield.finish(bf))
    st_0 = config.build("box16")
    h = st.h[0]
    E = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    S = oracle.State(st, 2)
    S0 = oracle.State(st_0, 2)
    for T in (S, S0):
        T.vxp[0, 0] = [7.5 * h, 8 * h, 8 * h, 0.0, 2e5, 0.0]    # left plane ix = 8
        T.vxp[0, 1] = [8.5 * h, 8 * h, 8 * h, 0.0, 2e5, 0.0]    # left plane ix = 9
        T.np_tot[0] = 2
    _push(st, S, E)
    _push(st_0, S0, E)
    np.testing.assert_array_equal(S.vxp[0, 0], S0.vxp[0, 0])
    assert abs(S.vxp[0, 1, 3]) > 1e3       # rotated by Bz = 0.05 T


def test_flag_B_pos_leaves_ions_unmagnetised():
    st = config.build("box16")
    bf = bfield.new_map(st)
    bf.Bi[..., 2] = 0.5
    bfield.attach(st, bfield.finish(bf), flag_B_pos=1)
    st_0 = config.build("box16")
    E = _fields(st_0)
    S = _push(st, _grid_particles(st), E, steps=3)
    S0 = _push(st_0, _grid_particles(st_0), E, steps=3)
    np.testing.assert_array_equal(S.vxp[1], S0.vxp[1])               # Ar+
    assert np.abs(S.vxp[0, :64, 3:6] - S0.vxp[0, :64, 3:6]).max() > 0  # e-


def test_map_builders():
    st = config.build("box16")
    bf = bfield.new_map(st)
    h = bf.h_B[0]
    np.testing.assert_allclose(bf.h_B, np.array(st.geom.box) / 16, rtol=0, atol=0)
    x0, Lx = 8 * h, 3 * h
    bfield.gaussian(bf, 0.02, x0, Lx, 2)
    # node ix sits at x = (ix-1) h_B: the peak is at ix = 9
    assert bf.Bi[4, 5, 9, 1] == pytest.approx(0.02, rel=0, abs=1e-18)
    assert bf.Bi[4, 5, 12, 1] == pytest.approx(0.02 * np.exp(-0.5), rel=1e-15)
    bfield.ee_magnets(bf, 0.01, x0=2e-3, z0=8 * h, d=4 * h)
    x = (7 - 1) * h
    z = (3 - 1) * h
    ex = np.exp(-np.pi * (2e-3 - x) / (4 * h))
    assert bf.Bi[3, 0, 7, 0] == pytest.approx(0.01 * np.sin(np.pi * (z - 8 * h) / (4 * h)) * ex, rel=1e-14)
    assert bf.Bi[3, 0, 7, 2] == pytest.approx(0.01 * np.cos(np.pi * (z - 8 * h) / (4 * h)) * ex, rel=1e-14)
    bfield.finish(bf)
    np.testing.assert_allclose(bf.Bi[..., 3], np.linalg.norm(bf.Bi[..., 0:3], axis=-1), rtol=1e-15)
    assert bf.Bmax == bf.Bi[..., 3].max()
    # the pseudo-1D Hall-thruster profile: Bx = 0, By independent of y and z
    ht = bfield.hall_thruster(bfield.new_map(st), -0.01, x0=0.75e-3, a=1e-3)
    assert not ht.Bi[..., 0].any()
    assert np.all(ht.Bi[..., 1] == ht.Bi[1:2, 1:2, :, 1])
    # the ELISE filter-field fit: the quartic up to 39 cm, the line beyond
    pg = bfield.new_map(st)
    pg.h_B[:] = 0.39 / 10.0
    bfield.pg_current(pg, 1.0, 1)
    x = 39.0
    # Src/Bfield.f90:85-92 writes the coefficients as single-precision
    # literals: the doubles of the fit are their float32 roundings
    a = [float(np.float32(v)) for v in (0.0175596, 0.0227362, 0.00193113, -8.51235e-05, 9.58673e-07)]
    b = [float(np.float32(v)) for v in (15.7416, -0.377132)]
    quart = a[0] + a[1] * x + a[2] * x ** 2 + a[3] * x ** 3 + a[4] * x ** 4
    assert pg.Bi[0, 0, 11, 0] == pytest.approx(quart, rel=1e-14)
    assert pg.Bi[0, 0, 12, 0] == pytest.approx(b[0] + b[1] * 42.9, rel=1e-14)
    exact = 0.0175596 + 0.0227362 * x + 0.00193113 * x ** 2 - 8.51235e-05 * x ** 3 + 9.58673e-07 * x ** 4
    assert 1e-9 < abs(quart - exact) / exact < 1e-6           # the single-precision rounding shows
    assert abs(quart - (b[0] + b[1] * x)) < 0.05               # nearly continuous at 39 cm


def test_read_map_file(tmp_path):
    st = config.build("box16")
    bf = bfield.new_map(st, n_B=(4, 4, 4))
    path = tmp_path / "Bz.dat"
    path.write_text("1 2 3 0.5\n4 4 4 -0.25\n1 2 3 0.25\n")
    bfield.read_map_file(bf, str(path), 3, scaling=2.0)
    assert bf.Bi[3, 2, 1, 2] == 1.5 and bf.Bi[4, 4, 4, 2] == -0.5
    assert np.count_nonzero(bf.Bi) == 2
    with pytest.raises(ValueError):
        bfield.attach(st, bfield.BField((4, 4, 4), bf.h_B, np.zeros((3, 3, 3, 4))))
