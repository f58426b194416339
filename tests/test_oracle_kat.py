"""Known-answer tests that pin the CPU oracle where the reference has no
golden vectors (its Fortran cannot be built here).

Each test states the analytic or independent answer it checks against.
"""
import math

import os

import numpy as np
import pytest

import oracle
from essaitemporaire_lepic_module_b200 import config, reactions
from essaitemporaire_lepic_module_b200.constants import EPS0, ME, QE


@pytest.fixture(autouse=True)
def one_thread(oracle_lib):
    oracle.set_threads(1)


def test_ran2_park_miller_known_values():
    """Park & Miller (1988): from seed 1 the first draw is 16807/(2^31-1) and
    the 10000th seed is 1043618065 (Src/ran2.f90 is this generator)."""
    r, s = oracle.ran2(1)
    assert s == 16807 and r == 16807 * (1.0 / 2147483647)
    seed = 1
    for _ in range(10000):
        _, seed = oracle.ran2(seed)
    assert seed == 1043618065


def _apply_A(u, st):
    """Discrete operator of Src/mg.h on interior nodes: (A u) = sum a_nb u_nb + ac u."""
    h = st.h
    aw = EPS0 / (h[0] * h[0])
    an = EPS0 / (h[1] * h[1])
    at = EPS0 / (h[2] * h[2])
    ac = -(an + an + aw + aw + at + at)
    Au = np.zeros_like(u)
    c = u[1:-1, 1:-1, 1:-1]
    Au[1:-1, 1:-1, 1:-1] = (aw * u[1:-1, 1:-1, :-2] + aw * u[1:-1, 1:-1, 2:] + an * u[1:-1, :-2, 1:-1] +
                            an * u[1:-1, 2:, 1:-1] + at * u[:-2, 1:-1, 1:-1] + at * u[2:, 1:-1, 1:-1] +
                            ac * c)
    return Au


def test_pdesolver_manufactured_solution():
    """phi_exact with Dirichlet walls; b = A phi_exact on plasma nodes; the
    multigrid must return phi_exact to the solver tolerance."""
    st = config.build("box32")
    n1, n2, n3 = st.n
    z, y, x = np.meshgrid(np.arange(n3 + 3), np.arange(n2 + 3), np.arange(n1 + 3), indexing="ij")
    ex = 5.0 * np.sin(np.pi * (x - 1) / n1) * np.sin(2 * np.pi * (y - 1) / n2) * np.sin(np.pi * (z - 1) / n3)
    plasma = st.geom.bcnd == -1
    ex = np.where(plasma, ex, 0.0)
    Au = _apply_A(ex, st)
    b = np.zeros((n3 + 2, n2 + 2, n1 + 2))
    b[:, :, :] = Au[:n3 + 2, :n2 + 2, :n1 + 2]
    b = np.where(plasma[:n3 + 2, :n2 + 2, :n1 + 2], b, 0.0)
    phi = np.zeros_like(ex)
    k, ktot, res = oracle.pdesolver(st, phi, b, eps=1e-12)
    assert res < 1e-12
    assert np.abs(phi - ex).max() <= 1e-9 * np.abs(ex).max()


def test_pdesolver_point_charge_matches_sparse_direct_solve():
    """A point charge in a grounded 16^3 box: multigrid vs scipy's direct
    sparse solve of the same 7-point operator."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    st = config.build("box16")
    n1, n2, n3 = st.n
    b = np.zeros((n3 + 2, n2 + 2, n1 + 2))
    b[n3 // 2 + 1, n2 // 2 + 1, n1 // 2 + 1] = -QE * 1e18
    phi = np.zeros((n3 + 3, n2 + 3, n1 + 3))
    oracle.pdesolver(st, phi, b, eps=1e-13)
    # direct solve on interior nodes 2..n
    idx = -np.ones((n3 + 3, n2 + 3, n1 + 3), dtype=np.int64)
    inner = st.geom.bcnd == -1
    idx[inner] = np.arange(inner.sum())
    h = st.h
    aw, an, at = EPS0 / h[0] ** 2, EPS0 / h[1] ** 2, EPS0 / h[2] ** 2
    ac = -(an + an + aw + aw + at + at)
    rows, cols, vals = [], [], []
    zz, yy, xx = np.nonzero(inner)
    for (dz, dy, dx, a) in ((0, 0, 0, ac), (0, 0, 1, aw), (0, 0, -1, aw), (0, 1, 0, an), (0, -1, 0, an),
                            (1, 0, 0, at), (-1, 0, 0, at)):
        j = idx[zz + dz, yy + dy, xx + dx]
        m = j >= 0
        rows.append(idx[zz, yy, xx][m])
        cols.append(j[m])
        vals.append(np.full(m.sum(), a))
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))))
    rhs = b[zz, yy, xx]
    sol = spl.spsolve(A, rhs)
    got = phi[zz, yy, xx]
    assert np.abs(got - sol).max() <= 1e-8 * np.abs(sol).max()


def test_boris_gyration_phase_and_radius():
    """One electron in a uniform Bz, E = 0: the Boris rotation advances the
    gyro-phase by 2 atan(wc dt / 2) per step exactly and keeps |v_perp|
    (Src/main.f90:708-712 quotes this phase error)."""
    st = config.build("penning_small")
    nmax = 4
    S = oracle.State(st, nmax)
    L = st.geom.box
    v0 = 3e5
    S.vxp[0, 0] = [L[0] / 2, L[1] / 2, L[2] / 2, v0, 0.0, 0.0]
    S.np_tot[0] = 1
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    ng1 = st.geom.ngrid + 1
    wc = QE * st.Bconst[2] / ME
    steps = 50
    for _ in range(steps):
        oracle.part_mover(st, Ei, S, np.zeros((ng1, 2, 1)), np.zeros((1, 4)), 1)
    vx, vy = S.vxp[0, 0, 3], S.vxp[0, 0, 4]
    phase = math.atan2(vy, vx)
    want = steps * 2 * math.atan(wc * st.dt / 2)        # electron (q<0): counter-clockwise
    want = math.atan2(math.sin(want), math.cos(want))
    assert abs(phase - want) < 1e-10
    assert abs(math.hypot(vx, vy) - v0) < 1e-9 * v0


def test_boris_exb_drift():
    """One electron in uniform Ex and Bz starting at the E x B drift velocity
    (0, -Ex/Bz, 0): the Boris step keeps it there (the rotation of the drift-
    frame velocity zero is zero) and the particle moves by v_d dt per step."""
    st = config.build("penning_small")
    nmax = 4
    S = oracle.State(st, nmax)
    L = st.geom.box
    Ex, Bz = 1e3, st.Bconst[2]
    vd = -Ex / Bz
    y0 = L[1] / 2
    S.vxp[0, 0] = [L[0] / 2, y0, L[2] / 2, 0.0, vd, 0.0]
    S.np_tot[0] = 1
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    Ei[..., 0] = Ex
    ng1 = st.geom.ngrid + 1
    steps = 50
    for _ in range(steps):
        oracle.part_mover(st, Ei, S, np.zeros((ng1, 2, 1)), np.zeros((1, 4)), 1)
    vx, vy, vz = S.vxp[0, 0, 3:6]
    assert abs(vx) <= 1e-9 * abs(vd) and abs(vz) <= 1e-9 * abs(vd)
    assert abs(vy - vd) <= 1e-9 * abs(vd)
    assert abs((S.vxp[0, 0, 1] - y0) - steps * st.dt * vd) <= 1e-9 * abs(steps * st.dt * vd)


def test_cic_charge_conservation_and_sort_invariants():
    """Sum over nodes of np/kq * h^3 equals N Nm; the counting sort is a
    permutation, Plist is the inclusive cumulative cell count, keys ascend."""
    st = config.build("box16")
    S = oracle.load_part(st, nmax=st.n_particles() + 16)
    vol = st.h[0] * st.h[1] * st.h[2]
    for p in range(st.ntype):
        tot = (S.np[p] / st.kq).sum() * vol
        assert abs(tot - S.np_tot[p] * st.Nm[p]) <= 1e-12 * S.np_tot[p] * st.Nm[p]
    before = S.vxp[0, :S.np_tot[0]].copy()
    pl = oracle.part_sorting(st, S, 1)
    after = S.vxp[0, :S.np_tot[0]]
    n = st.n
    ic = ((after[:, 0] / st.h[0]).astype(int) + n[0] * ((after[:, 1] / st.h[1]).astype(int) +
                                                        n[1] * (after[:, 2] / st.h[2]).astype(int)) + 1)
    assert np.all(np.diff(ic) >= 0)
    counts = np.bincount(ic, minlength=len(pl))
    np.testing.assert_array_equal(pl[1:], np.cumsum(counts[1:]))
    a = before[np.lexsort(before.T[::-1])]
    b = after[np.lexsort(after.T[::-1])]
    np.testing.assert_array_equal(a, b)


def test_mcc_constant_cross_section_rate():
    """Only e-Ar elastic with constant sigma: the expected number of
    collisions per call is sum_i n_g sigma |v_i - v_g| ns_coll dt; the
    oracle's count must fall within 4 sigma of it."""
    st = config.build("mcc32")
    T = st.tables
    # keep the elastic reaction only (index 1)
    keep = [0, 3]
    from essaitemporaire_lepic_module_b200.reactions import Tables
    st.tables = Tables(sig_Er=T.sig_Er, sig=T.sig[keep], sigv_mx=T.sigv_mx[:, keep],
                       sig_list=np.zeros((10, 2), dtype=np.int32), p_ncol=np.zeros(10, dtype=np.int32),
                       Eth=T.Eth[keep], col_info=T.col_info[keep])
    st.tables.sig_list[0, 0] = 1
    st.tables.sig_list[1, 0] = 2
    st.tables.p_ncol[0] = 1
    st.tables.p_ncol[1] = 1
    S = oracle.load_part(st, nmax=int(st.n_particles() * 1.2))
    v = S.vxp[0, :S.np_tot[0], 3:6]
    speed = np.sqrt((v ** 2).sum(axis=1))          # electrons >> gas thermal speed
    nu = st.np_mx[2] * 1e-19 * speed
    expect = (nu * st.wl.ns_coll * st.dt).sum()
    tot = 0.0
    calls = 3
    for c in range(calls):
        Sc = S.copy()
        Sc.iseed[0] = 777 + c
        _, cnt, _ = oracle.collisions(st, Sc)
        tot += cnt[0]
    assert abs(tot - calls * expect) <= 4 * math.sqrt(calls * expect) + 0.01 * calls * expect


def test_ordering_python_matches_c():
    """The host restatement of ordering() (reactions.py) and the oracle's C
    restatement produce the same merged grid, tables and (sigma v)_max."""
    st = config.build("mcc32")
    chem_tables = reactions.argon_tables_synthetic()
    import os
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "c.dat")
        reactions.write_dat(path, st.wl.ions, [("[Ar]", -39.95, 0.0, 0.02585, 1.0)], chem_tables)
        chem = reactions.read_dat(path, 2.0, st.ngas)
    T = reactions.ordering(chem)
    Er, sig, sv, sl, pn = oracle.ordering(chem)
    np.testing.assert_array_equal(T.sig_Er, Er)
    np.testing.assert_array_equal(T.sig, sig)
    np.testing.assert_allclose(T.sigv_mx, sv, rtol=1e-15, atol=0)
    np.testing.assert_array_equal(T.sig_list, sl)
    np.testing.assert_array_equal(T.p_ncol, pn)


def test_ordering_of_the_reference_argon_file():
    """The reference's own input_dir/argon.dat (fixture tests/golden/
    argon_chem.npz: e, Ar+, Ar; the e-Ar+ Coulomb collision with a charged
    target, e-Ar elastic, excitation and ionization, Ar+-Ar elastic and
    charge exchange): the host and oracle restatements of ordering() agree,
    and the parsed reactions are the file's."""
    from essaitemporaire_lepic_module_b200.constants import KB
    path = os.path.join(os.path.dirname(__file__), "golden", "argon_chem.npz")
    chem = reactions.chemistry_from_arrays(np.load(path), 6.0, 0.5 / (KB * 300.0))
    assert [s.name for s in chem.species] == ["[e]", "[Ar+]", "[Ar]"]
    assert chem.labels[0] == "[e]+[Ar+]->[e]+[Ar+]" and chem.col_info[0, 3] == 2   # charged target
    assert [int(r[2 + r[0] + r[1]]) for r in chem.col_info] == [1, 1, 3, 2, 1, 4]   # reaction types
    np.testing.assert_array_equal(chem.Eth, [0.0, 0.0, 11.5, 15.8, 0.0, 0.0])
    T = reactions.ordering(chem)
    Er, sig, sv, sl, pn = oracle.ordering(chem)
    np.testing.assert_array_equal(T.sig_Er, Er)
    np.testing.assert_array_equal(T.sig, sig)
    np.testing.assert_allclose(T.sigv_mx, sv, rtol=1e-15, atol=0)
    np.testing.assert_array_equal(T.sig_list, sl)
    np.testing.assert_array_equal(T.p_ncol, pn)
    assert list(pn[:2]) == [4, 2]


def _periodic_profile(n, m):
    """A function of the node index that is periodic with period n (node 1 and
    node n + 1 coincide, ghost 0 is node n)."""
    j = np.arange(n + 3) - 1.0
    return m[0] + np.cos(2 * np.pi * j / n) + m[1] * np.sin(4 * np.pi * j / n)


def test_pdesolver_periodic_manufactured_solution():
    """Walls at both x ends, periodic planes in y and z (Src/sors.f90:113-231,
    Src/mg.f90:314-805): phi_exact periodic in y and z with phi = 0 on the
    walls, b = A phi_exact; the multigrid returns phi_exact on every
    unknown node and on the periodic ghosts."""
    st = config.build("pbc16")
    n1, n2, n3 = st.n
    x = np.arange(n1 + 3) - 1.0
    fx = np.sin(np.pi * x / n1)
    fx[0] = fx[-1] = 0.0
    ex = (_periodic_profile(n3, (0.5, 0.3))[:, None, None] * _periodic_profile(n2, (0.2, -0.4))[None, :, None] *
          fx[None, None, :] * 3.0)
    # the unknowns and the ghost planes the solver refreshes (y and z indices
    # 0..n+1; the outer ghosts n+2 are not read)
    unknown = st.geom.bcnd <= 0
    unknown[n3 + 2, :, :] = False
    unknown[:, n2 + 2, :] = False
    ex = np.where(st.geom.bcnd >= 1, 0.0, ex)
    b = np.ascontiguousarray(_apply_A(ex, st)[:n3 + 2, :n2 + 2, :n1 + 2])
    phi = np.zeros_like(ex)
    k, ktot, res = oracle.pdesolver(st, phi, b, eps=1e-12)
    assert res < 1e-12
    assert np.abs(np.where(unknown, phi - ex, 0.0)).max() <= 1e-8 * np.abs(ex).max()
    # walls keep their Dirichlet value
    assert not np.where(st.geom.bcnd >= 1, phi, 0.0).any()


def test_pdesolver_neumann_plane_is_the_mirror_of_the_full_box():
    """The Neumann plane at x = 0 (Src/sors.f90:113-117, getres at ir = 1,
    Src/mg.f90:826-832) makes the half box the mirror image of a box twice as
    long in x with the source reflected about its middle plane: the two
    solutions agree on the half box (periodic planes in y and z in both)."""
    half = config.build("nmn16")
    full = config.build("pbc32x16")
    n1, n2, n3 = half.n
    x = np.arange(n1 + 2) - 1.0
    src = (np.exp(-(x ** 2) / (2 * 5.0 ** 2))[None, None, :] *
           _periodic_profile(n2, (1.5, 0.3))[None, :n2 + 2, None] *
           _periodic_profile(n3, (2.0, -0.2))[:n3 + 2, None, None]) * (-1.6e-19 * 1e15)
    b_half = np.ascontiguousarray(src)
    b_full = np.zeros((n3 + 2, n2 + 2, 2 * n1 + 2))
    for ip in range(1, 2 * n1 + 2):             # full node ip <-> half node |ip - (n1+1)| + 1
        b_full[:, :, ip] = src[:, :, abs(ip - (n1 + 1)) + 1]
    phi_h = half.geom.phi.copy()
    phi_f = full.geom.phi.copy()
    oracle.pdesolver(half, phi_h, b_half, eps=1e-13)
    oracle.pdesolver(full, phi_f, b_full, eps=1e-13)
    mirror = phi_f[:, :, n1 + 1:2 * n1 + 2]       # full x nodes n1+1..2 n1+1 = half nodes 1..n1+1
    mine = phi_h[:, :, 1:n1 + 2]
    unknown = half.geom.bcnd[:, :, 1:n1 + 2] <= 0
    unknown[n3 + 2, :, :] = False
    unknown[:, n2 + 2, :] = False
    assert np.abs(np.where(unknown, mine - mirror, 0.0)).max() <= 1e-7 * np.abs(mirror).max()
    assert np.abs(mirror).max() > 0


def test_eheating_rate_and_temperature():
    """Src/part_expmover.f90:484-568: of the electrons in the heating region
    a fraction nudt is heated (binomial, within 4 sigma), their new
    velocities are Maxwellian of thermal speed vt (<v^2> = 1.5 vt^2, within
    4 sigma), electrons outside the region are untouched, and P_loss(2)
    equals the energy change."""
    st = config.build("box16")
    hz = config.Heating(xl_pow=0.4e-3, xr_pow=1.2e-3, nu_h=1.5e9)
    S = oracle.load_part(st, nmax=st.n_particles() + 16)
    before = S.vxp[0, :S.np_tot[0]].copy()
    _, nreg = oracle.heat_stats(st, S, hz)
    nudt = config.heating_params(st, hz)["nudt"]
    vt = 2.0 * st.vt0[0]
    P_loss = np.zeros((st.ntype, 4))
    nh = oracle.eheating(st, S, vt, P_loss, hz)
    after = S.vxp[0, :S.np_tot[0]]
    assert abs(nh - nreg * nudt) <= 4 * math.sqrt(nreg * nudt * (1 - nudt))
    changed = np.any(after != before, axis=1)
    assert changed.sum() == nh
    ix = (before[:, 0] / st.h[0]).astype(int) + 1
    hp = config.heating_params(st, hz)
    assert not changed[(ix < hp["ixl_pow"]) | (ix > hp["ixr_pow"])].any()
    v2 = (after[changed, 3:6] ** 2).sum(axis=1)
    # v^2 / vt^2 of a 3D Maxwellian is Gamma(3/2): mean 1.5, variance 1.5
    assert abs(v2.mean() / vt ** 2 - 1.5) <= 4 * math.sqrt(1.5 / nh)
    dE = 0.5 * st.Nm[0] * st.mass[0] * ((after[:, 3:6] ** 2).sum() - (before[:, 3:6] ** 2).sum())
    assert abs(P_loss[0, 1] - dE) <= 1e-9 * abs(dE)
