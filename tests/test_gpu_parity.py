"""GPU parity tests: the C-ABI drop-ins and device API against the CPU
oracle on the same seeded inputs.

Bars (from the benchmark definition, written in each test):
  * calc_rho, calc_Efield, one push, Poisson solve (same inputs): bit-exact
    where the operation order is fixed, else <= 1e-12 relative;
  * deposition: <= 1e-12 relative (atomic summation order);
  * sort: per-cell counts (Plist) bit-exact, same particles in every cell;
  * collisionless trajectories after 100 steps: <= 1e-10 relative;
  * MCC: collision counts per process within 3 sigma.
"""
import numpy as np
import pytest

import oracle
from essaitemporaire_lepic_module_b200 import config, dropin
from tests.conftest import have_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / den


@pytest.fixture(scope="module")
def box16():
    oracle.set_threads(1)
    st = config.build("box16")
    S = oracle.load_part(st, nmax=st.n_particles() + 4096)
    dropin.set_commons(st)
    return st, S


@pytest.fixture(scope="module")
def mcc32():
    oracle.set_threads(1)
    st = config.build("mcc32")
    S = oracle.load_part(st, nmax=int(st.n_particles() * 1.3))
    T = st.tables
    dropin.set_commons(st, ncol=T.sig.shape[0], npt=T.sig_Er.shape[0], p_ncol=T.p_ncol)
    return st, S


def solved_fields(st, S):
    rhs = oracle.calc_rho(st, S.np.copy())
    phi = st.geom.phi.copy()
    oracle.pdesolver(st, phi, rhs)
    E = oracle.calc_efield(st, phi)
    return rhs, phi, E


def test_calc_rho_bit_exact(box16):
    st, S = box16
    dropin.set_commons(st)
    r_o = oracle.calc_rho(st, S.np.copy())
    r_g = dropin.calc_rho(st, S.np.copy())
    np.testing.assert_array_equal(r_g, r_o)


@pytest.mark.parametrize("name", ["box16", "box32", "poisson32", "penning_small", "pbc16", "nmn16"])
def test_pdesolver_matches_oracle(name):
    """Same schedule (V-cycles, sweeps per level) and phi to <= 1e-12
    (pbc16: periodic planes in y and z; nmn16: the Neumann plane at x = 0
    as well)."""
    st = config.build(name)
    dropin.set_commons(st)
    if st.rhs_blobs is not None:
        rhs = st.rhs_blobs
    else:
        # electrons alone: the co-located e/ion load makes the full rho zero
        S = oracle.load_part(st, nmax=st.n_particles() + 4096)
        npg = S.np.copy()
        npg[1:] = 0.0
        rhs = oracle.calc_rho(st, npg)
    for warm in (False, True):
        phi_o = st.geom.phi.copy()
        if warm:
            oracle.pdesolver(st, phi_o, rhs, eps=1e-6)
        phi_g = phi_o.copy()
        ko = oracle.pdesolver(st, phi_o, rhs)
        kg = dropin.pdesolver(st, phi_g, rhs)
        assert kg[0] == ko[0], (kg, ko)
        assert abs(kg[1] - ko[1]) == 0.0, (kg, ko)
        assert rel(phi_g, phi_o) <= 1e-12
        assert kg[2] < st.wl.eps


def test_efield_bit_exact(box16):
    st, S = box16
    dropin.set_commons(st)
    _, phi, E_o = solved_fields(st, S)
    E_g = dropin.calc_efield(st, phi)
    np.testing.assert_array_equal(E_g, E_o)


@pytest.mark.parametrize("cfg", ["box16", "mcc32"])
def test_part_mover_one_step_bit_exact(cfg, box16, mcc32):
    st, S = box16 if cfg == "box16" else mcc32
    dropin.set_commons(st)
    _, _, E = solved_fields(st, S)
    # a strong field so that some particles reach the walls in one step
    E = E * 1e3
    So = S.copy()
    Sg = S.copy()
    ng1 = st.geom.ngrid + 1
    pm_o, pl_o = np.zeros((ng1, 2, st.ntype)), np.zeros((st.ntype, 4))
    pm_g, pl_g = np.zeros((ng1, 2, st.ntype)), np.zeros((st.ntype, 4))
    for p in range(1, st.ntype + 1):
        oracle.part_mover(st, E, So, pm_o, pl_o, p)
        dropin.part_mover(st, E, Sg.vxp, Sg.np_tot, Sg.flag_dead, pm_g, pl_g, p)
    np.testing.assert_array_equal(Sg.np_tot, So.np_tot)
    for p in range(st.ntype):
        n = So.np_tot[p]
        np.testing.assert_array_equal(Sg.vxp[p, :n], So.vxp[p, :n])
    assert (So.np_tot < S.np_tot).any(), "test meant to exercise losses"
    np.testing.assert_allclose(pm_g, pm_o, rtol=1e-12, atol=0)
    np.testing.assert_allclose(pl_g, pl_o, rtol=1e-12, atol=0)


def test_charge_deposition(box16):
    st, S = box16
    dropin.set_commons(st)
    So = S.copy()
    So.np[:] = 0
    g = np.zeros_like(S.np)
    for p in range(1, st.ntype + 1):
        oracle.charge_deposition(st, So, p)
        dropin.charge_deposition(st, S.vxp, S.np_tot, g, p)
    assert rel(g, So.np) <= 1e-12
    # charge conservation: sum np/kq * h^3 = N Nm (exact up to rounding)
    vol = st.h[0] * st.h[1] * st.h[2]
    for p in range(st.ntype):
        tot = (g[p] / st.kq).sum() * vol
        assert abs(tot - S.np_tot[p] * st.Nm[p]) <= 1e-12 * S.np_tot[p] * st.Nm[p]


def test_part_sorting_counts_and_cells(mcc32):
    st, S = mcc32
    dropin.set_commons(st)
    So = S.copy()
    Sg = S.copy()
    for p in range(1, st.ntype + 1):
        pl_o = oracle.part_sorting(st, So, p)
        pl_g = dropin.part_sorting(st, Sg.vxp, Sg.np_tot, p)
        np.testing.assert_array_equal(pl_g, pl_o)
        n = So.np_tot[p - 1]
        a, b = So.vxp[p - 1, :n], Sg.vxp[p - 1, :n]
        # same particles in each cell segment (order inside a cell is free)
        starts = np.concatenate([[0], pl_o[1:]])
        cell_of = np.searchsorted(pl_o[1:], np.arange(n), side="right")
        ka = np.lexsort((a[:, 5], a[:, 4], a[:, 3], a[:, 2], a[:, 1], a[:, 0], cell_of))
        kb = np.lexsort((b[:, 5], b[:, 4], b[:, 3], b[:, 2], b[:, 1], b[:, 0], cell_of))
        np.testing.assert_array_equal(a[ka], b[kb])
        del starts


def test_collisions_statistics(mcc32):
    """Counts per process agree with the oracle's (ran2, with-replacement
    picks) within 3 sigma of the difference of two counts."""
    st, S = mcc32
    T = st.tables
    dropin.set_commons(st, ncol=T.sig.shape[0], npt=T.sig_Er.shape[0], p_ncol=T.p_ncol)
    tot_o = np.zeros(T.sig.shape[0])
    tot_g = np.zeros(T.sig.shape[0])
    for call in range(4):
        So = S.copy()
        So.iseed[0] = 1234567 + 77 * call
        _, cnt, _ = oracle.collisions(st, So)
        tot_o += cnt
        tot_g += _gpu_counts(st, S, 11 + 10 * call, 987654 + call)
    assert tot_o.sum() > 1000
    for r in range(len(tot_o)):
        if tot_o[r] + tot_g[r] == 0:
            continue
        sig = np.sqrt(tot_o[r] + tot_g[r])
        assert abs(tot_o[r] - tot_g[r]) <= 3 * sig + 1, (r, tot_o, tot_g)


def test_collisions_dropin(mcc32):
    """collisions_ through the Fortran-signature entry point: one region
    covering the box; every ionization appends one e- and one Ar+; the region
    counter sums 1/np_tot_rg per collision (Src/collisions.f90:1005-1013)."""
    st, S = mcc32
    Sg = S.copy()
    n1 = st.n[0]
    red, _ = oracle.dens_red(st, S.np.copy())
    cnt_col = np.zeros((1, 1, 65))
    before = Sg.np_tot.copy()
    dropin.collisions(st, 11, Sg.vxp, Sg.np_tot, Sg.flag_dead, np.array([4242], dtype=np.int32),
                      np_red=red, regions=[(1, n1 + 1)], cnt_col=cnt_col)
    added = Sg.np_tot - before
    assert added[0] == added[1]
    # unchanged particles stay bit-identical (only collided ones change)
    n = before[0]
    changed = np.any(Sg.vxp[0, :n] != S.vxp[0, :n], axis=1)
    assert 0 < changed.mean() < 0.2
    assert cnt_col[0, 0, :4].sum() > 0
    # ionization at Te = 2 eV is rare (a few per call): further calls until
    # some have happened, each adding e- and Ar+ in pairs
    total = int(added[0])
    for it in range(21, 211, 10):
        if total > 0:
            break
        b = Sg.np_tot.copy()
        dropin.collisions(st, it, Sg.vxp, Sg.np_tot, Sg.flag_dead, np.array([4242], dtype=np.int32),
                          np_red=red, regions=[(1, n1 + 1)], cnt_col=cnt_col)
        a = Sg.np_tot - b
        assert a[0] == a[1]
        total += int(a[0])
    assert total > 0


def _gpu_counts(st, S, it, seed):
    """Collision counts per reaction from the device API (same state)."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    sim = Simulation(st, cap=S.vxp.shape[1], seed=seed)
    sim.load_from_host(S.vxp, S.np_tot, S.np)
    sim.it = it
    sim.collisions()
    torch.cuda.synchronize()
    return sim.counts[:st.tables.sig.shape[0]].astype(float)


def test_box32_100_steps_at_its_own_size():
    """The plain FP64 benchmark case at its own size (32^3 cells, electrons
    and Ar+ at 16 per cell: 524,288 each, walls at 0 V, no B, no collisions):
    100 device steps of the step loop against 100 oracle steps in the
    reference's order from the same loaded particles -- particle counts
    equal, every position and velocity within 1e-10 of the largest, phi
    within 1e-10 of its largest value (the deposit's atomics sum in another
    order than the oracle: 1e-16 per step, grown over 100 steps), the
    multigrid schedule (V-cycles of the last solve) equal."""
    import os
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    oracle.set_threads(os.cpu_count() or 1)
    st = config.build("box32")
    assert st.n_particles() == 524288
    nmax = st.n_particles() + 4096
    S = oracle.load_part(st, nmax=nmax)
    sim = Simulation(st, cap=nmax)
    sim.load_from_host(S.vxp, S.np_tot, S.np)
    phi = st.geom.phi.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    for it in range(1, 101):
        Ei, mg_o, _ = oracle.step(st, S, phi, Ei, it)
        sim.step()
    torch.cuda.synchronize()
    assert list(sim.counts_host()) == list(S.np_tot)
    assert sim.mg_last[0] == mg_o[0], (sim.mg_last, mg_o)
    for p in range(st.ntype):
        g = sim.sp[p].to_vxp()
        o = S.vxp[p, :S.np_tot[p]]
        ko = np.lexsort((o[:, 2], o[:, 1], o[:, 0]))
        kg = np.lexsort((g[:, 2], g[:, 1], g[:, 0]))
        for c in range(6):
            assert rel(g[kg, c], o[ko, c]) <= 1e-10, (p, c, rel(g[kg, c], o[ko, c]))
    assert rel(sim.phi.cpu().numpy(), phi) <= 1e-10


@pytest.mark.parametrize("fused", [True, False])
def test_step_loop_trajectories_100_steps(fused):
    """Collisionless box: 100 device-resident steps vs 100 oracle steps in
    the reference order; positions/velocities within 1e-10 relative.
    fused: in-place push + deposition with hole filling (the step path), else
    the drop-in kernels (push, in-order compaction, deposition)."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    oracle.set_threads(1)
    st = config.build("box16")
    nmax = st.n_particles() + 4096
    S = oracle.load_part(st, nmax=nmax)
    sim = Simulation(st, cap=nmax, fused=fused)
    sim.load_from_host(S.vxp, S.np_tot, S.np)
    phi = st.geom.phi.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    steps = 100
    for it in range(1, steps + 1):
        Ei, _, _ = oracle.step(st, S, phi, Ei, it)
        sim.step()
    torch.cuda.synchronize()
    for p in range(st.ntype):
        g = sim.sp[p].to_vxp()
        o = S.vxp[p, :S.np_tot[p]]
        assert g.shape == o.shape
        ko = np.lexsort((o[:, 2], o[:, 1], o[:, 0]))
        kg = np.lexsort((g[:, 2], g[:, 1], g[:, 0]))
        for c in range(6):
            assert rel(g[kg, c], o[ko, c]) <= 1e-10, (p, c, rel(g[kg, c], o[ko, c]))
    assert rel(sim.phi.cpu().numpy(), phi) <= 1e-10
    # charge conservation of the deposit: sum np/kq h^3 = N Nm per species
    vol = st.h[0] * st.h[1] * st.h[2]
    kq = torch.as_tensor(st.kq, device=sim.dev)
    for p in range(st.ntype):
        tot = float((sim.np[p] / kq).sum()) * vol
        want = sim.sp[p].n() * st.Nm[p]
        assert abs(tot - want) <= 1e-12 * want
    # wall losses agree with the oracle's count of lost particles
    pm, _ = sim.loss_stats()
    assert np.allclose(pm[:, 0, :].sum(axis=0), S.np_tot * 0 + (np.array(
        [st.n_particles()] * st.ntype) - S.np_tot))


def test_load_uniform_moments():
    """GPU Philox loader: uniform positions, Maxwellian velocities with
    <v_i^2> = vt0^2 / 2 (load_gauss form), co-located species."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("mcc32")
    sim = Simulation(st)
    sim.load_uniform()
    torch.cuda.synchronize()
    n = st.n_particles()
    for p, s in enumerate(sim.sp):
        assert s.n() == n
        v = s.p[3:6, :n].cpu().numpy()
        var = (v ** 2).mean(axis=1)
        want = st.vt0[p] ** 2 / 2
        assert np.all(np.abs(var / want - 1) < 6 * np.sqrt(2.0 / n)), (var / want)
    a = sim.sp[0].p[0:3, :n]
    b = sim.sp[1].p[0:3, :n]
    assert torch.equal(a, b)
    # total deposited charge = N Nm per species
    vol = st.h[0] * st.h[1] * st.h[2]
    kq = torch.as_tensor(st.kq, device=sim.dev)
    for p in range(st.ntype):
        tot = float((sim.np[p] / kq).sum()) * vol
        assert abs(tot - n * st.Nm[p]) <= 1e-12 * n * st.Nm[p]


def test_step_host_pipelined_io():
    """Simulation.step_host: electrode potentials in, phi and counts out into
    pinned host buffers on a copy stream (two steps in flight) -- the same
    phi (1e-12, deposition order) and counts as plain steps."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("box16")
    nl = int(st.geom.ngrid)
    a = Simulation(st, seed=99)
    b = Simulation(st, seed=99)
    a.load_uniform()
    b.load_uniform()
    v = torch.zeros(nl + 2, dtype=torch.float64).pin_memory()
    for lab in range(1, nl + 1):
        v[lab] = float(st.wl.V[lab]) if lab < len(st.wl.V) else 0.0
    phis = [torch.empty(tuple(st.geom.phi.shape), dtype=torch.float64).pin_memory() for _ in range(2)]
    cnts = torch.zeros((6, st.ntype), dtype=torch.int32).pin_memory()
    ref_phi, ref_cnt = [], []
    done = [None, None]
    got = []
    for k in range(6):
        a.step()
        ref_phi.append(a.phi.cpu().numpy())
        ref_cnt.append(a.counts_host())
        if done[k % 2] is not None:
            done[k % 2].synchronize()
            got.append((k - 2, phis[k % 2].numpy().copy()))
        done[k % 2] = b.step_host(v, phis[k % 2], cnts[k])
    torch.cuda.synchronize()
    got += [(4, phis[0].numpy().copy()), (5, phis[1].numpy().copy())]
    # the first step's phi is round-off (co-located species: rho = 0), so the
    # bar is relative to the largest |phi| of the run
    scale = max(np.abs(r).max() for r in ref_phi)
    for k, ph in got:
        assert np.abs(ph - ref_phi[k]).max() <= 1e-12 * scale, k
    assert np.array_equal(cnts.numpy(), np.array(ref_cnt))


def test_mcc_moments_vs_oracle(mcc32):
    """Ten steps with MCC every step from the same particles, the oracle
    (serial ran2 picks) against the GPU FP64 step (Philox null collisions):
    per species the population, the mean kinetic energy and the mean position
    within 3 sigma of the sampling error (sigma of a mean: std / sqrt(N) of
    both runs; population: the square root of the particles each run created
    or lost)."""
    import os
    from essaitemporaire_lepic_module_b200.constants import QE
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st, S0 = mcc32
    oracle.set_threads(os.cpu_count() or 1)
    S = S0.copy()
    sim = Simulation(st, cap=S.vxp.shape[1], seed=777, ns_coll=1)
    sim.load_from_host(S.vxp, S.np_tot, S.np)
    phi = st.geom.phi.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    for it in range(1, 11):
        Ei, _, _ = oracle.step(st, S, phi, Ei, it, ns_coll=1)
        sim.step()
    oracle.set_threads(1)
    for p in range(st.ntype):
        g = sim.sp[p].to_vxp()
        o = S.vxp[p, :S.np_tot[p]]
        n0 = S0.np_tot[p]
        dn = abs(len(g) - len(o))
        assert dn <= 3.0 * np.sqrt(abs(len(g) - n0) + abs(len(o) - n0) + 1.0), (p, len(g), len(o), n0)
        m = abs(st.mass[p])
        eg = 0.5 * m * (g[:, 3:6] ** 2).sum(axis=1) / QE
        eo = 0.5 * m * (o[:, 3:6] ** 2).sum(axis=1) / QE
        qs = [(eg, eo)] + [(g[:, c], o[:, c]) for c in range(3)]
        for a, b in qs:
            sig = np.sqrt(a.var() / len(a) + b.var() / len(b))
            assert abs(a.mean() - b.mean()) <= 3.0 * sig, (p, a.mean(), b.mean(), sig)
