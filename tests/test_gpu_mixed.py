"""GPU tests of the mixed-precision form (int32 cell + FP32 offset/velocity
particles, FP32 V-cycles inside FP64 refinement) against the FP64 oracle.

Bars, written in each test:
  * Poisson: phi within 1e-6 (relative to max |phi|) of the FP64 solution at
    the workload tolerance; the FP64 refinement converges past FP32 precision
    (res/alpha < 1e-12) to within 1e-9 of the FP64 solution;
  * one push from the same particles: positions within 2e-6 h, velocities
    within 1e-5 relative (FP32 arithmetic), deposited density within 1e-6 of
    its maximum;
  * charge conservation of the deposit: N Nm to 1e-12 relative;
  * tiled and untiled deposit paths: the same particles bit for bit and the
    same grid to 1e-13;
  * MCC counts within 3 sigma of the oracle's.
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


def _sim(st, cap, **kw):
    from essaitemporaire_lepic_module_b200.sim import Simulation
    return Simulation(st, cap=cap, precision="mixed", **kw)


def _interior(st, S, margin=3):
    """Particles at least `margin` cells from every face (no loss in one step)."""
    h = np.asarray(st.h)
    n = np.asarray(st.n)
    T = S.copy()
    for p in range(st.ntype):
        v = S.vxp[p, :S.np_tot[p]]
        keep = np.all((v[:, 0:3] >= margin * h) & (v[:, 0:3] <= (n - margin + 1) * h), axis=1)
        m = int(keep.sum())
        T.vxp[p, :m] = v[keep]
        T.vxp[p, m:] = 0.0
        T.np_tot[p] = m
    return T


def _charge_ok(st, sim, tol=1e-12):
    import torch
    vol = st.h[0] * st.h[1] * st.h[2]
    kq = torch.as_tensor(st.kq, device=sim.dev)
    for p in range(st.ntype):
        tot = float((sim.np[p] / kq).sum()) * vol
        want = sim.sp[p].n() * st.Nm[p]
        assert abs(tot - want) <= tol * want, (p, tot, want)


def test_layout_roundtrip():
    """FP64 -> mixed -> FP64: cell exact, offsets and velocities to FP32."""
    import torch
    oracle.set_threads(1)
    st = config.build("box16")
    S = oracle.load_part(st, nmax=st.n_particles() + 4096)
    sim = _sim(st, S.vxp.shape[1])
    sim.load_from_host(S.vxp, S.np_tot, S.np)
    torch.cuda.synchronize()
    h = np.asarray(st.h)
    for p in range(st.ntype):
        g = sim.particles_f64(p).t().cpu().numpy()
        o = S.vxp[p, :S.np_tot[p]]
        assert g.shape == o.shape
        assert np.all(np.abs(g[:, 0:3] - o[:, 0:3]) <= 1.2e-7 * h)
        assert rel(g[:, 3:6], o[:, 3:6]) <= 1e-7
        cell_g = sim.sp[p].cell[:S.np_tot[p]].cpu().numpy()
        ix = (o[:, 0] / h[0]).astype(int)
        iy = (o[:, 1] / h[1]).astype(int)
        iz = (o[:, 2] / h[2]).astype(int)
        np.testing.assert_array_equal(cell_g, ix | (iy << 10) | (iz << 20))


def test_mixed_loader_matches_f64_loader():
    """The direct mixed loader draws the FP64 loader's particles (to FP32) and
    deposits their charge exactly."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("mcc32")
    a = Simulation(st, seed=9)
    b = Simulation(st, seed=9, precision="mixed")
    a.load_uniform()
    b.load_uniform()
    torch.cuda.synchronize()
    h = np.asarray(st.h)
    for p in range(st.ntype):
        n = a.sp[p].n()
        assert b.sp[p].n() == n
        x = a.sp[p].p[:, :n].cpu().numpy()
        y = b.particles_f64(p).cpu().numpy()
        assert np.all(np.abs(y[0:3] - x[0:3]).T <= 1.2e-7 * h)
        assert rel(y[3:6], x[3:6]) <= 1e-7
        assert rel(b.np[p].cpu().numpy(), a.np[p].cpu().numpy()) <= 1e-6
    _charge_ok(st, b)


def test_sort_tile_order():
    """The mixed sort: tile-major key order, tile offsets, same particles."""
    import torch
    oracle.set_threads(1)
    st = config.build("mcc32")
    S = oracle.load_part(st, nmax=int(st.n_particles() * 1.3))
    sim = _sim(st, S.vxp.shape[1])
    sim.load_from_host(S.vxp, S.np_tot, S.np)
    before = [(s.cell[:s.n()].clone(), s.p[:, :s.n()].clone()) for s in sim.sp]
    sim.sort()
    torch.cuda.synchronize()
    n1, n2, n3 = st.n
    ntx, nty = (n1 + 7) // 8, (n2 + 7) // 8
    for p, s in enumerate(sim.sp):
        n = s.n()
        c = s.cell[:n].cpu().numpy().astype(np.int64)
        cx, cy, cz = c & 1023, (c >> 10) & 1023, c >> 20
        key = ((cx // 8) + ntx * ((cy // 8) + nty * (cz // 8))) * 512 + (cx % 8) + 8 * ((cy % 8) + 8 * (cz % 8))
        assert np.all(np.diff(key) >= 0)
        toff = s.tile_off.cpu().numpy()
        tiles = key // 512
        want = np.searchsorted(tiles, np.arange(len(toff)), side="left")
        np.testing.assert_array_equal(toff, want)
        # same multiset of particles
        a = np.column_stack([before[p][0].cpu().numpy(), before[p][1].t().cpu().numpy()])
        b = np.column_stack([c, s.p[:, :n].t().cpu().numpy()])
        ka = np.lexsort(a.T[::-1])
        kb = np.lexsort(b.T[::-1])
        np.testing.assert_array_equal(a[ka], b[kb])


@pytest.mark.parametrize("cfg", ["box16", "penning_small"])
def test_push_deposit_one_step_vs_oracle(cfg):
    """One mixed push + deposit from the oracle's particles and field against
    the FP64 oracle (in-order, no losses: interior particles only)."""
    import torch
    oracle.set_threads(1)
    st = config.build(cfg)
    dropin.set_commons(st)
    S0 = oracle.load_part(st, nmax=st.n_particles() + 4096)
    S = _interior(st, S0)
    rhs = oracle.calc_rho(st, S0.np.copy())
    phi = st.geom.phi.copy()
    oracle.pdesolver(st, phi, rhs)
    E = oracle.calc_efield(st, phi)
    So = S.copy()
    ng1 = st.geom.ngrid + 1
    pm, pl = np.zeros((ng1, 2, st.ntype)), np.zeros((st.ntype, 4))
    So.np[:] = 0
    for p in range(1, st.ntype + 1):
        oracle.part_mover(st, E, So, pm, pl, p)
        oracle.charge_deposition(st, So, p)
    np.testing.assert_array_equal(So.np_tot, S.np_tot)
    sim = _sim(st, S.vxp.shape[1])
    sim.load_from_host(S.vxp, S.np_tot, S.np)
    sim.Ei.copy_(torch.as_tensor(E, device=sim.dev))
    sim.pack_e32()
    sim.move_deposit()
    torch.cuda.synchronize()
    h = np.asarray(st.h)
    for p in range(st.ntype):
        assert sim.sp[p].n() == So.np_tot[p]
        g = sim.particles_f64(p).t().cpu().numpy()
        o = So.vxp[p, :So.np_tot[p]]
        dx = np.abs(g[:, 0:3] - o[:, 0:3]) / h
        assert dx.max() <= 2e-6, dx.max()
        assert rel(g[:, 3:6], o[:, 3:6]) <= 1e-5, rel(g[:, 3:6], o[:, 3:6])
        assert rel(sim.np[p].cpu().numpy(), So.np[p]) <= 1e-6, rel(sim.np[p].cpu().numpy(), So.np[p])
    _charge_ok(st, sim)


def test_tiled_and_untiled_deposit_agree():
    """The tiled push (after a sort) and the untiled one (no sort) move every
    particle identically and deposit the same grid."""
    import torch
    oracle.set_threads(1)
    st = config.build("mcc32")
    S0 = oracle.load_part(st, nmax=int(st.n_particles() * 1.3))
    S = _interior(st, S0)
    E = np.random.default_rng(5).normal(0.0, 2e3, tuple(st.geom.bcnd.shape) + (3,))
    sims = []
    for tiled in (False, True):
        sim = _sim(st, S.vxp.shape[1])
        sim.load_from_host(S.vxp, S.np_tot, S.np)
        sim.Ei.copy_(torch.as_tensor(E, device=sim.dev))
        sim.pack_e32()
        if tiled:
            sim.sort()
        sim.move_deposit()
        torch.cuda.synchronize()
        sims.append(sim)
    a, b = sims
    for p in range(st.ntype):
        assert a.sp[p].n() == b.sp[p].n() == S.np_tot[p]
        A = np.column_stack([a.sp[p].cell[:a.sp[p].n()].cpu().numpy(), a.sp[p].p[:, :a.sp[p].n()].t().cpu().numpy()])
        B = np.column_stack([b.sp[p].cell[:b.sp[p].n()].cpu().numpy(), b.sp[p].p[:, :b.sp[p].n()].t().cpu().numpy()])
        ka = np.lexsort(A.T[::-1])
        kb = np.lexsort(B.T[::-1])
        np.testing.assert_array_equal(A[ka], B[kb])
        assert rel(b.np[p].cpu().numpy(), a.np[p].cpu().numpy()) <= 1e-13
    _charge_ok(st, a)
    _charge_ok(st, b)


def test_losses_vs_oracle():
    """A strong field drives particles into the walls in one step: the mixed
    push loses the same particles (up to FP32 rounding at the wall) and keeps
    the wall energy accounts."""
    import torch
    oracle.set_threads(1)
    st = config.build("box16")
    dropin.set_commons(st)
    S = oracle.load_part(st, nmax=st.n_particles() + 4096)
    rhs = oracle.calc_rho(st, S.np.copy())
    phi = st.geom.phi.copy()
    oracle.pdesolver(st, phi, rhs)
    E = oracle.calc_efield(st, phi) * 1e3
    So = S.copy()
    ng1 = st.geom.ngrid + 1
    pm, pl = np.zeros((ng1, 2, st.ntype)), np.zeros((st.ntype, 4))
    for p in range(1, st.ntype + 1):
        oracle.part_mover(st, E, So, pm, pl, p)
    lost_o = S.np_tot - So.np_tot
    assert lost_o.sum() > 0
    sim = _sim(st, S.vxp.shape[1])
    sim.load_from_host(S.vxp, S.np_tot, S.np)
    sim.sort()
    sim.Ei.copy_(torch.as_tensor(E, device=sim.dev))
    sim.pack_e32()
    sim.move_deposit()
    torch.cuda.synchronize()
    lost_g = S.np_tot - sim.counts_host()
    assert np.all(np.abs(lost_g - lost_o) <= np.maximum(2, 1e-3 * lost_o)), (lost_g, lost_o)
    pm_g, pl_g = sim.loss_stats()
    assert rel(pm_g[:, 1, :].sum(axis=0), pm[:, 1, :].sum(axis=0)) <= 1e-3
    _charge_ok(st, sim)


@pytest.mark.parametrize("name", ["box32", "poisson32", "penning_small"])
def test_pdesolver_mixed(name):
    """FP32 V-cycles in FP64 refinement: phi within 1e-6 of the FP64 solve
    at the workload tolerance, within 1e-9 when both are driven to 1e-12."""
    import torch
    oracle.set_threads(1)
    st = config.build(name)
    dropin.set_commons(st)
    if st.rhs_blobs is not None:
        rhs = st.rhs_blobs
    else:
        S = oracle.load_part(st, nmax=st.n_particles() + 4096)
        npg = S.np.copy()
        npg[1:] = 0.0
        rhs = oracle.calc_rho(st, npg)
    sim = _sim(st, 1024)
    for eps, tol in ((st.wl.eps, 1e-6), (1e-12, 1e-9)):
        phi_o = st.geom.phi.copy()
        oracle.pdesolver(st, phi_o, rhs, eps=eps)
        sim.phi.copy_(torch.as_tensor(st.geom.phi, device=sim.dev))
        sim.rhs.copy_(torch.as_tensor(rhs, device=sim.dev))
        it, _, res = sim.pdesolver_mixed(eps=eps)
        torch.cuda.synchronize()
        assert res < eps, (it, res)
        err = rel(sim.phi.cpu().numpy(), phi_o)
        assert err <= tol, (name, eps, err, it)


def test_collisions_mixed_statistics():
    """Collision counts per process against the oracle within 3 sigma."""
    import torch
    oracle.set_threads(1)
    st = config.build("mcc32")
    S = oracle.load_part(st, nmax=int(st.n_particles() * 1.3))
    T = st.tables
    dropin.set_commons(st, ncol=T.sig.shape[0], npt=T.sig_Er.shape[0], p_ncol=T.p_ncol)
    tot_o = np.zeros(T.sig.shape[0])
    tot_g = np.zeros(T.sig.shape[0])
    for call in range(4):
        So = S.copy()
        So.iseed[0] = 1234567 + 77 * call
        _, cnt, _ = oracle.collisions(st, So)
        tot_o += cnt
        sim = _sim(st, S.vxp.shape[1], seed=987654 + call)
        sim.load_from_host(S.vxp, S.np_tot, S.np)
        sim.it = 11 + 10 * call
        before = sim.counts_host()
        sim.collisions()
        torch.cuda.synchronize()
        tot_g += sim.counts[:T.sig.shape[0]]
        assert np.all(sim.counts_host() >= before)
    assert tot_o.sum() > 1000
    for r in range(len(tot_o)):
        if tot_o[r] + tot_g[r] == 0:
            continue
        sig = np.sqrt(tot_o[r] + tot_g[r])
        assert abs(tot_o[r] - tot_g[r]) <= 3 * sig + 1, (r, tot_o, tot_g)


def test_mixed_steps_with_mcc():
    """20 mixed steps with MCC on the Ar workload: charge conserved every
    step, populations and mean energies close to the FP64 device loop."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("mcc32")
    f64 = Simulation(st, seed=77)
    mx = Simulation(st, seed=77, precision="mixed")
    f64.load_uniform()
    mx.load_uniform()
    for _ in range(20):
        f64.step()
        mx.step()
        _charge_ok(st, mx)
    torch.cuda.synchronize()
    nf, nm = f64.counts_host(), mx.counts_host()
    assert np.all(np.abs(nm - nf) <= 0.01 * nf), (nm, nf)
    for p in range(st.ntype):
        ef = float((f64.sp[p].p[3:6, :nf[p]] ** 2).sum(dim=0).mean())
        em = float((mx.particles_f64(p)[3:6] ** 2).sum(dim=0).mean())
        assert abs(em / ef - 1) <= 1e-2, (p, em, ef)
    assert rel(mx.phi.cpu().numpy(), f64.phi.cpu().numpy()) <= 5e-2


def test_nonblocking_steps_match_blocking():
    """The step loop without waits (mixed solve launched without reading its
    refinements, the device error word snapshotted asynchronously) moves the
    same particles to the same phi as the blocking loop, and its solve
    history holds the same refinements."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("box32")
    runs = []
    for nb in (False, True):
        sim = Simulation(st, precision="mixed", seed=5, nonblocking=nb)
        sim.load_uniform()
        its = []
        for _ in range(12):
            sim.step()
            if not nb:
                its.append(sim.mg_last[0])
        if nb:
            its = sim.solve_history(12)
            sim.flush_checks()
        torch.cuda.synchronize()
        runs.append((sim.phi.cpu().numpy(), list(sim.counts_host()), its, sim.mg_last[0]))
    # the FP64 density sums are atomic (their rounding follows the thread
    # order), so two runs agree to rounding, not bit for bit
    (pa, ca, ia, la), (pb, cb, ib, lb) = runs
    assert all(abs(x - y) <= 1e-4 * x + 2 for x, y in zip(ca, cb)), (ca, cb)
    assert len(ib) == 12 and lb == ib[-1] and la == ia[-1]
    assert all(abs(x - y) <= 1 for x, y in zip(ia, ib)), (ia, ib)
    assert np.abs(pa - pb).max() <= 1e-6 * np.abs(pa).max()
