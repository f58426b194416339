"""GPU dielectric wall charging in the drop-in mover (part_mover_ with
flag_die = 1, Src/part_expmover.f90:302-348) against the CPU oracle on the
die16 box (a Y = const dielectric at y = ymax, an X = const one at
x = xmax): particles bit-identical, the surface-charge sums sum_q_xz /
sum_q_yz within 1e-12 of the largest node sum (the device adds with atomics,
the oracle in particle order), and the device step loop refuses the
geometry instead of ignoring the walls' charge."""
import numpy as np
import pytest

import oracle
from essaitemporaire_lepic_module_b200 import config, dropin
from tests.conftest import have_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]


def _sums(st):
    n1, n2, n3 = st.n
    return np.zeros((st.ntype, n3 + 3, n1 + 3)), np.zeros((st.ntype, n3 + 3, n2 + 3, 2))


def test_dielectric_dropin_vs_oracle():
    oracle.set_threads(1)
    st = config.build("die16")
    dropin.set_commons(st)
    So = oracle.load_part(st, nmax=st.n_particles() + 16)
    Sg = So.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    rng = np.random.default_rng(5)
    Ei[...] = rng.normal(0.0, 2e3, Ei.shape)
    ng1 = st.geom.ngrid + 1
    pm_o, pm_g = np.zeros((ng1, 2, st.ntype)), np.zeros((ng1, 2, st.ntype))
    pl_o, pl_g = np.zeros((st.ntype, 4)), np.zeros((st.ntype, 4))
    qo, qg = _sums(st), _sums(st)
    for _ in range(6):
        for p in range(1, st.ntype + 1):
            oracle.part_mover(st, Ei, So, pm_o, pl_o, p, sum_q=qo)
            dropin.part_mover(st, Ei, Sg.vxp, Sg.np_tot, Sg.flag_dead, pm_g, pl_g, p, sum_q=qg)
    np.testing.assert_array_equal(Sg.np_tot, So.np_tot)
    for p in range(st.ntype):
        np.testing.assert_array_equal(Sg.vxp[p, :So.np_tot[p]], So.vxp[p, :So.np_tot[p]])
    np.testing.assert_array_equal(pm_g[:, 0, :], pm_o[:, 0, :])
    assert pm_o[2, 0, 0] > 50 and pm_o[3, 0, 0] > 50
    for a, b in zip(qg, qo):
        scale = np.abs(b).max()
        assert scale > 0
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * scale)



@pytest.mark.parametrize("pbc", [0, 1])
def test_dielectric_phi_device_bit_exact(pbc):
    """lepic_dev_dielectric_phi (Src/main.f90:859-949) against the oracle on
    random surface charges: phi bit for bit, the sums cleared."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("die16")
    st.geom.flag_pbc = pbc
    rng = np.random.default_rng(11 + pbc)
    qo = _sums(st)
    for a in qo:
        a[...] = rng.normal(0.0, 1e-17, a.shape)
    sim = Simulation(st, cap=1000)
    sim.die[1].copy_(torch.as_tensor(qo[0]))
    sim.die[2].copy_(torch.as_tensor(qo[1]))
    phi_o = st.geom.phi.copy()
    oracle.dielectric_phi(st, phi_o, qo)
    sim.dielectric_phi()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(sim.phi.cpu().numpy(), phi_o)
    assert not sim.die[1].any() and not sim.die[2].any()
    assert (phi_o != st.geom.phi).sum() > 100


@pytest.mark.parametrize("fused", [True, False])
def test_step_loop_dielectric(fused):
    """20 device steps of the FP64 loop on die16 (surface charge summed by the
    push, the walls' potential raised before each field solve) against 20
    oracle steps: particles and phi within 1e-10, the walls charged."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    oracle.set_threads(1)
    st = config.build("die16")
    nmax = st.n_particles() + 4096
    S = oracle.load_part(st, nmax=nmax)
    sim = Simulation(st, cap=nmax, fused=fused)
    sim.load_from_host(S.vxp, S.np_tot, S.np)
    phi = st.geom.phi.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    for it in range(1, 21):
        Ei, _, _ = oracle.step(st, S, phi, Ei, it)
        sim.step()
    torch.cuda.synchronize()
    for p in range(st.ntype):
        g = sim.sp[p].to_vxp()
        o = S.vxp[p, :S.np_tot[p]]
        assert g.shape == o.shape
        ko = np.lexsort((o[:, 2], o[:, 1], o[:, 0]))
        kg = np.lexsort((g[:, 2], g[:, 1], g[:, 0]))
        scale = np.abs(o).max(axis=0)
        assert (np.abs(g[kg] - o[ko]) <= 1e-10 * scale).all(), p
    phg = sim.phi.cpu().numpy()
    assert np.abs(phg - phi).max() <= 1e-10 * np.abs(phi).max()
    n1, n2, n3 = st.n
    assert np.abs(phi[:, n2 + 1, :]).max() > 1e-3       # the Y plane charged
    assert np.abs(phi[:, :, n1 + 1]).max() > 1e-3       # the X plane charged
    for a, b in zip(sim.die[1:], S.sum_q):
        np.testing.assert_allclose(a.cpu().numpy(), b, rtol=0, atol=1e-10 * max(np.abs(b).max(), 1e-30))


def test_step_loop_dielectric_mixed():
    """The mixed step loop on die16: the surface charge of one step equals
    Nm q times the particles it lost on each dielectric label (1e-12), and
    after 10 steps the walls' potential is within 10 % of the FP64 loop's
    from the same particles (FP32 trajectories lose a few particles at other
    steps)."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    oracle.set_threads(1)
    st = config.build("die16")
    nmax = st.n_particles() + 4096
    S = oracle.load_part(st, nmax=nmax)
    runs = {}
    for prec in ("mixed", "f64"):
        sim = Simulation(st, cap=nmax, precision=prec)
        sim.load_from_host(S.vxp, S.np_tot, S.np)
        for _ in range(9):
            sim.step()
        pm0, _ = sim.loss_stats()
        sim.step()
        torch.cuda.synchronize()
        pm1, _ = sim.loss_stats()
        runs[prec] = sim.phi.cpu().numpy()
        if prec != "mixed":
            continue
        qxz, qyz = (t.cpu().numpy() for t in sim.die[1:])
        for p in range(st.ntype):
            k3 = st.Nm[p] * st.charge[p]
            d2, d3 = pm1[2, 0, p] - pm0[2, 0, p], pm1[3, 0, p] - pm0[3, 0, p]
            assert abs(qxz[p].sum() - k3 * d2) <= 1e-12 * abs(k3) * max(d2, 1)
            assert abs(qyz[p, ..., 0].sum() - k3 * d3) <= 1e-12 * abs(k3) * max(d3, 1)
            assert not qyz[p, ..., 1].any()
        assert pm1[2, 0, 0] > 20 and pm1[3, 0, 0] > 20
    wall = (st.geom.bcnd == 2) | (st.geom.bcnd == 3)
    a, b = runs["mixed"][wall], runs["f64"][wall]
    assert np.abs(b).max() > 1e-3
    assert np.abs(a - b).max() <= 0.1 * np.abs(b).max()


def test_dielectric_periodic_z_wrap_dropin():
    """the z wrap of a particle lost on a dielectric (periodic z planes): the
    drop-in's plane sums equal the oracle's"""
    from tests.test_dielectric import _corner_electron
    st = config.build("die16")
    st.geom.flag_pbc = 1
    dropin.set_commons(st)
    So = _corner_electron(st)
    Sg = So.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    ng1 = st.geom.ngrid + 1
    qo, qg = _sums(st), _sums(st)
    oracle.part_mover(st, Ei, So, np.zeros((ng1, 2, st.ntype)), np.zeros((st.ntype, 4)), 1, sum_q=qo)
    dropin.part_mover(st, Ei, Sg.vxp, Sg.np_tot, Sg.flag_dead, np.zeros((ng1, 2, st.ntype)),
                      np.zeros((st.ntype, 4)), 1, sum_q=qg)
    assert So.np_tot[0] == 0 and Sg.np_tot[0] == 0
    assert qo[0][0, 1:3].any()
    np.testing.assert_array_equal(qg[0], qo[0])
    np.testing.assert_array_equal(qg[1], qo[1])


@pytest.mark.parametrize("precision", ["mixed", "f64"])
def test_dielectric_periodic_corner_push(precision):
    """The step loop's push with periodic y and z planes: an electron that
    leaves through x = xmax (the X = const dielectric, label 3) while it
    crosses y = ymax and z = zmax.  As in Src/part_expmover.f90:250-348 the
    wall label and the y weight come from the clamped cell before any wrap
    (row n2+1) and only z wraps (row 1): sum_q_yz node for node equal to the
    oracle's (FP32 offsets in the mixed form: 1e-6 of the charge)."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    oracle.set_threads(1)
    st = config.build("die16")
    st.geom.flag_pbc = 1
    h, L = st.h, st.geom.box
    So = oracle.State(st, 4)
    So.vxp[0, 0] = [L[0] - 0.1 * h[0], L[1] - 0.1 * h[1], L[2] - 0.2 * h[2],
                    0.5 * h[0] / st.dt, 0.5 * h[1] / st.dt, 0.5 * h[2] / st.dt]
    So.np_tot[0] = 1
    sim = Simulation(st, cap=1024, precision=precision)
    sim.load_from_host(So.vxp, So.np_tot)
    sim.move_deposit()
    torch.cuda.synchronize()
    qo = _sums(st)
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    ng1 = st.geom.ngrid + 1
    oracle.part_mover(st, Ei, So, np.zeros((ng1, 2, st.ntype)), np.zeros((st.ntype, 4)), 1, sum_q=qo)
    assert So.np_tot[0] == 0 and int(sim.counts_host()[0]) == 0
    n2 = st.n[1]
    k3 = abs(st.Nm[0] * st.charge[0])
    assert np.abs(qo[1][0, 1:3, n2 + 1:n2 + 3, 0]).sum() > 0.99 * k3     # rows n2+1, n2+2 at z rows 1, 2
    qyz = sim.die[2].cpu().numpy()
    np.testing.assert_allclose(qyz[0], qo[1][0], rtol=0, atol=1e-6 * k3)
    assert not sim.die[1].cpu().numpy().any()
