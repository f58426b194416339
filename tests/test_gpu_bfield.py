"""GPU parity of the push with a B-field map (Src/part_expmover.f90:148-203)
against the CPU oracle on the same seeded inputs.

Two maps on the 16^3 box, each with regions below the 1e-5 T gate: a
Gaussian filter field By(x) plus a cusp field (Bx, Bz) of magnets beyond
the x = xmax wall, on the node grid (the E-field's cell and weights) and on
an 8 x 8 x 8 map grid of its own (index INT(x/h_B)+1, weights from h_B).

Bars: the drop-in push bit for bit (FP64, same expression order); 20 FP64
device-resident steps within 1e-10 relative; 3 mixed-form steps with phi
within 5e-5 of the oracle and every particle's velocity within 1e-4 of the
largest speed (particles matched by position to 1e-9 m; the same run without
the map leaves thousands of particles unmatched).
"""
import numpy as np
import pytest

import oracle
from essaitemporaire_lepic_module_b200 import bfield, config, dropin
from tests.conftest import have_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def mapped_box16(own):
    st = config.build("box16")
    bf = bfield.new_map(st, n_B=(8, 8, 8) if own else None)
    h = st.h[0]
    bfield.gaussian(bf, 0.05, x0=8 * h, Lx=1.5 * h, B_dir=2)
    bfield.ee_magnets(bf, 0.01, x0=20 * h, z0=8 * h, d=8 * h)
    bfield.attach(st, bfield.finish(bf))
    below = (bf.Bi[..., 3] <= bfield.GATE).mean()
    assert 0.05 < below < 0.8, below          # both branches of the gate are exercised
    return st


@pytest.mark.parametrize("own", [False, True])
def test_part_mover_bmap_bit_exact(own):
    oracle.set_threads(1)
    st = mapped_box16(own)
    dropin.set_commons(st)
    S = oracle.load_part(st, nmax=st.n_particles() + 4096)
    rng = np.random.default_rng(4)
    E = rng.normal(0, 3e4, tuple(st.geom.bcnd.shape) + (3,))
    So, Sg = S.copy(), S.copy()
    ng1 = st.geom.ngrid + 1
    pm_o, pl_o = np.zeros((ng1, 2, st.ntype)), np.zeros((st.ntype, 4))
    pm_g, pl_g = np.zeros((ng1, 2, st.ntype)), np.zeros((st.ntype, 4))
    for _ in range(3):
        for p in range(1, st.ntype + 1):
            oracle.part_mover(st, E, So, pm_o, pl_o, p)
            dropin.part_mover(st, E, Sg.vxp, Sg.np_tot, Sg.flag_dead, pm_g, pl_g, p)
    np.testing.assert_array_equal(Sg.np_tot, So.np_tot)
    for p in range(st.ntype):
        n = So.np_tot[p]
        np.testing.assert_array_equal(Sg.vxp[p, :n], So.vxp[p, :n])
    np.testing.assert_allclose(pm_g, pm_o, rtol=1e-12, atol=0)


@pytest.mark.parametrize("own", [False, True])
def test_step_loop_bmap_f64(own):
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    oracle.set_threads(1)
    st = mapped_box16(own)
    nmax = st.n_particles() + 4096
    S = oracle.load_part(st, nmax=nmax)
    sim = Simulation(st, cap=nmax)
    sim.load_from_host(S.vxp, S.np_tot, S.np)
    phi = st.geom.phi.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    for it in range(1, 21):
        Ei, _, _ = oracle.step(st, S, phi, Ei, it)
        sim.step()
    torch.cuda.synchronize()
    assert list(sim.counts_host()) == list(S.np_tot)
    for p in range(st.ntype):
        g = sim.sp[p].to_vxp()
        o = S.vxp[p, :S.np_tot[p]]
        kg = np.lexsort((g[:, 2], g[:, 1], g[:, 0]))
        ko = np.lexsort((o[:, 2], o[:, 1], o[:, 0]))
        for c in range(6):
            assert rel(g[kg, c], o[ko, c]) <= 1e-10, (p, c, rel(g[kg, c], o[ko, c]))
    assert rel(sim.phi.cpu().numpy(), phi) <= 1e-10


def _mixed_run(st, steps, nmax):
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    S0 = oracle.load_part(st, nmax=nmax)
    mx = Simulation(st, cap=nmax, precision="mixed")
    mx.load_from_host(S0.vxp, S0.np_tot, S0.np)
    for _ in range(steps):
        mx.step()
    torch.cuda.synchronize()
    return mx


@pytest.mark.parametrize("own", [False, True])
def test_step_loop_bmap_mixed(own):
    oracle.set_threads(1)
    st = mapped_box16(own)
    nmax = st.n_particles() + 4096
    S = oracle.load_part(st, nmax=nmax)
    phi = st.geom.phi.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    steps = 3
    for it in range(1, steps + 1):
        Ei, _, _ = oracle.step(st, S, phi, Ei, it)

    def errors(mx):
        from scipy.spatial import cKDTree
        dphi = rel(mx.phi.cpu().numpy(), phi)
        dv, nbad = 0.0, 0
        for p in range(st.ntype):
            g = mx.particles_f64(p).t().cpu().numpy()
            o = S.vxp[p, :S.np_tot[p]]
            # particle identity by position: FP32 offsets move a particle by
            # ~1e-11 m, the particles of a species are ~4e-5 m apart
            dist, j = cKDTree(o[:, 0:3]).query(g[:, 0:3])
            ok = dist <= 1e-9
            nbad = max(nbad, int((~ok).sum()))
            vmax = np.abs(o[:, 3:6]).max()
            if ok.any():
                dv = max(dv, np.abs(g[ok, 3:6] - o[j[ok], 3:6]).max() / vmax)
        return dphi, dv, nbad

    mx = _mixed_run(st, steps, nmax)
    assert np.abs(mx.counts_host() - S.np_tot).max() <= 2
    dphi, dv, nbad = errors(mx)
    assert dphi <= 5e-5, dphi
    assert nbad <= 2, nbad
    assert dv <= 1e-4, dv
    # the same particles pushed without a field end elsewhere: the map is
    # what the match tests
    st0 = config.build("box16")
    _, _, nbad0 = errors(_mixed_run(st0, steps, nmax))
    assert nbad0 > 1000, nbad0
