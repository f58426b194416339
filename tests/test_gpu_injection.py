"""GPU particle injection (Src/part_injection.f90) against the CPU oracle.

The events draw from Philox instead of the reference's serial ran2.  Bars:
the number of events equal to the oracle's to the one-event rounding draw
(the same current), every species injected by every event when n/n0 = 1,
the new particles inside the injection box (the disk of the beam and the
cathode), velocity moments within 4 sigma of the oracle's, P_loss(4) equal
to the injected kinetic energy (1e-9); in the step loop (both forms) the
new particles deposited with the others (the density integral equals the
particle count times Nm to 1e-12), and with opt_inj 2 as many electrons
injected as ions were lost.
"""
import math

import numpy as np
import pytest

import oracle
from essaitemporaire_lepic_module_b200 import config, dropin
from tests.conftest import have_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

BOX = dict(xl=0.4e-3, xr=1.2e-3, yl=0.2e-3, yr=1.4e-3, zl=0.2e-3, zr=1.4e-3)


def _inj(opt):
    return config.Injection(opt_inj=opt, I_inj=2.5e-3, THm=10.0, zg_sec=(0.2e-3, 1.4e-3), **BOX)


def _mean_close(a, b):
    s = math.sqrt(a.var() / len(a) + b.var() / len(b))
    return abs(a.mean() - b.mean()) <= 4 * s + 1e-300


@pytest.mark.parametrize("opt", [1, -1, 3, 4])
def test_part_injection_dropin(opt):
    oracle.set_threads(1)
    st = config.build("box16")
    dropin.set_commons(st)
    inj = _inj(opt)
    So = oracle.State(st, 20000)
    plo = np.zeros((st.ntype, 4))
    oracle.part_injection(st, So, inj, st.geom.phi, plo)
    vxp = np.zeros((st.ntype, 20000, 6))
    npt = np.zeros(st.ntype, dtype=np.int32)
    plg = np.zeros((st.ntype, 4))
    dropin.part_injection(st, inj, vxp, npt, st.geom.phi, plg)
    beam = abs(opt) in (3, 4)
    for p in range(st.ntype):
        if beam and p > 0:
            assert npt[p] == 0
            continue
        assert abs(int(npt[p]) - int(So.np_tot[p])) <= 1, (npt, So.np_tot)
        g = vxp[p, :npt[p]]
        o = So.vxp[p, :So.np_tot[p]]
        assert (g[:, 0] >= BOX["xl"]).all() and (g[:, 0] <= BOX["xr"]).all()
        assert (g[:, 1] >= BOX["yl"]).all() and (g[:, 1] <= BOX["yr"]).all()
        if beam:
            xm, ym = (BOX["xl"] + BOX["xr"]) / 2, (BOX["yl"] + BOX["yr"]) / 2
            R = min(BOX["xr"] - BOX["xl"], BOX["yr"] - BOX["yl"]) / 2
            assert ((g[:, 0] - xm) ** 2 + (g[:, 1] - ym) ** 2 <= R * R * (1 + 1e-12)).all()
            assert (g[:, 2] >= 0).all() and (g[:, 2] <= st.geom.box[2]).all()
        for c in range(3, 6):
            assert _mean_close(g[:, c], o[:, c]), (p, c, g[:, c].mean(), o[:, c].mean())
            assert _mean_close(g[:, c] ** 2, o[:, c] ** 2), (p, c)
        for c in range(3):
            assert _mean_close(g[:, c], o[:, c]), (p, c)
        ke = 0.5 * st.Nm[p] * st.mass[p] * (g[:, 3:6] ** 2).sum()
        assert abs(plg[p, 3] - ke) <= 1e-9 * ke


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_step_loop_injection(precision):
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    oracle.set_threads(1)
    st = config.build("box16")
    nmax = st.n_particles() + 30000
    S0 = oracle.load_part(st, nmax=nmax)
    sim = Simulation(st, cap=nmax, precision=precision, injection=_inj(1))
    sim.load_from_host(S0.vxp, S0.np_tot, S0.np)
    for _ in range(2):
        sim.step()
    torch.cuda.synchronize()
    n_ev = 2.5e-3 * st.dt / (1.602176634e-19 * st.Nm[0])
    assert np.all(np.abs(sim.injected - 2 * n_ev) <= 2), sim.injected
    vol = st.h[0] * st.h[1] * st.h[2]
    kq = torch.as_tensor(st.kq, device=sim.dev)
    for p in range(st.ntype):
        tot = float((sim.np[p] / kq).sum()) * vol
        want = sim.sp[p].n() * st.Nm[p]
        assert abs(tot - want) <= 1e-12 * want, (p, tot, want)


def test_step_loop_injection_replaces_lost_ions():
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    oracle.set_threads(1)
    st = config.build("box16")
    nmax = st.n_particles() + 30000
    S0 = oracle.load_part(st, nmax=nmax)
    inj = config.Injection(opt_inj=2, I_inj=0.0, **BOX)
    # 100 ions that cross the wall x = 0 in the first step
    S0.vxp[1, :100, 0] = 0.3 * st.h[0]
    S0.vxp[1, :100, 3] = -0.7 * st.h[0] / st.dt
    sim = Simulation(st, cap=nmax, injection=inj)
    sim.load_from_host(S0.vxp, S0.np_tot, S0.np)
    for _ in range(5):
        sim.step()
    torch.cuda.synchronize()
    pm, _ = sim.loss_stats()
    lost_ions = int(round(pm[:, 0, 1].sum()))
    assert lost_ions >= 100
    assert sim.injected[0] == lost_ions and sim.injected[1] == lost_ions
