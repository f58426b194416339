"""GPU tests of the adjoint window: the transposed operators against their
forward operators (dot-product identities), and the window gradient with
respect to the electrode potentials, B_z and the initial velocities against
central finite differences of the same FP64 forward window.

Bars: transposes to 1e-12 relative; gradients within 1e-4 relative of the
central differences (h = 1e-3 V, 1e-6 T); the default adjoint (FP32 V-cycles
in FP64 refinement for the adjoint Poisson solves) within 1e-4 relative of the
FP64 reference gradient."""
import ctypes as C

import numpy as np
import pytest

from essaitemporaire_lepic_module_b200 import config
from tests.conftest import have_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_efield_transpose():
    """<G phi, l> = <phi, G^T l> for the E operator with wall extrapolation."""
    import torch
    from essaitemporaire_lepic_module_b200._lib import check, lib
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("penning_small")
    sim = Simulation(st, cap=1024, fused=False)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    phi = torch.randn(sim.phi.shape, dtype=torch.float64, device="cuda", generator=g)
    lE = torch.randn(sim.Ei.shape, dtype=torch.float64, device="cuda", generator=g)
    sim.Ei.zero_()
    sim.phi.copy_(phi)
    sim.efield()
    lhs = float((sim.Ei * lE).sum())
    lphi = torch.zeros_like(phi)
    lE2 = lE.clone()
    check(lib().lepic_dev_adj_efield(C.byref(sim.grid), _p(lE2), _p(lphi), sim._s()), "adj_efield")
    rhs = float((phi * lphi).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs), (lhs, rhs)


@pytest.fixture(scope="module")
def window():
    from essaitemporaire_lepic_module_b200.adjoint import Window
    st = config.build("penning_small")
    win = Window(st, K=16, every=4)
    win.load_uniform(seed=4242)
    return win


def test_window_gradient_vs_central_differences(window):
    import torch
    from essaitemporaire_lepic_module_b200.adjoint import window_objective
    win = window
    V = torch.tensor([0.0, 200.0, 200.0], dtype=torch.float64, requires_grad=True)
    Bz = torch.tensor(0.1, dtype=torch.float64, requires_grad=True)
    v0 = win.x0[3:6].clone().requires_grad_(True)
    J = window_objective(win, V, Bz, v0)
    J.backward()
    gV, gB, gv = V.grad.numpy(), float(Bz.grad), v0.grad
    base = [0.0, 200.0, 200.0]

    def Jat(Vl, B, v=None):
        return win.forward(Vl, B, v)

    h = 1e-3
    for lab in range(3):
        Vp = list(base)
        Vm = list(base)
        Vp[lab] += h
        Vm[lab] -= h
        fd = (Jat(Vp, 0.1) - Jat(Vm, 0.1)) / (2 * h)
        print("dJ/dV", lab + 1, gV[lab], fd)
        assert abs(gV[lab] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(gV).max()), (lab, gV[lab], fd)
    hb = 1e-6
    fdb = (Jat(base, 0.1 + hb) - Jat(base, 0.1 - hb)) / (2 * hb)
    print("dJ/dBz", gB, fdb)
    assert abs(gB - fdb) <= 1e-4 * abs(fdb), (gB, fdb)
    # a random direction in the initial velocities
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    dirn = torch.randn(v0.shape, dtype=torch.float64, device="cuda", generator=g)
    hv = 1.0  # m/s, against velocities of ~1e6 m/s
    v = win.x0[3:6]
    fdv = (Jat(base, 0.1, v + hv * dirn) - Jat(base, 0.1, v - hv * dirn)) / (2 * hv)
    ad = float((gv * dirn).sum())
    print("dJ/dv0 . d", ad, fdv)
    assert abs(ad - fdv) <= 1e-4 * abs(fdv), (ad, fdv)
    print("timing", win.timing)


def test_mixed_adjoint_solve_matches_fp64_reference_gradient(window):
    """The adjoint with its Poisson solves as FP32 V-cycles inside FP64
    refinement (the default) against the FP64 reference gradient (FP64
    multigrid adjoint solves) of the same window: within 1e-4 relative."""
    import torch
    win = window
    base = [0.0, 200.0, 200.0]
    grads = {}
    for solver in ("f64", "mixed"):
        win.adjoint_solver = solver
        win.forward(base, 0.1)
        dV, dB, dv = win.backward()
        grads[solver] = (np.asarray(dV), dB, dv.clone())
    win.adjoint_solver = "mixed"
    rV, rB, rv = grads["f64"]
    mV, mB, mv = grads["mixed"]
    print("dV", rV, mV, "dBz", rB, mB)
    assert np.abs(mV - rV).max() <= 1e-4 * np.abs(rV).max()
    assert abs(mB - rB) <= 1e-4 * abs(rB)
    assert float((mv - rv).abs().max()) <= 1e-4 * float(rv.abs().max())
