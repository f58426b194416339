"""Order independence of the depositions (the races of the reference's
OpenMP build are avoided with per-thread copies; here atomics sum in whatever
order the threads run): the same particles deposited in their order and in a
random permutation give the same density, FP64 weights and the mixed form's
integer weights alike, to the rounding of the FP64 node sums (1e-13
relative); the mixed form's integer weights conserve the charge exactly in
either order."""
import ctypes as C

import numpy as np
import pytest

from essaitemporaire_lepic_module_b200 import config
from tests.conftest import have_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]


def _shuffle(s, perm, planes, extra=()):
    n = perm.numel()
    for t in planes:
        t[:, :n] = t[:, :n][:, perm]
    for t in extra:
        t[:n] = t[:n][perm]


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_deposit_is_order_independent(precision):
    import torch
    from essaitemporaire_lepic_module_b200._lib import check, lib
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("box32")
    sim = Simulation(st, precision=precision, seed=31)
    sim.load_uniform()
    g = torch.Generator(device="cuda")
    g.manual_seed(5)

    def deposit():
        out = torch.zeros_like(sim.np)
        for p, s in enumerate(sim.sp):
            if precision == "f64":
                check(lib().lepic_dev_charge_deposition(C.byref(sim.grid), C.byref(s.s), p + 1, C.byref(sim.P),
                                                        C.c_void_p(out[p].data_ptr()), sim._s()), "deposit")
            else:
                check(lib().lepic_dev_deposit_mixed(C.byref(sim.grid), C.byref(s.s), p + 1, C.byref(sim.P),
                                                    C.c_void_p(out[p].data_ptr()), s.n(), sim._s()), "deposit")
        torch.cuda.synchronize()
        return out

    a = deposit()
    for s in sim.sp:
        n = s.n()
        perm = torch.randperm(n, device="cuda", generator=g)
        if precision == "f64":
            _shuffle(s, perm, [s.p])
        else:
            _shuffle(s, perm, [s.p], [s.cell])
    b = deposit()
    scale = float(a.abs().max())
    assert float((a - b).abs().max()) <= 1e-13 * scale
    # charge per species: sum np / kq h^3 = N Nm
    vol = float(np.prod(st.h))
    kq = torch.as_tensor(st.kq, device="cuda")
    for p, s in enumerate(sim.sp):
        want = s.n() * st.Nm[p]
        for d in (a, b):
            assert abs(float((d[p] / kq).sum()) * vol - want) <= 1e-12 * want
