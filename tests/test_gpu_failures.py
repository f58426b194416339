"""Failure detection without faulting the GPU: bad inputs are made on the
host, the kernels record a status in the device error word instead of
trapping, the host turns it into LepicError with the status code, and the
context stays usable afterwards.

  * a particle in a cell outside the grid         -> LEPIC_ERR_CELL (22)
  * ionization products beyond the capacity       -> LEPIC_ERR_CAPACITY (1)
  * a refinement cap too small for the tolerance  -> LEPIC_ERR_NOT_CONVERGED (23)
  * a NaN in the right-hand side                  -> a non-zero status, then a
                                                     clean solve succeeds
  * a bounded device wait that nothing completes  -> LEPIC_ERR_TIMEOUT (25)
                                                     after its limit, then the
                                                     context runs a step
"""
import numpy as np
import pytest

from essaitemporaire_lepic_module_b200 import config
from tests.conftest import have_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]


def test_cell_outside_grid_raises_then_recovers():
    from essaitemporaire_lepic_module_b200._lib import LepicError
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("box16")
    sim = Simulation(st, precision="mixed")
    sim.load_uniform()
    sim.step()
    n1 = st.n[0]
    sim.sp[0].cell[7] = (n1 + 4) | (2 << 10) | (2 << 20)   # ix beyond the grid
    with pytest.raises(LepicError) as e:
        sim.step()
    assert e.value.code == 22
    sim.step()                                             # the bad particle became a hole


def test_capacity_overflow_in_collisions():
    import torch
    from essaitemporaire_lepic_module_b200._lib import LepicError
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("mcc32")
    n = st.n_particles()
    sim = Simulation(st, cap=n)
    sim.load_uniform()
    s = sim.sp[0]
    s.p[3:6, :n] *= 4.0             # 32 eV electrons: every call ionizes many
    torch.cuda.synchronize()
    sim.it = 11
    with pytest.raises(LepicError) as e:
        sim.collisions()
    assert e.value.code == 1
    sim.check_device()              # the error word was cleared by the raise


def _poisson_sim():
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("poisson32")
    sim = Simulation(st, cap=1024, precision="mixed")
    sim.rhs.copy_(torch.as_tensor(st.rhs_blobs, device="cuda"))
    sim.phi.copy_(torch.as_tensor(st.geom.phi, device="cuda"))
    return st, sim


def test_refinement_cap_reports_not_converged():
    from essaitemporaire_lepic_module_b200._lib import LepicError
    st, sim = _poisson_sim()
    with pytest.raises(LepicError) as e:
        sim.pdesolver_mixed(eps=1e-15, max_refine=1)
    assert e.value.code == 23
    it, _, res = sim.pdesolver_mixed()
    assert res < st.wl.eps


def test_nan_in_rhs_is_reported_and_the_next_solve_works():
    import torch
    from essaitemporaire_lepic_module_b200._lib import LepicError
    st, sim = _poisson_sim()
    good = sim.rhs.clone()
    sim.rhs.view(-1)[12345] = float("nan")
    with pytest.raises(LepicError):
        sim.pdesolver_mixed(max_refine=5)
    sim.rhs.copy_(good)
    sim.phi.copy_(torch.as_tensor(st.geom.phi, device="cuda"))
    it, _, res = sim.pdesolver_mixed()
    assert res < st.wl.eps and bool(torch.isfinite(sim.phi).all())


def test_bounded_wait_times_out_and_context_stays_usable():
    """An mbarrier phase that no copy completes: the wait gives up after its
    limit (50 ms here; the library's copy waits allow one second) and the
    kernel records LEPIC_ERR_TIMEOUT instead of hanging; the status is read
    once and cleared, and a step runs afterwards."""
    import ctypes as C
    import time
    import torch
    from essaitemporaire_lepic_module_b200._lib import lib
    from essaitemporaire_lepic_module_b200.sim import Simulation
    torch.cuda.synchronize()
    L = lib()
    t0 = time.perf_counter()
    assert L.lepic_dev_wait_selftest(50_000_000, None) == 0
    detail = C.c_int(-1)
    assert L.lepic_dev_check(None, C.byref(detail)) == 25
    elapsed = time.perf_counter() - t0
    assert 0.045 <= elapsed < 5.0, elapsed
    assert L.lepic_dev_check(None, C.byref(detail)) == 0          # read once, then cleared
    assert L.lepic_dev_wait_selftest(0, None) == 21                # limit out of range: LEPIC_ERR_ARG
    st = config.build("box16")
    sim = Simulation(st, precision="mixed")
    sim.load_uniform()
    sim.step()
    torch.cuda.synchronize()
    assert L.lepic_dev_check(None, C.byref(detail)) == 0


def test_nonblocking_loop_reports_failures_later():
    """Nonblocking mode (no wait in the step loop): a particle moved outside
    the grid is reported by a later step's check or at flush_checks, with
    the same status code, and the loop goes on afterwards."""
    from essaitemporaire_lepic_module_b200._lib import LepicError
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build("box16")
    sim = Simulation(st, precision="mixed", nonblocking=True)
    sim.load_uniform()
    sim.step()
    sim.flush_checks()
    n1 = st.n[0]
    sim.sp[0].cell[7] = (n1 + 4) | (2 << 10) | (2 << 20)
    with pytest.raises(LepicError) as e:
        for _ in range(4):
            sim.step()
        sim.flush_checks()
    assert e.value.code == 22
    sim.flush_checks()
    sim.step()
    sim.flush_checks()
