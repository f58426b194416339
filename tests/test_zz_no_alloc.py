"""The allocation-free Poisson solve (lepic_dev_pdesolver_noalloc).

It serves callers that cannot call cudaMalloc inside their time loop
because their device memory belongs to their own pool (a Fortran host that
hands every buffer in, or a framework allocator such as PyTorch's); its
scratch is one static device array per GPU.  This test calls it through the
C ABI and checks it against the allocating entry point lepic_dev_pdesolver
on the same inputs, on two calls in a row (a cold solve, then a warm-started
one that reuses the scratch left by the first), with the same bar as the
other Poisson parity tests: identical V-cycle count and sweep total, phi
within 1e-12 relative.  It also checks that a grid larger than the static
scratch is refused with LEPIC_ERR_SCRATCH_LIMIT.  The file name makes pytest
collect it last.
"""
import ctypes as C

import numpy as np
import pytest

from tests.conftest import have_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]


def _solve(entry, grid, phi, rhs, P, st, stream):
    k = C.c_int(0)
    ktot = C.c_double(0)
    res = C.c_double(0)
    rc = entry(C.byref(grid), C.c_void_p(phi.data_ptr()), C.c_void_p(rhs.data_ptr()), st.wl.ncycl,
               st.wl.eps, st.wl.omega, st.ng, C.byref(P), C.byref(k), C.byref(ktot), C.byref(res),
               stream)
    return rc, k.value, ktot.value, res.value


@pytest.mark.parametrize("name", ["poisson32", "poisson64"])
def test_noalloc_matches_allocating_solve_twice(name):
    import torch
    from essaitemporaire_lepic_module_b200 import config
    from essaitemporaire_lepic_module_b200._lib import LepicGrid, lib, phys_struct

    st = config.build(name)
    dev = torch.device("cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    bc = torch.as_tensor(np.ascontiguousarray(st.geom.bcnd), dtype=torch.int32, device=dev)
    rhs = torch.as_tensor(np.ascontiguousarray(st.rhs_blobs), dtype=torch.float64, device=dev)
    grid = LepicGrid()
    for a in range(3):
        grid.n[a] = st.n[a]
        grid.h[a] = float(st.h[a])
    grid.bcnd = bc.data_ptr()
    P = phys_struct(st)
    L = lib()
    phi_a = torch.as_tensor(np.ascontiguousarray(st.geom.phi), dtype=torch.float64, device=dev)
    phi_b = phi_a.clone()
    for call in range(2):   # cold solve, then a warm start from the previous phi
        ra = _solve(L.lepic_dev_pdesolver, grid, phi_a, rhs, P, st, stream)
        rb = _solve(L.lepic_dev_pdesolver_noalloc, grid, phi_b, rhs, P, st, stream)
        torch.cuda.synchronize()
        assert ra[0] == 0 and rb[0] == 0, (ra, rb)
        assert rb[1] == ra[1] and rb[2] == ra[2], (call, ra, rb)
        a = phi_a.cpu().numpy()
        b = phi_b.cpu().numpy()
        assert np.abs(b - a).max() <= 1e-12 * np.abs(a).max(), call
        assert rb[3] < st.wl.eps
        # perturb the source a little so the second call does real work
        rhs.mul_(1.01)


def test_noalloc_rejects_grid_beyond_limit():
    import torch
    from essaitemporaire_lepic_module_b200 import config
    from essaitemporaire_lepic_module_b200._lib import LepicGrid, lib, phys_struct

    st = config.build("box32")
    grid = LepicGrid()
    for a in range(3):
        grid.n[a] = 128
        grid.h[a] = float(st.h[a])
    grid.bcnd = None
    P = phys_struct(st)
    k = C.c_int(0)
    kt = C.c_double(0)
    r = C.c_double(0)
    rc = lib().lepic_dev_pdesolver_noalloc(C.byref(grid), None, None, 10, 1e-10, 1.4, 7, C.byref(P),
                                           C.byref(k), C.byref(kt), C.byref(r),
                                           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 24   # LEPIC_ERR_SCRATCH_LIMIT, raised before any device work


def test_noalloc_allocates_no_device_memory():
    """The property the entry point exists for: after one call has set the
    device up, further calls (two grid sizes, two calls each) leave the
    device's free memory unchanged -- no cudaMalloc behind the caller's
    back.  Every input is allocated before the first reading."""
    import torch
    from essaitemporaire_lepic_module_b200 import config
    from essaitemporaire_lepic_module_b200._lib import LepicGrid, lib, phys_struct

    dev = torch.device("cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    cases = []
    for name in ("poisson32", "poisson64"):
        st = config.build(name)
        bc = torch.as_tensor(np.ascontiguousarray(st.geom.bcnd), dtype=torch.int32, device=dev)
        rhs = torch.as_tensor(np.ascontiguousarray(st.rhs_blobs), dtype=torch.float64, device=dev)
        phi = torch.as_tensor(np.ascontiguousarray(st.geom.phi), dtype=torch.float64, device=dev)
        grid = LepicGrid()
        for a in range(3):
            grid.n[a] = st.n[a]
            grid.h[a] = float(st.h[a])
        grid.bcnd = bc.data_ptr()
        cases.append((st, grid, phi, rhs, phys_struct(st), bc))
    L = lib()
    st, grid, phi, rhs, P, _ = cases[0]
    assert _solve(L.lepic_dev_pdesolver_noalloc, grid, phi, rhs, P, st, stream)[0] == 0   # set-up call
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        for st, grid, phi, rhs, P, _ in reversed(cases):
            phi.zero_()
            assert _solve(L.lepic_dev_pdesolver_noalloc, grid, phi, rhs, P, st, stream)[0] == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
