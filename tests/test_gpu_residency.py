"""The drop-in call sequence of Src/main.f90's timestep, per-call copies vs
device-resident mirrors (lepic_gpu_set_residency).

Bars, written in each test:
  * the drop-in loop against the oracle's steps: positions / velocities and
    phi within 1e-10 relative after 20 steps (the trajectory bar);
  * resident vs per-call copies: the same bar (atomic deposition order
    differs from run to run, so not bit for bit), np_tot equal;
  * after the first step the resident loop moves fewer than 1e-3 of the
    per-call bytes between host and device;
  * host-appended particles (injection) reach the device through np_tot;
  * MCC under residency: counted collisions within 5 sigma of the copy mode.
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


def sorted_particles(vxp, n):
    a = vxp[:n]
    return a[np.lexsort((a[:, 2], a[:, 1], a[:, 0]))]


def run_loop(st, S, resident, steps, collide=False, inject=None, **kw):
    """MainLoop over copies of S; inject = (after_step, species, rows) appends
    rows behind np_tot on the host, the way part_injection does."""
    vxp, np_tot, fd, npg = S.vxp.copy(), S.np_tot.copy(), S.flag_dead.copy(), S.np.copy()
    ml = dropin.MainLoop(st, vxp, np_tot, fd, npg, resident=resident, collide=collide, **kw)
    traffic = []
    try:
        for s in range(1, steps + 1):
            a = dropin.mirror_stats()
            ml.step()
            b = dropin.mirror_stats()
            traffic.append((b[0] - a[0]) + (b[1] - a[1]))
            if inject is not None and s == inject[0]:
                p, rows = inject[1], inject[2]
                n0 = int(np_tot[p])
                vxp[p, n0:n0 + len(rows)] = rows
                np_tot[p] = n0 + len(rows)
        ml.sync()
        out = dict(vxp=vxp, np_tot=np_tot.copy(), np=npg.copy(), phi=ml.phi.copy(), Ei=ml.Ei.copy(),
                   traffic=traffic)
    finally:
        ml.close()
    return out


@pytest.fixture(scope="module")
def box16():
    oracle.set_threads(1)
    st = config.build("box16")
    S = oracle.load_part(st, nmax=st.n_particles() + 4096)
    return st, S


def test_dropin_loop_matches_oracle(box16):
    """20 timesteps of calls through the Fortran-signature entry points
    (resident) against 20 oracle steps in the reference order: 1e-10."""
    st, S0 = box16
    S = S0.copy()
    out = run_loop(st, S0, True, 20)
    phi = st.geom.phi.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    for it in range(1, 21):
        Ei, _, _ = oracle.step(st, S, phi, Ei, it)
    assert np.array_equal(out["np_tot"], S.np_tot)
    for p in range(st.ntype):
        g = sorted_particles(out["vxp"][p], S.np_tot[p])
        o = sorted_particles(S.vxp[p], S.np_tot[p])
        for c in range(6):
            assert rel(g[:, c], o[:, c]) <= 1e-10, (p, c, rel(g[:, c], o[:, c]))
    assert rel(out["phi"], phi) <= 1e-10
    assert rel(out["Ei"], Ei) <= 1e-10


def test_resident_matches_copy_mode_and_moves_little(box16):
    st, S0 = box16
    a = run_loop(st, S0, False, 12)
    b = run_loop(st, S0, True, 12)
    assert np.array_equal(a["np_tot"], b["np_tot"])
    for p in range(st.ntype):
        n = a["np_tot"][p]
        ga, gb = sorted_particles(a["vxp"][p], n), sorted_particles(b["vxp"][p], n)
        for c in range(6):
            assert rel(gb[:, c], ga[:, c]) <= 1e-10
    for k in ("phi", "Ei", "np"):
        assert rel(b[k], a[k]) <= 1e-10, k
    copy_bytes = np.mean(a["traffic"][1:])
    resident_bytes = np.mean(b["traffic"][1:])
    assert copy_bytes > 1e6
    assert resident_bytes < 1e-3 * copy_bytes, (resident_bytes, copy_bytes)


def test_injection_behind_np_tot_reaches_the_device(box16):
    st, S0 = box16
    rows = S0.vxp[0, :500].copy()
    rows[:, 0] = np.clip(rows[:, 0] * 0.5 + 0.25 * st.geom.box[0], 0.0, st.geom.box[0])
    a = run_loop(st, S0, False, 8, inject=(4, 0, rows))
    b = run_loop(st, S0, True, 8, inject=(4, 0, rows))
    c = run_loop(st, S0, True, 8)
    # the rows start mid-box: few of them reach a wall within 4 steps
    assert a["np_tot"][0] > c["np_tot"][0] + 400
    assert np.array_equal(a["np_tot"], b["np_tot"])
    for p in range(st.ntype):
        n = a["np_tot"][p]
        ga, gb = sorted_particles(a["vxp"][p], n), sorted_particles(b["vxp"][p], n)
        for c in range(6):
            assert rel(gb[:, c], ga[:, c]) <= 1e-10


def test_update_device_and_stale_mirror(box16):
    """A host write to a mirrored array is invisible to the GPU until
    lepic_gpu_update_device covers it."""
    import ctypes as C
    from essaitemporaire_lepic_module_b200._lib import lib
    st, _ = box16
    dropin.set_commons(st)
    dropin.set_residency(True)
    try:
        n = np.array(st.n, dtype=np.int32)
        h = np.asarray(st.h, dtype=np.float64).copy()
        bc = np.ascontiguousarray(st.geom.bcnd, dtype=np.int32).copy()
        x = np.linspace(0.0, 1.0, st.geom.bcnd.shape[2])
        phi = np.ascontiguousarray(np.broadcast_to(x, st.geom.bcnd.shape) * 10.0)
        Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
        pi, pd = dropin._pi, dropin._pd
        L = lib()
        L.calc_efield_(pi(n), pd(h), pd(phi), pd(Ei), pi(bc))
        assert L.lepic_gpu_last_error() == 0
        dropin.sync_to_host()
        E1 = Ei.copy()
        phi *= 2.0
        L.calc_efield_(pi(n), pd(h), pd(phi), pd(Ei), pi(bc))
        dropin.sync_to_host()
        assert np.array_equal(Ei, E1)          # stale: the mirror still holds phi
        assert L.lepic_gpu_update_device(C.c_void_p(phi.ctypes.data), phi.nbytes) == 0
        L.calc_efield_(pi(n), pd(h), pd(phi), pd(Ei), pi(bc))
        dropin.sync_to_host()
        assert np.abs(E1).max() > 0
        assert rel(Ei, 2.0 * E1) <= 1e-14
    finally:
        dropin.set_residency(False)
    assert dropin.mirror_stats()[2] == 0


def test_mcc_loop_resident():
    """MCC every step through collisions_ with resident particle mirrors and
    a region counter over the whole box (which reads np_red back from its
    mirror): the counted collisions, sum over processes of cnt_col times the
    region population, within 5 sigma of the per-call copy mode."""
    oracle.set_threads(1)
    st = config.build("mcc32")
    S0 = oracle.load_part(st, nmax=int(st.n_particles() * 1.3))
    reg = [(1, st.n[0] + 1)]
    res = {}
    for resident in (False, True):
        vxp, np_tot, fd, npg = S0.vxp.copy(), S0.np_tot.copy(), S0.flag_dead.copy(), S0.np.copy()
        ml = dropin.MainLoop(st, vxp, np_tot, fd, npg, resident=resident, collide=True, ns_coll=1,
                             regions=reg)
        try:
            for _ in range(6):
                ml.step()
            ml.sync()
            res[resident] = float(ml.cnt_col.sum()) * float(np_tot[0])
        finally:
            ml.close()
    a, b = res[False], res[True]
    assert a > 100 and b > 100, (a, b)
    assert abs(a - b) <= 5.0 * np.sqrt(a + b), (a, b)
