"""GPU part_mover_ with negative ions and secondary emission against the CPU
oracle (Src/part_expmover.f90:76, 278-301, 353-400, 416-470).

Negative ions (species 3 of neg16, with the Neumann plane at x = 0 and the
extraction grid at x = xmax): particles bit for bit, flag_cex compacted with
them, cnt_cex and cnt_dead exact, beam_div within 1e-12 (the device sums in
atomic order), p_mac and P_loss as the oracle.  Secondary emission (Ar+ of
box16 on the emissive wall): the ions bit for bit; the reference draws from its
serial ran2 stream and the device from Philox, so with gam_sec = 2 the number
of electrons and the multiset of their positions are exact, their velocities
are checked in distribution, and P_loss(4, 1) is the reference's sum over the
electrons the device emitted (1e-12); with gam_sec = 0.5 the count is within
4 sigma of the binomial expectation."""
import numpy as np
import pytest

import oracle
from essaitemporaire_lepic_module_b200 import dropin
from essaitemporaire_lepic_module_b200.constants import QE
from tests.conftest import have_gpu
from tests.test_mover_extras import neg_setup, sec_setup

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]


def _random(st, S, p, n, vmax, rng):
    L = np.asarray(st.geom.box)
    h = np.asarray(st.h)
    lo, hi = h, L - h
    S.vxp[p, :n, :3] = lo + (hi - lo) * rng.random((n, 3))
    S.vxp[p, :n, 3:] = rng.uniform(-vmax, vmax, (n, 3)) * h / st.dt
    S.np_tot[p] = n


def test_negative_ions_dropin_vs_oracle():
    oracle.set_threads(1)
    st = neg_setup()
    dropin.set_commons(st)
    rng = np.random.default_rng(21)
    nmax = 4096
    So = oracle.State(st, nmax)
    _random(st, So, 2, 3000, 8.0, rng)
    So.flag_dead[2, :3000] = (rng.random(3000) < 0.05).astype(np.int8)
    Xo = oracle.MoverExtra(nmax, tag_neg=3, tag_neu=4, num_grd=1)
    Xo.flag_cex[:3000] = rng.choice([0, 4, -4, 9], 3000)
    Sg = So.copy()
    Xg = dropin.MoverExtra(nmax, tag_neg=3, tag_neu=4, num_grd=1)
    Xg.flag_cex[:] = Xo.flag_cex
    Ei = rng.normal(0.0, 2e3, tuple(st.geom.bcnd.shape) + (3,))
    ng1 = st.geom.ngrid + 1
    pm_o, pm_g = np.zeros((ng1, 2, st.ntype)), np.zeros((ng1, 2, st.ntype))
    pl_o, pl_g = np.zeros((st.ntype, 4)), np.zeros((st.ntype, 4))
    for _ in range(3):
        oracle.part_mover(st, Ei, So, pm_o, pl_o, 3, extra=Xo)
        dropin.part_mover(st, Ei, Sg.vxp, Sg.np_tot, Sg.flag_dead, pm_g, pl_g, 3, extra=Xg)
    n = int(So.np_tot[2])
    assert Sg.np_tot[2] == n and 0 < n < 2500
    np.testing.assert_array_equal(Sg.vxp[2, :n], So.vxp[2, :n])
    np.testing.assert_array_equal(Xg.flag_cex[:n], Xo.flag_cex[:n])
    np.testing.assert_array_equal(Xg.cnt_cex, Xo.cnt_cex)
    assert Xo.cnt_cex[0] > 100 and Xo.cnt_cex[2] > 10
    assert Xg.cnt_dead[0] == Xo.cnt_dead[0] != 0.0
    np.testing.assert_allclose(Xg.beam_div, Xo.beam_div, rtol=0, atol=1e-12 * np.abs(Xo.beam_div).max())
    np.testing.assert_array_equal(pm_g[:, 0, :], pm_o[:, 0, :])
    assert pm_o[0, 0, 2] > 50                             # lost through the Neumann plane, label 0
    np.testing.assert_allclose(pm_g[:, 1, :], pm_o[:, 1, :], rtol=1e-12, atol=0)
    np.testing.assert_allclose(pl_g, pl_o, rtol=1e-12, atol=0)


@pytest.mark.parametrize("gam", [2.0, 0.5])
def test_secondary_emission_dropin_vs_oracle(gam):
    oracle.set_threads(1)
    st = sec_setup()
    dropin.set_commons(st)
    rng = np.random.default_rng(31)
    nmax = 16384
    L = st.geom.box
    zg = (0.25 * L[2], 0.75 * L[2])
    So = oracle.State(st, nmax)
    _random(st, So, 1, 3000, 8.0, rng)
    _random(st, So, 0, 500, 0.1, rng)
    Sg = So.copy()
    Xo = oracle.MoverExtra(nmax, gam_sec=gam, igrid_sec=1, THm=2.0, zg_sec=zg, iseed=777)
    Xg = dropin.MoverExtra(nmax, gam_sec=gam, igrid_sec=1, THm=2.0, zg_sec=zg, iseed=777)
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    ng1 = st.geom.ngrid + 1
    pm_o, pm_g = np.zeros((ng1, 2, st.ntype)), np.zeros((ng1, 2, st.ntype))
    pl_o, pl_g = np.zeros((st.ntype, 4)), np.zeros((st.ntype, 4))
    oracle.part_mover(st, Ei, So, pm_o, pl_o, 2, extra=Xo)
    dropin.part_mover(st, Ei, Sg.vxp, Sg.np_tot, Sg.flag_dead, pm_g, pl_g, 2, extra=Xg)
    ni = int(So.np_tot[1])
    assert Sg.np_tot[1] == ni
    np.testing.assert_array_equal(Sg.vxp[1, :ni], So.vxp[1, :ni])
    np.testing.assert_array_equal(Sg.vxp[0, :500], So.vxp[0, :500])      # the electrons already there
    lost = int(pm_o[1, 0, 1])
    assert lost == 3000 - ni and lost > 1000
    ne_g, ne_o = int(Sg.np_tot[0]) - 500, int(So.np_tot[0]) - 500
    eg = Sg.vxp[0, 500:500 + ne_g]
    if gam == 2.0:
        assert ne_g == ne_o == 2 * lost
        # positions: the ions' impact points on the cathode planes, as a multiset
        ko = np.lexsort(So.vxp[0, 500:500 + ne_o, :3].T[::-1])
        kg = np.lexsort(eg[:, :3].T[::-1])
        np.testing.assert_array_equal(eg[kg, :3], So.vxp[0, 500:500 + ne_o][ko, :3])
    else:
        sd = np.sqrt(lost * 0.25)
        assert abs(ne_g - 0.5 * lost) <= 4 * sd, (ne_g, lost)
    assert set(np.unique(eg[:, 2])) <= set(zg)
    # the normal velocity points away from the plane the ion moved towards
    assert (eg[eg[:, 2] == zg[0], 5] > 0).all() and (eg[eg[:, 2] == zg[1], 5] < 0).all()
    vt2 = 2.0 * QE * 2.0 / abs(st.mass[0])
    m = len(eg)
    for x2, name in ((eg[:, 5] ** 2, "vz^2"), (eg[:, 3] ** 2 + eg[:, 4] ** 2, "vx^2 + vy^2")):
        # both are vt^2 times an exponential variable: mean vt^2, sd vt^2
        assert abs(x2.mean() / vt2 - 1.0) <= 5.0 / np.sqrt(m), name
    want = 0.5 * st.Nm[0] * st.mass[0] * (eg[:, 3] ** 2 + 2 * eg[:, 5] ** 2).sum()
    np.testing.assert_allclose(pl_g[0, 3], want, rtol=1e-12)
    np.testing.assert_array_equal(pm_g[:, 0, :], pm_o[:, 0, :])
    assert int(Xg.iseed[0]) != 777
