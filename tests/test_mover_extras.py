"""The negative-ion bookkeeping and the secondary emission of the mover
(Src/part_expmover.f90:76, 278-301, 353-400, 416-470) in the CPU oracle:
known answers on hand-placed particles.

Negative ions (species tag_neg): a negative ion reaching x < 0 with the
Neumann plane is lost at label 0 instead of reflected; a killed one adds Nm q
to cnt_dead; one lost on the grid num_grd counts in cnt_cex(1), in cnt_cex(2)
when |flag_cex| = tag_neu, in cnt_cex(3) when flag_cex = -tag_neu, and adds
atan(vy/vx), atan(vz/vx) and their squares to beam_div; flag_cex follows the
in-order compaction.  Secondary emission: an ion lost on igrid_sec emits
INT(gam_sec) electrons (one more with probability gam_sec - INT(gam_sec)) at
its (x, y) on the cathode plane it moved towards, with the ran2 draws of the
reference's order, and P_loss(4, 1) grows by 0.5 Nm m (vx^2 + 2 vz^2)."""
import dataclasses

import numpy as np

import oracle
from essaitemporaire_lepic_module_b200 import config
from essaitemporaire_lepic_module_b200.constants import QE


def neg_setup():
    """nmn16 (Neumann plane at x = 0, wall label 1 at x = xmax) with e-, H+
    and H- (species 3, the negative ions)."""
    wl = dataclasses.replace(config.workload("nmn16"), name="neg16",
                             ions=[("[H+]", 1.008, 1.0, 0.1, 1.0), ("[H-]", 1.008, -1.0, 0.1, 0.2)])
    return config.build(wl)


def sec_setup():
    """box16 (label 1 on every wall) with e- and Ar+."""
    return config.build("box16")


def _mover(st, S, ptype, extra):
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    pm = np.zeros((st.geom.ngrid + 1, 2, st.ntype))
    pl = np.zeros((st.ntype, 4))
    oracle.part_mover(st, Ei, S, pm, pl, ptype, extra=extra)
    return pm, pl


def test_negative_ions_known_answers():
    st = neg_setup()
    h, L, dt = st.h, st.geom.box, st.dt
    S = oracle.State(st, 8)
    X = oracle.MoverExtra(8, tag_neg=3, tag_neu=4, num_grd=1)
    v1 = h[0] / dt
    S.vxp[2, 0] = [0.3 * h[0], 0.5 * L[1], 0.5 * L[2], -0.5 * v1, 0.0, 0.0]       # through x = 0
    S.vxp[2, 1] = [0.5 * L[0], 0.5 * L[1], 0.5 * L[2], 0.1 * v1, 0.0, 0.0]       # killed
    S.vxp[2, 2] = [L[0] - 0.2 * h[0], 0.5 * L[1], 0.5 * L[2], 0.5 * v1, 0.2 * v1, -0.1 * v1]  # onto num_grd
    S.vxp[2, 3] = [0.5 * L[0], 0.4 * L[1], 0.5 * L[2], 0.01 * v1, 0.0, 0.0]      # stays
    S.vxp[2, 4] = [L[0] - 0.2 * h[0], 0.3 * L[1], 0.5 * L[2], 0.5 * v1, 0.0, 0.3 * v1]  # onto num_grd
    S.vxp[2, 5] = [0.6 * L[0], 0.4 * L[1], 0.5 * L[2], 0.01 * v1, 0.0, 0.0]      # stays
    S.np_tot[2] = 6
    S.flag_dead[2, 1] = 1
    X.flag_cex[:6] = [7, 9, 4, 11, -4, 13]
    pm, pl = _mover(st, S, 3, X)
    assert S.np_tot[2] == 2
    assert list(X.flag_cex[:2]) == [11, 13]              # the kept particles' flags, in order
    assert pm[0, 0, 2] == 1 and pm[1, 0, 2] == 2          # label 0 (Neumann), label 1 (num_grd)
    assert X.cnt_dead[0] == st.Nm[2] * st.charge[2]
    assert list(X.cnt_cex) == [2, 2, 1]
    t1, t2 = np.arctan(0.2 / 0.5), np.arctan(0.0 / 0.5)
    u1, u2 = np.arctan(-0.1 / 0.5), np.arctan(0.3 / 0.5)
    np.testing.assert_allclose(X.beam_div, [t1 + t2, t1 * t1 + t2 * t2, u1 + u2, u1 * u1 + u2 * u2], rtol=1e-14)
    # a positive species at x < 0 is reflected as before
    S2 = oracle.State(st, 4)
    S2.vxp[1, 0] = [0.3 * h[0], 0.5 * L[1], 0.5 * L[2], -0.5 * v1, 0.0, 0.0]
    S2.np_tot[1] = 1
    _mover(st, S2, 2, oracle.MoverExtra(4, tag_neg=3, tag_neu=4, num_grd=1))
    assert S2.np_tot[1] == 1 and S2.vxp[1, 0, 3] > 0


def test_secondary_emission_known_answers():
    st = sec_setup()
    h, L, dt = st.h, st.geom.box, st.dt
    v1 = h[0] / dt
    zg = (0.25 * L[2], 0.75 * L[2])
    for gam, nexp in ((2.0, 2), (2.999999999, 3)):
        S = oracle.State(st, 16)
        S.vxp[1, 0] = [0.5 * L[0], 0.5 * L[1], 0.2 * h[2], 0.0, 0.0, -0.5 * v1]     # onto z = 0
        S.vxp[1, 1] = [0.4 * L[0], 0.5 * L[1], 0.5 * L[2], 0.0, 0.0, 0.001 * v1]    # stays
        S.np_tot[1] = 2
        S.vxp[0, 0] = [0.5 * L[0], 0.5 * L[1], 0.5 * L[2], 0.0, 0.0, 0.0]
        S.np_tot[0] = 1
        X = oracle.MoverExtra(16, gam_sec=gam, igrid_sec=1, THm=2.0, zg_sec=zg, iseed=4242)
        pm, pl = _mover(st, S, 2, X)
        assert S.np_tot[1] == 1 and S.np_tot[0] == 1 + nexp
        # the draws in the reference's order: the count, then per electron vz, vx/vy
        seed = 4242

        def draw():
            nonlocal seed
            r, seed = oracle.ran2(seed)
            return r

        r = draw()
        assert (r <= gam - int(gam)) == (nexp > int(gam))
        vt = np.sqrt(2.0 * QE * 2.0 / abs(st.mass[0]))
        e4 = 0.0
        for k in range(nexp):
            vz = 1.0 * vt * np.sqrt(-np.log(1.0 - draw()))     # -sign(vz_ion) = +1
            ra = draw()
            rb = draw()
            vp, th = vt * np.sqrt(-np.log(1.0 - ra)), 2.0 * np.pi * rb
            want = [0.5 * L[0], 0.5 * L[1], zg[0], vp * np.cos(th), vp * np.sin(th), vz]
            np.testing.assert_allclose(S.vxp[0, 1 + k], want, rtol=1e-13, atol=1e-300)
            e4 += 0.5 * st.Nm[0] * st.mass[0] * (want[3] ** 2 + 2 * vz * vz)
        np.testing.assert_allclose(pl[0, 3], e4, rtol=1e-13)
        assert int(X.iseed[0]) == seed
