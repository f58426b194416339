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

