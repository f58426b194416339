"""The collisions with the reference's hydrogen source chemistry
(input_dir/hydrogen.dat: 5 charged species, 2 neutrals, 60 reactions of the
five types, charged targets among them; the parsed tables come from the
fixture tests/golden/hydrogen_chem.npz) on the GPU against the CPU oracle,
from the same seeded particles.

Four reactions of the file have a table that is non-zero below their
threshold (e.g. [e]+[H2]->[e]+[H]+[H], sigma > 0 from 8.07 eV, Eth 10.5 eV);
when one of them is drawn below its threshold the reference stops the run
(negative centre-of-mass energy, Src/collisions.f90:769-775), as the oracle
and the GPU do (LEPIC_ERR_NEG_ENERGY).  The test keeps the other 56.

Bars (statistical: Philox per particle against the serial ran2): over six
calls, the collisions of every incident species and of every reaction the
oracle sees at least 30 times within 3 sigma; the incident particles that
find no charged target (no H- is loaded) within 3 sigma of the oracle's;
nu_max equal (1e-12); no drawn collision left undone (lost_claims 0).
"""
import dataclasses
import math
import os

import numpy as np
import pytest

import oracle
from essaitemporaire_lepic_module_b200 import config, reactions as rx
from essaitemporaire_lepic_module_b200.constants import KB
from tests.conftest import have_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

CALLS = 6
FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hydrogen_chem.npz")


def hydrogen_setup():
    wl = dataclasses.replace(config.workload("box16"), name="h2_16", gas_pressure=3.0, Te=4.0)
    ngas = wl.gas_pressure / (KB * wl.gas_T)
    chem = rx.chemistry_from_arrays(np.load(FIX), wl.Te, ngas)
    T = rx.ordering(chem)
    keep = [c for c in range(len(chem.labels))
            if not (T.Eth[c] > 0 and (T.sig[c][T.sig_Er < T.Eth[c]] > 0).any())]
    assert len(keep) == 56
    chem = rx.Chemistry(species=chem.species, labels=[chem.labels[c] for c in keep],
                        col_info=chem.col_info[keep], Eth=chem.Eth[keep], tables=[chem.tables[c] for c in keep])
    return config.build(wl, chem=chem)


def _sorted_copy(st, S0):
    S = S0.copy()
    S.Plist = np.zeros((st.ntype, oracle.pl_max_of(st) + 1), dtype=np.int32)
    for p in range(1, st.ntype + 1):
        if S.np_tot[p - 1] > 0:
            S.Plist[p - 1] = oracle.part_sorting(st, S, p)
    return S


def _close(a, b):
    return abs(a - b) <= 3 * math.sqrt(max(a + b, 1.0))


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_hydrogen_chemistry_vs_oracle(precision):
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    oracle.set_threads(4)
    st = hydrogen_setup()
    assert st.ntype == 5 and st.tables.sig.shape[0] == 56
    nmax = int(st.n_particles() * 1.5)
    S0 = oracle.load_part(st, nmax=nmax)
    ncol = st.tables.sig.shape[0]
    want = np.zeros(ncol, dtype=np.int64)
    miss_o = 0
    seed = S0.iseed.copy()
    nu_o = None
    for _ in range(CALLS):
        S = _sorted_copy(st, S0)
        S.iseed = seed
        err = np.zeros(st.ntype, dtype=np.int64)
        nu_o, cnt, _ = oracle.collisions(st, S, err)
        seed = S.iseed
        want += cnt
        miss_o += int(err.sum())
    got = np.zeros(ncol, dtype=np.int64)
    miss_g = 0
    for call in range(CALLS):
        sim = Simulation(st, cap=nmax, precision=precision, seed=500 + call)
        sim.load_from_host(S0.vxp, S0.np_tot, S0.np)
        sim.sort()
        sim.it = 11
        sim.collisions()
        torch.cuda.synchronize()
        got += sim.counts[:ncol]
        miss_g += sim._targets.missed
        assert sim._targets.lost_claims == 0
        np.testing.assert_allclose(sim.nu_max[:st.ntype], nu_o, rtol=1e-12, atol=0)
    ci = st.tables.col_info
    for p in range(1, st.ntype + 1):
        mine = [c for c in range(ncol) if ci[c, 2] == p]
        assert _close(got[mine].sum(), want[mine].sum()), (p, got[mine].sum(), want[mine].sum())
    for c in range(ncol):
        if want[c] >= 30:
            assert _close(got[c], want[c]), (c, st.tables and got[c], want[c])
    assert want.sum() > 500
    assert _close(miss_g, miss_o), (miss_g, miss_o)
