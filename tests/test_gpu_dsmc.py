"""GPU collisions with charged targets (DSMC, Src/collisions.f90:335-423,
524-531): e-Ar+ elastic collisions where the ion partner is a particle of
the Ar+ species in the electron's cell (the synthetic Coulomb-like table of
the dsmc16 workload), against the CPU oracle on the same seeded particles.

Bars: nu_max equal to the oracle's (1e-12; it uses the dens_red maximum of
the ion density); collision counts over several calls within 3 sigma of the
oracle's; the bookkeeping exact -- every drawn collision happens (no
collision is left over: lost_claims 0), every collision changes its
electron, the ions changed are the collisions less those that hit an ion
already hit in the same call (at most the replays), and no electron finds its
cell and neighbours without ions; the drop-in (Plist from part_sorting_,
np_red from dens_red_) the same; the device step loop of both forms with the
sort of the ions on every collision step; a dense case (dsmc32, about 1e5
collisions per call, several on one ion in many cells) against the oracle.
"""
import math

import numpy as np
import pytest

import oracle
from essaitemporaire_lepic_module_b200 import config, dropin
from tests.conftest import have_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

CALLS = 6


def _oracle_counts(st, S0, calls=CALLS):
    """counts of the e-Ar+ reaction over `calls` oracle calls (each from the
    same particles, the ran2 stream running on)"""
    out, nus = [], None
    seed = S0.iseed.copy()
    for _ in range(calls):
        S = S0.copy()
        S.iseed = seed
        S.Plist = np.zeros((st.ntype, oracle.pl_max_of(st) + 1), dtype=np.int32)
        for p in range(1, st.ntype + 1):
            S.Plist[p - 1] = oracle.part_sorting(st, S, p)
        err = np.zeros(st.ntype, dtype=np.int64)
        nus, cnt, _ = oracle.collisions(st, S, err)
        assert err.sum() == 0
        seed = S.iseed
        out.append(int(cnt[0]))
    return np.array(out), nus


def _within(a, b):
    """two samples of Poisson-like counts: means within 3 sigma"""
    sa = max(a.mean(), 1.0) / len(a)
    sb = max(b.mean(), 1.0) / len(b)
    return abs(a.mean() - b.mean()) <= 3 * math.sqrt(sa + sb)


def _device_calls(st, S0, nmax, precision, calls):
    """`calls` collision calls, each from the oracle's particles on a fresh
    device state (seeds 1000 + call): the e-Ar+ counts, with the bookkeeping
    checked per call; returns (counts, replays, nu_max)"""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    got, rep, nu = [], 0, None
    for call in range(calls):
        sim = Simulation(st, cap=nmax, precision=precision, seed=1000 + call)
        sim.load_from_host(S0.vxp, S0.np_tot, S0.np)
        sim.sort()
        before = [sim.particles_f64(p).t().cpu().numpy() for p in range(st.ntype)]
        sim.it = 11
        sim.collisions()
        torch.cuda.synchronize()
        after = [sim.particles_f64(p).t().cpu().numpy() for p in range(st.ntype)]
        n = int(sim.counts[0])
        got.append(n)
        nu = sim.nu_max[0]
        tg = sim._targets
        assert tg.missed == 0
        assert tg.lost_claims == 0, tg.lost_claims
        e_changed = np.any(after[0][:, 3:6] != before[0][:, 3:6], axis=1).sum()
        i_changed = np.any(after[1][:, 3:6] != before[1][:, 3:6], axis=1).sum()
        assert e_changed == n, (e_changed, n)
        # an ion hit twice in one call changes once; a second hit is always
        # a replay (its first round found the ion taken)
        assert n - tg.replayed <= i_changed <= n, (i_changed, n, tg.replayed)
        rep += tg.replayed
        # positions stay
        np.testing.assert_array_equal(after[1][:, 0:3], before[1][:, 0:3])
    return np.array(got), rep, nu


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_dsmc_counts_and_bookkeeping(precision):
    oracle.set_threads(1)
    st = config.build("dsmc16")
    nmax = int(st.n_particles() * 1.3)
    S0 = oracle.load_part(st, nmax=nmax)
    want, nu_o = _oracle_counts(st, S0)
    got, _, nu = _device_calls(st, S0, nmax, precision, CALLS)
    assert abs(nu - nu_o[0]) <= 1e-12 * nu_o[0]
    assert got.min() > 100
    assert _within(got, want), (got, want)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_dsmc_dense(precision):
    """About 1e5 e-Ar+ collisions per call on 1.3e6 ions (40 per cell): many
    ions are drawn by several electrons of one call, whose collisions then
    run in later rounds against the ion as the earlier collision left it, as
    in the reference's serial loop.  Counts over three calls within 3 sigma
    of the oracle's, nothing left over, replays seen."""
    oracle.set_threads(8)
    st = config.build("dsmc32")
    nmax = int(st.n_particles() * 1.3)
    S0 = oracle.load_part(st, nmax=nmax)
    want, nu_o = _oracle_counts(st, S0, calls=3)
    got, rep, nu = _device_calls(st, S0, nmax, precision, 3)
    assert abs(nu - nu_o[0]) <= 1e-12 * nu_o[0]
    assert want.min() >= 1e5 and got.min() >= 1e5, (got, want)
    assert rep > 1000, rep
    assert _within(got, want), (got, want)


def test_dsmc_dropin():
    oracle.set_threads(1)
    st = config.build("dsmc16")
    T = st.tables
    nmax = int(st.n_particles() * 1.3)
    S0 = oracle.load_part(st, nmax=nmax)
    want, _ = _oracle_counts(st, S0)
    dropin.set_commons(st, ncol=T.sig.shape[0], npt=T.sig_Er.shape[0], p_ncol=T.p_ncol)
    got = []
    for call in range(CALLS):
        S = S0.copy()
        iseed = np.array([777 + 13 * call], dtype=np.int32)
        pls = [dropin.part_sorting(st, S.vxp, S.np_tot, p) for p in range(1, st.ntype + 1)]
        be = S.vxp[0, :S.np_tot[0]].copy()
        bi = S.vxp[1, :S.np_tot[1]].copy()
        dropin.collisions(st, 11 + call, S.vxp, S.np_tot, S.flag_dead, iseed, np_red=S.np, Plist=pls)
        ne = int(np.any(S.vxp[0, :len(be), 3:6] != be[:, 3:6], axis=1).sum())
        ni = int(np.any(S.vxp[1, :len(bi), 3:6] != bi[:, 3:6], axis=1).sum())
        assert 0.9 * ne <= ni <= ne, (ni, ne)   # an ion hit twice changes once
        got.append(ne)
    got = np.array(got)
    assert got.min() > 100
    assert _within(got, want), (got, want)


@pytest.mark.parametrize("name,precision", [("dsmc16", "f64"), ("dsmc16", "mixed"), ("dsmcar16", "mixed")])
def test_dsmc_step_loop(name, precision):
    """21 device steps against 21 oracle steps from the same particles (two
    collision calls; the ions are sorted on every collision step so that their
    cell offsets are current): e-Ar+ collision totals within 3 sigma,
    populations within 1 %."""
    import torch
    from essaitemporaire_lepic_module_b200.sim import Simulation
    oracle.set_threads(4)
    st = config.build(name)
    nmax = int(st.n_particles() * 1.3)
    S0 = oracle.load_part(st, nmax=nmax)
    sim = Simulation(st, cap=nmax, precision=precision, sort_policy="adaptive")
    sim.load_from_host(S0.vxp, S0.np_tot, S0.np)
    S = S0.copy()
    phi = st.geom.phi.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    want = 0
    for it in range(1, 22):
        sim.step()
        Ei, _, mcc = oracle.step(st, S, phi, Ei, it)
        if mcc is not None:
            want += int(mcc[1][0])
    torch.cuda.synchronize()
    got = int(sim.counts[0])
    assert want > 200
    assert abs(got - want) <= 3 * math.sqrt(want + got), (got, want)
    assert sim._targets.missed == 0
    assert sim._targets.lost_claims == 0
    c = sim.counts_host()
    assert np.all(np.abs(c - S.np_tot) <= 0.01 * S0.np_tot), (c, S.np_tot)
