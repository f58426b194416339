"""Multi-rank host logic on CPU (gloo, world size 2): the per-step density
all-reduce of the sharded step (each rank holds its own particles over the
full grid, as the reference's MPI ranks do with Src/calc_rho.f90:102) and the
per-rank macroparticle weight."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    try:
        from datetime import timedelta
        from essaitemporaire_lepic_module_b200.sim import allreduce_density, rank_weight
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=timedelta(seconds=60))
        # (ntype, nodes) density grids: rank r deposits r + 1 on species 0
        # and 10 (r + 1) on species 1, on alternate nodes
        g = torch.zeros((2, 5, 6, 7), dtype=torch.float64)
        g[0, :, :, rank::2] = rank + 1.0
        g[1] = 10.0 * (rank + 1)
        allreduce_density(g)
        want0 = torch.zeros((5, 6, 7), dtype=torch.float64)
        for r in range(world):
            want0[:, :, r::2] += r + 1.0
        ok = bool(torch.equal(g[0], want0)) and bool(torch.all(g[1] == 10.0 * sum(range(1, world + 1))))
        # every rank ends with the same grids
        h = g.clone()
        dist.broadcast(h, src=0)
        ok = ok and bool(torch.equal(h, g))
        ok = ok and rank_weight(4.0, world) == 4.0 / world
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ok, ""))
    except Exception as ex:  # reported to the parent
        q.put((rank, False, repr(ex)))


def test_density_allreduce_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    for rank, ok, err in res:
        assert ok, (rank, err)


def test_rank_weight_keeps_density():
    from essaitemporaire_lepic_module_b200.sim import rank_weight
    Nm = 1.25e3
    for world in (1, 2, 4, 8):
        # world ranks of n particles at weight Nm / world deposit what n particles at Nm do
        assert np.isclose(world * rank_weight(Nm, world), Nm, rtol=0, atol=1e-12 * Nm)


def _sharded_worker(rank, world, port, q, steps):
    """Rank `rank` of the sharded step: its own population (seeded by rank)
    at weight Nm / world over the full grid; the density grids all-reduced
    before every field solve.  Rank 0 also runs one rank holding every
    population and compares."""
    try:
        from datetime import timedelta

        import oracle
        from essaitemporaire_lepic_module_b200 import config
        from essaitemporaire_lepic_module_b200.sim import allreduce_density, rank_weight
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=timedelta(seconds=120))
        oracle.build()
        oracle.set_threads(1)
        st = config.build("box16")
        st.Nm[:st.ntype] = rank_weight(st.Nm[:st.ntype], world)
        nmax = st.n_particles() + 4096

        def population(r):
            return oracle.load_part(st, nmax=nmax, seed=123456 + 7919 * r)

        def reduce_np(S):
            t = torch.from_numpy(S.np)
            allreduce_density(t)
            S.np[...] = t.numpy()

        S = population(rank)
        reduce_np(S)
        phi = st.geom.phi.copy()
        Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
        for it in range(1, steps + 1):
            Ei, _, _ = oracle.step(st, S, phi, Ei, it)     # ends with this rank's deposition
            reduce_np(S)
        # gather every rank's particles and potential on rank 0
        counts = [torch.zeros(st.ntype, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(counts, torch.from_numpy(S.np_tot.astype(np.int64)))
        mine = torch.from_numpy(np.ascontiguousarray(S.vxp))
        parts = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(parts, mine)
        phis = [torch.zeros(phi.shape, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(phis, torch.from_numpy(phi))
        ok, msg = True, ""
        if rank == 0:
            # every rank solved the same field
            for r in range(1, world):
                ok = ok and bool(torch.equal(phis[r], phis[0]))
            # one rank holding every population at the same weight
            A = oracle.State(st, world * nmax)
            for r in range(world):
                P = population(r)
                for p in range(st.ntype):
                    n0, n = A.np_tot[p], P.np_tot[p]
                    A.vxp[p, n0:n0 + n] = P.vxp[p, :n]
                    A.np_tot[p] += n
                A.np += P.np
            phi1 = st.geom.phi.copy()
            Ei1 = np.zeros_like(Ei)
            for it in range(1, steps + 1):
                Ei1, _, _ = oracle.step(st, A, phi1, Ei1, it)
            dphi = np.abs(phi1 - phi).max() / np.abs(phi1).max()
            drho = np.abs(A.np - S.np).max() / np.abs(A.np).max()
            ok = ok and dphi <= 1e-12 and drho <= 1e-12
            for p in range(st.ntype):
                g = np.concatenate([parts[r].numpy()[p, :int(counts[r][p])] for r in range(world)])
                o = A.vxp[p, :A.np_tot[p]]
                ok = ok and g.shape == o.shape
                if ok:
                    kg = np.lexsort((g[:, 2], g[:, 1], g[:, 0]))
                    ko = np.lexsort((o[:, 2], o[:, 1], o[:, 0]))
                    err = (np.abs(g[kg] - o[ko]) / np.abs(o).max(axis=0)).max()
                    ok = ok and err <= 1e-10
                    msg += f"species {p}: {len(o)} particles, err {err:.1e}; "
            msg += f"phi {dphi:.1e} rho {drho:.1e}"
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ok, msg))
    except Exception as ex:  # reported to the parent
        import traceback
        q.put((rank, False, traceback.format_exc()))


def test_sharded_step_matches_one_rank():
    """The sharded timestep of the multi-GPU design, run on two CPU ranks
    through the oracle's step (Src/main.f90:853-1277): each rank advances its
    own population at weight Nm/2 and the density grids are all-reduced
    after every deposition (the MPI_ALLREDUCE of Src/calc_rho.f90:102).
    After 12 steps (a sort included) both ranks hold the same potential, and
    it equals (1e-12) the potential of one rank holding both populations at
    the same weight; the density grids agree to 1e-12, every particle to
    1e-10 (only the summation order of the density differs)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_sharded_worker, args=(r, world, port, q, 12)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    for rank, ok, msg in res:
        assert ok, (rank, msg)
