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
