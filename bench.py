#!/usr/bin/env python
"""Benchmark of the PIC-MCC timestep hot path on B200.

Metric: particle-steps/s (all species, all ranks) of the full timestep of
Src/main.f90:853-1277 -- rho, multigrid Poisson, E, sort (every nsort), MCC
(every ns_coll), push + loss + compaction, deposition -- on the 128^3
workload with 2 x 1.34e8 particles, Bz = 0.01 T and Ar MCC.  Inputs are
synthetic (seeded Philox loader on the device, analytic cross sections).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value:  device-resident steps, CUDA events around exactly K steps, max
        over ranks.  Particle arrays (2 x 6.4 GB FP64 SoA plus sort buffers)
        are far larger than L2, so no flush is needed.
e2e:    the same steps through the public host API: every step copies the
        host-owned wall potentials (pinned) in and the potential grid and
        particle counts out.
roofline: the dominant kernel's algorithmic bytes (96 B per FP64
        particle-step: read and write x,y,z,vx,vy,vz) over its average
        event-timed duration, against the measured HBM copy bandwidth.
cpu_baseline: the FP64 CPU oracle (the reference restated in C++) on the
        host cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s (PIC-MCC timestep, FP64 form)"
UNIT = "particle-steps/s"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(workload, steps=10, ppc=4):
    """The CPU FP64 oracle on a bounded sample: the workload's grid with
    `ppc` particles per cell and species, steps it=2..steps+1 (one sort and
    one MCC call per 10 steps, the reference cadence)."""
    import oracle
    from essaitemporaire_lepic_module_b200 import config
    wl = config.workload(workload)
    wl.ppc = ppc
    st = config.build(wl)
    threads = oracle.set_threads(os.cpu_count() or 1)
    S = oracle.load_part(st, nmax=int(st.n_particles() * 1.3) + 1024)
    phi = st.geom.phi.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    ntot = 0
    t0 = time.perf_counter()
    for it in range(2, steps + 2):
        ntot += int(S.np_tot.sum())
        Ei, _, _ = oracle.step(st, S, phi, Ei, it)
    dt = time.perf_counter() - t0
    return {"value": ntot / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{workload} grid {st.n}, {ppc} ppc/species ({st.n_particles()} per species), "
                      f"{steps} steps it=2..{steps + 1} incl. 1 sort + 1 MCC call, {dt:.1f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cb = cpu_baseline(args.workload, steps=args.cpu_steps, ppc=args.cpu_ppc)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.cpu_steps, "warmup": 0,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "sample": cb["sample"]},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from essaitemporaire_lepic_module_b200 import _lib, config
    from essaitemporaire_lepic_module_b200.sim import Simulation

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    st = config.build(args.workload)
    sim = Simulation(st, seed=20240601 + 7919 * rank, nsort=args.nsort, fused=not args.unfused)
    sim.load_uniform()
    torch.cuda.synchronize()
    n_start = int(sim.counts_host().sum())
    for _ in range(args.warmup):
        sim.step()
    torch.cuda.synchronize()

    # ------------------------------------------------------------ value
    _lib.timing(enable=True)
    _lib.timing(reset=True)
    clk = ClockSampler(local)
    clk.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nps = 0
    vcycles = []
    e0.record()
    for _ in range(args.steps):
        nps += int(sum(s.n() for s in sim.sp))
        sim.step()
        vcycles.append(sim.mg_last[0] - 1)
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        c = torch.tensor([nps], device="cuda", dtype=torch.float64)
        dist.all_reduce(c)
        nps = float(c.item())
    timers = _lib.timing()
    _lib.timing(enable=False)
    value = nps / (ms / 1e3)

    # --------------------------------------------------------- roofline
    peak, peak_kind = measured_peaks()
    kname = "push_deposit_f64" if "push_deposit_f64" in timers else "push_f64"
    push = timers.get(kname, (0.0, 0))
    top = max(timers.items(), key=lambda kv: kv[1][0]) if timers else ("push_f64", push)
    per_launch_particles = nps / max(push[1], 1)
    bytes_per_launch = 96.0 * per_launch_particles
    achieved = bytes_per_launch / (push[0] / max(push[1], 1) / 1e3) / 1e9 if push[1] else None

    # ------------------------------------------------------------- e2e
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    phi_host = torch.empty(tuple(st.geom.phi.shape), dtype=torch.float64).pin_memory()
    phi_host.copy_(torch.as_tensor(st.geom.phi))
    wall = torch.as_tensor(st.geom.bcnd >= 1, device=sim.dev)
    out_phi = torch.empty_like(phi_host).pin_memory()
    out_cnt = torch.empty(len(sim.sp), dtype=torch.int32).pin_memory()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        dphi = phi_host.to(sim.dev, non_blocking=True)
        sim.phi[wall] = dphi[wall]
        sim.step()
        out_phi.copy_(sim.phi, non_blocking=True)
        out_cnt.copy_(torch.cat([s.count for s in sim.sp]), non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    n_now = int(out_cnt.sum())
    e2e_val = n_now * e2e_steps / e2e_s * (world if world > 1 else 1)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": list(st.n), "species": st.ntype,
                   "particles_per_species": st.n_particles(), "Bz_T": st.Bconst[2],
                   "mcc": "Ar 1 Pa 300 K, every 10 steps", "sort_every": sim.nsort,
                   "l2": "inputs larger than L2 (12.9 GB particle state)",
                   "particles_at_start": n_start},
        "mg_vcycles_per_solve": float(np.mean(vcycles)) if vcycles else None,
        "gpu_launches": int(sum(v[1] for v in timers.values())),
        "kernel_ms": {k: round(v[0], 3) for k, v in sorted(timers.items())},
        "kernel_launches": {k: v[1] for k, v in sorted(timers.items())},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": None,
                     "algorithmic_bytes_per_launch": bytes_per_launch,
                     "top_kernel": top[0]},
        "e2e": {"value": e2e_val, "unit": UNIT, "steps": e2e_steps,
                "h2d_bytes_per_step": int(phi_host.numel() * 8),
                "d2h_bytes_per_step": int(out_phi.numel() * 8 + out_cnt.numel() * 4)},
        "clocks": clocks,
    }
    if args.cpu_baseline and world == 1:
        try:
            line["cpu_baseline"] = cpu_baseline(args.workload, steps=args.cpu_steps, ppc=args.cpu_ppc)
        except Exception as ex:  # reported, never silently dropped
            line["cpu_baseline"] = {"error": repr(ex)}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mcc128")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--cpu-ppc", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--nsort", type=int, default=None, help="sort cadence (default: the reference's 10)")
    ap.add_argument("--unfused", action="store_true", help="separate push/compact/deposit kernels")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
