#!/usr/bin/env python
"""Benchmark of the PIC-MCC timestep hot path on B200.

Metric: particle-steps/s (all species, all ranks) of the full timestep of
Src/main.f90:853-1277 -- rho, multigrid Poisson, E, sort (every nsort), MCC
(every ns_coll), push + loss + compaction, deposition -- on the 128^3
workload with 2 x 1.34e8 particles, Bz = 0.01 T and Ar MCC.  Inputs are
synthetic (seeded Philox loader on the device, analytic cross sections).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value:  the mixed form (int32 cell + FP32 particles, FP32 V-cycles in FP64
        refinement): device-resident steps, CUDA events around exactly K
        steps, max over ranks.  The FP64 form is timed the same way first and
        reported under "f64" with the ratio "mixed_over_f64"; phi_err_vs_f64
        compares the last mixed solve with the FP64 multigrid solution of the
        same rhs converged to 1e-12 (phi_err_detail also gives the FP64 form's
        own distance from it at the workload tolerance).
        Particle arrays (>= 7.5 GB) are far larger than L2, so no flush is
        needed.
e2e:    the same steps through the public host API: every step copies the
        host's electrode potentials (pinned) in and the potential grid and
        particle counts out.
roofline: the dominant kernel's algorithmic bytes (mixed: 57 B per
        particle-step = read and write cell + 6 FP32 planes, read the flag;
        FP64: 96 B = read and write x,y,z,vx,vy,vz) over its average
        event-timed duration, against the measured HBM copy bandwidth.
cpu_baseline: the FP64 CPU oracle (the reference restated in C++) on the
        host cores, on a bounded sample of the same workload.
poisson: the Poisson stress configuration (256^3, two electrodes at +-100 V, 64
        Gaussian blobs): cold and warm solve times of the FP64 multigrid and of
        the mixed solve, and phi of the mixed solve against the FP64 one.
large:  the large mixed-precision configuration (192^3 cells, e- + Ar+ at 128
        ppc = 2 x 9.06e8 FP32 particles, the MCC of the 128^3 workload; the
        FP64 form does not fit in HBM): after 3 warm-up steps, 500 steps timed
        with CUDA events as one region (50 electron sorts and 50 MCC calls),
        with its roofline, clocks and phi error against the FP64 multigrid;
        then the differentiable window of the next 32 steps (collisions
        recorded and replayed): the gradient of the potential at the box
        centre after them with respect to the wall potential, B_z and the
        electrons' initial velocities, forward and backward times.
mixed_vs_f64_error: the mixed form against the FP64 form after 10 and 100
        steps from the same particles (64^3 workload, collisions replayed): phi
        (every step), E, per-particle positions and velocities, density and
        energy moments.
adjoint: forward and backward time of the differentiable K-step window on the
        Penning workload (96x96x192, 5.7e7 electrons, K = 64, checkpoints every
        8 steps): gradient of the final mean electron energy with respect to the
        electrode potentials, B_z and the initial velocities.
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

METRIC = "particle-steps/s (PIC-MCC timestep), mixed form vs FP64 form"
UNIT = "particle-steps/s"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons during the timed region:
    NVML read every 20 ms on a thread (read-only queries), nvidia-smi's
    200 ms loop when NVML is unavailable."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index=0):
        self.index = index
        self.rows = []           # (sm_mhz, max_mhz, set of reason names)
        self.proc = None
        self.nvml = None
        self.stop_flag = threading.Event()

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            self.nvml = (pynvml, h, bits)
            self.t = threading.Thread(target=self._poll_nvml, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read_smi, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _poll_nvml(self):
        pynvml, h, bits = self.nvml
        while not self.stop_flag.is_set():
            try:
                sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
                r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), {nm for nm, b in bits.items() if r & b}))
            except Exception:
                pass
            self.stop_flag.wait(0.02)

    def _read_smi(self):
        for line in self.proc.stdout:
            r = [v.strip() for v in line.split(",")]
            if len(r) < 9 or not r[1].replace(".", "").isdigit():
                continue
            self.rows.append((float(r[1]), float(r[2]) if r[2].replace(".", "").isdigit() else 0.0,
                              {nm for nm, v in zip(self.NAMES, r[5:9]) if v.lower().startswith("active")}))

    def stop(self):
        if self.nvml is None and self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.stop_flag.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        self.t.join(timeout=2)
        rows = list(self.rows)
        sm = [r[0] for r in rows]
        reasons = set()
        for r in rows:
            reasons |= r[2]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(r[1] for r in rows) if rows else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml 20 ms" if self.nvml is not None else "nvidia-smi 200 ms"}


def cpu_baseline(workload, steps=10, ppc=4, warmup=0):
    """The CPU FP64 oracle on a bounded sample: the workload's grid with
    `ppc` particles per cell and species, `warmup` untimed steps, then
    `steps` timed ones (one sort and one MCC call per 10 steps, the
    reference cadence)."""
    import oracle
    from essaitemporaire_lepic_module_b200 import config
    wl = config.workload(workload)
    wl.ppc = ppc
    st = config.build(wl)
    threads = oracle.set_threads(os.cpu_count() or 1)
    S = oracle.load_part(st, nmax=int(st.n_particles() * 1.3) + 1024)
    phi = st.geom.phi.copy()
    Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    for it in range(2, warmup + 2):
        Ei, _, _ = oracle.step(st, S, phi, Ei, it)
    first = warmup + 2
    ntot = 0
    t0 = time.perf_counter()
    for it in range(first, first + steps):
        ntot += int(S.np_tot.sum())
        Ei, _, _ = oracle.step(st, S, phi, Ei, it)
    dt = time.perf_counter() - t0
    nsort = sum(1 for it in range(first, first + steps) if it % 10 == 1)
    ncoll = nsort if st.tables is not None else 0
    return {"value": ntot / dt, "unit": UNIT, "cores": threads, "kind": "port", "ms_per_step": 1e3 * dt / steps,
            "sample": f"{workload} grid {st.n}, {ppc} ppc/species ({st.n_particles()} per species), "
                      f"{steps} timed steps it={first}..{first + steps - 1} after {warmup} warm-up, incl. {nsort} "
                      f"sort(s) + {ncoll} MCC call(s), {dt:.1f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # the driver's --steps / --warmup, each step a bounded sample (cpu_ppc particles per cell)
    cb = cpu_baseline(args.workload, steps=args.steps, ppc=args.cpu_ppc, warmup=args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cb["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "sample": cb["sample"]},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _timed_steps(sim, steps, world, dist, torch):
    """Exactly `steps` steps between CUDA events (device time, max over ranks)."""
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the particles each step pushes (the counts before it), summed on the
    # device: no host read of the counts inside the timed region
    acc = torch.zeros(1, dtype=torch.int64, device="cuda")
    counts = [s.count for s in sim.sp]
    vcycles = []
    c0 = sim._mg_count
    e0.record()
    for _ in range(steps):
        for c in counts:
            acc += c
        sim.step()
        if not sim.nonblocking:
            vcycles.append(sim.mg_last[0])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if sim.nonblocking:
        # the solves' refinements, copied out in stream order during the
        # steps; statuses recorded by the last steps' kernels are read here
        vcycles = sim.solve_history(steps) if sim._mg_count - c0 == steps else [sim.mg_last[0]]
        sim.flush_checks()
    nps = int(acc.item())
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        c = torch.tensor([nps], device="cuda", dtype=torch.float64)
        dist.all_reduce(c)
        nps = float(c.item())
    return nps, ms, vcycles


def _e2e(sim, st, steps, world, dist, torch):
    """Steps through the public API with host buffers (Simulation.step_host):
    every step the host's electrode potentials (one per wall label, pinned)
    go in and are applied to the wall nodes, and the potential grid and the
    particle counts come out into pinned host buffers, inside the timed
    region; each step's copy out overlaps the next step, and the region ends
    when the last copy has landed."""
    nl = int(st.geom.ngrid)
    v_host = torch.zeros(nl + 2, dtype=torch.float64).pin_memory()
    for lab in range(1, nl + 1):
        v_host[lab] = float(st.wl.V[lab]) if lab < len(st.wl.V) else 0.0
    phi_host = [torch.empty(tuple(st.geom.phi.shape), dtype=torch.float64).pin_memory() for _ in range(2)]
    cnt_host = torch.zeros((max(steps, 2), len(sim.sp)), dtype=torch.int32).pin_memory()
    # warm-up: the first calls create the device snapshots and the copy stream
    for k in range(2):
        sim.step_host(v_host, phi_host[k], cnt_host[k])
    n0 = int(sim.counts_host().sum())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    done = [None, None]
    for k in range(steps):
        if done[k % 2] is not None:
            done[k % 2].synchronize()  # the host buffer of two steps ago is free again
        done[k % 2] = sim.step_host(v_host, phi_host[k % 2], cnt_host[k])
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    # particles pushed by each step: the count before it
    nps = n0 + int(cnt_host[:steps - 1].sum())
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
        c = torch.tensor([nps], device="cuda", dtype=torch.float64)
        dist.all_reduce(c)
        nps = float(c.item())
    return {"value": nps / e2e_s, "unit": UNIT, "steps": steps,
            "h2d_bytes_per_step": int(v_host.numel() * 8),
            "d2h_bytes_per_step": int(phi_host[0].numel() * 8 + cnt_host.shape[1] * 4)}


# DRAM bytes per particle of each push kernel from an ncu capture of one launch
# on the 96^3 workload (5.7e7 particles per species); the traffic grows in
# proportion to the particles, so a launch's traffic is this times its
# particles
MEASURED_TRAFFIC_PER_PARTICLE = {"push_mixed": 56.7, "deposit_mixed_tiles": 17.5, "push_deposit_f64": 96.6}


def _roofline(timers, kname, bytes_per_particle, nps):
    peak, peak_kind = measured_peaks()
    push = timers.get(kname, (0.0, 0))
    top = max(timers.items(), key=lambda kv: kv[1][0]) if timers else (kname, push)
    per_launch_particles = nps / max(push[1], 1)
    bytes_per_launch = bytes_per_particle * per_launch_particles
    achieved = bytes_per_launch / (push[0] / max(push[1], 1) / 1e3) / 1e9 if push[1] else None
    tpp = MEASURED_TRAFFIC_PER_PARTICLE.get(kname)
    return {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
            "traffic": tpp * per_launch_particles if tpp else None,
            "traffic_source": "ncu DRAM bytes per particle at 96^3 x particles per launch" if tpp else None,
            "algorithmic_bytes_per_launch": bytes_per_launch,
            "algorithmic_bytes_per_particle": bytes_per_particle, "top_kernel": top[0]}


def _run_form(args, st, precision, rank, world, dist, torch, e2e=True):
    from essaitemporaire_lepic_module_b200 import _lib
    from essaitemporaire_lepic_module_b200.sim import Simulation
    cap = int(st.n_particles() * args.cap_factor) + 1024 if args.cap_factor else None
    sim = Simulation(st, cap=cap, seed=20240601 + 7919 * rank, nsort=args.nsort, fused=not args.unfused,
                     precision=precision, comm=True if world > 1 else None, sort_policy=args.sort_policy,
                     ns_coll=args.ns_coll, nonblocking=True)
    sim.load_uniform()
    torch.cuda.synchronize()
    n_start = int(sim.counts_host().sum())
    # the sampler starts before the warm-up so that nvidia-smi's start-up
    # does not stall the timed steps; it samples through them
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clk.start()
    for _ in range(args.warmup):
        sim.step()
    torch.cuda.synchronize()
    _lib.timing(enable=True)
    _lib.timing(reset=True)
    clk.rows.clear()
    nps, ms, iters = _timed_steps(sim, args.steps, world, dist, torch)
    clocks = clk.stop()
    timers = _lib.timing()
    _lib.timing(enable=False)
    out = {"sim": sim, "nps": nps, "ms": ms, "iters": iters, "timers": timers, "clocks": clocks,
           "n_start": n_start, "value": nps / (ms / 1e3)}
    if e2e:
        out["e2e"] = _e2e(sim, st, max(1, min(args.steps, args.e2e_steps)), world, dist, torch)
    return out


def _fp64_solve(sim, st, torch, eps, ncycl):
    """Cold FP64 multigrid solve of sim.rhs (walls at their potentials)."""
    import ctypes as C
    from essaitemporaire_lepic_module_b200._lib import lib
    phi = torch.as_tensor(st.geom.phi, device=sim.dev).clone()
    k, kt, res = C.c_int(0), C.c_double(0), C.c_double(0)
    wl = st.wl
    rc = lib().lepic_dev_pdesolver(C.byref(sim.grid), C.c_void_p(phi.data_ptr()), C.c_void_p(sim.rhs.data_ptr()),
                                   ncycl, eps, wl.omega, st.ng, C.byref(sim.P), C.byref(k), C.byref(kt),
                                   C.byref(res), sim._s())
    torch.cuda.synchronize()
    return phi, rc, res.value


def _phi_err(sim, st, torch):
    """phi of the last mixed step (FP32 V-cycles in FP64 refinement, warm
    start, workload tolerance) against the FP64 multigrid solution of the same
    right-hand side converged to 1e-12; next to it the FP64 form's own
    distance from that solution at the workload tolerance.  max |dphi| /
    max |phi|."""
    tight, _, res = _fp64_solve(sim, st, torch, 1e-12, 400)
    at_tol, _, _ = _fp64_solve(sim, st, torch, st.wl.eps, st.wl.ncycl)
    scale = float(tight.abs().max())
    return {"mixed": float((sim.phi - tight).abs().max()) / scale,
            "f64_at_tolerance": float((at_tol - tight).abs().max()) / scale,
            "reference_residual": res}


def run_poisson(workload, warm=10):
    """The Poisson stress configuration: a cold solve and `warm` warm solves
    (the source scaled by 1 + 1e-3 k, starting from the previous phi) in the
    FP64 multigrid and in the mixed solve (FP32 V-cycles in FP64 refinement),
    each to the workload tolerance; phi of the mixed cold solve against the
    FP64 one."""
    import torch
    from essaitemporaire_lepic_module_b200 import config
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build(workload)
    out = {"workload": f"{workload} {list(st.n)} grid, electrodes + {st.wl.blobs} Gaussian blobs, "
                       f"tolerance {st.wl.eps:g}"}
    rhs0 = torch.as_tensor(st.rhs_blobs, device="cuda")
    phis = {}
    for form in ("f64", "mixed"):
        sim = Simulation(st, cap=1024, precision=form)
        sim.phi.copy_(torch.as_tensor(st.geom.phi, device="cuda"))
        sim.rhs.copy_(rhs0)
        sim.pdesolver()  # warm-up (allocations), then the timed cold solve
        sim.phi.copy_(torch.as_tensor(st.geom.phi, device="cuda"))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        it_cold = sim.pdesolver()[0]
        e1.record()
        torch.cuda.synchronize()
        cold_ms = e0.elapsed_time(e1)
        phis[form] = sim.phi.clone()
        its = []
        e0.record()
        for k in range(1, warm + 1):
            sim.rhs.copy_(rhs0 * (1.0 + 1e-3 * k))
            its.append(sim.pdesolver()[0])
        e1.record()
        torch.cuda.synchronize()
        out[form] = {"cold_ms": cold_ms, "cold_cycles": it_cold, "warm_ms": e0.elapsed_time(e1) / warm,
                     "warm_cycles": float(np.mean(its))}
        del sim
        torch.cuda.empty_cache()
    ref = phis["f64"]
    out["phi_err_mixed_vs_f64"] = float((phis["mixed"] - ref).abs().max() / ref.abs().max())
    out["cold_speedup"] = out["f64"]["cold_ms"] / out["mixed"]["cold_ms"]
    out["warm_speedup"] = out["f64"]["warm_ms"] / out["mixed"]["warm_ms"]
    return out


def run_adjoint(workload, K, every):
    """Adjoint/forward cost of the differentiable window: the gradient of the
    final mean electron energy with respect to the electrode potentials, B_z
    and the initial velocities (discrete adjoint of the FP64 window, adjoint
    Poisson solves in FP32 V-cycles inside FP64 refinement, checkpoints every
    `every` steps, recomputed), and its distance from the FP64 reference
    gradient (FP64 multigrid adjoint solves)."""
    import torch
    from essaitemporaire_lepic_module_b200 import config
    from essaitemporaire_lepic_module_b200.adjoint import Window, window_objective
    st = config.build(workload)
    win = Window(st, K=K, every=every)
    win.load_uniform(seed=20240611)
    V0 = [float(st.wl.V[lab]) if lab < len(st.wl.V) else 0.0 for lab in range(1, win.nlabel + 1)]
    V = torch.tensor(V0, dtype=torch.float64, requires_grad=True)
    Bz = torch.tensor(float(st.Bconst[2]), dtype=torch.float64, requires_grad=True)
    v0 = win.x0[3:6].clone().requires_grad_(True)
    from essaitemporaire_lepic_module_b200 import _lib
    win.forward(V0, float(Bz.detach()))  # warm-up (allocations)
    J = window_objective(win, V, Bz, v0)
    _lib.timing(enable=True)
    _lib.timing(reset=True)
    J.backward()
    timers = _lib.timing()
    _lib.timing(enable=False)
    t = dict(win.timing)
    # the FP64 reference gradient: the same window with FP64 multigrid adjoint solves
    win.adjoint_solver = "f64"
    win.forward(V0, float(Bz.detach()))
    rV, rB, rv = win.backward()
    tf = dict(win.timing)
    win.adjoint_solver = "mixed"
    gV = np.array([float(x) for x in V.grad])
    ref_err = {"dJ_dV": float(np.abs(gV - rV).max() / max(np.abs(rV).max(), 1e-300)),
               "dJ_dBz": float(abs(float(Bz.grad) - rB) / max(abs(rB), 1e-300)),
               "dJ_dv0": float((v0.grad - rv).abs().max() / max(float(rv.abs().max()), 1e-300))}
    out = {"workload": f"{workload} {list(st.n)} cells, {win.n} particles of species 1, K={K}, "
                       f"checkpoint every {every}, FP64 forward, adjoint Poisson solves FP32 V-cycles in "
                       f"FP64 refinement",
           "grad_rel_err_vs_fp64_reference": ref_err,
           "fp64_adjoint": {"forward_ms": tf["forward_ms"], "backward_ms": tf["backward_ms"],
                            "backward_over_forward": tf["backward_ms"] / tf["forward_ms"]},
           "observable": "mean kinetic energy (eV) after K steps",
           "J": float(J), "dJ_dV_by_label": [float(x) for x in V.grad], "dJ_dBz": float(Bz.grad),
           "dJ_dv0_norm": float(v0.grad.norm()),
           "forward_ms": t["forward_ms"], "backward_ms": t["backward_ms"],
           "backward_over_forward": t["backward_ms"] / t["forward_ms"],
           "backward_kernel_ms": {k: round(v[0], 3) for k, v in sorted(timers.items())}}
    del win, v0
    torch.cuda.empty_cache()
    return out


def run_large(args):
    """The large mixed-precision configuration: `--large-steps` steps of the
    mixed form timed as one region after 3 warm-up steps."""
    import torch
    from essaitemporaire_lepic_module_b200 import config
    st = config.build(args.large_workload)
    a = argparse.Namespace(**vars(args))
    a.warmup, a.steps = 3, args.large_steps
    R = _run_form(a, st, "mixed", 0, 1, None, torch, e2e=False)
    perr = _phi_err(R["sim"], st, torch)
    timers = R["timers"]
    out = {"workload": f"{args.large_workload} {list(st.n)} cells, {st.ntype} species x {st.n_particles()} "
                       f"FP32 particles, MCC every {st.wl.ns_coll} steps, 3 warm-up + {a.steps} timed steps",
           "value": R["value"], "unit": UNIT, "steps": a.steps, "ms_per_step": R["ms"] / a.steps,
           "particles_at_start": R["n_start"],
           "particles_at_end": int(R["sim"].counts_host().sum()),
           "phi_err_vs_f64": perr["mixed"], "phi_err_detail": perr,
           "poisson_iters_per_solve": float(np.mean(R["iters"])) if R["iters"] else None,
           "roofline": _roofline(timers, "push_mixed", 57.0, R["nps"]),
           "roofline_deposit": _roofline(timers, "deposit_mixed_tiles", 17.0, R["nps"]),
           "kernel_ms": {k: round(v[0], 3) for k, v in sorted(timers.items())},
           "kernel_launches": {k: v[1] for k, v in sorted(timers.items())},
           "clocks": R["clocks"]}
    if args.large_adjoint:
        out["adjoint"] = run_window_adjoint(R["sim"], st, K=32, observable="probe",
                                            production_ms_per_step=R["ms"] / a.steps)
    del R
    torch.cuda.empty_cache()
    return out


def run_window_adjoint(sim, st, K, observable, production_ms_per_step):
    """The differentiable window of the collisional step over the next K steps
    of `sim` (mixed form, in place): the first forward records the collisions,
    the backward replays them; gradient of the observable with respect to the
    wall potentials, B_z and the electrons' initial velocities."""
    import torch
    from essaitemporaire_lepic_module_b200 import _lib
    from essaitemporaire_lepic_module_b200.adjoint import CollisionWindow
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    win = CollisionWindow(sim, K=K, sort=True)     # the particles in cell order for the tiled scatters
    torch.cuda.synchronize()
    setup_ms = 1e3 * (time.perf_counter() - t0)
    V = [float(st.wl.V[lab]) if lab < len(st.wl.V) else 0.0 for lab in range(1, win.nlabel + 1)]
    Bz = float(st.Bconst[2])
    _lib.timing(enable=True)
    _lib.timing(reset=True)
    J = win.forward(V, Bz, observable=observable)
    fwd = _lib.timing()
    _lib.timing(reset=True)
    gV, gB, gv = win.backward()
    bwd = _lib.timing()
    _lib.timing(enable=False)
    t = dict(win.timing)
    events = sum(b - a for a, b in win.ev_range.values())
    out = {"window": f"{K} steps after the timed run, {win.ntype} species, {sum(win.count0)} particles (FP32, "
                     f"slots kept), MCC every {win.ns_coll} steps with {events} collisions recorded and replayed, "
                     f"no particle checkpoints (pushes and collisions undone in the backward pass)",
           "observable": {"probe": "phi at the box centre after the window (V)",
                          "energy": "mean electron kinetic energy after the window (eV)",
                          "flux": "kinetic energy carried to the walls in the window (J)"}[observable],
           "J": J, "dJ_dV_by_label": [float(x) for x in gV], "dJ_dBz": gB, "dJ_dv0_norm": float(gv.norm()),
           "setup_ms": setup_ms, "setup": "one sort of every species by cell, then the window's stores",
           "forward_ms": t["forward_ms"], "backward_ms": t["backward_ms"],
           "backward_over_forward": t["backward_ms"] / t["forward_ms"],
           "production_forward_ms": production_ms_per_step * K,
           "backward_over_production_forward": t["backward_ms"] / (production_ms_per_step * K),
           "forward_kernel_ms": {k: round(v[0], 3) for k, v in sorted(fwd.items())},
           "backward_kernel_ms": {k: round(v[0], 3) for k, v in sorted(bwd.items())}}
    del win
    torch.cuda.empty_cache()
    return out


def run_precision(workload, steps=(10, 100)):
    """The mixed form against the FP64 form after N steps from the same
    particles: both run the collisional window (particles keep their slots, so
    each particle is compared with itself), the mixed one recording its
    collisions and the FP64 one replaying them; the errors of phi (every step),
    E, positions, velocities and the species' density and energy moments."""
    import torch
    from essaitemporaire_lepic_module_b200 import config
    from essaitemporaire_lepic_module_b200.adjoint import CollisionWindow
    from essaitemporaire_lepic_module_b200.constants import QE
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build(workload)
    sim = Simulation(st, precision="mixed", seed=20240612)
    sim.load_uniform()
    for _ in range(3):
        sim.step()
    torch.cuda.synchronize()
    V = [float(st.wl.V[lab]) if lab < len(st.wl.V) else 0.0 for lab in range(1, st.geom.ngrid + 1)]
    Bz = float(st.Bconst[2])
    out = {"workload": f"{workload} {list(st.n)} cells, {st.ntype} species, {sum(s.n() for s in sim.sp)} particles, "
                       f"Bz {Bz} T, MCC every {st.wl.ns_coll} steps (the mixed run's collisions replayed by the "
                       f"FP64 run)"}
    h = st.h
    for K in steps:
        w64 = CollisionWindow(sim, K=K, fp64=True)
        w32 = CollisionWindow(sim, K=K, keep_initial=True)
        w32.forward(V, Bz)
        w64.use_log_of(w32)
        w64.forward(V, Bz)
        dphi = [float((w32.phis[n] - w64.phis[n]).abs().max() / w64.phis[n].abs().max()) for n in range(K)]
        Es = []
        for w in (w32, w64):
            sim.phi.copy_(w.phis[K - 1])
            sim.efield()
            Es.append(sim.Ei.clone())
        res = {"phi_rel_err_last_step": dphi[-1], "phi_rel_err_max_over_steps": max(dphi),
               "E_rel_err_last_step": float((Es[0] - Es[1]).abs().max() / Es[1].abs().max()),
               "collisions_replayed": sum(b - a for a, b in w32.ev_range.values())}
        for p in range(st.ntype):
            a, b = w32.stores[p], w64.stores[p]
            n = int(b["count"].item())
            both = ((a["bl"][:n] >> 16) == 0x7fff) & ((b["bl"][:n] >> 16) == 0x7fff)
            xa = torch.stack([((a["cell"][:n] >> (10 * k)) & 1023).double() + a["p"][k, :n].double()
                              for k in range(3)])
            xb = torch.stack([((b["cell"][:n] >> (10 * k)) & 1023).double() + b["p"][k, :n] for k in range(3)])
            dx = (xa - xb)[:, both].abs()
            va, vb = a["p"][3:6, :n].double(), b["p"][3:6, :n]
            vmax = float(vb.abs().max())
            m = abs(st.mass[p])
            ke_a = float((0.5 * m * (va[:, both] ** 2).sum(dim=0)).mean() / QE)
            ke_b = float((0.5 * m * (vb[:, both] ** 2).sum(dim=0)).mean() / QE)
            mom_a = [float((xa[k, both] * h[k]).mean()) for k in range(3)]
            mom_b = [float((xb[k, both] * h[k]).mean()) for k in range(3)]
            res[st.names[p]] = {
                "particles_compared": int(both.sum()), "lost_in_one_form_only": int((((a["bl"][:n] >> 16) == 0x7fff)
                                                                                    != ((b["bl"][:n] >> 16) == 0x7fff)).sum()),
                "position_err_max_cells": float(dx.max()), "position_err_rms_cells": float((dx ** 2).mean().sqrt()),
                "velocity_rel_err_max": float((va - vb)[:, both].abs().max()) / vmax,
                "energy_moment_rel_err": abs(ke_a - ke_b) / ke_b,
                "density_moment_err_m": max(abs(x - y) for x, y in zip(mom_a, mom_b))}
        out[f"after_{K}_steps"] = res
        for d, (c0, p0, n0) in zip(w32.stores, w32.initial):
            d["cell"].copy_(c0)
            d["p"].copy_(p0)
            d["count"].copy_(n0)
        del w32, w64
        torch.cuda.empty_cache()
    del sim
    torch.cuda.empty_cache()
    return out


def run_dropin(workload, steps=4, warm=1):
    """The reference-facing path: Src/main.f90's timestep as calls to the
    Fortran-signature entry points over host arrays in the reference layouts
    (FP64), once with per-call copies (a Fortran build that only relinks) and
    once with device-resident mirrors (lepic_gpu_set_residency).  Wall-clock
    particle-steps/s with every host<->device copy inside the timed region;
    the resident run creates its mirrors in the warm-up step and ends the
    timed steps with lepic_gpu_sync_to_host, so the host arrays are current
    at both ends.  Initial particles come from the GPU loader."""
    import torch
    from essaitemporaire_lepic_module_b200 import config, dropin
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build(workload)
    nmax = int(st.n_particles() * 1.25)
    sim = Simulation(st, cap=nmax, precision="f64")
    sim.load_uniform()
    vxp0 = np.zeros((st.ntype, nmax, 6))
    np_tot0 = np.zeros(st.ntype, dtype=np.int32)
    for p in range(st.ntype):
        v = sim.sp[p].to_vxp()
        vxp0[p, :len(v)] = v
        np_tot0[p] = len(v)
    np0 = np.ascontiguousarray(sim.np.cpu().numpy())
    del sim
    torch.cuda.empty_cache()
    out = {"workload": f"{workload} {list(st.n)} grid, {int(np_tot0.sum())} particles in host arrays "
                       f"vxp(6, nmax, {st.ntype}), FP64, MCC every {st.wl.ns_coll} steps",
           "timing": "wall clock over the drop-in calls, host<->device copies included"}
    for mode in ("copy", "resident"):
        vxp, np_tot = vxp0.copy(), np_tot0.copy()
        fd = np.zeros((st.ntype, nmax), dtype=np.int8)
        npg = np0.copy()
        ml = dropin.MainLoop(st, vxp, np_tot, fd, npg, resident=(mode == "resident"))
        try:
            for _ in range(warm):
                ml.step()
            ml.sync()
            torch.cuda.synchronize()
            a = dropin.mirror_stats()
            t0 = time.perf_counter()
            nps = 0
            for _ in range(steps):
                nps += int(np_tot.sum())
                ml.step()
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            ml.sync()
            torch.cuda.synchronize()
            t = time.perf_counter() - t0
            b = dropin.mirror_stats()
        finally:
            ml.close()
        out[mode] = {"value": nps / t, "unit": UNIT, "ms_per_step": 1e3 * t / steps, "steps": steps,
                     "step_ms_without_final_sync": 1e3 * (t1 - t0) / steps,
                     "final_sync_ms": 1e3 * (t - (t1 - t0)),
                     "h2d_bytes_per_step": int((b[0] - a[0]) / steps),
                     "d2h_bytes_per_step": int((b[1] - a[1]) / steps)}
    out["resident_over_copy"] = out["resident"]["value"] / out["copy"]["value"]
    return out


def run_profile_step(args):
    """One step bracketed by cudaProfilerStart/Stop for `ncu --profile-from-start off`
    (the steps before it run unprofiled): step `--profile-step` of the workload in
    the form `--precision` (f64 or mixed)."""
    import torch
    from essaitemporaire_lepic_module_b200 import config
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build(args.workload)
    form = "mixed" if args.precision == "both" else args.precision
    sim = Simulation(st, precision=form, sort_policy=args.sort_policy)
    sim.load_uniform()
    for _ in range(args.profile_step - 1):
        sim.step()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    sim.step()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profiled_step": sim.it, "form": form, "workload": args.workload,
                      "particles": [s.n() for s in sim.sp]}), flush=True)


def run_profile_poisson(args):
    """One warm solve of the Poisson workload `--profile-poisson` (the source
    scaled by 1.001 after a cold solve) in the form `--precision`, bracketed
    by cudaProfilerStart/Stop for `ncu --profile-from-start off`."""
    import torch
    from essaitemporaire_lepic_module_b200 import config
    from essaitemporaire_lepic_module_b200.sim import Simulation
    st = config.build(args.profile_poisson)
    form = "mixed" if args.precision == "both" else args.precision
    sim = Simulation(st, cap=1024, precision=form)
    sim.phi.copy_(torch.as_tensor(st.geom.phi, device="cuda"))
    rhs0 = torch.as_tensor(st.rhs_blobs, device="cuda")
    sim.rhs.copy_(rhs0)
    cold = sim.pdesolver()
    sim.rhs.copy_(rhs0 * 1.001)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    warm = sim.pdesolver()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profiled": "warm solve", "workload": args.profile_poisson, "form": form,
                      "cold": list(cold), "warm": list(warm)}), flush=True)


def run_profile_window(args):
    """The collisional window of `--profile-window` steps (forward, then the
    backward pass) on the mixed-precision workload `--workload` after
    `--warmup` plain steps, bracketed by cudaProfilerStart/Stop."""
    import torch
    from essaitemporaire_lepic_module_b200 import config
    from essaitemporaire_lepic_module_b200.sim import Simulation
    from essaitemporaire_lepic_module_b200.adjoint import CollisionWindow
    st = config.build(args.workload)
    sim = Simulation(st, precision="mixed", sort_policy=args.sort_policy)
    sim.load_uniform()
    for _ in range(args.warmup):
        sim.step()
    w = CollisionWindow(sim, K=args.profile_window, sort=True)
    V = [float(st.wl.V[lab]) if lab < len(st.wl.V) else 0.0 for lab in range(1, st.geom.ngrid + 1)]
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    J = w.forward(V, float(st.Bconst[2]), observable="probe")
    g = w.backward()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profiled": "collisional window", "workload": args.workload, "K": args.profile_window,
                      "J": J, "dJ_dBz": g[1], "timing_ms": w.timing}), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from essaitemporaire_lepic_module_b200 import config

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    st = config.build(args.workload)
    forms = ["f64", "mixed"] if args.precision == "both" else [args.precision]
    res = {}
    for f in forms:
        res[f] = _run_form(args, st, f, rank, world, dist, torch, e2e=(f == forms[-1]) or args.e2e_all)
        if f != forms[-1]:
            del res[f]["sim"]
            torch.cuda.empty_cache()
    head = forms[-1]
    R = res[head]
    perr = _phi_err(R["sim"], st, torch) if head == "mixed" else None
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    kname = "push_mixed" if head == "mixed" else (
        "push_deposit_f64" if "push_deposit_f64" in R["timers"] else "push_f64")
    bpp = 57.0 if head == "mixed" else 96.0
    timers = R["timers"]
    line = {
        "metric": METRIC, "value": R["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": R["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 particles + f64 grids" if head == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": args.workload, "form": head, "grid": list(st.n), "species": st.ntype,
                   "particles_per_species": st.n_particles(), "Bz_T": st.Bconst[2],
                   "mcc": f"Ar 1 Pa 300 K, every {R['sim'].ns_coll} steps", "sort_every": R["sim"].sort_every,
                   "sort_policy": R["sim"].sort_policy,
                   "l2": "inputs larger than L2 (>= 7.5 GB particle state)",
                   "particles_at_start": R["n_start"]},
        "phi_err_vs_f64": perr["mixed"] if perr else None,
        "phi_err_detail": perr,
        "poisson_iters_per_solve": float(np.mean(R["iters"])) if R["iters"] else None,
        "gpu_launches": int(sum(v[1] for v in timers.values())),
        "kernel_ms": {k: round(v[0], 3) for k, v in sorted(timers.items())},
        "kernel_launches": {k: v[1] for k, v in sorted(timers.items())},
        "roofline": _roofline(timers, kname, bpp, R["nps"]),
        "roofline_deposit": _roofline(timers, "deposit_mixed_tiles", 17.0, R["nps"]) if head == "mixed" else None,
        "e2e": R["e2e"],
        "clocks": R["clocks"],
    }
    if "f64" in res and head != "f64":
        F = res["f64"]
        fk = "push_deposit_f64" if "push_deposit_f64" in F["timers"] else "push_f64"
        line["f64"] = {"value": F["value"], "ms_per_step": F["ms"] / args.steps,
                       "poisson_vcycles_per_solve": float(np.mean(F["iters"])) if F["iters"] else None,
                       "kernel_ms": {k: round(v[0], 3) for k, v in sorted(F["timers"].items())},
                       "roofline": _roofline(F["timers"], fk, 96.0, F["nps"]), "clocks": F["clocks"]}
        if "e2e" in F:
            line["f64"]["e2e"] = F["e2e"]
        line["mixed_over_f64"] = R["value"] / F["value"]
    del res
    R = None
    torch.cuda.empty_cache()
    if args.large and world == 1:
        line["large"] = run_large(args)
    if args.precision_leg and world == 1:
        line["mixed_vs_f64_error"] = run_precision(args.precision_workload)
    if args.poisson:
        line["poisson"] = run_poisson(args.poisson_workload)
    if args.adjoint:
        line["adjoint"] = run_adjoint(args.adjoint_workload, args.adjoint_k, args.adjoint_every)
    if args.dropin:
        line["dropin"] = run_dropin(args.dropin_workload, args.dropin_steps)
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
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--cpu-ppc", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--nsort", type=int, default=None, help="sort cadence (default: the reference's 10)")
    ap.add_argument("--ns-coll", type=int, default=None,
                    help="MCC every N steps (default: the workload's cadence, 10 as in the reference)")
    ap.add_argument("--sort-policy", default="adaptive", choices=["adaptive", "reference"],
                    help="adaptive: species slower than half a cell per nsort steps are sorted 10x less "
                         "often (both forms); reference: every species every nsort steps")
    ap.add_argument("--unfused", action="store_true", help="FP64: separate push/compact/deposit kernels")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "f64"],
                    help="both: time the FP64 form, then the mixed form (the headline)")
    ap.add_argument("--e2e-all", action="store_true", help="also measure e2e for the FP64 form")
    ap.add_argument("--cap-factor", type=float, default=None,
                    help="particle capacity per species / particles loaded (default 1.25)")
    ap.add_argument("--no-large", dest="large", action="store_false",
                    help="skip the large mixed-precision configuration (192^3, 2 x 9.06e8 particles)")
    ap.add_argument("--large-workload", default="mcc192")
    ap.add_argument("--large-steps", type=int, default=500)
    ap.add_argument("--no-large-adjoint", dest="large_adjoint", action="store_false",
                    help="skip the differentiable window after the large run")
    ap.add_argument("--no-precision", dest="precision_leg", action="store_false",
                    help="skip the mixed-vs-FP64 error after 10 and 100 steps")
    ap.add_argument("--precision-workload", default="mcc64")
    ap.add_argument("--no-poisson", dest="poisson", action="store_false",
                    help="skip the Poisson stress measurement")
    ap.add_argument("--poisson-workload", default="poisson256")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false",
                    help="skip the adjoint window measurement")
    ap.add_argument("--adjoint-workload", default="penning")
    ap.add_argument("--adjoint-k", type=int, default=64)
    ap.add_argument("--adjoint-every", type=int, default=8)
    ap.add_argument("--no-dropin", dest="dropin", action="store_false",
                    help="skip the drop-in (Fortran-signature) loop, per-call copies vs resident")
    ap.add_argument("--dropin-workload", default="mcc64")
    ap.add_argument("--dropin-steps", type=int, default=10)
    ap.add_argument("--profile-step", type=int, default=0,
                    help="run only up to this step, the last one between cudaProfilerStart/Stop (for ncu)")
    ap.add_argument("--profile-poisson", default=None,
                    help="run only one warm solve of this Poisson workload between cudaProfilerStart/Stop")
    ap.add_argument("--profile-window", type=int, default=0,
                    help="run only a collisional window of this many steps (forward + backward) on --workload "
                         "after --warmup steps, between cudaProfilerStart/Stop")
    args = ap.parse_args()
    if args.profile_poisson:
        run_profile_poisson(args)
    elif args.profile_window > 0:
        run_profile_window(args)
    elif args.profile_step > 0:
        run_profile_step(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
