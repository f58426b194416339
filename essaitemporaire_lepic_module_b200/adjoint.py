"""Differentiable K-step window of the collisionless FP64 timestep.

No counterpart in the reference: the gradient of a scalar observable of the
particles after K steps (the mean kinetic energy of one species, in eV) with
respect to the electrode potentials (one per wall label), the magnetic field
amplitude B_z and the initial velocities.  The forward window runs the
reference's step (Src/main.f90:853-1277 without sort and collisions:
deposition, rho, multigrid Poisson, E, gather + Boris + leapfrog) with the
window kernels of liblepic_gpu.so, particles keeping their slots (a particle
that reaches a wall stops being pushed and deposited).  The backward pass is
the discrete adjoint of that step (adjoint push, gather and deposition as
each other's transposes, E = -grad phi transposed, and the adjoint Poisson
solve -- by default FP32 V-cycles inside FP64 refinement, to the same
residual test as the FP64 multigrid, or the FP64 multigrid itself), in reverse, from checkpoints of the
particle state taken every `every` steps (sqrt(K) by default) and recomputed
forward one segment at a time.

    win = Window(st, K=64, every=8)
    win.load_uniform(seed)
    J = window_objective(win, V, Bz, v0)     # torch scalar, FP64
    J.backward()                             # dV, dBz and dv0 into .grad
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from ._lib import LepicWinEvent, LepicWinSpecies, check, lib
from .constants import QE
from .sim import Simulation


def _p(t):
    return C.c_void_p(t.data_ptr())


class Window:
    """K-step differentiable window of species `ptype` (1-based) of a
    collisionless workload; the other species are not moved (their charge
    stays where it was loaded)."""

    def __init__(self, st, K, every=None, ptype=1, cap=None, device="cuda", adjoint_solver="mixed"):
        if st.geom.flag_pbc or st.geom.flag_nmn or st.geom.flag_die:
            raise ValueError("the adjoint window supports Dirichlet (metal) walls only")
        self.st = st
        self.K = int(K)
        self.every = int(every) if every else max(1, int(round(math.sqrt(self.K))))
        self.ptype = int(ptype)
        if adjoint_solver not in ("mixed", "f64"):
            raise ValueError(f"adjoint_solver must be 'mixed' or 'f64', not {adjoint_solver!r}")
        # the adjoint Poisson solves: FP32 V-cycles inside FP64 refinement
        # ("mixed", converged to the same residual test as the FP64
        # multigrid) or the FP64 multigrid itself ("f64", the reference
        # gradient); the forward window always runs the FP64 step
        self.adjoint_solver = adjoint_solver
        self.sim = Simulation(st, cap=cap, device=device, fused=False)
        self.dev = self.sim.dev
        self.nlabel = int(st.geom.ngrid)
        self.bcnd = self.sim.bcnd
        self.x0 = None
        self.timing = {}

    # ------------------------------------------------------------ set-up
    def _adopt(self, p0):
        """The window's own particle order: sorted by cell, so that the
        deposition and its transposes of neighbouring threads touch
        neighbouring nodes.  `order` maps window slots to the input order."""
        h = self.st.h
        n1, n2, _ = self.st.n
        ix = (p0[0] / h[0]).long()
        iy = (p0[1] / h[1]).long()
        iz = (p0[2] / h[2]).long()
        self.order = torch.argsort(ix + n1 * (iy + n2 * iz))
        self.x0 = p0[:, self.order].contiguous()
        self.n = int(p0.shape[1])

    def load_uniform(self, seed=None):
        """Initial state from the GPU loader (positions, Maxwellian v)."""
        self.sim.load_uniform(seed=seed)
        s = self.sim.sp[self.ptype - 1]
        self._adopt(s.p[:, :s.n()])
        self.np_fixed = self.sim.np.clone()
        self.np_fixed[self.ptype - 1].zero_()

    def load(self, p0):
        """Initial state (6, n) FP64 device tensor x, y, z, vx, vy, vz of the
        species; the other species carry no charge.  The window keeps the
        particles in its own order (x0, initial velocities and their
        gradients are in that order; `order` maps it to p0's)."""
        self._adopt(p0)
        self.np_fixed = torch.zeros_like(self.sim.np)

    def _s(self):
        return self.sim._s()

    def _set_params(self, V, Bz):
        st = self.st
        phi = torch.as_tensor(st.geom.phi, device=self.dev).clone()
        for lab in range(1, self.nlabel + 1):
            phi[self.bcnd == lab] = float(V[lab - 1])
        self.phi0 = phi
        self.sim.P.Bconst[2] = float(Bz)

    # ------------------------------------------------------------ forward
    def _step(self, p, alive):
        """One window step: deposit, rho, Poisson, E, push."""
        sim, L = self.sim, lib()
        n = self.n
        sim.np.copy_(self.np_fixed)
        check(L.lepic_dev_win_deposit(C.byref(sim.grid), _p(p), p.shape[1], n, _p(alive), self.ptype,
                                      C.byref(sim.P), C.c_void_p(sim.np[self.ptype - 1].data_ptr()),
                                      self._s()), "win_deposit")
        sim.calc_rho()
        sim.pdesolver()
        sim.efield()
        check(L.lepic_dev_win_push(C.byref(sim.grid), _p(sim.Ei), _p(p), p.shape[1], n, _p(alive), self.ptype,
                                   C.byref(sim.P), self._s()), "win_push")

    def _objective(self, p, alive):
        st = self.st
        m = abs(st.mass[self.ptype - 1])
        a = alive.to(torch.float64)
        na = float(a.sum())
        ke = 0.5 * m * (p[3:6] ** 2).sum(dim=0) / QE
        return float((ke * a).sum()) / na, na

    def forward(self, V, Bz, v0=None):
        """Run the window; returns J = mean kinetic energy (eV) of the
        species' particles still alive after K steps."""
        if self.x0 is None:
            raise RuntimeError("load the initial state first")
        self._set_params(V, Bz)
        p = self.x0.clone()
        if v0 is not None:
            p[3:6] = v0
        alive = torch.ones(self.n, dtype=torch.int8, device=self.dev)
        self.sim.phi.copy_(self.phi0)
        self.ckpt = []
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for it in range(self.K):
            if it % self.every == 0:
                self.ckpt.append((p.clone(), alive.clone(), self.sim.phi.clone()))
            self._step(p, alive)
        ev1.record()
        torch.cuda.synchronize()
        self.timing["forward_ms"] = ev0.elapsed_time(ev1)
        self.p_final, self.alive_final = p, alive
        J, self.n_alive = self._objective(p, alive)
        self.V, self.Bz = [float(v) for v in V], float(Bz)
        return J

    # ------------------------------------------------------------ backward
    def backward(self, gJ=1.0):
        """Adjoint of the last forward: (dJ/dV per label, dJ/dBz, dJ/dv0)."""
        sim, L, st = self.sim, lib(), self.st
        n = self.n
        dev = self.dev
        m = abs(st.mass[self.ptype - 1])
        lam = torch.zeros((6, n), dtype=torch.float64, device=dev)
        a = self.alive_final.to(torch.float64)
        lam[3:6] = (gJ * m / (QE * self.n_alive)) * self.p_final[3:6] * a
        lE = torch.zeros_like(sim.Ei)
        lphi = torch.zeros_like(sim.phi)
        mu = torch.zeros_like(sim.phi)
        lnp = torch.zeros_like(sim.phi)
        b = torch.zeros_like(sim.rhs)
        dV = torch.zeros(max(self.nlabel, 1), dtype=torch.float64, device=dev)
        dBz = torch.zeros(1, dtype=torch.float64, device=dev)
        wl = st.wl
        n1, n2, n3 = st.n
        h = st.h
        from .constants import EPS0
        ac = 2.0 * EPS0 * (1.0 / h[0] ** 2 + 1.0 / h[1] ** 2 + 1.0 / h[2] ** 2)
        alpha = (n1 + 1) * (n2 + 1) * (n3 + 1) * ac
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        nseg = len(self.ckpt)
        for seg in reversed(range(nseg)):
            n0 = seg * self.every
            n1s = min(self.K, n0 + self.every)
            p, alive, phi = (t.clone() for t in self.ckpt[seg])
            sim.phi.copy_(phi)
            states = []
            for it in range(n0, n1s):
                pn, an = p.clone(), alive.clone()
                self._step(p, alive)
                states.append((pn, an, sim.Ei.clone()))
            alive_after = alive
            for it in reversed(range(n0, n1s)):
                pn, an, En = states[it - n0]
                lE.zero_()
                check(L.lepic_dev_adj_push(C.byref(sim.grid), _p(En), _p(pn), n, n, _p(an), _p(alive_after),
                                           _p(lam), n, self.ptype, C.byref(sim.P), _p(lE), _p(dBz), self._s()),
                      "adj_push")
                check(L.lepic_dev_adj_efield(C.byref(sim.grid), _p(lE), _p(lphi), self._s()), "adj_efield")
                check(L.lepic_dev_adj_rhs(C.byref(sim.grid), _p(lphi), _p(b), self._s()), "adj_rhs")
                # warm start: mu of the later step (walls stay 0)
                r0 = float(b.abs().sum()) / alpha
                if r0 > 0.0:
                    k, kt, res = C.c_int(0), C.c_double(0), C.c_double(0)
                    if self.adjoint_solver == "mixed":
                        m = sim.mg_mixed
                        check(L.lepic_dev_pdesolver_mixed(C.byref(sim.grid), _p(mu), _p(b), wl.eps * r0,
                                                          m["omega"], st.ng, C.byref(sim.P), m["max_refine"],
                                                          m["nu_fine_pre"], m["nu_fine_post"], m["nu_pre"],
                                                          m["nu_post"], m["coarse_sweeps"],
                                                          C.byref(k), C.byref(res), self._s()),
                              "adjoint pdesolver (mixed)")
                    else:
                        check(L.lepic_dev_pdesolver(C.byref(sim.grid), _p(mu), _p(b), wl.ncycl, wl.eps * r0,
                                                    wl.omega, st.ng, C.byref(sim.P), C.byref(k), C.byref(kt),
                                                    C.byref(res), self._s()), "adjoint pdesolver")
                check(L.lepic_dev_adj_walls(C.byref(sim.grid), C.byref(sim.P), self.ptype, _p(lphi), _p(mu),
                                            _p(lnp), _p(dV), self.nlabel, self._s()), "adj_walls")
                check(L.lepic_dev_adj_deposit(C.byref(sim.grid), _p(pn), n, n, _p(an), _p(lnp), _p(lam), n,
                                              self.ptype, C.byref(sim.P), self._s()), "adj_deposit")
                alive_after = an
            del states
        ev1.record()
        torch.cuda.synchronize()
        self.timing["backward_ms"] = ev0.elapsed_time(ev1)
        return dV.cpu().numpy()[:self.nlabel].copy(), float(dBz.item()), lam[3:6].clone()


class _WindowFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, V, Bz, v0, window):
        J = window.forward(V.detach().cpu().numpy(), float(Bz), v0.detach())
        ctx.window = window
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        dV, dBz, dv0 = ctx.window.backward(float(gJ))
        return (torch.as_tensor(dV, dtype=torch.float64), torch.tensor(dBz, dtype=torch.float64), dv0, None)


def window_objective(window, V, Bz, v0):
    """J(V, Bz, v0) through the window as a torch.autograd.Function:
    V (nlabel,) FP64 CPU tensor of wall potentials by label, Bz FP64 scalar
    tensor, v0 (3, n) FP64 device tensor of initial velocities."""
    return _WindowFn.apply(V, Bz, v0, window)


# ----------------------------------------------------------------------------
# The differentiable window of the collisional step
# ----------------------------------------------------------------------------
_ALIVE_BL = -1 & 0xffff | (0x7fff << 16)     # born -1 (present at the start), not lost


class CollisionWindow:
    """K-step differentiable window of the full collisional step (no
    counterpart in the reference) on the particles of a mixed-precision
    Simulation: every charged species is deposited and pushed, the
    null-collision MCC against the neutral gas runs every ns_coll steps
    (Src/main.f90:1116-1122) and its collisions are recorded, so that every
    later pass -- the backward pass, finite differences, the FP64 reference --
    replays exactly those events (which particle, which reaction, the target's
    velocity and the scattering directions; the velocities themselves follow
    from the replayed state).

    Observables (scalar J):
      "energy"  mean kinetic energy (eV) of species 1 after K steps,
      "probe"   the potential (V) at the node nearest the box centre after K
                steps (a field solve of the final charge),
      "flux"    the kinetic energy (J) carried to the walls by the
                macroparticles lost during the window (P_loss(1) of
                Src/part_expmover.f90:290-296 summed over the steps).
    Gradients: dJ/dV per wall label, dJ/dB_z (uniform B) and dJ/dv0 (the
    initial velocities of species 1, in its slot order).

    fp64=False runs in place on the simulation's FP32 stores (the adjoint in
    the particle-state arrays the sort uses as its second buffer, the window
    history in the second cell array) with FP32 pushes and the mixed Poisson
    solve; fp64=True runs on FP64 copies of the same initial particles with
    the FP64 multigrid: the FP64 reference of the same events.  The backward
    pass needs no particle checkpoints: it undoes each push (the inverse
    Boris rotation), each collision (from its record), and keeps only the
    potential of every step.

    sort=True sorts the simulation's particles by cell first (every species),
    which the FP32 kernels' tile-by-tile scatter is fast on; a second window
    on the same initial state (the FP64 reference) must then be made with
    sort=False, after the first, so that both see the same slots."""

    def __init__(self, sim, K, fp64=False, ns_coll=None, first_it=None, log_cap=None, keep_initial=False,
                 seed=None, sort=False):
        st = sim.st
        if not sim.mixed:
            raise ValueError("the collisional window runs on a mixed-precision Simulation")
        if st.geom.flag_pbc or st.geom.flag_nmn or st.geom.flag_die:
            raise ValueError("the collisional window supports Dirichlet (metal) walls only")
        if st.bfield is not None:
            raise ValueError("the collisional window differentiates a uniform B, not a B-field map")
        if sort:
            sim.sort()
        self.sim, self.st, self.K, self.fp64 = sim, st, int(K), bool(fp64)
        self.dev = sim.dev
        self.ntype = st.ntype
        self.nlabel = int(st.geom.ngrid)
        self.ns_coll = int(ns_coll or st.wl.ns_coll)
        self.first_it = int(sim.it + 1 if first_it is None else first_it)
        self.seed = int(sim.seed if seed is None else seed)
        self.ws = (LepicWinSpecies * self.ntype)()
        self.stores = []
        for p in range(self.ntype):
            sp = sim.sp[p]
            if self.fp64:
                d = dict(cell=sp.cell.clone(), p=sp.p.to(torch.float64), lam=torch.zeros((6, sp.cap),
                         dtype=torch.float64, device=self.dev), bl=torch.empty(sp.cap, dtype=torch.int32,
                         device=self.dev), count=sp.count.clone())
            else:
                d = dict(cell=sp.cell, p=sp.p, lam=sp.p_alt, bl=sp.cell_alt, count=sp.count)
            d["cap"] = sp.cap
            self.stores.append(d)
            w = self.ws[p]
            w.cell, w.p, w.lam = d["cell"].data_ptr(), d["p"].data_ptr(), d["lam"].data_ptr()
            w.bl, w.count, w.cap, w.fp64 = d["bl"].data_ptr(), d["count"].data_ptr(), d["cap"], int(self.fp64)
            if not self.fp64:
                # the tiles of the simulation's last sort: the FP32 deposit and
                # push adjoint scatter tile by tile (fast when the particles
                # are still in that sort's order, correct in any order)
                d["tile_off"] = sp.tile_off.clone()
                w.tile_off = d["tile_off"].data_ptr()
                w.tile_end = int(d["tile_off"][-1].item())
        self.count0 = [int(d["count"].item()) for d in self.stores]
        self.initial = None
        if keep_initial:
            self.initial = [(d["cell"].clone(), d["p"].clone(), d["count"].clone()) for d in self.stores]
        n1, n2, n3 = st.n
        self.centre = (n3 // 2 + 1, n2 // 2 + 1, n1 // 2 + 1)
        self.phis = torch.empty((self.K + 1,) + tuple(sim.phi.shape), dtype=torch.float64, device=self.dev)
        self.wall_acc = torch.zeros(self.ntype, dtype=torch.float64, device=self.dev)
        # records: about 0.35 % of the particles collide per call at 1 Pa (the
        # electrons' null-collision probability is 1.4 %); the default leaves
        # room for 3 % per call, at most 8 GB of records (a call that finds
        # the log full raises LEPIC_ERR_CAPACITY)
        calls = sum(1 for n in range(self.K) if (self.first_it + n) > 1
                    and (self.first_it + n) % self.ns_coll == 1 % self.ns_coll)
        cap = log_cap or min(4096 + int(0.03 * sum(self.count0) * max(calls, 1)),
                             (8 << 30) // C.sizeof(LepicWinEvent))
        self.log = torch.zeros(cap * C.sizeof(LepicWinEvent), dtype=torch.uint8, device=self.dev)
        self.log_cap = cap
        self.nlog = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.ev_range = {}            # step -> (first record, end)
        self.recorded = False
        self.timing = {}
        self.counts = np.zeros(64, dtype=np.int64)

    # ------------------------------------------------------------ helpers
    def _s(self):
        return self.sim._s()

    def _E(self):
        return self.sim.Ei if self.fp64 else self.sim.E32

    def _events(self, step):
        a, b = self.ev_range.get(step, (0, 0))
        return C.c_void_p(self.log.data_ptr() + a * C.sizeof(LepicWinEvent)), b - a

    def use_log_of(self, other):
        """Replay the collisions another window of the same initial state
        recorded (the FP64 reference of a mixed window)."""
        self.log = other.log.clone()
        self.log_cap = other.log_cap
        self.ev_range = dict(other.ev_range)
        self.recorded = True

    def _solve(self, u, rhs, eps=None):
        """A u = rhs on plasma nodes (u holds the wall values and the start):
        the FP64 multigrid for the FP64 window, FP32 V-cycles in FP64
        refinement for the mixed one."""
        sim, st = self.sim, self.st
        eps = st.wl.eps if eps is None else eps
        if self.fp64:
            k, kt, res = C.c_int(0), C.c_double(0), C.c_double(0)
            check(lib().lepic_dev_pdesolver(C.byref(sim.grid), _p(u), _p(rhs), st.wl.ncycl, eps, st.wl.omega,
                                            st.ng, C.byref(sim.P), C.byref(k), C.byref(kt), C.byref(res),
                                            self._s()), "pdesolver")
        else:
            m = sim.mg_mixed
            it, res = C.c_int(0), C.c_double(0)
            check(lib().lepic_dev_pdesolver_mixed(C.byref(sim.grid), _p(u), _p(rhs), eps, m["omega"], st.ng,
                                                  C.byref(sim.P), m["max_refine"], m["nu_fine_pre"],
                                                  m["nu_fine_post"], m["nu_pre"], m["nu_post"], m["coarse_sweeps"],
                                                  C.byref(it), C.byref(res), self._s()), "pdesolver_mixed")

    def _field(self):
        self.sim.calc_rho()
        self._solve(self.sim.phi, self.sim.rhs)

    def _efield(self):
        sim = self.sim
        check(lib().lepic_dev_calc_efield(C.byref(sim.grid), _p(sim.phi), _p(sim.Ei), self._s()), "calc_efield")
        if not self.fp64:
            sim.pack_e32()

    def _deposit(self, step):
        sim, L = self.sim, lib()
        sim.np.zero_()
        for p in range(self.ntype):
            if self.st.charge[p] != 0.0:
                check(L.lepic_dev_cw_deposit(C.byref(sim.grid), C.byref(self.ws[p]), p + 1, C.byref(sim.P), step,
                                             _p(sim.np[p]), self._s()), "cw_deposit")

    def _set_params(self, V, Bz):
        st, sim = self.st, self.sim
        phi = torch.as_tensor(st.geom.phi, device=self.dev).clone()
        for lab in range(1, self.nlabel + 1):
            phi[sim.bcnd == lab] = float(V[lab - 1])
        self.phi0 = phi
        sim.P.Bconst[2] = float(Bz)
        if float(Bz) != 0.0:
            sim.P.flag_B = 1

    # ------------------------------------------------------------ forward
    def forward(self, V, Bz, v0=None, observable="energy"):
        """Run the window from its initial state; returns J.  The first call
        records the collisions, later calls replay them."""
        if observable not in ("energy", "probe", "flux"):
            raise ValueError(f"observable must be energy, probe or flux, not {observable!r}")
        sim, L, st = self.sim, lib(), self.st
        self.observable = observable
        self._set_params(V, Bz)
        if self.initial is not None:
            for d, (c0, p0, n0) in zip(self.stores, self.initial):
                d["cell"].copy_(c0)
                d["p"].copy_(p0)
                d["count"].copy_(n0)
        for d in self.stores:
            d["bl"].fill_(_ALIVE_BL)
        if v0 is not None:
            self.stores[0]["p"][3:6, :self.count0[0]] = v0.to(self.stores[0]["p"].dtype)
        self.wall_acc.zero_()
        sim.phi.copy_(self.phi0)
        record = not self.recorded
        if record:
            self.nlog.zero_()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for n in range(self.K):
            self._deposit(n)
            self._field()
            self.phis[n].copy_(sim.phi)
            self._efield()
            it = self.first_it + n
            if st.tables is not None and it > 1 and it % self.ns_coll == 1 % self.ns_coll:
                if record:
                    a = int(self.nlog.item())
                    nu = (C.c_double * 10)()
                    cnt = (C.c_longlong * 64)()
                    # Pmax = nu_max ns_coll dt with the window's own cadence
                    # (Src/collisions.f90:122)
                    ns0 = sim.P.ns_coll
                    sim.P.ns_coll = self.ns_coll
                    try:
                        check(L.lepic_dev_win_collisions(C.byref(sim.grid), self.ws, self.ntype,
                                                         C.byref(sim._tables), C.byref(sim.P),
                                                         C.c_ulonglong(self.seed), C.c_ulonglong(it), n,
                                                         _p(self.log), self.log_cap, _p(self.nlog), nu, cnt,
                                                         self._s()),
                              "win_collisions")
                    finally:
                        sim.P.ns_coll = ns0
                    self.counts[:64] += np.array(cnt[:], dtype=np.int64)
                    self.ev_range[n] = (a, int(self.nlog.item()))
                else:
                    evp, ne = self._events(n)
                    check(L.lepic_dev_cw_replay(C.byref(sim.grid), self.ws, self.ntype, C.byref(sim.P), evp, ne,
                                                self._s()), "cw_replay")
            for p in range(self.ntype):
                if st.charge[p] != 0.0:
                    check(L.lepic_dev_cw_push(C.byref(sim.grid), _p(self._E()), C.byref(self.ws[p]), p + 1,
                                              C.byref(sim.P), n, _p(self.wall_acc[p:]), self._s()), "cw_push")
        if observable == "probe":
            self._deposit(self.K)
            self._field()
            self.phis[self.K].copy_(sim.phi)
        ev1.record()
        torch.cuda.synchronize()
        self.recorded = True
        self.timing["forward_ms"] = ev0.elapsed_time(ev1)
        self.V, self.Bz = [float(v) for v in V], float(Bz)
        return self._objective()

    def _alive(self, p):
        d = self.stores[p]
        n = int(d["count"].item())
        return n, ((d["bl"][:n] >> 16) == 0x7fff)

    def _objective(self):
        st = self.st
        if self.observable == "energy":
            n, a = self._alive(0)
            v = self.stores[0]["p"][3:6, :n].to(torch.float64)
            m = abs(st.mass[0])
            self.n_alive = int(a.sum())
            ke = 0.5 * m * (v ** 2).sum(dim=0) / QE
            return float((ke * a).sum()) / self.n_alive
        if self.observable == "probe":
            k, j, i = self.centre
            return float(self.phis[self.K][k, j, i])
        return float(self.wall_acc.sum())

    # ------------------------------------------------------------ backward
    def backward(self, gJ=1.0):
        """Adjoint of the last forward: (dJ/dV per label, dJ/dBz, dJ/dv0)."""
        sim, L, st = self.sim, lib(), self.st
        dev = self.dev
        wl = st.wl
        for d in self.stores:
            d["lam"].zero_()
        dV = torch.zeros(max(self.nlabel, 1), dtype=torch.float64, device=dev)
        dBz = torch.zeros(1, dtype=torch.float64, device=dev)
        lE = torch.zeros_like(sim.Ei)
        lphi = torch.zeros_like(sim.phi)
        mu = torch.zeros_like(sim.phi)
        lnp = torch.zeros_like(sim.phi)
        b = torch.zeros_like(sim.rhs)
        from .constants import EPS0
        h = st.h
        n1, n2, n3 = st.n
        ac = 2.0 * EPS0 * (1.0 / h[0] ** 2 + 1.0 / h[1] ** 2 + 1.0 / h[2] ** 2)
        alpha = (n1 + 1) * (n2 + 1) * (n3 + 1) * ac

        def field_adjoint():
            # lphi -> mu (A mu = lphi on plasma nodes) and dJ/dV; the deposit
            # adjoint of the step's particles follows with mu (fused into the
            # previous step's backward kernels, or last for step 0)
            check(L.lepic_dev_adj_rhs(C.byref(sim.grid), _p(lphi), _p(b), self._s()), "adj_rhs")
            r0 = float(b.abs().sum()) / alpha
            if r0 > 0.0:
                self._solve(mu, b, eps=wl.eps * r0)   # warm start: mu of the later step (walls 0)
            check(L.lepic_dev_adj_walls(C.byref(sim.grid), C.byref(sim.P), 1, _p(lphi), _p(mu), _p(lnp), _p(dV),
                                        self.nlabel, self._s()), "adj_walls")

        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        wflux = 0.0
        if self.observable == "energy":
            n, a = self._alive(0)
            m = abs(st.mass[0])
            d = self.stores[0]
            d["lam"][3:6, :n] = ((gJ * m / (QE * self.n_alive)) * d["p"][3:6, :n].to(torch.float64)
                                 * a.to(torch.float64)).to(d["lam"].dtype)
        have_mu = False
        if self.observable == "probe":
            lphi.zero_()
            k, j, i = self.centre
            lphi[k, j, i] = gJ
            field_adjoint()
            have_mu = True
        elif self.observable == "flux":
            wflux = gJ
        for n in reversed(range(self.K)):
            sim.phi.copy_(self.phis[n])
            self._efield()
            lE.zero_()
            # the deposit adjoint of step n + 1, the push of step n undone and
            # its adjoint, per species in one pass over the particles
            for p in range(self.ntype):
                if st.charge[p] != 0.0:
                    check(L.lepic_dev_cw_back(C.byref(sim.grid), _p(self._E()), C.byref(self.ws[p]), p + 1,
                                              C.byref(sim.P), n, _p(mu) if have_mu else None, C.c_double(wflux),
                                              _p(lE), _p(dBz), self._s()), "cw_back")
            if n in self.ev_range:
                evp, ne = self._events(n)
                check(L.lepic_dev_cw_adj_collide(C.byref(sim.grid), self.ws, self.ntype, C.byref(sim.P), evp, ne,
                                                 self._s()), "cw_adj_collide")
            check(L.lepic_dev_adj_efield(C.byref(sim.grid), _p(lE), _p(lphi), self._s()), "adj_efield")
            field_adjoint()
            have_mu = True
        for p in range(self.ntype):
            if st.charge[p] != 0.0:
                check(L.lepic_dev_cw_adj_deposit(C.byref(sim.grid), C.byref(self.ws[p]), p + 1, C.byref(sim.P), 0,
                                                 _p(mu), self._s()), "cw_adj_deposit")
        ev1.record()
        torch.cuda.synchronize()
        self.timing["backward_ms"] = ev0.elapsed_time(ev1)
        # dJ/dv0 is a view of the adjoint planes (the window's precision),
        # valid until the window's next pass
        lam = self.stores[0]["lam"]
        return dV.cpu().numpy()[:self.nlabel].copy(), float(dBz.item()), lam[3:6, :self.count0[0]]


class _CollisionWindowFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, V, Bz, v0, window, observable):
        J = window.forward(V.detach().cpu().numpy(), float(Bz), v0.detach(), observable=observable)
        ctx.window = window
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        dV, dBz, dv0 = ctx.window.backward(float(gJ))
        return (torch.as_tensor(dV, dtype=torch.float64), torch.tensor(dBz, dtype=torch.float64),
                dv0.to(torch.float64).clone(), None, None)


def collision_window_objective(window, V, Bz, v0, observable="energy"):
    """J(V, Bz, v0) through a CollisionWindow as a torch.autograd.Function:
    V (nlabel,) FP64 CPU tensor of wall potentials by label, Bz FP64 scalar
    tensor, v0 (3, n) FP64 device tensor of the initial velocities of
    species 1 (its slot order)."""
    return _CollisionWindowFn.apply(V, Bz, v0, window, observable)
