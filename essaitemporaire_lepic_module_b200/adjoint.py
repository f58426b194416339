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

from ._lib import check, lib
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
