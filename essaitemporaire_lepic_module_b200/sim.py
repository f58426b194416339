"""Device-resident PIC-MCC time stepping on one B200 (FP64 and mixed forms).

``Simulation`` keeps every array of the hot path in HBM (torch tensors used
as plain device buffers) and advances the legacy timestep of
Src/main.f90:853-1277 through the C ABI of liblepic_gpu.so:

    calc_rho -> pdesolver -> calc_Efield -> part_sorting (every nsort)
    -> collisions (every ns_coll, it > 1) -> part_mover -> charge_deposition

Layout in HBM (reference index bases, column-major like the Fortran arrays):
    bcnd, kq, phi          (n3+3, n2+3, n1+3) int32 / float64
    Ei                     (n3+3, n2+3, n1+3, 3) float64, component fastest
    np                     (ntype, n3+3, n2+3, n1+3) float64
    rhs                    (n3+2, n2+2, n1+2) float64
    particles per species  SoA (6, cap) float64 = x, y, z, vx, vy, vz
                           + second buffer (sort target), int32 keys,
                           int8 dead flags, device int32 count

Mixed form (precision="mixed"): particles are int32 cell + (6, cap) float32
= fx, fy, fz (in-cell offsets), vx, vy, vz (28 B instead of 48 B), the push
reads an FP32 copy E32 of the field, and the Poisson solve is FP32 V-cycles
inside FP64 iterative refinement to the same residual tolerance.  rho, phi,
E and the charge grids stay FP64.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import (LepicGrid, LepicSpeciesF64, LepicSpeciesMixed, LepicTables, LepicTargets, check, lib,
                   phys_struct)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def allreduce_density(np_grids, group=None):
    """Sum the per-rank density grids over the ranks of `group` in place:
    every rank holds its own particles over the full grid, and the field
    needs the density of all of them (the MPI_ALLREDUCE of rho of
    Src/calc_rho.f90:102).  One collective of the (ntype, nodes) FP64 grids."""
    import torch.distributed as dist
    dist.all_reduce(np_grids, op=dist.ReduceOp.SUM, group=group)
    return np_grids


def sort_intervals(st, nsort, policy="reference"):
    """Steps between sorts of each species.  "reference": every species every
    nsort steps (Src/main.f90:1071-1080).  "adaptive": the order only serves
    the push's memory locality, so a species whose thermal displacement in
    nsort steps, vt0 dt nsort / h, stays below half a cell is sorted up to
    ten times less often (a multiple of nsort); fast species keep nsort."""
    if not nsort:
        return [0] * st.ntype
    if policy == "reference":
        return [int(nsort)] * st.ntype
    if policy != "adaptive":
        raise ValueError(f"sort policy must be 'reference' or 'adaptive', not {policy!r}")
    hmin = float(min(st.h))
    out = []
    for p in range(st.ntype):
        d = float(st.vt0[p]) * float(st.dt) * nsort / hmin
        m = 10 if d <= 0.05 else max(1, min(10, int(0.5 / d)))
        out.append(int(nsort) * m)
    return out


def rank_weight(Nm, world):
    """Macroparticle weight of each of `world` ranks that each load a full
    set of particles of weight Nm: Nm / world keeps the plasma density."""
    return Nm / float(world)


class Species:
    """One species' FP64 particle store on the device."""

    def __init__(self, cap, device):
        self.cap = int(cap)
        self.p = torch.zeros((6, self.cap), dtype=torch.float64, device=device)
        self.p_alt = torch.zeros((6, self.cap), dtype=torch.float64, device=device)
        self.count = torch.zeros(1, dtype=torch.int32, device=device)
        self.key = torch.zeros(self.cap, dtype=torch.int32, device=device)
        self.flag_dead = torch.zeros(self.cap, dtype=torch.int8, device=device)
        self.s = LepicSpeciesF64()
        self._sync_struct()

    def _sync_struct(self):
        s = self.s
        s.p, s.p_alt = self.p.data_ptr(), self.p_alt.data_ptr()
        s.count, s.key = self.count.data_ptr(), self.key.data_ptr()
        s.flag_dead, s.cap = self.flag_dead.data_ptr(), self.cap

    def after_call(self):
        """The sort swaps the two buffers inside the struct; follow it."""
        if self.s.p != self.p.data_ptr():
            self.p, self.p_alt = self.p_alt, self.p
        self._sync_struct()

    def n(self):
        return int(self.count.item())

    def to_vxp(self):
        """Host copy in the reference layout vxp(6, 1:np) -> (np, 6)."""
        n = self.n()
        return self.p[:, :n].t().contiguous().cpu().numpy()


def tiles_of(n):
    """Number of 8x8x8-cell tiles the mixed sort orders particles by."""
    return ((n[0] + 7) // 8) * ((n[1] + 7) // 8) * ((n[2] + 7) // 8)


class SpeciesMixed:
    """One species' mixed-precision particle store (cell + FP32 planes)."""

    def __init__(self, cap, device, n):
        self.cap = (int(cap) + 3) // 4 * 4
        self.cell = torch.zeros(self.cap, dtype=torch.int32, device=device)
        self.p = torch.zeros((6, self.cap), dtype=torch.float32, device=device)
        self.cell_alt = torch.zeros(self.cap, dtype=torch.int32, device=device)
        self.p_alt = torch.zeros((6, self.cap), dtype=torch.float32, device=device)
        self.count = torch.zeros(1, dtype=torch.int32, device=device)
        self.flag_dead = torch.zeros(self.cap, dtype=torch.int8, device=device)
        self.tile_off = torch.zeros(tiles_of(n) + 1, dtype=torch.int32, device=device)
        self.cell_off = None        # per-cell starts of the last sort (charged targets)
        self.s = LepicSpeciesMixed()
        self._sync_struct()

    def keep_cell_offsets(self, n):
        """Have every sort keep the start of each cell (for charged-target
        collisions): LEPIC_TILES(n) * 512 + 1 ints."""
        if self.cell_off is None:
            self.cell_off = torch.zeros(tiles_of(n) * 512 + 1, dtype=torch.int32, device=self.count.device)
            self._sync_struct()

    def _sync_struct(self):
        s = self.s
        s.cell, s.p = self.cell.data_ptr(), self.p.data_ptr()
        s.cell_alt, s.p_alt = self.cell_alt.data_ptr(), self.p_alt.data_ptr()
        s.count, s.flag_dead, s.cap = self.count.data_ptr(), self.flag_dead.data_ptr(), self.cap
        s.tile_off = self.tile_off.data_ptr()
        s.cell_off = None if self.cell_off is None else self.cell_off.data_ptr()

    def after_call(self):
        if self.s.p != self.p.data_ptr():
            self.p, self.p_alt = self.p_alt, self.p
            self.cell, self.cell_alt = self.cell_alt, self.cell
        self._sync_struct()

    def n(self):
        return int(self.count.item())


class Simulation:
    """Device-resident timestep.  With `comm` (a torch.distributed process
    group, or True for the default group) each rank holds its own particles
    at weight Nm / world, the density grids are all-reduced after every
    deposition and every rank solves the same field."""

    def __init__(self, st, cap=None, device="cuda", seed=123456, nsort=None, ns_coll=None,
                 fused=True, precision="f64", mg_mixed=None, comm=None, sort_policy="reference",
                 check_every=1, heating=None, injection=None, nonblocking=False):
        if precision not in ("f64", "mixed"):
            raise ValueError(f"precision must be 'f64' or 'mixed', not {precision!r}")
        if st.geom.flag_die and not st.Ca > 0.0:
            raise ValueError("dielectric walls need a capacitance Ca > 0")
        self.st = st
        self.mixed = precision == "mixed"
        self.precision = precision
        self.fused = fused or self.mixed
        # FP32 V-cycle parameters of the mixed Poisson solve: over-relaxed
        # red-black smoothing (omega 1.3) reduces the smooth error modes that
        # the L1 residual test hardly sees; one pre- and three post-sweeps on
        # the finest level (its sweeps are the dearest, the last one also
        # accumulates u), two and two on the coarser levels; at the workloads'
        # tolerance phi lands within ~1e-8 of the converged FP64 solution in
        # 4-5 refinements
        self.mg_mixed = dict(max_refine=60, nu_fine_pre=1, nu_fine_post=3, nu_pre=2, nu_post=2,
                             coarse_sweeps=4, omega=1.3)
        if mg_mixed:
            self.mg_mixed.update(mg_mixed)
        self._acc = None
        self.dev = torch.device(device)
        self.stream = torch.cuda.current_stream(self.dev)
        self.nsort = st.wl.nsort if nsort is None else nsort
        self.ns_coll = st.wl.ns_coll if ns_coll is None else ns_coll
        self.sort_every = sort_intervals(st, self.nsort, sort_policy)
        self.sort_policy = sort_policy
        # steps between reads of the device error word (0: never); a kernel
        # that met a bad cell, a full particle array or a collision-table
        # overflow raises LepicError at the next read
        self.check_every = int(check_every)
        # nonblocking: the step loop never waits for the device.  The mixed
        # solve is launched without waiting (its refinements and residual
        # are copied into pinned host memory in stream order, read when
        # mg_last or solve_history() is asked for), and the device error
        # word is snapshotted into pinned memory and read at a later step,
        # so a failure surfaces one or two steps after the step that met it
        # (flush_checks() waits for the last snapshot).
        self.nonblocking = bool(nonblocking)
        self._mg_ring = 8192
        self._mg_count = 0
        self._mg_last_sync = None
        self._mg_it = self._mg_res = None
        self._err_host = None
        self._err_ev = None
        self._err_pending = False
        self.seed = int(seed)
        self.Bmap = None
        if getattr(st, "bfield", None) is not None:
            # the B-field map, resident for the run (Bi(4, 0:nB1+2, ...))
            self.Bmap = torch.as_tensor(np.ascontiguousarray(st.bfield.Bi), dtype=torch.float64,
                                        device=self.dev)
        self.P = phys_struct(st, bmap_ptr=None if self.Bmap is None else self.Bmap.data_ptr())
        # the collision probability of a call covers the steps since the last
        # one (Pmax = nu_max ns_coll dt, Src/collisions.f90:122)
        self.P.ns_coll = self.ns_coll
        self.comm = comm
        if comm is not None:
            import torch.distributed as dist
            self._group = None if comm is True else comm
            world = dist.get_world_size(self._group)
            for p in range(st.ntype):
                self.P.Nm[p] = rank_weight(st.Nm[p], world)
        self.die = None
        if st.geom.flag_die:
            # dielectric walls: dtype(0:ngrid) and the surface-charge sums of
            # every species, sum_q_xz (ntype, n3+3, n1+3) and sum_q_yz
            # (ntype, n3+3, n2+3, 2), which the pushes add to
            n1, n2, n3 = st.n
            f64 = dict(dtype=torch.float64, device=self.dev)
            self.die = (torch.as_tensor(st.geom.dtype_array(), device=self.dev),
                        torch.zeros((st.ntype, n3 + 3, n1 + 3), **f64),
                        torch.zeros((st.ntype, n3 + 3, n2 + 3, 2), **f64))
            self.P.dtype, self.P.sum_q_xz, self.P.sum_q_yz = (t.data_ptr() for t in self.die)
        g = st.geom
        T = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=self.dev)
        self.bcnd = T(g.bcnd, torch.int32)
        self.kq = T(st.kq, torch.float64)
        self.phi = T(g.phi, torch.float64)
        n1, n2, n3 = st.n
        self.cw = torch.zeros((n3 + 2) * (n2 + 2) * (n1 + 2), dtype=torch.uint8, device=self.dev)
        self.Ei = torch.zeros(tuple(g.bcnd.shape) + (3,), dtype=torch.float64, device=self.dev)
        self.np = torch.zeros((st.ntype,) + tuple(g.bcnd.shape), dtype=torch.float64, device=self.dev)
        self.rhs = torch.zeros((n3 + 2, n2 + 2, n1 + 2), dtype=torch.float64, device=self.dev)
        self.grid = LepicGrid()
        for a in range(3):
            self.grid.n[a] = st.n[a]
            self.grid.h[a] = float(st.h[a])
        self.grid.bcnd = self.bcnd.data_ptr()
        self.grid.kq = self.kq.data_ptr()
        self.grid.cell_wall = self.cw.data_ptr()
        nn = (C.c_int * 3)(*st.n)
        check(lib().lepic_dev_cell_wall(nn, C.c_void_p(self.bcnd.data_ptr()),
                                        C.c_void_p(self.cw.data_ptr()), self._s()), "cell_wall")
        if cap is None:
            cap = int(st.n_particles() * 1.25) + 1024
        self.cap = cap
        if self.mixed:
            self.sp = [SpeciesMixed(cap, self.dev, st.n) for _ in range(st.ntype)]
            self.E32 = torch.zeros(tuple(g.bcnd.shape) + (4,), dtype=torch.float32, device=self.dev)
        else:
            self.sp = [Species(cap, self.dev) for _ in range(st.ntype)]
        self.sp_arr = (LepicSpeciesF64 * max(st.ntype, 1))()
        self.it = 0
        self.p_mac = np.zeros((st.geom.ngrid + 1, 2, st.ntype))
        self.P_loss = np.zeros((st.ntype, 4))
        self.mg_last = None
        self.counts = np.zeros(64, dtype=np.int64)
        self.nu_max = np.zeros(10)
        self._tables = None
        if st.tables is not None:
            self._setup_tables()
        # Maxwellian electron heating (Src/main.f90:1206-1240): a config.Heating
        # particle injection after the push (Src/main.f90:1261-1267): a config.Injection
        self.inj = None
        if injection is not None:
            from .dropin import inject_struct
            self.inj = injection
            self._I = inject_struct(st, injection)
            if comm is not None:
                # every rank holds the whole population at weight Nm / world
                import torch.distributed as dist
                self._I.I_inj = injection.I_inj / dist.get_world_size(None if comm is True else comm)
            self._inj_calls = 0
            self._inj_lost_seen = 0.0
            self.injected = np.zeros(st.ntype, dtype=np.int64)
        self.heat = None
        if heating is not None:
            from .dropin import heat_struct
            self.heat = heating
            self._H, self.heat_params = heat_struct(st, heating)
            self._heat_acc = torch.zeros(3, dtype=torch.float64, device=self.dev)   # dE, heated, vt
            self._heat_stats = torch.zeros(2, dtype=torch.float64, device=self.dev)  # sum Ek, Nh
            self._heat_stats_ok = False
            self._heat_calls = 0

    def _s(self):
        return C.c_void_p(self.stream.cuda_stream)

    def _setup_tables(self):
        T = self.st.tables
        ncol, npt = T.sig.shape
        d = self.dev
        self._tsig = torch.as_tensor(np.ascontiguousarray(T.sig), device=d)
        self._tEr = torch.as_tensor(np.ascontiguousarray(T.sig_Er), device=d)
        self._tEth = torch.as_tensor(np.ascontiguousarray(T.Eth), device=d)
        self._ci_h = np.ascontiguousarray(T.col_info.T, dtype=np.int32)      # col_info(ncol,10)
        self._tci = torch.as_tensor(self._ci_h, device=d)
        self._sl_h = np.ascontiguousarray(T.sig_list.T, dtype=np.int32)      # sig_list(10,ncol)
        self._pn_h = np.ascontiguousarray(T.p_ncol, dtype=np.int32)
        self._sv_h = np.ascontiguousarray(T.sigv_mx.T, dtype=np.float64)     # sigv_mx(10,ncol)
        t = LepicTables()
        t.ncol, t.npt, t.npt_mx = ncol, npt, npt
        t.sig_Er, t.sig, t.sig_Eth = self._tEr.data_ptr(), self._tsig.data_ptr(), self._tEth.data_ptr()
        t.col_info = self._tci.data_ptr()
        t.sig_list = self._sl_h.ctypes.data
        t.p_ncol = self._pn_h.ctypes.data
        t.sigv_mx = self._sv_h.ctypes.data
        t.col_info_h = self._ci_h.ctypes.data
        self._tables = t
        # charged target species (DSMC): sorted on every collision step, their
        # per-cell offsets kept (Src/collisions.f90:335-423)
        st = self.st
        self.dsmc_targets = sorted({int(T.col_info[c, 2 + T.col_info[c, 0] - 1]) - 1
                                    for c in range(ncol)
                                    if st.charge[int(T.col_info[c, 2 + T.col_info[c, 0] - 1]) - 1] != 0.0})
        self._targets = None
        if self.dsmc_targets:
            self._targets = LepicTargets()
            if self.mixed:
                for q in self.dsmc_targets:
                    self.sp[q].keep_cell_offsets(st.n)

    # ----------------------------------------------------------- loading
    def _f64_stage(self):
        """FP64 species stores the mixed form loads through."""
        return [Species(self.cap, self.dev) for _ in range(self.st.ntype)]

    def _adopt_f64(self, f64):
        """Convert FP64 species (positions x, y, z) into the mixed stores."""
        for s64, sm in zip(f64, self.sp):
            n = s64.n()
            check(lib().lepic_dev_f64_to_mixed(C.byref(self.grid), C.byref(s64.s), C.byref(sm.s),
                                               C.c_longlong(n), self._s()), "f64_to_mixed")

    def load_from_host(self, vxp, np_tot, np_grids=None):
        """Initial state from host arrays in the reference layout
        (vxp (ntype, nmax, 6), np_tot, np grids)."""
        dst = self._f64_stage() if self.mixed else self.sp
        for p, s in enumerate(dst):
            n = int(np_tot[p])
            assert n <= s.cap
            s.p[:, :n] = torch.as_tensor(np.ascontiguousarray(vxp[p, :n, :].T), device=self.dev)
            s.count.fill_(n)
        if np_grids is not None:
            self.np.copy_(torch.as_tensor(np.ascontiguousarray(np_grids), device=self.dev))
        else:
            self._deposit_f64(dst)
        if self.mixed:
            self._adopt_f64(dst)

    def load_uniform(self, n_per_species=None, seed=None):
        """GPU Philox loader + initial deposition."""
        n = self.st.n_particles() if n_per_species is None else int(n_per_species)
        if self.mixed:
            arr = (LepicSpeciesMixed * len(self.sp))(*[s.s for s in self.sp])
            check(lib().lepic_dev_load_uniform_mixed(C.byref(self.grid), arr, len(self.sp), C.c_longlong(n),
                                                     C.byref(self.P), C.c_ulonglong(seed or self.seed),
                                                     self._s()), "load_uniform_mixed")
            self.np.zero_()
            for p, s in enumerate(self.sp):
                check(lib().lepic_dev_deposit_mixed(C.byref(self.grid), C.byref(s.s), p + 1, C.byref(self.P),
                                                    C.c_void_p(self.np[p].data_ptr()), n, self._s()),
                      "deposit_mixed")
            self._reduce_density()
            return
        arr = (LepicSpeciesF64 * len(self.sp))(*[s.s for s in self.sp])
        check(lib().lepic_dev_load_uniform(C.byref(self.grid), arr, len(self.sp), C.c_longlong(n),
                                           C.byref(self.P), C.c_ulonglong(seed or self.seed),
                                           self._s()), "load_uniform")
        self._deposit_f64(self.sp)

    def save_bak(self, path, time=0.0):
        """Particle backup in the reference's DATA.BAK/particlesNNN.bak format
        (Src/main.f90:1294-1330): time, np_tot and every species' vxp."""
        from .checkpoint import write_particles_bak
        arrs = [self.particles_f64(p).t().contiguous().cpu().numpy() for p in range(len(self.sp))]
        write_particles_bak(path, time, [a.shape[0] for a in arrs], arrs)

    def load_bak(self, path):
        """Restart from a particle backup of the reference's format
        (Src/restart.f90:62-70, one process): particles loaded, density
        deposited; returns the backup's time."""
        from .checkpoint import read_particles_bak
        time, npt, arrs, _ = read_particles_bak(path, len(self.sp))
        nmax = max(1, int(npt.max()))
        vxp = np.zeros((len(self.sp), nmax, 6))
        for p, a in enumerate(arrs):
            vxp[p, :len(a)] = a
        self.load_from_host(vxp, npt[:, 0])
        return time

    def particles_f64(self, p):
        """Species p as FP64 (6, n) x, y, z, vx, vy, vz on the device."""
        s = self.sp[p]
        n = s.n()
        if not self.mixed:
            return s.p[:, :n]
        out = torch.empty((6, max(n, 1)), dtype=torch.float64, device=self.dev)
        check(lib().lepic_dev_mixed_to_f64(C.byref(self.grid), C.byref(s.s), _ptr(out),
                                           C.c_longlong(out.shape[1]), C.c_longlong(n), self._s()),
              "mixed_to_f64")
        return out[:, :n]

    # ----------------------------------------------------------- kernels
    def calc_rho(self):
        check(lib().lepic_dev_calc_rho(C.byref(self.grid), _ptr(self.np), _ptr(self.rhs),
                                       self.st.ntype, C.byref(self.P), self._s()), "calc_rho")

    def dielectric_phi(self):
        """Src/main.f90:859-949: the dielectric walls' potential rises by
        the surface charge the pushes summed since the last call (summed over
        the ranks first, the MPI_ALLREDUCE of Src/main.f90:888-892); the
        sums restart from zero."""
        if self.comm is not None:
            import torch.distributed as dist
            for t in self.die[1:]:
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self._group)
        check(lib().lepic_dev_dielectric_phi(C.byref(self.grid), _ptr(self.phi), C.byref(self.P),
                                             self.st.geom.ngrid, C.c_double(self.st.Ca), self._s()),
              "dielectric_phi")

    def pdesolver(self, eps=None, omega=None, ng=None, ncycl=None):
        # the FP32 V-cycles cover Dirichlet walls; with periodic planes or the
        # Neumann plane the mixed form solves with the FP64 multigrid
        g = self.st.geom
        if self.mixed and not (g.flag_pbc or g.flag_nmn):
            return self.pdesolver_mixed(eps=eps, ng=ng)
        wl = self.st.wl
        k = C.c_int(0)
        ktot = C.c_double(0)
        res = C.c_double(0)
        check(lib().lepic_dev_pdesolver(C.byref(self.grid), _ptr(self.phi), _ptr(self.rhs),
                                        wl.ncycl if ncycl is None else ncycl,
                                        wl.eps if eps is None else eps,
                                        wl.omega if omega is None else omega,
                                        self.st.ng if ng is None else ng, C.byref(self.P),
                                        C.byref(k), C.byref(ktot), C.byref(res), self._s()),
              "pdesolver")
        self.mg_last = (k.value, ktot.value, res.value)
        return self.mg_last

    def pdesolver_mixed(self, eps=None, ng=None, **kw):
        """FP32 V-cycles inside FP64 refinement; returns (refinements, 0, res)
        (None in nonblocking mode: see mg_last)."""
        wl = self.st.wl
        m = dict(self.mg_mixed)
        m.update(kw)
        if self.nonblocking:
            self._pdesolver_mixed_nowait(eps, ng, m)
            return None
        it = C.c_int(0)
        res = C.c_double(0)
        check(lib().lepic_dev_pdesolver_mixed(C.byref(self.grid), _ptr(self.phi), _ptr(self.rhs),
                                              wl.eps if eps is None else eps, m["omega"],
                                              self.st.ng if ng is None else ng, C.byref(self.P),
                                              m["max_refine"], m["nu_fine_pre"], m["nu_fine_post"],
                                              m["nu_pre"], m["nu_post"], m["coarse_sweeps"],
                                              C.byref(it), C.byref(res),
                                              self._s()), "pdesolver_mixed")
        self.mg_last = (it.value, 0.0, res.value)
        return self.mg_last

    def _pdesolver_mixed_nowait(self, eps, ng, m):
        """The mixed solve without a wait; its refinements and residual go to
        slot (count mod ring) of the pinned history."""
        wl = self.st.wl
        if self._mg_it is None:
            self._mg_it = torch.zeros(self._mg_ring, dtype=torch.int32).pin_memory()
            self._mg_res = torch.zeros(self._mg_ring, dtype=torch.float64).pin_memory()
        check(lib().lepic_dev_pdesolver_mixed(C.byref(self.grid), _ptr(self.phi), _ptr(self.rhs),
                                              wl.eps if eps is None else eps, m["omega"],
                                              self.st.ng if ng is None else ng, C.byref(self.P),
                                              m["max_refine"], m["nu_fine_pre"], m["nu_fine_post"],
                                              m["nu_pre"], m["nu_post"], m["coarse_sweeps"],
                                              None, None, self._s()), "pdesolver_mixed")
        k = self._mg_count % self._mg_ring
        check(lib().lepic_dev_pdesolver_mixed_stats(C.c_void_p(self._mg_it[k:].data_ptr()),
                                                    C.c_void_p(self._mg_res[k:].data_ptr()), self._s()),
              "pdesolver_mixed_stats")
        self._mg_count += 1
        self._mg_last_sync = None

    @property
    def mg_last(self):
        """(refinements or V-cycles, ktot, residual) of the last solve; in
        nonblocking mode reading it waits for the stream."""
        if self._mg_last_sync is None and self._mg_count:
            self.stream.synchronize()
            k = (self._mg_count - 1) % self._mg_ring
            self._mg_last_sync = (int(self._mg_it[k]), 0.0, float(self._mg_res[k]))
        return self._mg_last_sync

    @mg_last.setter
    def mg_last(self, v):
        self._mg_last_sync = v

    def solve_history(self, n):
        """Refinements of the last n nonblocking mixed solves (waits for the
        stream)."""
        self.stream.synchronize()
        n = min(n, self._mg_count, self._mg_ring)
        idx = [(self._mg_count - n + j) % self._mg_ring for j in range(n)]
        return [int(self._mg_it[k]) for k in idx]

    def efield(self):
        check(lib().lepic_dev_calc_efield(C.byref(self.grid), _ptr(self.phi), _ptr(self.Ei),
                                          self._s()), "calc_efield")
        if self.mixed:
            self.pack_e32()

    def pack_e32(self):
        """FP32 copy of the current E (one float4 per node) for the mixed push."""
        check(lib().lepic_dev_pack_e32(_ptr(self.Ei), _ptr(self.E32), C.c_longlong(self.Ei.numel() // 3),
                                       self._s()), "pack_e32")

    def sort(self, species=None):
        """Counting sort by cell of the given species (0-based; all by default)."""
        todo = [self.sp[p] for p in (range(len(self.sp)) if species is None else species)]
        if self.mixed:
            for s in todo:
                check(lib().lepic_dev_sort_mixed(C.byref(self.grid), C.byref(s.s), -1,
                                                 self._s()), "sort_mixed")
                s.after_call()
            return
        pl_max = self.st.n[0] + self.st.n[0] * (self.st.n[1] + self.st.n[1] * self.st.n[2]) + 1
        if not hasattr(self, "_plist_sp"):
            # per-species cell offsets (Plist) of the last sort
            self._plist_sp = [torch.zeros(pl_max + 1, dtype=torch.int32, device=self.dev) for _ in self.sp]
        for s in todo:
            q = self.sp.index(s)
            check(lib().lepic_dev_part_sorting(C.byref(self.grid), C.byref(s.s), _ptr(self._plist_sp[q]),
                                               pl_max, self._s()), "part_sorting")
            s.after_call()

    def collisions(self):
        if self._tables is None:
            return
        nu = (C.c_double * 10)()
        cnt = (C.c_longlong * 64)()
        tg = self._targets
        if tg is not None:
            # dens_red before the collisions (Src/main.f90:1194): np_mx of the
            # charged species for nu_max; the density grids and the offsets of
            # the target species' sort of this step
            mx = (C.c_double * 10)()
            check(lib().lepic_dev_dens_red(C.byref(self.grid), _ptr(self.np), None, self.st.ntype, mx,
                                           self._s()), "dens_red")
            for q in range(self.st.ntype):
                self.P.np_mx[q] = mx[q]
            for q in self.dsmc_targets:
                tg.np[q] = self.np[q].data_ptr()
                tg.cell_off[q] = (self.sp[q].cell_off.data_ptr() if self.mixed else self._plist_sp[q].data_ptr())
        if self.mixed:
            arr = (LepicSpeciesMixed * len(self.sp))(*[s.s for s in self.sp])
            fn, name = lib().lepic_dev_collisions_mixed, "collisions_mixed"
            if tg is not None:
                fn, name = lib().lepic_dev_collisions_mixed_targets, "collisions_mixed_targets"
        else:
            arr = (LepicSpeciesF64 * len(self.sp))(*[s.s for s in self.sp])
            fn, name = lib().lepic_dev_collisions, "collisions"
            if tg is not None:
                fn, name = lib().lepic_dev_collisions_targets, "collisions_targets"
        args = [C.byref(self.grid), arr, len(self.sp), C.byref(self._tables), C.byref(self.P),
                C.c_ulonglong(self.seed), C.c_ulonglong(self.it), nu, cnt]
        if tg is not None:
            args.append(C.byref(tg))
        check(fn(*args, self._s()), name)
        self.counts[:64] += np.array(cnt[:], dtype=np.int64)
        self.nu_max[:] = nu[:]

    def move(self):
        pm = np.zeros((self.st.geom.ngrid + 1, 2, self.st.ntype))
        pl = np.zeros((self.st.ntype, 4))
        for p, s in enumerate(self.sp):
            if self.st.charge[p] == 0.0:
                continue
            check(lib().lepic_dev_part_mover(C.byref(self.grid), _ptr(self.Ei), C.byref(s.s), p + 1,
                                             self.st.ntype, self.st.geom.ngrid, C.byref(self.P),
                                             pm.ctypes.data_as(_lib.P_dbl),
                                             pl.ctypes.data_as(_lib.P_dbl), self._s()), "part_mover")
        self.p_mac += pm
        self.P_loss += pl

    def deposit(self):
        if self.mixed:
            raise RuntimeError("the mixed form deposits inside the fused push (move_deposit)")
        self._deposit_f64(self.sp)

    def _deposit_f64(self, sps):
        self.np.zero_()
        for p, s in enumerate(sps):
            check(lib().lepic_dev_charge_deposition(C.byref(self.grid), C.byref(s.s), p + 1,
                                                    C.byref(self.P), C.c_void_p(self.np[p].data_ptr()),
                                                    self._s()), "charge_deposition")
        self._reduce_density()

    def _reduce_density(self):
        if self.comm is not None:
            allreduce_density(self.np, self._group)

    def move_deposit(self, reduce=True):
        """Fused in-place push + deposition of every species (the step path);
        lost particles are removed by hole filling.  reduce: all-reduce the
        density grids over the ranks (deferred while an injection follows)."""
        st = self.st
        if self._acc is None:
            self._acc = torch.zeros((st.ntype, 2 + 2 * (st.geom.ngrid + 1)), dtype=torch.float64,
                                    device=self.dev)
        # no host read of the counts: the FP64 push launches over the capacity
        # and its threads read the count on the device; the mixed push walks
        # its tiles and a grid-stride tail
        self.np.zero_()
        for p, s in enumerate(self.sp):
            if st.charge[p] == 0.0:
                continue
            if self.mixed:
                check(lib().lepic_dev_push_deposit_mixed(
                    C.byref(self.grid), _ptr(self.E32), C.byref(s.s), p + 1, st.geom.ngrid,
                    C.byref(self.P), C.c_void_p(self.np[p].data_ptr()),
                    C.c_void_p(self._acc[p].data_ptr()), -1, self._s()),
                    "push_deposit_mixed")
                continue
            check(lib().lepic_dev_push_deposit(C.byref(self.grid), _ptr(self.Ei), C.byref(s.s), p + 1,
                                               st.geom.ngrid, C.byref(self.P),
                                               C.c_void_p(self.np[p].data_ptr()),
                                               C.c_void_p(self._acc[p].data_ptr()), -1,
                                               self._s()), "push_deposit")
        if reduce:
            self._reduce_density()

    def loss_stats(self):
        """(p_mac (ngrid+1, 2, ntype), P_loss (ntype, 4)) accumulated so far."""
        pm = self.p_mac.copy()
        pl = self.P_loss.copy()
        if self._acc is not None:
            a = self._acc.cpu().numpy()
            ng1 = self.st.geom.ngrid + 1
            for p in range(self.st.ntype):
                pl[p, 0] += a[p, 0]
                pl[p, 2] += a[p, 1]
                pm[:, 0, p] += a[p, 2:2 + 2 * ng1:2]
                pm[:, 1, p] += a[p, 3:3 + 2 * ng1:2]
        return pm, pl

    def step(self):
        """One timestep in the reference's order (Src/main.f90:853-1277)."""
        self.it += 1
        it = self.it
        self.calc_rho()
        if self.die is not None:
            self.dielectric_phi()
        self.pdesolver()
        self.efield()
        due = [p for p, k in enumerate(self.sort_every) if k and it % k == 1 % k]
        mcc = self._tables is not None and it > 1 and it % self.ns_coll == 1 % self.ns_coll
        if mcc and self._targets is not None:
            # charged targets are picked from the cells of this step's sort
            due = sorted(set(due) | set(self.dsmc_targets))
        if due:
            self.sort(due)
        if mcc:
            self.collisions()
        hp = self.heat_params if self.heat is not None else None
        if hp is not None and hp["flag_heat"] and it % hp["ns_heat"] == 0:
            self.eheating()
        inj_due = self.inj is not None and it % max(int(self.inj.ns_inj), 1) == 0
        if self.fused:
            self.move_deposit(reduce=not inj_due)
        else:
            self.move()
            self.deposit()
        if inj_due:
            self.inject()
            if self.fused:
                self._reduce_density()
        if hp is not None and self.heat.Pabs > 0 and (it + 1) % hp["ns_heat"] == 0:
            self.heat_stats()
        if self.check_every and it % self.check_every == 0:
            self.check_device()

    # ---------------------------------------------------------- injection
    def inject(self):
        """Src/part_injection.f90 after the push; the new particles are
        deposited into the density grids as well (the fused push has already
        deposited the others).  opt_inj 2: as many events as ions were lost to
        the walls since the last injection."""
        st = self.st
        nev = -1
        if abs(int(self.inj.opt_inj)) == 2:
            pm, _ = self.loss_stats()
            lost = float(pm[:, 0, 1].sum()) if st.ntype > 1 else 0.0
            nev = int(round(lost - self._inj_lost_seen))
            self._inj_lost_seen = lost
        pl4 = (C.c_double * 10)()
        got = (C.c_longlong * 10)()
        nps = (C.c_void_p * 10)(*[self.np[p].data_ptr() for p in range(st.ntype)])
        if self.mixed:
            arr = (LepicSpeciesMixed * len(self.sp))(*[s.s for s in self.sp])
            fn = lib().lepic_dev_inject_mixed
        else:
            arr = (LepicSpeciesF64 * len(self.sp))(*[s.s for s in self.sp])
            fn = lib().lepic_dev_inject
        check(fn(C.byref(self.grid), arr, st.ntype, C.byref(self.P), C.byref(self._I), nev,
                 C.c_ulonglong(self.seed ^ 0x696E6A), C.c_ulonglong(self._inj_calls), nps, _ptr(self.phi), pl4, got,
                 self._s()), "inject")
        self._inj_calls += 1
        for p in range(st.ntype):
            self.P_loss[p, 3] += pl4[p]
            self.injected[p] += got[p]

    # ------------------------------------------------------------ heating
    def heat_stats(self):
        """Kinetic energy and number of the electrons in the heating region
        after the push (Src/part_expmover.f90:658-681), for the next heating
        step's self-consistent temperature."""
        self._heat_stats.zero_()
        s = self.sp[0]
        fn = lib().lepic_dev_heat_stats_mixed if self.mixed else lib().lepic_dev_heat_stats
        check(fn(C.byref(self.grid), C.byref(s.s), C.byref(self.P), C.byref(self._H),
                 _ptr(self._heat_stats), self._s()), "heat_stats")
        self._heat_stats_ok = True

    def eheating(self):
        """Src/part_expmover.f90:484-568 on the electrons: thermal speed vt0 of
        the electrons, or with Pabs > 0 the self-consistent one of
        Src/main.f90:1224-1226 from the last statistics (computed on the
        device)."""
        s = self.sp[0]
        use_stats = self.heat.Pabs > 0 and self._heat_stats_ok and not self.heat.flag_inj
        fn = lib().lepic_dev_eheating_mixed if self.mixed else lib().lepic_dev_eheating
        check(fn(C.byref(self.grid), C.byref(s.s), C.byref(self.P), C.byref(self._H), float(self.st.vt0[0]),
                 _ptr(self._heat_stats) if use_stats else None, C.c_ulonglong(self.seed ^ 0x68656174),
                 C.c_ulonglong(self._heat_calls), _ptr(self._heat_acc), self._s()), "eheating")
        self._heat_calls += 1

    def heating_totals(self):
        """(energy added by heating so far (J, P_loss(2) of the electrons),
        electrons heated so far, thermal speed of the last heating call)."""
        a = self._heat_acc.cpu().numpy()
        return float(a[0]), int(a[1]), float(a[2])

    def check_device(self):
        """Read and clear the device error word; raise LepicError when a
        kernel recorded a status since the last read.  In nonblocking mode
        the word is snapshotted into pinned memory without a wait and the
        previous snapshot is read if the stream has passed it."""
        if self.nonblocking:
            if self._err_host is None:
                self._err_host = torch.zeros(2, dtype=torch.int32).pin_memory()
                self._err_ev = torch.cuda.Event()
            if self._err_pending:
                if not self._err_ev.query():
                    return
                self._err_pending = False
                rc, det = int(self._err_host[0]), int(self._err_host[1])
                if rc:
                    check(rc, f"device status at or before step {self.it} (detail {det})")
            check(lib().lepic_dev_check_async(self._s(), C.c_void_p(self._err_host.data_ptr())),
                  "check_async")
            self._err_ev.record(self.stream)
            self._err_pending = True
            return
        detail = C.c_int(0)
        rc = lib().lepic_dev_check(self._s(), C.byref(detail))
        if rc:
            check(rc, f"device status after step {self.it} (detail {detail.value})")

    def flush_checks(self):
        """Nonblocking mode: wait for the last snapshot of the error word and
        read it, then read the word itself."""
        if self._err_pending:
            self._err_ev.synchronize()
            self._err_pending = False
            rc, det = int(self._err_host[0]), int(self._err_host[1])
            if rc:
                check(rc, f"device status at or before step {self.it} (detail {det})")
        detail = C.c_int(0)
        rc = lib().lepic_dev_check(self._s(), C.byref(detail))
        if rc:
            check(rc, f"device status after step {self.it} (detail {detail.value})")

    def step_host(self, potentials=None, phi_out=None, counts_out=None):
        """One step with host input and output, pipelined.  `potentials`
        (FP64, one value per wall label 0..ngrid+1, pinned host memory) are
        copied in and set on the wall nodes before the step; after it phi and
        the particle counts are snapshotted on the device and copied into the
        pinned host tensors `phi_out` (the shape of the node grid) and
        `counts_out` (one int32 per species) on a separate copy stream, so
        the copy overlaps the next step.  Returns the CUDA event after which
        `phi_out` and `counts_out` hold this step's values (and may be
        reused); two steps may be in flight."""
        if potentials is not None:
            if getattr(self, "_wall", None) is None:
                nl = int(self.st.geom.ngrid)
                self._label = self.bcnd.long().clamp(0, nl + 1)
                self._wall = self.bcnd >= 1
            v = potentials.to(self.dev, non_blocking=True)
            torch.where(self._wall, v[self._label], self.phi, out=self.phi)
        self.step()
        done = torch.cuda.Event()
        if phi_out is None and counts_out is None:
            done.record(self.stream)
            return done
        if getattr(self, "_io", None) is None:
            self._io = [(torch.empty_like(self.phi), torch.empty(len(self.sp), dtype=torch.int32, device=self.dev),
                         None) for _ in range(2)]
            self._io_slot = 0
            self._copy_stream = torch.cuda.Stream(self.dev)
        slot = self._io_slot
        self._io_slot ^= 1
        snap_phi, snap_cnt, prev = self._io[slot]
        if prev is not None:
            self.stream.wait_event(prev)  # the copy of two steps ago has read this snapshot
        snap_phi.copy_(self.phi)
        torch.cat([sp.count for sp in self.sp], out=snap_cnt)
        ready = torch.cuda.Event()
        ready.record(self.stream)
        self._copy_stream.wait_event(ready)
        with torch.cuda.stream(self._copy_stream):
            if phi_out is not None:
                phi_out.copy_(snap_phi, non_blocking=True)
            if counts_out is not None:
                counts_out.copy_(snap_cnt, non_blocking=True)
            done.record(self._copy_stream)
        snap_phi.record_stream(self._copy_stream)
        snap_cnt.record_stream(self._copy_stream)
        self._io[slot] = (snap_phi, snap_cnt, done)
        return done

    def counts_host(self):
        return np.array([s.n() for s in self.sp])
