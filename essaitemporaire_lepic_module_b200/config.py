"""Synthetic workloads of the PIC-MCC benchmark and their derived constants.

Each workload mirrors what the reference derives from ``conditions.inp``,
``geometry.inp``, ``boundary.inp`` and the chemistry file in Src/main.f90:
thermal velocities ``vt0 = sqrt(2 q T / m)`` and macroparticle weights
``Nm = n0 h1 h2 h3 / np_cell`` (Src/main.f90:535-548), the multigrid level
count ``ng = log2(min n)`` for power-of-two grids (Src/main.f90:243-260), the
loaded-cell count (Src/main.f90:637-648), the collision frequency caps
``nu_uplim`` (Src/main.f90:565-566) and the cadences ``nsort = ns_coll = 10``
(Src/main.f90:550-551).  The time step is given directly instead of through
``kt`` so that every consumer sees the same double.

Workloads (sizes from the benchmark definition; ``*_small`` are the same
set-ups shrunk so the FP64 CPU oracle finishes in seconds):
  box32      32^3 cells, e- + Ar+ 16 ppc, walls 0 V, no B, no collisions
  mcc128     128^3 cells, e- + Ar+ 64 ppc, Bz = 0.01 T, Ar 1 Pa / 300 K MCC
             (mcc96, mcc64, mcc32, mcc16: the same on smaller grids, for
             profiling captures and tests)
  poisson256 256^3 grid, two 16^3 electrodes at +-100 V, 64 Gaussian blobs
             (poisson128, poisson64, poisson32: the same on smaller grids)
  penning    96x96x192 cells, e- 32 ppc, Bz = 0.1 T, end plates +200 V
             (electrode labels 2 and 3), side walls 0 V (label 1)
  mcc192     192^3 cells, e- + Ar+ 128 ppc (mixed precision only)
  pbc16      16^3 cells, e- + Ar+ 16 ppc, walls at both x ends, periodic
             planes in y and z (pbc32x16: 32 cells in x)
  nmn16      the same with the Neumann (symmetry) plane at x = 0
  dsmc16     16^3 box, e- + Ar+ 16 ppc, e-Ar+ elastic collisions with
             charged targets (dsmcar16: with the Ar MCC as well; dsmc32:
             32^3 box, 40 ppc and a cross section 20 times larger, about
             1e5 collisions per call, several on one ion in many cells)
"""
from __future__ import annotations

import math
import os
import tempfile
from dataclasses import dataclass, field

import numpy as np

from . import reactions as rx
from .constants import AMU, EPS0, KB, ME, PI, QE
from .geometry import count_cells, generate_boundary

NPART = 10


@dataclass
class Workload:
    name: str
    n: tuple
    dx: float                       # m (cubic cells)
    segments: list                  # geometry.inp rows in cm (box filled in)
    V: list                         # wall potentials, V[0] unused
    ions: list                      # [(name, mass_amu, charge_e, T_eV, n/n0)]
    Te: float
    n0: float
    ppc: int
    dt: float
    steps: int
    B: tuple = (0.0, 0.0, 0.0)
    gas_pressure: float = 0.0       # Pa (0: collisionless)
    gas_T: float = 300.0            # K
    eps: float = 1e-10
    omega: float = 1.4
    ng: int = 0                     # 0: log2(min n) for power-of-two grids
    ns_coll: int = 10
    nsort: int = 10
    ncycl: int = 20000
    blobs: int = 0                  # Poisson-only source: number of Gaussian blobs
    blob_seed: int = 3
    mixed_only: bool = False
    neumann_x: bool = False         # x = 0 is a Neumann (symmetry) plane
    coulomb: float = 0.0            # > 0: e-Ar+ elastic (charged target, DSMC) of this sigma0 (m^2)
    Ca: float = 0.0                 # capacitance of the dielectric walls, F/m^2


def _box(n, dx):
    return [0.0, 0.0, 0.0, n[0] * dx * 100.0, n[1] * dx * 100.0, n[2] * dx * 100.0]


def _ar_ion(T=0.026):
    return [("[Ar+]", 39.95, 1.0, T, 1.0)]


def workload(name: str) -> Workload:
    """Return one of the named workloads."""
    if name in ("box32", "box16"):
        n = (32, 32, 32) if name == "box32" else (16, 16, 16)
        return Workload(name, n, 1e-4, [_box(n, 1e-4) + [1]], [0.0, 0.0], _ar_ion(),
                        Te=2.0, n0=1e15, ppc=16, dt=2e-11, steps=200)
    if name in ("mcc128", "mcc32", "mcc64", "mcc96", "mcc16"):
        n = {"mcc128": (128,) * 3, "mcc32": (32,) * 3, "mcc64": (64,) * 3, "mcc96": (96,) * 3, "mcc16": (16,) * 3}[name]
        return Workload(name, n, 1e-4, [_box(n, 1e-4) + [1]], [0.0, 0.0], _ar_ion(),
                        Te=2.0, n0=1e15, ppc=64 if name != "mcc32" else 32, dt=2e-11, steps=500,
                        B=(0.0, 0.0, 0.01), gas_pressure=1.0, gas_T=300.0)
    if name in ("dsmc16", "dsmcar16", "dsmc32"):
        # e-Ar+ elastic collisions with charged targets (dsmcar16: on top of
        # the Ar MCC of mcc128; dsmc32: dense, nu_max at its cap nu_uplim)
        n = (32, 32, 32) if name == "dsmc32" else (16, 16, 16)
        return Workload(name, n, 1e-4, [_box(n, 1e-4) + [1]], [0.0, 0.0], _ar_ion(),
                        Te=2.0, n0=1e15, ppc=40 if name == "dsmc32" else 16, dt=2e-11, steps=200,
                        B=(0.0, 0.0, 0.01), gas_pressure=1.0 if name == "dsmcar16" else 0.0, gas_T=300.0,
                        coulomb=4e-12 if name == "dsmc32" else 2e-13)
    if name in ("pbc16", "pbc32x16", "nmn16"):
        # walls at both x ends (nmn16: the Neumann plane at x = 0 instead),
        # periodic planes in y and z (a box segment, then label 0 over it)
        n = {"pbc16": (16, 16, 16), "pbc32x16": (32, 16, 16), "nmn16": (16, 16, 16)}[name]
        return Workload(name, n, 1e-4, [_box(n, 1e-4) + [1], _box(n, 1e-4) + [0]], [0.0, 0.0], _ar_ion(),
                        Te=2.0, n0=1e15, ppc=16, dt=2e-11, steps=200, neumann_x=(name == "nmn16"))
    if name == "die16":
        # metal box plus two dielectric walls: the y = ymax plane (label 2,
        # a Y = const dielectric) and the x = xmax plane (label 3, the first
        # X = const dielectric)
        n = (16, 16, 16)
        box = _box(n, 1e-4)
        X, Y, Z = box[3], box[4], box[5]
        seg = [box + [1], [0.0, Y, 0.0, X, -Y, Z, -2], [X, 0.0, 0.0, -X, Y, Z, -3]]
        return Workload(name, n, 1e-4, seg, [0.0, 0.0, 0.0, 0.0], _ar_ion(), Te=2.0, n0=1e15, ppc=16,
                        dt=2e-11, steps=200, Ca=2e-8)
    if name in ("mcc192",):
        n = (192, 192, 192)
        return Workload(name, n, 1e-4, [_box(n, 1e-4) + [1]], [0.0, 0.0], _ar_ion(),
                        Te=2.0, n0=1e15, ppc=128, dt=2e-11, steps=500,
                        B=(0.0, 0.0, 0.01), gas_pressure=1.0, gas_T=300.0, mixed_only=True)
    if name in ("poisson256", "poisson128", "poisson64", "poisson32"):
        m = {"poisson256": 256, "poisson128": 128, "poisson64": 64, "poisson32": 32}[name]
        n = (m, m, m)
        dxc = 1e-4 * 100.0
        e = 16 * m // 256 if m >= 128 else max(m // 16, 2)
        c1, c2 = m // 3, 2 * m // 3
        seg = [_box(n, 1e-4) + [1]]
        for (cx, lab) in ((c1, 2), (c2, 3)):
            lo = (cx - e // 2 + 0.5) * dxc
            hi = (cx + e // 2 + 0.5) * dxc
            mid_lo = (m // 2 - e // 2 + 0.5) * dxc
            mid_hi = (m // 2 + e // 2 + 0.5) * dxc
            seg.append([lo, mid_lo, mid_lo, hi, mid_hi, mid_hi, -lab])
        return Workload(name, n, 1e-4, seg, [0.0, 0.0, 100.0, -100.0], [], Te=2.0, n0=1e15, ppc=0,
                        dt=2e-11, steps=1, blobs=64)
    if name in ("penning", "penning_small"):
        n = (96, 96, 192) if name == "penning" else (16, 16, 32)
        box = _box(n, 1e-4)
        X, Y, Z = box[3], box[4], box[5]
        # end plates as separate electrodes (labels 2 at z = 0 and 3 at z = zmax)
        # so that each has its own voltage parameter
        seg = [box + [1], [0.0, 0.0, 0.0, X, Y, 0.0, -2], [0.0, 0.0, Z, X, Y, Z, -3]]
        return Workload(name, n, 1e-4, seg, [0.0, 0.0, 200.0, 200.0], [], Te=5.0, n0=1e15, ppc=32,
                        dt=1e-11, steps=64, B=(0.0, 0.0, 0.1), ng=6 if name == "penning" else 5)
    raise KeyError(name)


@dataclass
class Setup:
    """Everything the hot path needs, derived like the reference does."""
    wl: Workload
    geom: object
    n: tuple
    h: np.ndarray
    ntype: int
    n_neu: int
    names: list
    charge: np.ndarray
    mass: np.ndarray
    Ti: np.ndarray
    vt0: np.ndarray
    Nm: np.ndarray
    np_mx: np.ndarray
    nu_uplim: np.ndarray
    ni0: np.ndarray
    dt: float
    x_load: float
    n_cell: int
    np_cell: int
    ng: int
    flag_B: int
    Bconst: np.ndarray
    kq: np.ndarray
    tables: object = None           # reactions.Tables or None (collisionless)
    ngas: float = 0.0
    rhs_blobs: np.ndarray = None    # Poisson-only source (-rho), (n3+2, n2+2, n1+2)
    extra: dict = field(default_factory=dict)
    bfield: object = None           # bfield.BField (a B-field map) or None (uniform Bconst)
    flag_B_pos: int = 0             # 1: positive ions not magnetised
    Ca: float = 0.0                 # dielectric walls: capacitance per cell (F), Src/main.f90:572

    @property
    def ncells(self):
        return int(self.n[0] * self.n[1] * self.n[2])

    def n_particles(self, ptype=1):
        """Expected number loaded per species (all ni0 = 1)."""
        return int(round(float(np.float32(self.np_cell * self.n_cell))))


@dataclass
class Heating:
    """Maxwellian electron heating (Src/read_input.f90:37, 72-74): the region
    xl_pow..xr_pow in x (m), the absorbed power Pabs (W; <= 0: no
    self-consistent temperature, the heating speed stays vt0 of the
    electrons) and the heating frequency nu_h (1/s; < 0: no heating); with
    flag_circxh the region is also limited to r <= R_ahp (flag_ahp = 0) or
    r >= R_ahp (flag_ahp = 1) about the box axis."""
    xl_pow: float
    xr_pow: float
    Pabs: float = -1.0
    nu_h: float = 1.0e7
    flag_circxh: int = 0
    flag_ahp: int = 0
    R_ahp: float = 0.0
    flag_inj: int = 0


@dataclass
class Injection:
    """Particle injection (Src/read_input.f90:75, Src/part_injection.f90):
    opt_inj 1 (uniform in the box xl..zr, m), -1 (cosine / flat-top profile),
    2 (as many events as ions lost to the walls), +-3 (electron beam of energy
    THm eV), +-4 (cathode emission at the planes zg_sec); I_inj the injected
    current (A); every ns_inj steps; ni0: the probability that an event
    injects each species (default: the set-up's n/n0)."""
    opt_inj: int
    I_inj: float
    xl: float
    xr: float
    yl: float
    yr: float
    zl: float
    zr: float
    ns_inj: int = 1
    THm: float = 0.0
    zg_sec: tuple = (0.0, 0.0)
    n_cath: int = 1
    dir_sec: int = 1
    tag_beam: int = 0
    ni0: tuple = None


def heating_params(st, hz):
    """What Src/main.f90 derives from the heating input: ns_heat from
    kt = dt vt0(1) / min(h) (:548-554), nudt = nu_h ns_heat dt (:564), the
    cell range ixl_pow..ixr_pow (:610-614) and flag_heat (nu_h >= 0)."""
    kt = st.dt * st.vt0[0] / float(min(st.h))
    ns_heat = 4
    if 0.05 <= kt < 0.1:
        ns_heat = 20
    if kt < 0.05:
        ns_heat = 40
    xmax = float(st.geom.box[0])
    xr = min(hz.xr_pow, xmax)
    xl = max(hz.xl_pow, 0.0)
    return dict(ns_heat=ns_heat, nudt=hz.nu_h * ns_heat * st.dt, ixl_pow=int(xl / st.h[0]) + 1,
                ixr_pow=int(xr / st.h[0]) + 1, flag_heat=0 if hz.nu_h < 0 else 1)


def mg_levels(n, ng_default):
    a = [math.log10(float(np.float32(v))) / math.log10(2.0) for v in n]
    if all(abs(round(x) - x) <= 1e-3 for x in a):
        return int(round(min(a)))
    for v in n:
        if v % (2 ** (ng_default - 1)):
            raise ValueError("Incorrect number of grid levels in MG")
    return ng_default


def build(wl: Workload | str, chem=None) -> Setup:
    """The set-up of a workload; chem: a reactions.Chemistry that replaces
    the workload's own species and reactions (e.g. a chemistry file of the
    reference read with reactions.read_dat)."""
    if isinstance(wl, str):
        wl = workload(wl)
    n = tuple(wl.n)
    segs = [list(s) for s in wl.segments]
    box = list(segs[0][3:6])
    if wl.neumann_x:
        box[0] = -box[0]            # a negative xmax selects the Neumann plane
    geom = generate_boundary(n, box, segs, wl.V)
    h = geom.h.copy()
    ngas = 0.0
    if wl.gas_pressure > 0:
        ngas = wl.gas_pressure / (KB * wl.gas_T)
    neutrals = []
    if ngas > 0:
        neutrals = [("[Ar]", -39.95, 0.0, KB * wl.gas_T / QE, 1.0)]
    reacts = rx.argon_tables_synthetic() if ngas > 0 else []
    if wl.coulomb > 0:
        reacts = [rx.coulomb_table_synthetic(wl.coulomb)] + reacts
    if chem is None:
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "chem.dat")
            rx.write_dat(path, wl.ions, neutrals, reacts)
            chem = rx.read_dat(path, wl.Te, ngas)
    ntype = chem.ntype
    n_neu = chem.n_neu
    charge = np.zeros(NPART)
    mass = np.zeros(NPART)
    Ti = np.zeros(NPART)
    ni0 = np.zeros(NPART)
    names = []
    for i, s in enumerate(chem.species):
        charge[i], mass[i], Ti[i], ni0[i] = s.charge, s.mass, s.T, s.ni0
        names.append(s.name)
    vt0 = np.zeros(NPART)
    Nm = np.zeros(NPART)
    np_cell = wl.ppc
    for p in range(ntype + n_neu):
        vt0[p] = math.sqrt(2.0 * QE * Ti[p] / abs(mass[p]))
        if abs(charge[p]) > 0:
            Nm[p] = wl.n0 * h[0] * h[1] * h[2] / abs(np_cell) if np_cell else 0.0
        else:
            Nm[p] = ngas * h[0] * h[1] * h[2] / abs(np_cell) if np_cell else 0.0
    np_mx = np.zeros(NPART)
    np_mx[ntype:ntype + n_neu] = ni0[ntype:ntype + n_neu]
    nu_uplim = np.zeros(NPART)
    nu_uplim[0] = 5e8
    nu_uplim[1:ntype] = 1e7
    x_load = float(geom.box[0])
    ix_pe = int(x_load / h[0]) + 1
    n_cell = count_cells(geom.bcnd, n, min(ix_pe, n[0] + 1))
    ng = mg_levels(n, wl.ng or 6)
    kq = np.where(geom.bcnd != -1, 2.0, 1.0)
    tables = rx.ordering(chem) if len(chem.tables) else None
    st = Setup(wl=wl, geom=geom, n=n, h=h, ntype=ntype, n_neu=n_neu, names=names, charge=charge,
               mass=mass, Ti=Ti, vt0=vt0, Nm=Nm, np_mx=np_mx, nu_uplim=nu_uplim, ni0=ni0,
               dt=wl.dt, x_load=x_load, n_cell=n_cell, np_cell=np_cell, ng=ng,
               flag_B=1 if any(b != 0.0 for b in wl.B) else 0,
               Bconst=np.array(wl.B, dtype=np.float64), kq=kq, tables=tables, ngas=ngas)
    if wl.blobs:
        st.rhs_blobs = gaussian_blobs(n, h, wl.blobs, wl.blob_seed)
    if geom.flag_die:
        st.Ca = wl.Ca * h[0] * h[2]     # Farads per grid cell (Src/main.f90:572)
    return st


def gaussian_blobs(n, h, nblobs, seed):
    """-rho of a sum of Gaussian charge blobs (seeded centres, widths 2-8
    cells, amplitudes uniform in +-1e16 e/m^3), on the rhs grid (0:n+1)^3."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n1, n2, n3 = n
    cx = rng.uniform(0, n1, nblobs)
    cy = rng.uniform(0, n2, nblobs)
    cz = rng.uniform(0, n3, nblobs)
    sg = rng.uniform(2.0, 8.0, nblobs)
    amp = rng.uniform(-1e16, 1e16, nblobs)
    z = np.arange(n3 + 2) - 1.0
    y = np.arange(n2 + 2) - 1.0
    x = np.arange(n1 + 2) - 1.0
    rho = np.zeros((n3 + 2, n2 + 2, n1 + 2))
    for k in range(nblobs):
        gz = np.exp(-((z - cz[k]) ** 2) / (2 * sg[k] ** 2))
        gy = np.exp(-((y - cy[k]) ** 2) / (2 * sg[k] ** 2))
        gx = np.exp(-((x - cx[k]) ** 2) / (2 * sg[k] ** 2))
        rho += amp[k] * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    rhs = -QE * rho
    rhs[0, :, :] = rhs[:, 0, :] = 0.0
    rhs[:, :, 0] = 0.0
    return np.ascontiguousarray(rhs)
