"""ctypes wrapper of the CPU FP64 oracle -- TEST INFRASTRUCTURE ONLY.

The oracle is the parity checker for the GPU path: a strict-IEEE C++
restatement of the reference's legacy routines (see lepic_oracle.cpp).  Only
tests/, the smoke check and bench.py's CPU-baseline leg use it; the product
package never imports it.

Parity pins: the geometry mask and the E-field stencil are pinned against
the reference's committed output planes (tests/golden/).  The other routines
are "parity unpinned" against the reference's own binary (no Fortran
compiler here) and are pinned by analytic known-answer tests.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liblepic_oracle.so")

P_int = C.POINTER(C.c_int)
P_dbl = C.POINTER(C.c_double)
P_i8 = C.POINTER(C.c_int8)
P_ll = C.POINTER(C.c_longlong)


class OTables(C.Structure):
    _fields_ = [("ncol", C.c_int), ("npt", C.c_int), ("npt_mx", C.c_int),
                ("sig_Er", P_dbl), ("sig", P_dbl), ("sig_Eth", P_dbl), ("col_info", P_int),
                ("sig_list", P_int), ("p_ncol", P_int), ("sigv_mx", P_dbl)]


class OHeat(C.Structure):
    _fields_ = [("ixl_pow", C.c_int), ("ixr_pow", C.c_int), ("flag_circxh", C.c_int), ("flag_ahp", C.c_int),
                ("R_ahp", C.c_double), ("nudt", C.c_double), ("Pabs", C.c_double)]


def _oheat(st, hz):
    from essaitemporaire_lepic_module_b200.config import heating_params
    hp = heating_params(st, hz)
    H = OHeat()
    H.ixl_pow, H.ixr_pow = hp["ixl_pow"], hp["ixr_pow"]
    H.flag_circxh, H.flag_ahp = int(hz.flag_circxh), int(hz.flag_ahp)
    H.R_ahp, H.nudt, H.Pabs = float(hz.R_ahp), hp["nudt"], float(hz.Pabs)
    return H


def eheating(st, S, vt, P_loss, hz):
    """Src/part_expmover.f90:484-568 on species 1 of S (serial ran2 on
    S.iseed); P_loss (ntype, 4); returns the number of electrons heated."""
    h = np.ascontiguousarray(st.h)
    H = _oheat(st, hz)
    nh = C.c_int(0)
    P = ophys(st)
    lib().oracle_eheating(_pd(h), _pd(S.vxp), C.c_int(S.vxp.shape[1]), _pi(S.iseed), _pi(S.np_tot),
                          C.c_double(vt), _pd(P_loss), C.byref(P), C.byref(H), C.byref(nh))
    return nh.value


class OInject(C.Structure):
    _fields_ = [("opt_inj", C.c_int), ("ns_inj", C.c_int), ("n_cath", C.c_int), ("dir_sec", C.c_int),
                ("tag_beam", C.c_int), ("flag_pbcz", C.c_int), ("I_inj", C.c_double),
                ("xl", C.c_double), ("xr", C.c_double), ("yl", C.c_double), ("yr", C.c_double),
                ("zl", C.c_double), ("zr", C.c_double), ("THm", C.c_double), ("zg_sec", C.c_double * 2)]


def part_injection(st, S, inj, phi, P_loss, N_inj_ions=0):
    """Src/part_injection.f90 on S (serial ran2 on S.iseed); P_loss (ntype, 4)."""
    I = OInject()
    I.opt_inj, I.ns_inj, I.n_cath = int(inj.opt_inj), int(inj.ns_inj), int(inj.n_cath)
    I.dir_sec, I.tag_beam, I.flag_pbcz = int(inj.dir_sec), int(inj.tag_beam), int(st.geom.flag_pbcz)
    I.I_inj = float(inj.I_inj)
    I.xl, I.xr, I.yl, I.yr, I.zl, I.zr = (float(v) for v in (inj.xl, inj.xr, inj.yl, inj.yr, inj.zl, inj.zr))
    I.THm = float(inj.THm)
    I.zg_sec[0], I.zg_sec[1] = (float(v) for v in inj.zg_sec)
    n = np.array(st.n, dtype=np.int32)
    h = np.ascontiguousarray(st.h)
    bc = np.ascontiguousarray(st.geom.bcnd, dtype=np.int32)
    ni0 = np.ascontiguousarray(st.ni0 if inj.ni0 is None else np.array(inj.ni0), dtype=np.float64)
    P = ophys(st)
    rc = lib().oracle_part_injection(_pi(n), _pd(h), _pi(bc), _pd(S.vxp), C.c_int(st.ntype),
                                     C.c_int(S.vxp.shape[1]), _pi(S.np_tot), _pi(S.iseed), C.c_int(N_inj_ions),
                                     _pd(P_loss), _pd(np.ascontiguousarray(phi)), _pd(ni0), C.byref(P), C.byref(I))
    if rc:
        raise RuntimeError(f"oracle part_injection status {rc}")


def heat_stats(st, S, hz):
    """Src/part_expmover.f90:658-681: (sum Ek, Nh) of the electrons in the
    heating region."""
    h = np.ascontiguousarray(st.h)
    H = _oheat(st, hz)
    s = C.c_double(0)
    nh = C.c_int(0)
    P = ophys(st)
    lib().oracle_heat_stats(_pd(h), _pd(S.vxp), C.c_int(S.vxp.shape[1]), _pi(S.np_tot), C.byref(P),
                            C.byref(H), C.byref(s), C.byref(nh))
    return s.value, nh.value


def build():
    """Compile the oracle with its Makefile (strict IEEE)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


_L = None


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.oracle_ran2.restype = C.c_double
        L.oracle_ran2.argtypes = [P_int]
        L.oracle_set_threads.restype = C.c_int
        L.oracle_set_threads.argtypes = [C.c_int]
        _L = L
    return _L


def _pd(a):
    return a.ctypes.data_as(P_dbl)


def _pi(a):
    return a.ctypes.data_as(P_int)


def ophys(st):
    """OPhys has the layout of lepic_phys_t; reuse the package's struct."""
    from essaitemporaire_lepic_module_b200._lib import phys_struct
    return phys_struct(st)


def set_threads(n):
    return lib().oracle_set_threads(int(n))


def ran2(seed):
    s = C.c_int(seed)
    r = lib().oracle_ran2(C.byref(s))
    return r, s.value


class State:
    """Particle state in the reference layout: vxp (ntype, nmax, 6)."""

    def __init__(self, st, nmax):
        self.vxp = np.zeros((st.ntype, nmax, 6))
        self.np_tot = np.zeros(st.ntype, dtype=np.int32)
        self.flag_dead = np.zeros((st.ntype, nmax), dtype=np.int8)
        self.np = np.zeros((st.ntype,) + tuple(st.geom.bcnd.shape))
        self.iseed = np.array([123456], dtype=np.int32)
        self.Plist = None          # (ntype, pl_max+1) per-cell offsets of the last sort
        n1, n2, n3 = st.n
        # surface-charge sums of the dielectric walls (sum_q_xz, sum_q_yz) C-order
        self.sum_q = (np.zeros((st.ntype, n3 + 3, n1 + 3)), np.zeros((st.ntype, n3 + 3, n2 + 3, 2)))

    def copy(self):
        o = object.__new__(State)
        o.vxp = self.vxp.copy()
        o.np_tot = self.np_tot.copy()
        o.flag_dead = self.flag_dead.copy()
        o.np = self.np.copy()
        o.iseed = self.iseed.copy()
        o.Plist = None if self.Plist is None else self.Plist.copy()
        o.sum_q = tuple(a.copy() for a in self.sum_q)
        return o


def load_part(st, nmax, seed=123456):
    """Src/load_part.f90 with one thread (seed 123456*iproc, iproc = 1)."""
    S = State(st, nmax)
    S.iseed[0] = seed
    n = np.array(st.n, dtype=np.int32)
    h = np.ascontiguousarray(st.h)
    bc = np.ascontiguousarray(st.geom.bcnd, dtype=np.int32)
    kq = np.ascontiguousarray(st.kq)
    ni0 = np.ascontiguousarray(st.ni0[:st.ntype])
    P = ophys(st)
    rc = lib().oracle_load_part(_pi(n), _pd(h), _pi(bc), _pd(S.np), _pd(S.vxp), C.c_int(st.ntype),
                                C.c_int(nmax), _pd(kq), _pd(ni0), _pi(S.np_tot), _pi(S.iseed),
                                C.byref(P))
    if rc:
        raise RuntimeError(f"oracle load_part status {rc}")
    return S


def calc_rho(st, np_grids):
    n = np.array(st.n, dtype=np.int32)
    rhs = np.zeros((st.n[2] + 2, st.n[1] + 2, st.n[0] + 2))
    bc = np.ascontiguousarray(st.geom.bcnd, dtype=np.int32)
    P = ophys(st)
    lib().oracle_calc_rho(_pi(n), _pd(np_grids), _pd(rhs), _pi(bc), C.c_int(st.ntype), C.byref(P))
    return rhs


def dens_red(st, np_grids):
    n = np.array(st.n, dtype=np.int32)
    red = np.zeros_like(np_grids)
    mx = np.zeros(10)
    bc = np.ascontiguousarray(st.geom.bcnd, dtype=np.int32)
    lib().oracle_dens_red(_pi(n), _pd(np_grids), _pd(red), _pi(bc), C.c_int(st.ntype), _pd(mx))
    return red, mx[:st.ntype]


def pdesolver(st, phi, rhs, eps=None, omega=None, ng=None, ncycl=None):
    wl = st.wl
    eps = wl.eps if eps is None else eps
    omega = wl.omega if omega is None else omega
    ng = st.ng if ng is None else ng
    ncycl = wl.ncycl if ncycl is None else ncycl
    n = np.array(st.n, dtype=np.int32)
    h = np.ascontiguousarray(st.h)
    bc = np.ascontiguousarray(st.geom.bcnd, dtype=np.int32)
    k = C.c_int(0)
    ktot = C.c_double(0)
    res = C.c_double(0)
    P = ophys(st)
    assert phi.flags["C_CONTIGUOUS"]
    rc = lib().oracle_pdesolver(_pd(phi), _pd(np.ascontiguousarray(rhs)), _pi(bc), _pd(h), _pi(n),
                                C.c_int(ncycl), C.c_double(eps), C.c_double(omega), C.byref(k),
                                C.byref(ktot), C.byref(res), C.c_int(ng), C.byref(P))
    if rc:
        raise RuntimeError(f"oracle pdesolver status {rc}")
    return k.value, ktot.value, res.value


def calc_efield(st, phi, Ei=None):
    n = np.array(st.n, dtype=np.int32)
    h = np.ascontiguousarray(st.h)
    bc = np.ascontiguousarray(st.geom.bcnd, dtype=np.int32)
    if Ei is None:
        Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    E = np.ascontiguousarray(Ei).copy()
    lib().oracle_calc_efield(_pi(n), _pd(h), _pd(np.ascontiguousarray(phi)), _pd(E), _pi(bc))
    return E


class OMoverExtra(C.Structure):
    _fields_ = [("tag_neg", C.c_int), ("tag_neu", C.c_int), ("num_grd", C.c_int),
                ("flag_cex", P_int), ("cnt_cex", P_int), ("cnt_dead", P_dbl), ("beam_div", P_dbl),
                ("gam_sec", C.c_double), ("THm", C.c_double), ("zg_sec", C.c_double * 2),
                ("igrid_sec", C.c_int), ("iseed", P_int)]


class MoverExtra:
    """The negative-ion bookkeeping and secondary emission of the mover
    (Src/part_expmover.f90:76, 278-301, 353-400, 416-470): the COMMON values
    and the caller's arrays (flag_cex of the tag_neg species, cnt_cex(3),
    cnt_dead, beam_div(4), the ran2 seed)."""

    def __init__(self, nmax, tag_neg=0, tag_neu=0, num_grd=0, gam_sec=0.0, igrid_sec=0, THm=0.0,
                 zg_sec=(0.0, 0.0), iseed=-1):
        self.flag_cex = np.zeros(nmax, dtype=np.int32)
        self.cnt_cex = np.zeros(3, dtype=np.int32)
        self.cnt_dead = np.zeros(1)
        self.beam_div = np.zeros(4)
        self.iseed = np.array([iseed], dtype=np.int32)
        self.tag_neg, self.tag_neu, self.num_grd = tag_neg, tag_neu, num_grd
        self.gam_sec, self.igrid_sec, self.THm, self.zg_sec = gam_sec, igrid_sec, THm, tuple(zg_sec)

    def copy(self):
        c = MoverExtra(len(self.flag_cex), self.tag_neg, self.tag_neu, self.num_grd, self.gam_sec,
                       self.igrid_sec, self.THm, self.zg_sec, int(self.iseed[0]))
        for a in ("flag_cex", "cnt_cex", "cnt_dead", "beam_div", "iseed"):
            getattr(c, a)[...] = getattr(self, a)
        return c

    def struct(self):
        return OMoverExtra(self.tag_neg, self.tag_neu, self.num_grd, _pi(self.flag_cex), _pi(self.cnt_cex),
                           _pd(self.cnt_dead), _pd(self.beam_div), self.gam_sec, self.THm,
                           (C.c_double * 2)(*self.zg_sec), self.igrid_sec, _pi(self.iseed))


def part_mover(st, Ei, S, p_mac, P_loss, ptype, ngrid=None, sum_q=None, extra=None):
    """sum_q: (sum_q_xz (ntype, n3+3, n1+3), sum_q_yz (ntype, n3+3, n2+3, 2))
    C-order, accumulated for the dielectric walls (flag_die = 1).  extra:
    a MoverExtra (negative ions, secondary emission into species 1)."""
    ngrid = st.geom.ngrid if ngrid is None else ngrid
    n = np.array(st.n, dtype=np.int32)
    h = np.ascontiguousarray(st.h)
    bc = np.ascontiguousarray(st.geom.bcnd, dtype=np.int32)
    P = ophys(st)
    X = extra.struct() if extra is not None else None
    rc = lib().oracle_part_mover(_pi(n), _pd(h), _pd(np.ascontiguousarray(Ei)), _pd(p_mac),
                                 _pd(P_loss), _pd(S.vxp), _pi(bc), C.c_int(S.vxp.shape[1]),
                                 C.c_int(st.ntype), C.c_int(ngrid), S.flag_dead.ctypes.data_as(P_i8),
                                 _pi(S.np_tot), C.c_int(ptype), C.byref(P), *_die_args(st, sum_q),
                                 C.byref(X) if X is not None else None)
    if rc:
        raise RuntimeError(f"oracle part_mover status {rc}")


def _die_args(st, sum_q):
    if sum_q is None or not st.geom.flag_die:
        return (None, None, None)
    qxz, qyz = sum_q
    assert qxz.flags["C_CONTIGUOUS"] and qyz.flags["C_CONTIGUOUS"]
    assert qxz.dtype == np.float64 and qyz.dtype == np.float64
    return (_pi(st.geom.dtype_array()), _pd(qxz), _pd(qyz))   # data_as keeps the array alive


def charge_deposition(st, S, ptype):
    n = np.array(st.n, dtype=np.int32)
    h = np.ascontiguousarray(st.h)
    kq = np.ascontiguousarray(st.kq)
    P = ophys(st)
    lib().oracle_charge_deposition(_pi(n), _pd(h), _pd(S.vxp), C.c_int(S.vxp.shape[1]),
                                   C.c_int(st.ntype), _pd(kq), _pd(S.np), _pi(S.np_tot),
                                   C.c_int(ptype), C.byref(P))


def part_sorting(st, S, ptype):
    n = np.array(st.n, dtype=np.int32)
    h = np.ascontiguousarray(st.h)
    pl_max = st.n[0] + st.n[0] * (st.n[1] + st.n[1] * st.n[2]) + 1
    Plist = np.zeros(pl_max + 1, dtype=np.int32)
    lib().oracle_part_sorting(_pd(S.vxp), C.c_int(S.vxp.shape[1]), C.c_int(st.ntype), _pi(n),
                              _pd(h), _pi(Plist), C.c_int(pl_max), _pi(S.np_tot), C.c_int(ptype))
    return Plist


def tables_struct(T, keep):
    """OTables over the package's reactions.Tables (arrays kept alive in
    `keep`)."""
    ncol, npt = T.sig.shape
    sig = np.ascontiguousarray(T.sig)                      # (ncol, npt) == sig(npt, ncol)
    Er = np.ascontiguousarray(T.sig_Er)
    Eth = np.ascontiguousarray(T.Eth)
    ci = np.ascontiguousarray(T.col_info.T, dtype=np.int32)  # col_info(ncol,10)
    sl = np.ascontiguousarray(T.sig_list.T, dtype=np.int32)  # sig_list(10,ncol)
    pn = np.ascontiguousarray(T.p_ncol, dtype=np.int32)
    sv = np.ascontiguousarray(T.sigv_mx.T)                   # sigv_mx(10,ncol)
    keep.extend([sig, Er, Eth, ci, sl, pn, sv])
    return OTables(ncol, npt, npt, _pd(Er), _pd(sig), _pd(Eth), _pi(ci), _pi(sl), _pi(pn), _pd(sv))


def pl_max_of(st):
    return st.n[0] + st.n[0] * (st.n[1] + st.n[1] * st.n[2]) + 1


def collisions(st, S, err=None, ns_coll=None):
    """Src/collisions.f90 with one thread, after dens_red (Src/main.f90:1194:
    np_mx of the charged species is the maximum of their density over the
    plasma nodes); charged targets (DSMC) are picked with the per-cell
    offsets S.Plist of the last sort.  Returns (nu_max, counts, Nc); err
    (int64[ntype]) counts the incident particles that found no target."""
    keep = []
    T = tables_struct(st.tables, keep)
    n = np.array(st.n, dtype=np.int32)
    h = np.ascontiguousarray(st.h)
    P = ophys(st)
    if ns_coll is not None:
        P.ns_coll = ns_coll          # Pmax = nu_max ns_coll dt (Src/collisions.f90:122)
    _, mx = dens_red(st, S.np)
    for p in range(st.ntype):
        P.np_mx[p] = mx[p]
    nu = np.zeros(10)
    cnt = np.zeros(64, dtype=np.int64)
    Nc = np.zeros(10, dtype=np.int32)
    pl_max = pl_max_of(st)
    if S.Plist is None:
        S.Plist = np.zeros((st.ntype, pl_max + 1), dtype=np.int32)
    if err is None:
        err = np.zeros(st.ntype, dtype=np.int64)
    rc = lib().oracle_collisions(_pd(S.vxp), _pi(n), _pd(h), C.c_int(st.ntype),
                                 C.c_int(S.vxp.shape[1]), C.byref(T), S.flag_dead.ctypes.data_as(P_i8),
                                 _pi(S.np_tot), _pi(S.iseed), C.byref(P), _pd(nu),
                                 cnt.ctypes.data_as(P_ll), _pi(Nc), _pi(S.Plist), C.c_int(pl_max),
                                 _pd(S.np), err.ctypes.data_as(P_ll))
    if rc:
        raise RuntimeError(f"oracle collisions status {rc}")
    return nu[:st.ntype], cnt[:T.ncol], Nc[:st.ntype]


def ordering(chem, npt_mx=4000):
    """Src/read_reactions.f90:ordering in C for a reactions.Chemistry."""
    ncol = len(chem.tables)
    mx = max(len(t[0]) for t in chem.tables) + 1
    E = np.zeros((ncol, mx))
    Sg = np.zeros((ncol, mx))
    npts = np.zeros(ncol, dtype=np.int32)
    for c, (e, s) in enumerate(chem.tables):
        E[c, :len(e)] = e
        Sg[c, :len(s)] = s
        npts[c] = len(e)
    Eth = np.ascontiguousarray(chem.Eth)
    ci = np.ascontiguousarray(chem.col_info.T, dtype=np.int32)
    mass = np.zeros(10)
    for i, s in enumerate(chem.species):
        mass[i] = s.mass
    from essaitemporaire_lepic_module_b200.constants import QE
    sig_Er = np.zeros(npt_mx)
    sig = np.zeros((ncol, npt_mx))
    npt_out = C.c_int(0)
    sl = np.zeros((ncol, 10), dtype=np.int32)
    pn = np.zeros(10, dtype=np.int32)
    sv = np.zeros((ncol, 10))
    rc = lib().oracle_ordering(C.c_int(ncol), _pi(npts), _pd(E), _pd(Sg), C.c_int(mx), _pd(Eth),
                               _pi(ci), _pd(mass), C.c_int(chem.ntype), C.c_double(QE), _pd(sig_Er),
                               _pd(sig), C.c_int(npt_mx), C.byref(npt_out), _pi(sl), _pi(pn), _pd(sv))
    if rc:
        raise RuntimeError(f"oracle ordering status {rc}")
    k = npt_out.value
    return sig_Er[:k], sig[:, :k], sv.T, sl.T, pn


def dielectric_phi(st, phi, sum_q):
    """Src/main.f90:859-949 (one rank): phi of the dielectric walls' nodes
    rises by the surface charges over the capacitance per cell st.Ca; the
    sums are cleared."""
    qxz, qyz = sum_q
    assert phi.flags["C_CONTIGUOUS"] and qxz.flags["C_CONTIGUOUS"] and qyz.flags["C_CONTIGUOUS"]
    n = np.array(st.n, dtype=np.int32)
    bc = np.ascontiguousarray(st.geom.bcnd, dtype=np.int32)
    lib().oracle_dielectric_phi(_pi(n), _pd(phi), _pi(bc), _pi(st.geom.dtype_array()),
                                C.c_int(st.geom.ngrid), _pd(qxz), _pd(qyz), C.c_int(st.ntype),
                                C.c_double(st.Ca), C.c_int(st.geom.flag_pbc))


def step(st, S, phi, Ei, it, p_mac=None, P_loss=None, nsort=10, ns_coll=10, mg=None):
    """One legacy timestep in the order of Src/main.f90:853-1277:
    calc_rho -> (dielectric walls' potential) -> pdesolver -> calc_Efield ->
    (sort) -> (collisions) -> part_mover -> charge_deposition.  Returns
    (Ei, mg result, MCC result)."""
    rhs = calc_rho(st, S.np)
    if st.geom.flag_die:
        dielectric_phi(st, phi, S.sum_q)
    mg_out = pdesolver(st, phi, rhs, **(mg or {}))
    Ei = calc_efield(st, phi, Ei)
    if nsort and it % nsort == 1 % nsort:
        for p in range(1, st.ntype + 1):
            if S.np_tot[p - 1] > 0:
                pl = part_sorting(st, S, p)
                if S.Plist is None:
                    S.Plist = np.zeros((st.ntype, len(pl)), dtype=np.int32)
                S.Plist[p - 1] = pl
    mcc = None
    if st.tables is not None and it > 1 and it % ns_coll == 1 % ns_coll:
        mcc = collisions(st, S, ns_coll=ns_coll)
    ng1 = st.geom.ngrid + 1
    if p_mac is None:
        p_mac = np.zeros((ng1, 2, st.ntype))
    if P_loss is None:
        P_loss = np.zeros((st.ntype, 4))
    for p in range(1, st.ntype + 1):
        if st.charge[p - 1] != 0.0:
            part_mover(st, Ei, S, p_mac, P_loss, p, sum_q=S.sum_q)
    for p in range(1, st.ntype + 1):
        S.np[p - 1] = 0.0
        if S.np_tot[p - 1] > 0:
            charge_deposition(st, S, p)
    return Ei, mg_out, mcc
