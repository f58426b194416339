"""Python mirror of the reference's hot-path routines, calling the GPU drop-ins.

Each function has the name and argument meaning of the legacy Fortran
routine it stands for and passes numpy arrays in the reference's layouts to
the C ABI of liblepic_gpu.so (the same entry points a Fortran build links).
Errors raise ``LepicError`` (the reference calls stop_calculation).

Array layouts (C-order numpy views of the Fortran arrays):
  node grid    (n3+3, n2+3, n1+3)            bcnd, kq, phi
  rhs grid     (n3+2, n2+2, n1+2)
  Ei           (n3+3, n2+3, n1+3, 3)
  np           (ntype, n3+3, n2+3, n1+3)
  vxp          (ntype, nmax, 6)
  u (pdesolver) (n3+4, n2+3, n1+3): z from -1 like phi_dom
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, commons, lib
from .constants import AMU, C_LIGHT, EPS0, PI, QE


def _i(v):
    return C.byref(C.c_int(int(v)))


def _d(v):
    return C.byref(C.c_double(float(v)))


def _pi(a):
    return a.ctypes.data_as(_lib.P_int)


def _pd(a):
    return a.ctypes.data_as(_lib.P_dbl)


def heat_struct(st, hz):
    """lepic_heat_t of a config.Heating on the set-up st."""
    from .config import heating_params
    hp = heating_params(st, hz)
    H = _lib.LepicHeat()
    H.ixl_pow, H.ixr_pow = hp["ixl_pow"], hp["ixr_pow"]
    H.flag_circxh, H.flag_ahp = int(hz.flag_circxh), int(hz.flag_ahp)
    H.R_ahp, H.nudt, H.Pabs, H.nu_h = float(hz.R_ahp), hp["nudt"], float(hz.Pabs), float(hz.nu_h)
    return H, hp


def set_commons(st, ncol=0, npt=0, p_ncol=None, heating=None):
    """Fill the library's COMMON blocks the way read_input/read_reactions/main
    fill the Fortran ones (Src/main.f90:124-579); heating: a config.Heating."""
    cm = commons()
    pi_, d1, d2, d3, cs = (cm["part_info_int"], cm["part_info_dp_1"], cm["part_info_dp_2"],
                           cm["part_info_dp_3"], cm["constants"])
    C.memset(C.addressof(pi_), 0, C.sizeof(pi_))
    C.memset(C.addressof(d1), 0, C.sizeof(d1))
    C.memset(C.addressof(d2), 0, C.sizeof(d2))
    C.memset(C.addressof(d3), 0, C.sizeof(d3))
    pi_.np_cell = st.np_cell
    pi_.ncol = ncol
    pi_.sig_npt_mx = npt
    pi_.n_cell = st.n_cell
    pi_.flag_B = st.flag_B
    pi_.flag_B_pos = int(getattr(st, "flag_B_pos", 0))
    bf = getattr(st, "bfield", None)
    pi_.flag_gridB = int(bf is not None and tuple(bf.n_B) != tuple(st.n))
    pi_.ns_coll = st.wl.ns_coll
    pi_.flag_pbc = st.geom.flag_pbc
    pi_.flag_nmn = st.geom.flag_nmn
    pi_.flag_die = st.geom.flag_die
    pi_.iz_pl = st.n[2] // 2 + 1            # the XY plot plane (Src/main.f90:570)
    if p_ncol is not None:
        for i in range(len(p_ncol)):
            pi_.p_ncol[i] = int(p_ncol[i])
    for i in range(_lib.NPART):
        d1.charge[i] = st.charge[i]
        d1.mass[i] = st.mass[i]
        d1.Ti[i] = st.Ti[i]
        d1.vt0[i] = st.vt0[i]
        d2.Nm[i] = st.Nm[i]
        d3.np_mx[i] = st.np_mx[i]
        d3.nu_uplim[i] = st.nu_uplim[i]
    d1.k_eps0 = 1.0
    d1.gam_sec = -1.0
    d2.Pabs = -1.0
    d2.n0 = st.wl.n0
    d2.ngas = st.ngas
    d2.dt = st.dt
    d2.xmax, d2.ymax, d2.zmax = (float(v) for v in st.geom.box)
    d2.x_load = st.x_load
    cs.qe, cs.eps0, cs.c, cs.pi, cs.amu = QE, EPS0, C_LIGHT, PI, AMU
    if heating is not None:
        H, hp = heat_struct(st, heating)
        pi_.ixl_pow, pi_.ixr_pow = H.ixl_pow, H.ixr_pow
        pi_.flag_circxh, pi_.flag_ahp = H.flag_circxh, H.flag_ahp
        pi_.ns_heat, pi_.flag_heat, pi_.flag_inj = hp["ns_heat"], hp["flag_heat"], int(heating.flag_inj)
        d2.R_ahp, d2.nudt, d2.Pabs, d2.nu_h = H.R_ahp, H.nudt, H.Pabs, H.nu_h


def inject_struct(st, inj):
    """lepic_inject_t of a config.Injection on the set-up st."""
    I = _lib.LepicInject()
    I.opt_inj, I.ns_inj, I.n_cath = int(inj.opt_inj), int(inj.ns_inj), int(inj.n_cath)
    I.dir_sec, I.tag_beam, I.flag_pbcz = int(inj.dir_sec), int(inj.tag_beam), int(st.geom.flag_pbcz)
    I.I_inj = float(inj.I_inj)
    I.xl, I.xr, I.yl, I.yr, I.zl, I.zr = (float(v) for v in (inj.xl, inj.xr, inj.yl, inj.yr, inj.zl, inj.zr))
    I.THm = float(inj.THm)
    I.zg_sec[0], I.zg_sec[1] = (float(v) for v in inj.zg_sec)
    ni0 = st.ni0 if inj.ni0 is None else inj.ni0
    for i in range(st.ntype):
        I.ni0[i] = float(ni0[i])
    return I


def part_injection(st, inj, vxp, np_tot, phi, P_loss, N_inj_ions=0, iseed=123456):
    """Src/part_injection.f90:1 -- appends to vxp (ntype, nmax, 6) behind
    np_tot; P_loss (ntype, 4) C-order, P_loss[p, 3] gains the injected power."""
    cm = commons()
    pi_, d1, d2 = cm["part_info_int"], cm["part_info_dp_1"], cm["part_info_dp_2"]
    pi_.opt_inj, pi_.ns_inj, pi_.n_cath = int(inj.opt_inj), int(inj.ns_inj), int(inj.n_cath)
    pi_.dir_sec, pi_.tag_beam, pi_.flag_pbcz = int(inj.dir_sec), int(inj.tag_beam), int(st.geom.flag_pbcz)
    pi_.flag_inj = 1
    d1.THm = float(inj.THm)
    d1.zg_sec[0], d1.zg_sec[1] = (float(v) for v in inj.zg_sec)
    n = _lib.np_i(st.n)
    h = np.ascontiguousarray(st.h, dtype=np.float64)
    bc = _lib.np_i(st.geom.bcnd)
    assert vxp.flags["C_CONTIGUOUS"] and np_tot.dtype == np.int32 and P_loss.flags["C_CONTIGUOUS"]
    ni0 = np.ascontiguousarray(st.ni0 if inj.ni0 is None else np.array(inj.ni0), dtype=np.float64)
    f = np.ascontiguousarray(phi, dtype=np.float64)
    zi = np.zeros(16, dtype=np.int32)
    N_inj = np.zeros((1, st.ntype), dtype=np.int32)
    if st.ntype > 1:
        N_inj[0, 1] = int(N_inj_ions)
    seed = np.array([iseed], dtype=np.int32)
    lib().part_injection_(_pi(n), _pd(h), _pi(bc), _pd(vxp), _pi(zi), _pi(zi), _pi(zi), _i(st.ntype),
                          _i(vxp.shape[1]), _d(inj.I_inj), _d(inj.xl), _d(inj.xr), _d(inj.yl), _d(inj.yr),
                          _d(inj.zl), _d(inj.zr), _pi(np_tot), _i(1), _pi(seed), _i(1), _pi(N_inj), _i(1),
                          _pd(P_loss), _pd(f), _pd(ni0))
    check(lib().lepic_gpu_last_error(), "part_injection")


def eheating(st, vxp, np_tot, vt, P_loss, iseed=123456):
    """Src/part_expmover.f90:484 -- heats species 1 of vxp (ntype, nmax, 6)
    in place; P_loss (ntype, 4) C-order, P_loss[0, 1] gains the energy."""
    h = np.ascontiguousarray(st.h, dtype=np.float64)
    assert vxp.flags["C_CONTIGUOUS"] and np_tot.dtype == np.int32 and P_loss.flags["C_CONTIGUOUS"]
    seed = np.array([iseed], dtype=np.int32)
    lib().eheating_(_pd(h), _pd(vxp), _i(vxp.shape[1]), _i(st.ntype), _i(1), _pi(seed), _pi(np_tot),
                    _d(vt), _i(1), _pd(P_loss))
    check(lib().lepic_gpu_last_error(), "eheating")


def calc_rho(st, np_grids):
    """Src/calc_rho.f90:1 -- returns rhs = -rho on (n3+2, n2+2, n1+2)."""
    n = _lib.np_i(st.n)
    npg = np.ascontiguousarray(np_grids, dtype=np.float64)
    rhs = np.zeros((st.n[2] + 2, st.n[1] + 2, st.n[0] + 2))
    bc = _lib.np_i(st.geom.bcnd)
    lib().calc_rho_(_pi(n), _pd(npg), _pd(rhs), _pi(bc), _i(st.ntype), _i(1), _i(1), _i(0))
    check(lib().lepic_gpu_last_error(), "calc_rho")
    np_grids[...] = npg
    return rhs


def dens_red(st, np_grids):
    """Src/calc_rho.f90:116 -- returns (np_red, np_mx[ntype])."""
    n = _lib.np_i(st.n)
    npg = np.ascontiguousarray(np_grids, dtype=np.float64)
    red = np.zeros_like(npg)
    bc = _lib.np_i(st.geom.bcnd)
    lib().dens_red_(_pi(n), _pd(npg), _pd(red), _pi(bc), _i(st.ntype), _i(1), _i(1))
    check(lib().lepic_gpu_last_error(), "dens_red")
    d3 = commons()["part_info_dp_3"]
    return red, np.array([d3.np_mx[i] for i in range(st.ntype)])


def pdesolver(st, phi, rhs, eps=None, omega=None, ng=None, ncycl=None):
    """Src/pdesolver.f90:1 -- solves in place into phi (n3+3, n2+3, n1+3);
    returns (k, ktot, res) like the reference."""
    wl = st.wl
    eps = wl.eps if eps is None else eps
    omega = wl.omega if omega is None else omega
    ng = st.ng if ng is None else ng
    ncycl = wl.ncycl if ncycl is None else ncycl
    n = _lib.np_i(st.n)
    u = np.zeros((st.n[2] + 4, st.n[1] + 3, st.n[0] + 3))
    u[1:] = phi
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    bc = _lib.np_i(st.geom.bcnd)
    h = np.ascontiguousarray(st.h, dtype=np.float64)
    k = C.c_int(0)
    ktot = C.c_double(0)
    res = C.c_double(0)
    lib().pdesolver_(_pd(u), _pd(b), _pi(bc), _pd(h), _pi(n), _i(ncycl), _d(eps), _d(omega),
                     C.byref(k), C.byref(ktot), C.byref(res), _i(ng), _i(0), _i(1))
    check(lib().lepic_gpu_last_error(), "pdesolver")
    phi[...] = u[1:]
    return k.value, ktot.value, res.value


def calc_efield(st, phi, Ei=None):
    """Src/Efield.f90:1 -- returns Ei (n3+3, n2+3, n1+3, 3); nodes the
    routine does not write keep the values of the Ei passed in."""
    n = _lib.np_i(st.n)
    if Ei is None:
        Ei = np.zeros(tuple(st.geom.bcnd.shape) + (3,))
    E = np.ascontiguousarray(Ei, dtype=np.float64)
    f = np.ascontiguousarray(phi, dtype=np.float64)
    bc = _lib.np_i(st.geom.bcnd)
    h = np.ascontiguousarray(st.h, dtype=np.float64)
    lib().calc_efield_(_pi(n), _pd(h), _pd(f), _pd(E), _pi(bc))
    check(lib().lepic_gpu_last_error(), "calc_efield")
    return E


def _bi(st):
    """(Bi, n_B, h_B) as the reference passes them to part_mover: the map of
    st.bfield, else Bi(4, 0:3, 0:3, 0:3) with n_B = 1 holding the uniform
    field at (1, 1, 1)."""
    bf = getattr(st, "bfield", None)
    if bf is not None:
        return (np.ascontiguousarray(bf.Bi, dtype=np.float64), np.array(bf.n_B, dtype=np.int32),
                np.ascontiguousarray(bf.h_B, dtype=np.float64))
    Bi = np.zeros((4, 4, 4, 4))
    Bi[1, 1, 1, 0:3] = st.Bconst
    return Bi, np.array([1, 1, 1], dtype=np.int32), np.ascontiguousarray(st.h, dtype=np.float64)


class MoverExtra:
    """The negative-ion bookkeeping and secondary emission of part_mover_
    (Src/part_expmover.f90:76, 278-301, 353-400, 416-470): the COMMON values
    (tag_neg, tag_neu, num_grd; gam_sec, igrid_sec, THm, zg_sec) and the
    caller's arrays flag_cex(1:nmax), cnt_cex(3), cnt_dead, beam_div(4) and the
    ran2 seed iseed."""

    def __init__(self, nmax, tag_neg=0, tag_neu=0, num_grd=0, gam_sec=0.0, igrid_sec=0, THm=0.0,
                 zg_sec=(0.0, 0.0), iseed=-1):
        self.flag_cex = np.zeros(nmax, dtype=np.int32)
        self.cnt_cex = np.zeros(3, dtype=np.int32)
        self.cnt_dead = np.zeros(1)
        self.beam_div = np.zeros(4)
        self.iseed = np.array([iseed], dtype=np.int32)
        self.tag_neg, self.tag_neu, self.num_grd = int(tag_neg), int(tag_neu), int(num_grd)
        self.gam_sec, self.igrid_sec, self.THm = float(gam_sec), int(igrid_sec), float(THm)
        self.zg_sec = tuple(float(z) for z in zg_sec)

    def set_commons(self):
        cm = commons()
        pi_, d1 = cm["part_info_int"], cm["part_info_dp_1"]
        pi_.tag_neg, pi_.tag_neu, pi_.num_grd, pi_.igrid_sec = self.tag_neg, self.tag_neu, self.num_grd, \
            self.igrid_sec
        d1.gam_sec = self.gam_sec if self.gam_sec > 0.0 else -1.0
        d1.THm = self.THm
        d1.zg_sec[0], d1.zg_sec[1] = self.zg_sec


def part_mover(st, Ei, vxp, np_tot, flag_dead, p_mac, P_loss, ptype, ngrid=None, sum_q=None, extra=None):
    """Src/part_expmover.f90:1 -- in place on vxp / np_tot / flag_dead /
    p_mac (ntype, 2, 0:ngrid) C-order (ngrid+1, 2, ntype) / P_loss (ntype, 4).
    sum_q: (sum_q_xz, sum_q_yz), the surface charges of the dielectric walls
    (flag_die = 1), C-order (ntype, n3+3, n1+3) and (ntype, n3+3, n2+3, 2),
    accumulated for ptype.  extra: a MoverExtra (negative ions, secondary
    emission into species 1); its COMMON values are set for the call."""
    ngrid = st.geom.ngrid if ngrid is None else ngrid
    n = _lib.np_i(st.n)
    h = np.ascontiguousarray(st.h, dtype=np.float64)
    E = np.ascontiguousarray(Ei, dtype=np.float64)
    Bi, nB, hB = _bi(st)
    bc = _lib.np_i(st.geom.bcnd)
    nmax = vxp.shape[1]
    assert vxp.flags["C_CONTIGUOUS"] and np_tot.dtype == np.int32 and flag_dead.dtype == np.int8
    dummy_i = np.zeros(16, dtype=np.int32)
    dummy_d = np.zeros(16)
    qxz = qyz = dummy_d
    dt = dummy_i
    if st.geom.flag_die:
        n1, n2, n3 = st.n
        if sum_q is None:
            sum_q = (np.zeros((st.ntype, n3 + 3, n1 + 3)), np.zeros((st.ntype, n3 + 3, n2 + 3, 2)))
        qxz, qyz = sum_q
        assert qxz.shape == (st.ntype, n3 + 3, n1 + 3) and qyz.shape == (st.ntype, n3 + 3, n2 + 3, 2)
        assert qxz.flags["C_CONTIGUOUS"] and qyz.flags["C_CONTIGUOUS"] and qxz.dtype == np.float64
        dt = st.geom.dtype_array()
    cex, ccex, cdead, bdiv, seed = dummy_i, dummy_i, dummy_d, dummy_d, dummy_i
    if extra is not None:
        extra.set_commons()
        assert len(extra.flag_cex) >= nmax
        cex, ccex, cdead, bdiv, seed = extra.flag_cex, extra.cnt_cex, extra.cnt_dead, extra.beam_div, extra.iseed
    try:
        lib().part_mover_(_pi(n), _pd(h), _pd(E), _pd(Bi), _pd(p_mac), _pd(P_loss), _pd(vxp), _pi(bc),
                          _i(nmax), _i(st.ntype), _i(ngrid), flag_dead.ctypes.data_as(_lib.P_i8), _i(1),
                          _pi(np_tot), _i(1), _i(ptype), _pi(cex), _pi(ccex), _pd(cdead),
                          _pd(bdiv), _pd(qxz), _pd(qyz), _pi(dt), _pi(seed), _pi(nB),
                          _pd(hB))
    finally:
        if extra is not None:
            MoverExtra(1).set_commons()   # back to no negative ions, no emission
    check(lib().lepic_gpu_last_error(), "part_mover")


def charge_deposition(st, vxp, np_tot, np_grids, ptype):
    """Src/part_expmover.f90:570 -- accumulates into np_grids[ptype-1];
    returns the heating-region statistics (sum_dEk, Nh) (non-zero for
    ptype 1 with Pabs > 0 in the COMMON blocks)."""
    n = _lib.np_i(st.n)
    h = np.ascontiguousarray(st.h, dtype=np.float64)
    kq = np.ascontiguousarray(st.kq, dtype=np.float64)
    assert np_grids.flags["C_CONTIGUOUS"]
    s = np.zeros(1)
    nh = np.zeros(1, dtype=np.int32)
    lib().charge_deposition_(_pi(n), _pd(h), _pd(vxp), _i(vxp.shape[1]), _i(st.ntype), _pd(kq),
                             _pd(np_grids), _i(1), _pi(np_tot), _pd(s), _pi(nh), _i(1), _i(ptype))
    check(lib().lepic_gpu_last_error(), "charge_deposition")
    return float(s[0]), int(nh[0])


def pl_max_of(n):
    """Src/main.f90:227."""
    return n[0] + n[0] * (n[1] + n[1] * n[2]) + 1


def part_sorting(st, vxp, np_tot, ptype):
    """Src/sorting.f90:97 -- sorts species ptype in place, returns Plist
    (0:pl_max) of that species."""
    n = _lib.np_i(st.n)
    h = np.ascontiguousarray(st.h, dtype=np.float64)
    pl_max = pl_max_of(st.n)
    Plist = np.zeros((st.ntype, pl_max + 1), dtype=np.int32)
    dummy = np.zeros(1)
    lib().part_sorting_(_pd(vxp), _pd(dummy), _i(vxp.shape[1]), _i(st.ntype), _pi(n), _pd(h),
                        _pi(Plist), _i(pl_max), _i(1), _pi(np_tot), _i(ptype))
    check(lib().lepic_gpu_last_error(), "part_sorting")
    return Plist[ptype - 1].copy()


def collisions(st, it, vxp, np_tot, flag_dead, iseed, np_red=None, ncol_mx=65, npt_mx=1300,
               regions=(), cnt_col=None, Plist=None, P_loss=None, sour=None):
    """Src/collisions.f90:1 -- in place on vxp / np_tot / flag_dead.
    regions: [(ixl, ixr)] x-ranges of the counting regions (n_rg of them)
    sharing the y/z range of the whole grid, like conditions.inp's regions.
    Charged targets (DSMC) need Plist, the per-species cell offsets of the
    last part_sorting (ntype rows of pl_max+1), and np_red, the densities:
    dens_red runs on np_red first, as in Src/main.f90:1194, to set np_mx.
    P_loss (ntype, 4), accumulated: column 3 gains the kinetic energy change
    of every particle the collisions set (created ones from zero).  sour:
    (sour_xy (ntype, n2+3, n1+3), sour_xz (ntype, n3+3, n1+3)) int32,
    accumulated: the particles created in the cells of the plot planes
    iz = n3/2+1 and iy = n2/2+1.
    Returns the per-species nu_max written to COMMON /part_info_dp_3/."""
    T = st.tables
    ncol = T.sig.shape[0]
    npt = T.sig_Er.shape[0]
    set_commons(st, ncol=ncol, npt=npt, p_ncol=T.p_ncol)
    cm = commons()
    n_rg = len(regions)
    pi_ = cm["part_info_int"]
    pi_.n_rg = n_rg
    for g, (lo, hi) in enumerate(regions):
        pi_.ixl_rg[g], pi_.ixr_rg[g] = int(lo), int(hi)
    pi_.iyl_rg, pi_.iyr_rg, pi_.izl_rg, pi_.izr_rg = 1, st.n[1] + 1, 1, st.n[2] + 1
    n = _lib.np_i(st.n)
    h = np.ascontiguousarray(st.h, dtype=np.float64)
    sig = np.zeros((ncol_mx, npt_mx))
    sig[:ncol, :npt] = T.sig
    sig_Er = np.zeros(npt_mx)
    sig_Er[:npt] = T.sig_Er
    sig_list = np.zeros((ncol_mx, 10), dtype=np.int32)
    sig_list[:ncol, :] = T.sig_list.T
    sig_Eex = np.zeros((2, ncol_mx))
    sig_Eex[0, :ncol] = T.Eth
    sigv = np.zeros((ncol_mx, 10))
    sigv[:ncol, :] = T.sigv_mx.T
    col_info = np.zeros((10, ncol_mx), dtype=np.int32)
    col_info[:, :ncol] = T.col_info.T
    if cnt_col is None:
        cnt_col = np.zeros((max(n_rg, 1), 1, ncol_mx))
    if np_red is None:
        np_red = np.zeros((st.ntype,) + tuple(st.geom.bcnd.shape))
    else:
        np_red = np.ascontiguousarray(np_red, dtype=np.float64)
        dens_red(st, np_red)
    zi = np.zeros(16, dtype=np.int32)
    zd = np.zeros(16)
    n1, n2, n3 = st.n
    if P_loss is None:
        P_loss = np.zeros((st.ntype, 4))
    assert P_loss.shape == (st.ntype, 4) and P_loss.dtype == np.float64 and P_loss.flags.c_contiguous
    if sour is None:
        sour = (np.zeros((st.ntype, n2 + 3, n1 + 3), dtype=np.int32),
                np.zeros((st.ntype, n3 + 3, n1 + 3), dtype=np.int32))
    sxy, sxz = sour
    assert sxy.shape == (st.ntype, n2 + 3, n1 + 3) and sxz.shape == (st.ntype, n3 + 3, n1 + 3)
    assert sxy.dtype == np.int32 and sxz.dtype == np.int32 and sxy.flags.c_contiguous and sxz.flags.c_contiguous
    if Plist is None:
        pl, plm = np.zeros(1, dtype=np.int32), 0
    else:
        pl = np.ascontiguousarray(np.stack([np.asarray(r, dtype=np.int32) for r in Plist]))
        plm = pl.shape[1] - 1
    lib().collisions_(_i(it), _pd(vxp), _pi(n), _pd(h), _i(st.ntype), _i(vxp.shape[1]), _pd(sig),
                      _pd(sig_Er), _pi(sig_list), _pd(sig_Eex), _i(ncol_mx), _i(npt_mx), _pd(cnt_col),
                      _pd(P_loss), _pi(sxy), _pi(sxz), _pi(pl), _i(plm), _pd(sigv), _pi(col_info), _pd(np_red),
                      flag_dead.ctypes.data_as(_lib.P_i8), _pi(zi), _i(1), _pi(np_tot), _pi(iseed),
                      _i(1), _i(0), _pd(zd), _pd(zd), _pd(zd), _i(0))
    check(lib().lepic_gpu_last_error(), "collisions")
    d3 = cm["part_info_dp_3"]
    return np.array([d3.nu_max[i] for i in range(st.ntype)])


# ---------------------------------------------------------------- residency
def set_residency(on):
    """lepic_gpu_set_residency: device mirrors of the drop-ins' host arrays
    kept between calls (on) or per-call copies (off; syncs and frees)."""
    check(lib().lepic_gpu_set_residency(1 if on else 0), "set_residency")


def sync_to_host():
    check(lib().lepic_gpu_sync_to_host(), "sync_to_host")


def mirror_stats():
    """(bytes host->device, bytes device->host, live mirrors) of the drop-in
    layer since the library loaded."""
    h2d, d2h, m = C.c_longlong(0), C.c_longlong(0), C.c_int(0)
    check(lib().lepic_gpu_mirror_stats(C.byref(h2d), C.byref(d2h), C.byref(m)), "mirror_stats")
    return h2d.value, d2h.value, m.value


def _vp(a, offset_bytes=0):
    return C.c_void_p(a.ctypes.data + offset_bytes)


class MainLoop:
    """The timestep of Src/main.f90:853-1280 through the drop-ins only, over
    persistent host arrays in the reference layouts -- the calls a Fortran
    build linked against liblepic_gpu.so makes:

        calc_rho -> pdesolver -> phi = phi_dom (the one-rank MPI_ALLGATHERV,
        main.f90:977) -> calc_Efield -> part_sorting (MOD(it,nsort) = 1)
        -> dens_red + collisions (it > 1, MOD(it,ns_coll) = 1)
        -> part_mover (charged species) -> np(:,:,:,p) = 0 + charge_deposition

    The arrays passed in (vxp (ntype, nmax, 6), np_tot int32 (ntype),
    flag_dead int8 (ntype, nmax), np_grids (ntype, n3+3, n2+3, n1+3)) are
    used in place.  resident=True turns the library's residency on: the
    arrays stay on the GPU between calls, the loop's two host statements on
    them run as lepic_gpu_mirror_copy / lepic_gpu_mirror_zero, and sync()
    brings the host arrays up to date."""

    def __init__(self, st, vxp, np_tot, flag_dead, np_grids, resident=False, iseed=4242,
                 nsort=None, ns_coll=None, collide=True, ncol_mx=65, npt_mx=1300, regions=()):
        assert vxp.flags["C_CONTIGUOUS"] and vxp.dtype == np.float64
        assert np_tot.dtype == np.int32 and flag_dead.dtype == np.int8
        assert np_grids.flags["C_CONTIGUOUS"] and np_grids.dtype == np.float64
        self.st = st
        self.vxp, self.np_tot, self.flag_dead, self.np = vxp, np_tot, flag_dead, np_grids
        self.resident = bool(resident)
        self.nsort = st.wl.nsort if nsort is None else nsort
        self.ns_coll = st.wl.ns_coll if ns_coll is None else ns_coll
        self.it = 0
        n1, n2, n3 = st.n
        N1, N2, N3 = n1 + 3, n2 + 3, n3 + 3
        self.n = _lib.np_i(st.n).copy()
        self.h = np.ascontiguousarray(st.h, dtype=np.float64).copy()
        self.bcnd = _lib.np_i(st.geom.bcnd).copy()
        self.kq = np.ascontiguousarray(st.kq, dtype=np.float64).copy()
        self.rhs = np.zeros((n3 + 2, n2 + 2, n1 + 2))
        self.phi_dom = np.zeros((n3 + 4, N2, N1))          # z from -1
        self.phi_dom[1:] = st.geom.phi
        self.phi = np.ascontiguousarray(st.geom.phi, dtype=np.float64).copy()
        self.Ei = np.zeros((N3, N2, N1, 3))
        self.np_red = np.zeros_like(np_grids)
        self.pl_max = pl_max_of(st.n)
        self.Plist = np.zeros((st.ntype, self.pl_max + 1), dtype=np.int32)
        ngrid = st.geom.ngrid
        self.ngrid = ngrid
        self.p_mac = np.zeros((ngrid + 1, 2, st.ntype))
        self.P_loss = np.zeros((st.ntype, 4))
        self.Bi, self.nB, self.hB = _bi(st)
        self.iseed = np.array([iseed], dtype=np.int32)
        self.zi = np.zeros(16, dtype=np.int32)
        self.zd = np.zeros(16)
        self.sour_xy = np.zeros((st.ntype, N2, N1), dtype=np.int32)   # sour_xy(0:n1+2, 0:n2+2, ntype, 1)
        self.sour_xz = np.zeros((st.ntype, N3, N1), dtype=np.int32)   # sour_xz(0:n1+2, 0:n3+2, ntype, 1)
        self.collide = bool(collide) and st.tables is not None
        self.regions = list(regions)  # [(ixl, ixr)]: MCC region counters in cnt_col
        self.ncol = self.npt = 0
        if self.collide:
            T = st.tables
            self.ncol, self.npt = T.sig.shape[0], T.sig_Er.shape[0]
            self.p_ncol = T.p_ncol
            self.ncol_mx, self.npt_mx = ncol_mx, npt_mx
            self.sig = np.zeros((ncol_mx, npt_mx))
            self.sig[:self.ncol, :self.npt] = T.sig
            self.sig_Er = np.zeros(npt_mx)
            self.sig_Er[:self.npt] = T.sig_Er
            self.sig_list = np.zeros((ncol_mx, 10), dtype=np.int32)
            self.sig_list[:self.ncol, :] = T.sig_list.T
            self.sig_Eex = np.zeros((2, ncol_mx))
            self.sig_Eex[0, :self.ncol] = T.Eth
            self.sigv = np.zeros((ncol_mx, 10))
            self.sigv[:self.ncol, :] = T.sigv_mx.T
            self.col_info = np.zeros((10, ncol_mx), dtype=np.int32)
            self.col_info[:, :self.ncol] = T.col_info.T
            self.cnt_col = np.zeros((max(len(self.regions), 1), 1, ncol_mx))
        set_residency(self.resident)

    def _commons(self):
        if self.collide:
            set_commons(self.st, ncol=self.ncol, npt=self.npt, p_ncol=self.p_ncol)
            pi_ = commons()["part_info_int"]
            # the loop's MCC cadence, which sets Pmax = nu_max ns_coll dt
            # (Src/collisions.f90:122)
            pi_.ns_coll = self.ns_coll
            pi_.n_rg = len(self.regions)
            for g, (lo, hi) in enumerate(self.regions):
                pi_.ixl_rg[g], pi_.ixr_rg[g] = int(lo), int(hi)
            pi_.iyl_rg, pi_.iyr_rg, pi_.izl_rg, pi_.izr_rg = 1, self.st.n[1] + 1, 1, self.st.n[2] + 1
        else:
            set_commons(self.st)

    def step(self):
        st, L = self.st, lib()
        self.it += 1
        it = self.it
        self._commons()
        nt = st.ntype
        nmax = self.vxp.shape[1]
        wl = st.wl
        L.calc_rho_(_pi(self.n), _pd(self.np), _pd(self.rhs), _pi(self.bcnd), _i(nt), _i(1), _i(1), _i(0))
        check(L.lepic_gpu_last_error(), "calc_rho")
        k, ktot, res = C.c_int(0), C.c_double(0), C.c_double(0)
        L.pdesolver_(_pd(self.phi_dom), _pd(self.rhs), _pi(self.bcnd), _pd(self.h), _pi(self.n),
                     _i(wl.ncycl), _d(wl.eps), _d(wl.omega), C.byref(k), C.byref(ktot), C.byref(res),
                     _i(st.ng), _i(0), _i(1))
        check(L.lepic_gpu_last_error(), "pdesolver")
        plane = self.phi_dom.shape[1] * self.phi_dom.shape[2] * 8
        check(L.lepic_gpu_mirror_copy(_vp(self.phi), _vp(self.phi_dom, plane), self.phi.nbytes), "phi gather")
        L.calc_efield_(_pi(self.n), _pd(self.h), _pd(self.phi), _pd(self.Ei), _pi(self.bcnd))
        check(L.lepic_gpu_last_error(), "calc_efield")
        if self.nsort and it % self.nsort == 1 % self.nsort:
            for p in range(1, nt + 1):
                if self.np_tot[p - 1] > 0:
                    L.part_sorting_(_pd(self.vxp), _pd(self.zd), _i(nmax), _i(nt), _pi(self.n), _pd(self.h),
                                    _pi(self.Plist), _i(self.pl_max), _i(1), _pi(self.np_tot), _i(p))
                    check(L.lepic_gpu_last_error(), "part_sorting")
        if self.collide and it > 1 and it % self.ns_coll == 1 % self.ns_coll:
            L.dens_red_(_pi(self.n), _pd(self.np), _pd(self.np_red), _pi(self.bcnd), _i(nt), _i(1), _i(1))
            check(L.lepic_gpu_last_error(), "dens_red")
            L.collisions_(_i(it), _pd(self.vxp), _pi(self.n), _pd(self.h), _i(nt), _i(nmax), _pd(self.sig),
                          _pd(self.sig_Er), _pi(self.sig_list), _pd(self.sig_Eex), _i(self.ncol_mx),
                          _i(self.npt_mx), _pd(self.cnt_col), _pd(self.P_loss), _pi(self.sour_xy),
                          _pi(self.sour_xz), _pi(self.Plist), _i(self.pl_max), _pd(self.sigv), _pi(self.col_info),
                          _pd(self.np_red), self.flag_dead.ctypes.data_as(_lib.P_i8), _pi(self.zi), _i(1),
                          _pi(self.np_tot), _pi(self.iseed), _i(1), _i(0), _pd(self.zd), _pd(self.zd),
                          _pd(self.zd), _i(0))
            check(L.lepic_gpu_last_error(), "collisions")
        for p in range(1, nt + 1):
            if st.charge[p - 1] != 0.0:
                L.part_mover_(_pi(self.n), _pd(self.h), _pd(self.Ei), _pd(self.Bi), _pd(self.p_mac),
                              _pd(self.P_loss), _pd(self.vxp), _pi(self.bcnd), _i(nmax), _i(nt),
                              _i(self.ngrid), self.flag_dead.ctypes.data_as(_lib.P_i8), _i(1),
                              _pi(self.np_tot), _i(1), _i(p), _pi(self.zi), _pi(self.zi), _pd(self.zd),
                              _pd(self.zd), _pd(self.zd), _pd(self.zd), _pi(self.zi), _pi(self.zi),
                              _pi(self.nB), _pd(self.hB))
                check(L.lepic_gpu_last_error(), "part_mover")
        for p in range(1, nt + 1):
            check(L.lepic_gpu_mirror_zero(_vp(self.np[p - 1]), self.np[p - 1].nbytes), "np = 0")
            if self.np_tot[p - 1] > 0:
                L.charge_deposition_(_pi(self.n), _pd(self.h), _pd(self.vxp), _i(nmax), _i(nt), _pd(self.kq),
                                     _pd(self.np), _i(1), _pi(self.np_tot), _pd(self.zd), _pi(self.zi), _i(1),
                                     _i(p))
                check(L.lepic_gpu_last_error(), "charge_deposition")
        return k.value, res.value

    def sync(self):
        """Host arrays up to date (no-op without residency)."""
        sync_to_host()

    def close(self):
        """Sync, free the mirrors and turn residency off."""
        set_residency(False)
