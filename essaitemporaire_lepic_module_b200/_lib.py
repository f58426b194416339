"""ctypes binding of ``liblepic_gpu.so`` (the C ABI declared in
include/lepic_gpu.h).

The library is the only compute path: if it is missing this module raises
immediately instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblepic_gpu.so")

NPART = 10
NM_RG = 5

P_int = C.POINTER(C.c_int)
P_dbl = C.POINTER(C.c_double)
P_i8 = C.POINTER(C.c_int8)


class LepicPhys(C.Structure):
    """lepic_phys_t (also the layout of the CPU oracle's OPhys)."""
    _fields_ = [("ntype", C.c_int), ("n_neu", C.c_int),
                ("charge", C.c_double * NPART), ("mass", C.c_double * NPART),
                ("vt0", C.c_double * NPART), ("Nm", C.c_double * NPART),
                ("np_mx", C.c_double * NPART), ("nu_uplim", C.c_double * NPART),
                ("dt", C.c_double), ("xmax", C.c_double), ("ymax", C.c_double),
                ("zmax", C.c_double), ("x_load", C.c_double),
                ("qe", C.c_double), ("eps0", C.c_double), ("pi", C.c_double),
                ("flag_B", C.c_int), ("flag_B_pos", C.c_int), ("flag_pbc", C.c_int),
                ("flag_nmn", C.c_int), ("ns_coll", C.c_int), ("n_cell", C.c_int),
                ("np_cell", C.c_int), ("Bconst", C.c_double * 3),
                ("Bmap", C.c_void_p), ("n_B", C.c_int * 3), ("h_B", C.c_double * 3),
                ("dtype", C.c_void_p), ("sum_q_xz", C.c_void_p), ("sum_q_yz", C.c_void_p)]


class LepicGrid(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("h", C.c_double * 3), ("bcnd", C.c_void_p),
                ("kq", C.c_void_p), ("cell_wall", C.c_void_p)]


class LepicSpeciesF64(C.Structure):
    _fields_ = [("p", C.c_void_p), ("p_alt", C.c_void_p), ("count", C.c_void_p),
                ("key", C.c_void_p), ("flag_dead", C.c_void_p), ("cap", C.c_int)]


class LepicSpeciesMixed(C.Structure):
    _fields_ = [("cell", C.c_void_p), ("p", C.c_void_p), ("cell_alt", C.c_void_p),
                ("p_alt", C.c_void_p), ("count", C.c_void_p), ("flag_dead", C.c_void_p),
                ("tile_off", C.c_void_p), ("cap", C.c_int), ("cell_off", C.c_void_p)]


class LepicWinSpecies(C.Structure):
    """lepic_win_species_t: one species of the differentiable collisional window."""
    _fields_ = [("cell", C.c_void_p), ("p", C.c_void_p), ("lam", C.c_void_p), ("bl", C.c_void_p),
                ("count", C.c_void_p), ("cap", C.c_int), ("fp64", C.c_int), ("tile_off", C.c_void_p),
                ("tile_end", C.c_int), ("pad", C.c_int)]


class LepicWinEvent(C.Structure):
    """lepic_win_event_t: one recorded collision of the window."""
    _fields_ = [("step", C.c_int), ("P", C.c_int), ("i", C.c_int), ("r", C.c_int),
                ("rt", C.c_int), ("nby", C.c_int), ("ind", C.c_int), ("pad", C.c_int),
                ("by", C.c_int * 4), ("slot", C.c_int * 4), ("e1", C.c_float * 12),
                ("tv", C.c_double * 3), ("vold", C.c_double * 3), ("m_t", C.c_double), ("Eth", C.c_double),
                ("sum_mass", C.c_double), ("pad2", C.c_double)]


class LepicTargets(C.Structure):
    """lepic_targets_t: charged-target (DSMC) inputs and counters."""
    _fields_ = [("np", C.c_void_p * NPART), ("cell_off", C.c_void_p * NPART),
                ("missed", C.c_longlong), ("lost_claims", C.c_longlong), ("replayed", C.c_longlong)]


class LepicHeat(C.Structure):
    """lepic_heat_t: electron heating region and rate."""
    _fields_ = [("ixl_pow", C.c_int), ("ixr_pow", C.c_int), ("flag_circxh", C.c_int), ("flag_ahp", C.c_int),
                ("R_ahp", C.c_double), ("nudt", C.c_double), ("Pabs", C.c_double), ("nu_h", C.c_double)]


class LepicInject(C.Structure):
    """lepic_inject_t: particle injection."""
    _fields_ = [("opt_inj", C.c_int), ("ns_inj", C.c_int), ("n_cath", C.c_int), ("dir_sec", C.c_int),
                ("tag_beam", C.c_int), ("flag_pbcz", C.c_int), ("I_inj", C.c_double),
                ("xl", C.c_double), ("xr", C.c_double), ("yl", C.c_double), ("yr", C.c_double),
                ("zl", C.c_double), ("zr", C.c_double), ("THm", C.c_double), ("zg_sec", C.c_double * 2),
                ("ni0", C.c_double * NPART)]


class LepicTables(C.Structure):
    _fields_ = [("ncol", C.c_int), ("npt", C.c_int), ("npt_mx", C.c_int),
                ("sig_Er", C.c_void_p), ("sig", C.c_void_p), ("sig_Eth", C.c_void_p),
                ("col_info", C.c_void_p), ("sig_list", C.c_void_p), ("p_ncol", C.c_void_p),
                ("sigv_mx", C.c_void_p), ("col_info_h", C.c_void_p)]


_I = C.c_int
_D = C.c_double


class PartInfoInt(C.Structure):
    _fields_ = [(nm, _I) for nm in ("np_cell ncol sig_npt_mx flag_pdf n_cell nbak flag_restart "
                                     "ixl_pow ixr_pow flag_B ns_heat ns_coll").split()] + \
        [("p_ncol", _I * NPART), ("nscol", _I), ("p_nscol", _I * NPART)] + \
        [(nm, _I) for nm in ("n_rg flag_pbc n_holes flag_grd ind_g nB cnt_seg tag_neg cnt_neg "
                             "tag_neu flag_nmn num_grd ptype_pdf ns_flx nhy nhz").split()] + \
        [("ixl_rg", _I * NM_RG), ("ns_inj", _I), ("ixr_rg", _I * NM_RG)] + \
        [(nm, _I) for nm in ("iyl_rg iyr_rg izl_rg izr_rg flag_heat flag_inj opt_inj flag_B_pos "
                             "ixg ix_PE omp_rank_max mpi_rank_max flag_die flag_thr ix_pl iz_pl "
                             "ix_thr flag_convP").split()] + \
        [("ig_die", _I * 5)] + \
        [(nm, _I) for nm in ("flag_pbcz tag_beam every cnt_plt flag_bak igrid_sec dir_sec n_cath "
                             "flag_circxh flag_ahp flag_gridB plt_src flag_RFpot").split()]


class PartInfoDp1(C.Structure):
    _fields_ = [("charge", _D * NPART), ("mass", _D * NPART), ("Ti", _D * NPART),
                ("vt0", _D * NPART), ("k_eps0", _D), ("B_scale", _D * 5), ("B0", _D * 5),
                ("dL", _D * 5), ("x0", _D * 5), ("y0", _D * 5), ("z0", _D * 5)] + \
        [(nm, _D) for nm in "jne RNeta THm x_thr y_thr tseq tseq_init tseq_final gam_sec".split()] + \
        [("zg_sec", _D * 2)]


class PartInfoDp2(C.Structure):
    _fields_ = [("Pabs", _D), ("n0", _D), ("ngas", _D), ("Nm", _D * NPART)] + \
        [(nm, _D) for nm in "dt xmax ymax zmax x_load nu_h Lgy Lgz Sg Lhy Lhz xg1 Bmax nudt R_ahp".split()]


class PartInfoDp3(C.Structure):
    _fields_ = [("np_mx", _D * NPART), ("nu_max", _D * NPART), ("nu_uplim", _D * NPART)]


class Constants(C.Structure):
    _fields_ = [(nm, _D) for nm in "qe eps0 c pi amu".split()]


_lib = None


def lib():
    """Load liblepic_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m essaitemporaire_lepic_module_b200.build`"
            " (the CUDA library is the only compute path; there is no fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sigs = {
        "lepic_gpu_last_error": ([], _I),
        "lepic_gpu_strerror": ([_I], C.c_char_p),
        "lepic_build_info": ([], C.c_char_p),
        "lepic_gpu_set_residency": ([_I], _I),
        "lepic_gpu_residency": ([], _I),
        "lepic_gpu_sync_to_host": ([], _I),
        "lepic_gpu_update_host": ([vp, C.c_size_t], _I),
        "lepic_gpu_update_device": ([vp, C.c_size_t], _I),
        "lepic_gpu_release": ([vp, C.c_size_t], _I),
        "lepic_gpu_release_all": ([], _I),
        "lepic_gpu_mirror_zero": ([vp, C.c_size_t], _I),
        "lepic_gpu_mirror_copy": ([vp, vp, C.c_size_t], _I),
        "lepic_gpu_mirror_stats": ([C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), P_int], _I),
        "lepic_dev_info": ([P_int, C.c_char_p, _I], _I),
        "lepic_dev_check": ([vp, P_int], _I),
        "lepic_dev_wait_selftest": ([C.c_longlong, vp], _I),
        "lepic_dev_check_async": ([vp, vp], _I),
        "lepic_dev_calc_rho": ([C.POINTER(LepicGrid), vp, vp, _I, C.POINTER(LepicPhys), vp], _I),
        "lepic_dev_calc_efield": ([C.POINTER(LepicGrid), vp, vp, vp], _I),
        "lepic_dev_pdesolver": ([C.POINTER(LepicGrid), vp, vp, _I, _D, _D, _I, C.POINTER(LepicPhys),
                                 P_int, P_dbl, P_dbl, vp], _I),
        "lepic_dev_pdesolver_noalloc": ([C.POINTER(LepicGrid), vp, vp, _I, _D, _D, _I,
                                         C.POINTER(LepicPhys), P_int, P_dbl, P_dbl, vp], _I),
        "lepic_dev_part_mover": ([C.POINTER(LepicGrid), vp, C.POINTER(LepicSpeciesF64), _I, _I, _I,
                                  C.POINTER(LepicPhys), P_dbl, P_dbl, vp], _I),
        "lepic_dev_push_deposit": ([C.POINTER(LepicGrid), vp, C.POINTER(LepicSpeciesF64), _I, _I,
                                    C.POINTER(LepicPhys), vp, vp, _I, vp], _I),
        "lepic_dev_charge_deposition": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesF64), _I,
                                         C.POINTER(LepicPhys), vp, vp], _I),
        "lepic_dev_part_sorting": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesF64), vp, _I, vp], _I),
        "lepic_dev_collisions": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesF64), _I,
                                  C.POINTER(LepicTables), C.POINTER(LepicPhys), C.c_ulonglong,
                                  C.c_ulonglong, P_dbl, C.POINTER(C.c_longlong), vp], _I),
        "lepic_dev_push_deposit_mixed": ([C.POINTER(LepicGrid), vp, C.POINTER(LepicSpeciesMixed), _I,
                                          _I, C.POINTER(LepicPhys), vp, vp, _I, vp], _I),
        "lepic_dev_sort_mixed": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesMixed), _I, vp], _I),
        "lepic_dev_pack_e32": ([vp, vp, C.c_longlong, vp], _I),
        "lepic_dev_load_uniform_mixed": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesMixed), _I, C.c_longlong,
                                          C.POINTER(LepicPhys), C.c_ulonglong, vp], _I),
        "lepic_dev_deposit_mixed": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesMixed), _I,
                                     C.POINTER(LepicPhys), vp, _I, vp], _I),
        "lepic_dev_f64_to_mixed": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesF64),
                                    C.POINTER(LepicSpeciesMixed), C.c_longlong, vp], _I),
        "lepic_dev_mixed_to_f64": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesMixed), vp,
                                    C.c_longlong, C.c_longlong, vp], _I),
        "lepic_dev_pdesolver_mixed": ([C.POINTER(LepicGrid), vp, vp, _D, _D, _I, C.POINTER(LepicPhys),
                                       _I, _I, _I, _I, _I, _I, P_int, P_dbl, vp], _I),
        "lepic_dev_pdesolver_mixed_stats": ([vp, vp, vp], _I),
        "lepic_dev_collisions_mixed": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesMixed), _I,
                                        C.POINTER(LepicTables), C.POINTER(LepicPhys), C.c_ulonglong,
                                        C.c_ulonglong, P_dbl, C.POINTER(C.c_longlong), vp], _I),
        "lepic_dev_collisions_targets": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesF64), _I,
                                          C.POINTER(LepicTables), C.POINTER(LepicPhys), C.c_ulonglong,
                                          C.c_ulonglong, P_dbl, C.POINTER(C.c_longlong), C.POINTER(LepicTargets),
                                          vp], _I),
        "lepic_dev_collisions_mixed_targets": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesMixed), _I,
                                                C.POINTER(LepicTables), C.POINTER(LepicPhys), C.c_ulonglong,
                                                C.c_ulonglong, P_dbl, C.POINTER(C.c_longlong),
                                                C.POINTER(LepicTargets), vp], _I),
        "lepic_dev_win_push": ([C.POINTER(LepicGrid), vp, vp, _I, _I, vp, _I, C.POINTER(LepicPhys), vp], _I),
        "lepic_dev_win_deposit": ([C.POINTER(LepicGrid), vp, _I, _I, vp, _I, C.POINTER(LepicPhys), vp, vp], _I),
        "lepic_dev_adj_push": ([C.POINTER(LepicGrid), vp, vp, _I, _I, vp, vp, vp, _I, _I, C.POINTER(LepicPhys),
                                vp, vp, vp], _I),
        "lepic_dev_adj_efield": ([C.POINTER(LepicGrid), vp, vp, vp], _I),
        "lepic_dev_adj_rhs": ([C.POINTER(LepicGrid), vp, vp, vp], _I),
        "lepic_dev_adj_walls": ([C.POINTER(LepicGrid), C.POINTER(LepicPhys), _I, vp, vp, vp, vp, _I, vp], _I),
        "lepic_dev_adj_deposit": ([C.POINTER(LepicGrid), vp, _I, _I, vp, vp, vp, _I, _I, C.POINTER(LepicPhys),
                                   vp], _I),
        "lepic_dev_cw_deposit": ([C.POINTER(LepicGrid), C.POINTER(LepicWinSpecies), _I, C.POINTER(LepicPhys),
                                  _I, vp, vp], _I),
        "lepic_dev_cw_back": ([C.POINTER(LepicGrid), vp, C.POINTER(LepicWinSpecies), _I, C.POINTER(LepicPhys),
                               _I, vp, C.c_double, vp, vp, vp], _I),
        "lepic_dev_cw_push": ([C.POINTER(LepicGrid), vp, C.POINTER(LepicWinSpecies), _I, C.POINTER(LepicPhys),
                               _I, vp, vp], _I),
        "lepic_dev_cw_reverse": ([C.POINTER(LepicGrid), vp, C.POINTER(LepicWinSpecies), _I,
                                  C.POINTER(LepicPhys), _I, vp], _I),
        "lepic_dev_cw_adj_push": ([C.POINTER(LepicGrid), vp, C.POINTER(LepicWinSpecies), _I,
                                   C.POINTER(LepicPhys), _I, _D, vp, vp, vp], _I),
        "lepic_dev_cw_adj_deposit": ([C.POINTER(LepicGrid), C.POINTER(LepicWinSpecies), _I,
                                      C.POINTER(LepicPhys), _I, vp, vp], _I),
        "lepic_dev_win_collisions": ([C.POINTER(LepicGrid), C.POINTER(LepicWinSpecies), _I,
                                      C.POINTER(LepicTables), C.POINTER(LepicPhys), C.c_ulonglong, C.c_ulonglong,
                                      _I, vp, _I, vp, P_dbl, C.POINTER(C.c_longlong), vp], _I),
        "lepic_dev_cw_replay": ([C.POINTER(LepicGrid), C.POINTER(LepicWinSpecies), _I, C.POINTER(LepicPhys),
                                 vp, _I, vp], _I),
        "lepic_dev_cw_adj_collide": ([C.POINTER(LepicGrid), C.POINTER(LepicWinSpecies), _I,
                                      C.POINTER(LepicPhys), vp, _I, vp], _I),
        "lepic_dev_eheating": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesF64), C.POINTER(LepicPhys),
                               C.POINTER(LepicHeat), C.c_double, vp, C.c_ulonglong, C.c_ulonglong, vp, vp], _I),
        "lepic_dev_eheating_mixed": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesMixed), C.POINTER(LepicPhys),
                                     C.POINTER(LepicHeat), C.c_double, vp, C.c_ulonglong, C.c_ulonglong, vp,
                                     vp], _I),
        "lepic_dev_heat_stats": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesF64), C.POINTER(LepicPhys),
                                  C.POINTER(LepicHeat), vp, vp], _I),
        "lepic_dev_heat_stats_mixed": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesMixed), C.POINTER(LepicPhys),
                                        C.POINTER(LepicHeat), vp, vp], _I),
        "eheating_": ([P_dbl, P_dbl, P_int, P_int, P_int, P_int, P_int, P_dbl, P_int, P_dbl], None),
        "part_injection_": ([P_int, P_dbl, P_int, P_dbl, P_int, P_int, P_int, P_int, P_int, P_dbl, P_dbl, P_dbl,
                             P_dbl, P_dbl, P_dbl, P_dbl, P_int, P_int, P_int, P_int, P_int, P_int, P_dbl, P_dbl,
                             P_dbl], None),
        "lepic_dev_inject": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesF64), _I, C.POINTER(LepicPhys),
                              C.POINTER(LepicInject), C.c_longlong, C.c_ulonglong, C.c_ulonglong, vp, vp, P_dbl,
                              C.POINTER(C.c_longlong), vp], _I),
        "lepic_dev_inject_mixed": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesMixed), _I, C.POINTER(LepicPhys),
                                    C.POINTER(LepicInject), C.c_longlong, C.c_ulonglong, C.c_ulonglong, vp, vp,
                                    P_dbl, C.POINTER(C.c_longlong), vp], _I),
        "lepic_dev_load_uniform": ([C.POINTER(LepicGrid), C.POINTER(LepicSpeciesF64), _I,
                                    C.c_longlong, C.POINTER(LepicPhys), C.c_ulonglong, vp], _I),
        "lepic_dev_cell_wall": ([P_int, vp, vp, vp], _I),
        "lepic_dev_dielectric_phi": ([C.POINTER(LepicGrid), vp, C.POINTER(LepicPhys), _I, C.c_double, vp], _I),
        "lepic_dev_dens_red": ([C.POINTER(LepicGrid), vp, vp, _I, P_dbl, vp], _I),
        "lepic_timing_enable": ([_I], None),
        "lepic_timing_reset": ([], None),
        "lepic_timing_read": ([C.c_char_p, _I, P_dbl, C.POINTER(C.c_longlong), _I], _I),
        "calc_rho_": ([P_int, P_dbl, P_dbl, P_int, P_int, P_int, P_int, P_int], None),
        "dens_red_": ([P_int, P_dbl, P_dbl, P_int, P_int, P_int, P_int], None),
        "pdesolver_": ([P_dbl, P_dbl, P_int, P_dbl, P_int, P_int, P_dbl, P_dbl, P_int, P_dbl, P_dbl,
                        P_int, P_int, P_int], None),
        "calc_efield_": ([P_int, P_dbl, P_dbl, P_dbl, P_int], None),
        "part_mover_": ([P_int, P_dbl, P_dbl, P_dbl, P_dbl, P_dbl, P_dbl, P_int, P_int, P_int, P_int,
                         P_i8, P_int, P_int, P_int, P_int, P_int, P_int, P_dbl, P_dbl, P_dbl, P_dbl,
                         P_int, P_int, P_int, P_dbl], None),
        "charge_deposition_": ([P_int, P_dbl, P_dbl, P_int, P_int, P_dbl, P_dbl, P_int, P_int, P_dbl,
                                P_int, P_int, P_int], None),
        "part_sorting_": ([P_dbl, P_dbl, P_int, P_int, P_int, P_dbl, P_int, P_int, P_int, P_int, P_int],
                          None),
        "collisions_": ([P_int, P_dbl, P_int, P_dbl, P_int, P_int, P_dbl, P_dbl, P_int, P_dbl, P_int,
                         P_int, P_dbl, P_dbl, P_int, P_int, P_int, P_int, P_dbl, P_int, P_dbl, P_i8,
                         P_int, P_int, P_int, P_int, P_int, P_int, P_dbl, P_dbl, P_dbl, P_int], None),
    }
    for name, (args, res) in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def commons():
    """The library's COMMON-block structs (Fortran layout)."""
    L = lib()
    return dict(part_info_int=PartInfoInt.in_dll(L, "part_info_int_"),
                part_info_dp_1=PartInfoDp1.in_dll(L, "part_info_dp_1_"),
                part_info_dp_2=PartInfoDp2.in_dll(L, "part_info_dp_2_"),
                part_info_dp_3=PartInfoDp3.in_dll(L, "part_info_dp_3_"),
                constants=Constants.in_dll(L, "constants_"))


def exported_symbols():
    """Names declared in include/lepic_gpu.h that the library must export."""
    return ["lepic_gpu_last_error", "lepic_gpu_strerror", "lepic_build_info", "lepic_dev_info", "lepic_dev_check",
            "lepic_dev_wait_selftest", "lepic_dev_check_async", "lepic_dev_pdesolver_mixed_stats",
            "lepic_gpu_set_residency", "lepic_gpu_residency", "lepic_gpu_sync_to_host",
            "lepic_gpu_update_host", "lepic_gpu_update_device", "lepic_gpu_release",
            "lepic_gpu_release_all", "lepic_gpu_mirror_zero", "lepic_gpu_mirror_copy",
            "lepic_gpu_mirror_stats",
            "lepic_dev_calc_rho", "lepic_dev_calc_efield", "lepic_dev_pdesolver",
            "lepic_dev_pdesolver_noalloc",
            "lepic_dev_part_mover", "lepic_dev_push_deposit", "lepic_dev_charge_deposition", "lepic_dev_part_sorting",
            "lepic_dev_collisions", "lepic_dev_push_deposit_mixed", "lepic_dev_sort_mixed",
            "lepic_dev_pack_e32", "lepic_dev_load_uniform_mixed", "lepic_dev_deposit_mixed", "lepic_dev_f64_to_mixed", "lepic_dev_mixed_to_f64",
            "lepic_dev_pdesolver_mixed", "lepic_dev_collisions_mixed", "lepic_dev_load_uniform",
            "lepic_dev_win_push", "lepic_dev_win_deposit", "lepic_dev_adj_push", "lepic_dev_adj_efield",
            "lepic_dev_adj_rhs", "lepic_dev_adj_walls", "lepic_dev_adj_deposit", "lepic_dev_cell_wall",
            "lepic_dev_cw_deposit", "lepic_dev_cw_back", "lepic_dev_cw_push", "lepic_dev_cw_reverse", "lepic_dev_cw_adj_push",
            "lepic_dev_cw_adj_deposit", "lepic_dev_win_collisions", "lepic_dev_cw_replay",
            "lepic_dev_cw_adj_collide",
            "lepic_dev_dielectric_phi",
            "lepic_dev_dens_red", "lepic_timing_enable", "lepic_timing_reset", "lepic_timing_read",
            "calc_rho_", "dens_red_", "pdesolver_", "calc_efield_",
            "part_mover_", "charge_deposition_", "part_sorting_", "collisions_", "eheating_",
            "lepic_dev_eheating", "lepic_dev_eheating_mixed", "lepic_dev_heat_stats", "lepic_dev_heat_stats_mixed",
            "lepic_dev_collisions_targets", "lepic_dev_collisions_mixed_targets",
            "part_injection_", "lepic_dev_inject", "lepic_dev_inject_mixed",
            "part_info_int_", "part_info_dp_1_", "part_info_dp_2_", "part_info_dp_3_", "constants_"]


def timing(enable=None, reset=False):
    """Per-kernel device timers: returns {name: (total_ms, launches)}."""
    L = lib()
    if enable is not None:
        L.lepic_timing_enable(1 if enable else 0)
    if reset:
        L.lepic_timing_reset()
        return {}
    buf = C.create_string_buffer(8192)
    ms = (C.c_double * 128)()
    cnt = (C.c_longlong * 128)()
    k = L.lepic_timing_read(buf, 8192, ms, cnt, 128)
    names = buf.value.decode().split("\n")[:k]
    return {nm: (ms[i], cnt[i]) for i, nm in enumerate(names)}


class LepicError(RuntimeError):
    """A status code from the GPU library (the reference's stop_calculation)."""

    def __init__(self, code, where=""):
        msg = lib().lepic_gpu_strerror(int(code)).decode()
        super().__init__(f"{where}: lepic status {code} ({msg})" if where else f"lepic status {code} ({msg})")
        self.code = int(code)


def check(rc, where=""):
    if rc:
        raise LepicError(rc, where)


def phys_struct(st, cls=LepicPhys, bmap_ptr=None):
    """Fill a LepicPhys (or the oracle's OPhys, same layout) from a Setup.
    With a B-field map (st.bfield) the map's pointer is ``bmap_ptr`` (a
    device address for the device API); by default the host array's, which
    only the CPU oracle may read."""
    from .constants import EPS0, PI, QE
    P = cls()
    P.ntype = st.ntype
    P.n_neu = st.n_neu
    for i in range(NPART):
        P.charge[i] = st.charge[i]
        P.mass[i] = st.mass[i]
        P.vt0[i] = st.vt0[i]
        P.Nm[i] = st.Nm[i]
        P.np_mx[i] = st.np_mx[i]
        P.nu_uplim[i] = st.nu_uplim[i]
    P.dt = st.dt
    P.xmax, P.ymax, P.zmax = (float(v) for v in st.geom.box)
    P.x_load = st.x_load
    P.qe, P.eps0, P.pi = QE, EPS0, PI
    P.flag_B = st.flag_B
    P.flag_B_pos = int(getattr(st, "flag_B_pos", 0))
    P.flag_pbc = st.geom.flag_pbc
    P.flag_nmn = st.geom.flag_nmn
    P.ns_coll = st.wl.ns_coll
    P.n_cell = st.n_cell
    P.np_cell = st.np_cell
    for i in range(3):
        P.Bconst[i] = st.Bconst[i]
    bf = getattr(st, "bfield", None)
    if bf is not None:
        for i in range(3):
            P.n_B[i] = int(bf.n_B[i])
            P.h_B[i] = float(bf.h_B[i])
        P.Bmap = int(bmap_ptr) if bmap_ptr is not None else bf.Bi.ctypes.data
    return P


def as_ptr(a, ctype):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ctype))


def np_i(a):
    return np.ascontiguousarray(a, dtype=np.int32)
