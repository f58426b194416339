"""Host-side logic and the C ABI surface (no GPU needed).

* liblepic_gpu.so loads and exports every function and COMMON block that
  include/lepic_gpu.h declares (no compute call is made);
* the COMMON-block structs have the Fortran member order of
  Src/particle_info.h (sizes checked against a member count);
* the workloads derive the constants the reference derives.
"""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

from essaitemporaire_lepic_module_b200 import _lib, config, reactions
from essaitemporaire_lepic_module_b200.constants import QE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lepic_gpu.h")


def header_names():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    funcs = set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src))
    funcs -= {"if", "for", "while", "return", "sizeof"}
    externs = set(re.findall(r"extern\s+\w+\s+([A-Za-z_][A-Za-z0-9_]*)\s*;", src))
    # only declarations (names followed by an argument list at top level)
    decl = set(re.findall(r"^\s*(?:const\s+)?(?:int|void|char|double)\s*\*?\s*([A-Za-z_]\w*)\s*\(",
                          src, flags=re.M))
    return decl, externs


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    decl, externs = header_names()
    assert len(decl) >= 20
    for name in sorted(decl | externs):
        assert hasattr(L, name), f"{name} declared in lepic_gpu.h but not exported"
    assert set(_lib.exported_symbols()) <= (decl | externs)


def test_common_blocks_match_fortran_layout():
    # /part_info_int/ : 12 ints + p_ncol(10) + nscol + p_nscol(10) + 16 ints
    # + ixl_rg(5) + ns_inj + ixr_rg(5) + 18 ints + ig_die(5) + 13 ints
    n_int = 12 + 10 + 1 + 10 + 16 + 5 + 1 + 5 + 18 + 5 + 13
    assert C.sizeof(_lib.PartInfoInt) == 4 * n_int
    # /part_info_dp_1/ : charge,mass,Ti,vt0 (4x10) + k_eps0 + 6 x (5) + 9 + zg_sec(2)
    assert C.sizeof(_lib.PartInfoDp1) == 8 * (40 + 1 + 30 + 9 + 2)
    # /part_info_dp_2/ : Pabs,n0,ngas + Nm(10) + 15
    assert C.sizeof(_lib.PartInfoDp2) == 8 * (3 + 10 + 15)
    assert C.sizeof(_lib.PartInfoDp3) == 8 * 30
    assert C.sizeof(_lib.Constants) == 8 * 5
    cm = _lib.commons()
    # the library's storage is reachable (weak definitions)
    cm["constants"].qe = QE
    assert cm["constants"].qe == QE


def test_status_strings():
    L = _lib.lib()
    for code in (0, 1, 2, 3, 4, 5, 6, 7, 20, 21, 22, 23, 24):
        assert L.lepic_gpu_strerror(code).decode() != "unknown status"
    assert L.lepic_gpu_last_error() == 0


@pytest.mark.parametrize("name,n_cell,ng", [("box16", 16 ** 3, 4), ("box32", 32 ** 3, 5),
                                            ("mcc32", 32 ** 3, 5), ("penning_small", 16 * 16 * 32, 4)])
def test_workload_constants(name, n_cell, ng):
    st = config.build(name)
    assert st.n_cell == n_cell
    assert st.ng == ng
    h3 = st.h[0] * st.h[1] * st.h[2]
    for p in range(st.ntype):
        # Src/main.f90:535-548
        assert st.vt0[p] == math.sqrt(2.0 * QE * st.Ti[p] / abs(st.mass[p]))
        assert st.Nm[p] == st.wl.n0 * h3 / st.np_cell
    assert st.n_particles() == st.np_cell * st.n_cell


def test_electrode_and_end_plate_geometry():
    st = config.build("poisson64")
    labels, counts = np.unique(st.geom.bcnd, return_counts=True)
    assert set(labels) == {-1, 1, 2, 3}
    V = st.wl.V
    assert np.all(st.geom.phi[st.geom.bcnd == 2] == V[2])
    assert np.all(st.geom.phi[st.geom.bcnd == 3] == V[3])
    assert np.all(st.geom.phi[st.geom.bcnd == -1] == 0.0)
    pen = config.build("penning_small")
    n1, n2, n3 = pen.n
    assert np.all(pen.geom.bcnd[0:2] == 2) and np.all(pen.geom.bcnd[n3 + 1:] == 3)
    assert np.all(pen.geom.phi[pen.geom.bcnd == 2] == 200.0)
    assert np.all(pen.geom.phi[pen.geom.bcnd == 3] == 200.0)
    assert np.all(pen.geom.bcnd[2:n3, 2:n2 + 1, 2:n1 + 1] == -1)


def test_chemistry_roundtrip(tmp_path):
    path = tmp_path / "argon.dat"
    reactions.write_dat(str(path), [("[Ar+]", 39.95, 1.0, 0.026, 1.0)],
                        [("[Ar]", -39.95, 0.0, 0.02585, 1.0)], reactions.argon_tables_synthetic())
    chem = reactions.read_dat(str(path), 2.0, 2.4e20)
    assert [s.name for s in chem.species] == ["[e]", "[Ar+]", "[Ar]"]
    assert chem.ntype == 2 and chem.n_neu == 1
    ion = chem.col_info[2]          # [e]+[Ar]->[e]+[Ar+]+[e]
    assert list(ion[:9]) == [2, 3, 1, 3, 1, 2, 1, 2, 2]
    cx = chem.col_info[3]           # [Ar+]+[Ar]->[Ar+]+[Ar]
    assert list(cx[:8]) == [2, 2, 2, 3, 2, 3, 4, 0]
    T = reactions.ordering(chem)
    assert np.all(np.diff(T.sig_Er) > 0)
    # (sigma v)_max of the constant elastic cross section is at the top energy
    mu = 9.10938188e-31 * 39.95 * 1.66053886e-27 / (9.10938188e-31 + 39.95 * 1.66053886e-27)
    vmax = math.sqrt(2 * T.sig_Er[-1] * QE / mu)
    assert abs(T.sigv_mx[0, 0] - 1e-19 * vmax) <= 1e-12 * 1e-19 * vmax


def test_residency_switch_and_host_statements_without_mirrors():
    """With residency off, lepic_gpu_mirror_zero / _copy are the host
    statements they stand for (np(...) = 0, the one-rank phi gather); the
    switch and the registry calls make no CUDA call while no mirror exists."""
    L = _lib.lib()
    assert L.lepic_gpu_residency() == 0
    a = np.arange(64, dtype=np.float64)
    b = np.zeros(64)
    vp = lambda x, off=0: C.c_void_p(x.ctypes.data + off)
    assert L.lepic_gpu_mirror_copy(vp(b), vp(a), a.nbytes) == 0
    assert np.array_equal(a, b)
    assert L.lepic_gpu_mirror_zero(vp(b, 8 * 16), 8 * 16) == 0
    assert np.all(b[16:32] == 0) and np.array_equal(b[:16], a[:16]) and np.array_equal(b[32:], a[32:])
    # overlapping copy ranges are refused
    assert L.lepic_gpu_mirror_copy(vp(a, 8), vp(a), 16 * 8) == 21
    assert L.lepic_gpu_set_residency(1) == 0 and L.lepic_gpu_residency() == 1
    assert L.lepic_gpu_sync_to_host() == 0
    h2d, d2h, m = C.c_longlong(0), C.c_longlong(0), C.c_int(-1)
    assert L.lepic_gpu_mirror_stats(C.byref(h2d), C.byref(d2h), C.byref(m)) == 0
    assert m.value == 0
    assert L.lepic_gpu_set_residency(0) == 0 and L.lepic_gpu_residency() == 0
