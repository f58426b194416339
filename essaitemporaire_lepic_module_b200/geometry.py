"""Wall-label mask and Dirichlet potential of the simulation box.

Restates Src/generate_boundary.f90:1-453 of the reference (metal walls,
solid electrode blocks, periodic planes, the left-hand Neumann plane and the
dielectric-plane labels; cylindrical segments and grid holes are out of
scope and rejected).  Lengths come in centimetres like ``geometry.inp`` and
are converted to metres at the end (Src/generate_boundary.f90:392-395).

Arrays are returned in the reference's column-major layout: a numpy array of
shape ``(n3+3, n2+3, n1+3)`` in C order is the Fortran array
``bcnd(0:n1+2, 0:n2+2, 0:n3+2)``; index it as ``a[iz, iy, ix]``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Geometry:
    n: tuple                   # cells (n1, n2, n3)
    h: np.ndarray              # cell size in metres
    box: np.ndarray            # (xmax, ymax, zmax) in metres
    bcnd: np.ndarray           # int32 (n3+3, n2+3, n1+3): -1 plasma, >=1 wall label, 0 periodic, -2 Neumann
    phi: np.ndarray            # float64 potential with the Dirichlet wall values
    dtype: dict = field(default_factory=dict)   # wall label -> 1 metal, 2..4 dielectric
    flag_pbc: int = 0
    flag_pbcz: int = 0
    flag_nmn: int = 0
    flag_die: int = 0
    ngrid: int = 1

    def dtype_array(self) -> np.ndarray:
        """dtype(0:ngrid) as the reference passes it: 0 for unused labels."""
        a = np.zeros(self.ngrid + 1, dtype=np.int32)
        for g, t in self.dtype.items():
            if 0 <= g <= self.ngrid:
                a[g] = t
        return a


def generate_boundary(n, box_cm, segments, V):
    """Build the mask like Src/generate_boundary.f90 does from geometry.inp.

    n        -- cells (n1, n2, n3)
    box_cm   -- first line of geometry.inp: xmax, ymax, zmax in cm (xmax < 0
                selects the left-hand Neumann plane)
    segments -- rows (xl, yl, zl, xr, yr, zr, ind) in cm: ind > 0 draws a box
                whose x-range becomes walls labelled ind and whose interior
                becomes plasma; ind < 0 paints a solid block labelled |ind|;
                ind = 0 draws periodic planes.  xr < 0 / yr < 0 mark
                dielectric planes, zr < 0 makes the z = 1, n3+1 planes
                periodic where they touch plasma.
    V        -- wall potentials V[1..ngrid] (index 0 unused), volts.
    """
    n1, n2, n3 = (int(v) for v in n)
    xmax, ymax, zmax = (float(v) for v in box_cm)
    flag_nmn = 1 if xmax < 0 else 0
    xmax = abs(xmax)
    if ymax < 0 or zmax < 0:
        raise ValueError("cylindrical segments are not supported")
    h = np.array([xmax / n1, ymax / n2, zmax / n3], dtype=np.float64)
    bcnd = np.zeros((n3 + 3, n2 + 3, n1 + 3), dtype=np.int32)
    u = np.zeros((n3 + 3, n2 + 3, n1 + 3), dtype=np.float64)
    dtype = {}
    flag_pbc = flag_pbcz = flag_die = 0
    cnt_yz_planes = 0
    ngrid = len(V) - 1
    for seg in segments:
        xl, yl, zl, xr, yr, zr, ind = seg
        ind = int(ind)
        dtype[abs(ind)] = 1
        if yl < 0:
            raise ValueError("cylindrical segments are not supported")
        if ind == 0:
            flag_pbc = 1
        if xr < 0:
            xr = abs(xr)
            dtype[abs(ind)] = 3 if cnt_yz_planes == 0 else 4
            cnt_yz_planes += 1
            flag_die = 1
        if yr < 0:
            yr = abs(yr)
            dtype[abs(ind)] = 2
            flag_die = 1
        if zr < 0:
            zr = abs(zr)
            dtype[abs(ind)] = -dtype[abs(ind)]
            flag_pbc = 1
            flag_pbcz = 1
        if abs(ind) > ngrid:
            raise ValueError("insufficient number of wall labels")
        ixl = int(xl / h[0]) + 1
        if ixl <= 1:
            ixl = 0
        ixr = int(xr / h[0]) + 1
        if ixr >= n1:
            ixr = n1 + 2
        iyl = int(yl / h[1]) + 1
        if iyl <= 1:
            iyl = 0
        iyr = int(yr / h[1]) + 1
        if iyr >= n2:
            iyr = n2 + 2
        izl = int(zl / h[2]) + 1
        if izl <= 1:
            izl = 0
        izr = int(zr / h[2]) + 1
        if izr >= n3:
            izr = n3 + 2
        if ind == 0:
            ixl = max(ixl, 2)
            ixr = min(ixr, n1)
        if ind >= 0:
            bcnd[:, :, ixl:ixr + 1] = ind
            if ind > 0:
                u[:, :, ixl:ixr + 1] = V[ind]
            ixl, ixr = max(ixl, 2), min(ixr, n1)
            iyl, iyr = max(iyl, 2), min(iyr, n2)
            izl, izr = max(izl, 2), min(izr, n3)
            bcnd[izl:izr + 1, iyl:iyr + 1, ixl:ixr + 1] = -1
            u[izl:izr + 1, iyl:iyr + 1, ixl:ixr + 1] = 0.0
        else:
            bcnd[izl:izr + 1, iyl:iyr + 1, ixl:ixr + 1] = abs(ind)
            if abs(ind) > 0:
                u[izl:izr + 1, iyl:iyr + 1, ixl:ixr + 1] = V[abs(ind)]
    if flag_nmn:
        bcnd[:, :, 0:2] = -2
        u[:, :, 0:2] = 0.0
    if flag_pbc:
        ig = bcnd[1, :, :]
        neg = np.vectorize(lambda g: dtype.get(int(g), 0) < 0)(ig) & (bcnd[2, :, :] == -1)
        for iz in (0, 1, n3 + 1, n3 + 2):
            bcnd[iz][neg] = 0
    dtype = {k: abs(v) for k, v in dtype.items()}
    return Geometry(n=(n1, n2, n3), h=h * 1e-2, box=np.array([xmax, ymax, zmax]) * 1e-2,
                    bcnd=bcnd, phi=u, dtype=dtype, flag_pbc=flag_pbc, flag_pbcz=flag_pbcz,
                    flag_nmn=flag_nmn, flag_die=flag_die, ngrid=ngrid)


def count_cells(bcnd, n, ix_pe):
    """Cells with at least one plasma node, Src/main.f90:637-648."""
    n1, n2, n3 = n
    b = bcnd
    cnt = 0
    pl = (b == -1)
    any8 = (pl[1:n3 + 1, 1:n2 + 1, 1:ix_pe + 1] | pl[1:n3 + 1, 1:n2 + 1, 2:ix_pe + 2] |
            pl[1:n3 + 1, 2:n2 + 2, 2:ix_pe + 2] | pl[1:n3 + 1, 2:n2 + 2, 1:ix_pe + 1] |
            pl[2:n3 + 2, 1:n2 + 1, 1:ix_pe + 1] | pl[2:n3 + 2, 1:n2 + 1, 2:ix_pe + 2] |
            pl[2:n3 + 2, 2:n2 + 2, 2:ix_pe + 2] | pl[2:n3 + 2, 2:n2 + 2, 1:ix_pe + 1])
    cnt = int(any8.sum())
    return cnt


def read_mco(path):
    """Read a reference ``.mco`` 2D plane (header n1 n2, rows top-down).

    Returns an array ``a[j, i]`` with j the row coordinate counted from the
    bottom (index 1 of the reference) -- i.e. rows are flipped back.
    """
    with open(path) as f:
        head = f.readline().split()
        n1, n2 = int(head[0]), int(head[1])
        vals = [float(v) for v in f.read().split()]
    a = np.array(vals, dtype=np.float64).reshape(n2 + 1, n1 + 1)
    return a[::-1, :].copy()
