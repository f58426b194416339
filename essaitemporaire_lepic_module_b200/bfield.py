"""B-field maps of the push, built like the reference builds them.

The legacy driver fills ``Bi(4, 0:n_B(1)+2, 0:n_B(2)+2, 0:n_B(3)+2)`` once
at start-up (Src/main.f90:361-431): each magnet entry of the input adds a
profile to one or more components, then ``Bi(4, ...) = |B|``.  The push reads
it (Src/part_expmover.f90:148-203): on the node grid (``n_B = n``) with the
E-field's cell and weights, on any other ``n_B`` at index ``INT(x/h_B)+1``
with weights from ``h_B = (xmax, ymax, zmax) / n_B``; a particle whose left
map node has ``|B| <= 1e-5 T`` takes the leapfrog step.  ``n_B(1) = 1`` is the
uniform field ``Bi(1:3, 1, 1, 1)`` (``Setup.Bconst``).

``BField.Bi`` is a C-ordered array of shape (nB3+3, nB2+3, nB1+3, 4), which
is the memory layout of the Fortran array.

    bf = new_map(st, n_B=st.n)              # on the node grid
    gaussian(bf, B0=0.01, x0=8e-4, Lx=2e-4, B_dir=3)
    finish(bf)                               # |B| and Bmax
    attach(st, bf)                           # st.bfield, st.flag_B = 1
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GATE = 1.0e-5   # T: below it a particle is not magnetised (Src/part_expmover.f90:158)


@dataclass
class BField:
    n_B: tuple
    h_B: np.ndarray
    Bi: np.ndarray
    Bmax: float = 0.0

    def nodes(self):
        """Node coordinates (x, y, z) of the map, ``(i-1) h_B`` per axis."""
        return tuple((np.arange(self.n_B[a] + 3) - 1.0) * self.h_B[a] for a in range(3))


def new_map(st, n_B=None):
    """An empty map on ``n_B`` (default: the node grid) over the box of ``st``."""
    n_B = tuple(int(v) for v in (st.n if n_B is None else n_B))
    if n_B[0] < 2 or min(n_B) < 1:
        raise ValueError("a map needs n_B(1) > 1 (n_B(1) = 1 is the uniform field)")
    box = np.array([float(v) for v in st.geom.box], dtype=np.float64)
    h_B = box / np.array(n_B, dtype=np.float64)        # Src/main.f90:364-366
    Bi = np.zeros((n_B[2] + 3, n_B[1] + 3, n_B[0] + 3, 4))
    return BField(n_B, h_B, Bi)


def read_map_file(bf, path, B_dir, scaling=1.0):
    """Src/Bfield.f90:1-41 (read_Bfield_map): rows ``ix iy iz B`` (T), added
    times ``scaling`` to component ``B_dir`` (1..3) at node (ix, iy, iz);
    at most (nB1+3)(nB2+3)(nB3+3) rows are read."""
    nmax = bf.Bi.shape[0] * bf.Bi.shape[1] * bf.Bi.shape[2]
    with open(path) as f:
        for k, line in enumerate(f):
            if k >= nmax:
                break
            parts = line.split()
            if len(parts) < 4:
                break
            ix, iy, iz = (int(v) for v in parts[:3])
            bf.Bi[iz, iy, ix, B_dir - 1] += float(parts[3]) * scaling
    return bf


def gaussian(bf, B0, x0, Lx, B_dir):
    """Src/Bfield.f90:44-68 (gaussian_Bfield): ``B0 exp(-(x-x0)^2 / (2 Lx^2))``
    along x, uniform in y and z, added to component ``B_dir``."""
    x = bf.nodes()[0]
    bf.Bi[:, :, :, B_dir - 1] += (B0 * np.exp(-(x - x0) ** 2 / (2 * Lx ** 2)))[None, None, :]
    return bf


# Franzen et al., Plasma Phys. Control. Fusion 56 (2014) 025007, Fig. 5: the
# filter-field profile of the ELISE source in G against x in cm, a quartic up
# to 39 cm and a straight line beyond (the fit of Src/Bfield.f90:83-92).  The
# reference writes the coefficients as default-real (single precision)
# literals, so its doubles hold their float32 roundings; so do these.
_PG_QUARTIC = tuple(float(np.float32(v)) for v in (0.0175596, 0.0227362, 0.00193113, -8.51235e-05, 9.58673e-07))
_PG_LINE = tuple(float(np.float32(v)) for v in (15.7416, -0.377132))


def pg_current(bf, B0, B_dir):
    """Src/Bfield.f90:71-118 (PG_current): ``B0`` times the fitted profile of
    x (in cm), added to component ``B_dir``."""
    x = bf.nodes()[0] * 1.0e2
    a, b = _PG_QUARTIC, _PG_LINE
    quart = a[0] + a[1] * x + a[2] * x ** 2 + a[3] * x ** 3 + a[4] * x ** 4
    prof = np.where(x <= 39.0, quart, b[0] + b[1] * x)
    bf.Bi[:, :, :, B_dir - 1] += (B0 * prof)[None, None, :]
    return bf


def ee_magnets(bf, B0, x0, z0, d):
    """Src/Bfield.f90:120-149 (EE_magnets): the cusp field of a row of
    magnets at x0 with period 2d in z, centred on z0:
    ``Bx += B0 sin(pi (z-z0)/d) exp(-pi (x0-x)/d)``,
    ``Bz += B0 cos(pi (z-z0)/d) exp(-pi (x0-x)/d)``."""
    x, _, z = bf.nodes()
    ex = np.exp(-np.pi * (x0 - x) / d)[None, None, :]
    arg = (np.pi * (z - z0) / d)[:, None, None]
    bf.Bi[:, :, :, 0] += B0 * np.sin(arg) * ex
    bf.Bi[:, :, :, 2] += B0 * np.cos(arg) * ex
    return bf


def _bx_magnet(x, y, a):
    # Src/Bfield.f90:200-214: x component of the field of a magnet pair
    return 0.5 * (a * x / (x ** 2 + (y + a) ** 2) - a * x / (x ** 2 + (y - a) ** 2))


def _by_magnet(x, y, a):
    # Src/Bfield.f90:216-230: y component of the same
    return 0.5 * (a * (y + a) / (x ** 2 + (y + a) ** 2) - a * (y - a) / (x ** 2 + (y - a) ** 2))


def hall_thruster(bf, B0, x0, a):
    """Src/Bfield.f90:151-197 (Bfield_Hall_thruster): two magnet pairs (the
    second at x0 - 2d, strength ratio 0.75, d = 1.5 cm) about the channel
    axis y0 = 2 cm; ``B0 < 0`` gives the pseudo-1D variant (y0 = 0, Bx = 0,
    By uniform in y and z at its value at iy = iz = 1)."""
    d, y0, alpha = 1.5e-2, 2.0e-2, 0.75
    B1 = abs(B0) / (1 - alpha * a ** 2 / (4.0 * d ** 2 + a ** 2))
    B2 = alpha * B1
    if B0 < 0:
        y0 = 0.0
    x, y, _ = bf.nodes()
    X, Y = x[None, :], y[:, None]
    bf.Bi[:, :, :, 0] += (B1 * _bx_magnet(X - x0, Y - y0, a) - B2 * _bx_magnet(X - x0 + 2 * d, Y - y0, a))[None]
    bf.Bi[:, :, :, 1] += (B1 * _by_magnet(X - x0, Y - y0, a) - B2 * _by_magnet(X - x0 + 2 * d, Y - y0, a))[None]
    if B0 < 0:
        bf.Bi[:, :, :, 0] = 0.0
        bf.Bi[:, :, :, 1] = bf.Bi[1, 1, :, 1][None, None, :]
    return bf


def finish(bf):
    """Src/main.f90:420-431: ``Bi(4, ...) = |B|`` and ``Bmax``."""
    B = bf.Bi
    B[..., 3] = np.sqrt(B[..., 0] * B[..., 0] + B[..., 1] * B[..., 1] + B[..., 2] * B[..., 2])
    bf.Bmax = float(B[..., 3].max())
    return bf


def attach(st, bf, flag_B_pos=None):
    """Give the set-up ``st`` the map ``bf`` (after ``finish``): the push of
    every species then reads it.  ``flag_B_pos = 1`` leaves positive ions
    unmagnetised (a negative magnet count in the reference's input)."""
    bf.Bi = np.ascontiguousarray(bf.Bi, dtype=np.float64)
    if bf.Bi.shape != (bf.n_B[2] + 3, bf.n_B[1] + 3, bf.n_B[0] + 3, 4):
        raise ValueError(f"B-field map of shape {bf.Bi.shape} for n_B = {tuple(bf.n_B)}")
    if not np.all(np.isfinite(bf.Bi)):
        raise ValueError("B-field map has non-finite values")
    st.bfield = bf
    st.flag_B = 1
    if flag_B_pos is not None:
        st.flag_B_pos = int(flag_B_pos)
    return st
