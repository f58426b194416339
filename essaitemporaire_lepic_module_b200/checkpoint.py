"""Particle backups in the reference's own file format, for checkpoint and
restart across the two codes.

The legacy driver backs the particles up every nbak steps into
DATA.BAK/particlesNNN.bak (Src/main.f90:1294-1330) and a restart reads them
back (Src/restart.f90:62-70).  The file is Fortran unformatted sequential
(the record layout of gfortran and ifort): each WRITE statement is one record
framed by a 4-byte little-endian length before and after it.  The records are

    time                                        real(8)
    np_tot(1:ntype, 1:nproc)                    integer(4), column-major
    vxp(1:6, 1:np_tot(ptype,iproc), ptype, iproc)
                                                real(8), one record per
                                                (iproc, ptype), iproc outer
    flag_cex(1:np_tot(tag_neg,iproc), iproc)    integer(4), after each
                                                iproc's species when
                                                tag_neg > 0

A record longer than 2**31 - 9 bytes (a species of more than ~4.5e7
particles) is split into subrecords the way gfortran writes them: a negative
leading length means that the record continues in the next subrecord, a
negative trailing length that the subrecord continues an earlier one.

    write_particles_bak(path, time, np_tot, vxp)   # vxp: list of (n, 6) FP64
    time, np_tot, vxp, flag_cex = read_particles_bak(path, ntype, nproc=1)
    sim.save_bak(path, time) / sim.load_bak(path)  # Simulation helpers
"""
from __future__ import annotations

import struct

import numpy as np

MAX_SUBRECORD = 2 ** 31 - 9


def _write_record(f, arr, max_sub=MAX_SUBRECORD):
    arr = np.ascontiguousarray(arr)
    if arr.size == 0:
        f.write(struct.pack("<ii", 0, 0))
        return
    data = memoryview(arr.reshape(-1)).cast("B")
    n = len(data)
    off, first = 0, True
    while off < n:
        chunk = min(n - off, max_sub)
        last = off + chunk >= n
        f.write(struct.pack("<i", chunk if last else -chunk))
        f.write(data[off:off + chunk])
        f.write(struct.pack("<i", chunk if first else -chunk))
        off += chunk
        first = False


def _read_record(f, dtype, count=None):
    """One record as a numpy array of `dtype` (`count` items when known, so
    that large records are read straight into their array)."""
    parts = []
    out = None if count is None else np.empty(count, dtype=dtype)
    view = None if out is None else (memoryview(out).cast("B") if count else memoryview(bytearray(0)))
    got, first = 0, True
    while True:
        head = f.read(4)
        if len(head) < 4:
            raise ValueError("truncated record (missing length)")
        h = struct.unpack("<i", head)[0]
        length = abs(h)
        if view is not None:
            if got + length > len(view):
                raise ValueError(f"record longer than the {len(view)} bytes expected")
            if f.readinto(view[got:got + length]) != length:
                raise ValueError("truncated record")
        else:
            b = f.read(length)
            if len(b) != length:
                raise ValueError("truncated record")
            parts.append(b)
        got += length
        t = struct.unpack("<i", f.read(4))[0]
        if abs(t) != length or (t < 0) == first:
            raise ValueError("inconsistent record markers")
        first = False
        if h >= 0:
            break
    if out is not None:
        if got != len(view):
            raise ValueError(f"record of {got} bytes, expected {len(view)}")
        return out
    return np.frombuffer(b"".join(parts), dtype=dtype)


def write_particles_bak(path, time, np_tot, vxp, flag_cex=None, max_sub=MAX_SUBRECORD):
    """np_tot: (ntype,) or (ntype, nproc) counts; vxp: one (n, 6) FP64 array
    per (iproc, ptype), iproc outer, n = np_tot[ptype, iproc];
    flag_cex: one int32 array per iproc (written after that iproc's species)
    or None (tag_neg = 0)."""
    npt = np.asarray(np_tot, dtype=np.int32)
    if npt.ndim == 1:
        npt = npt[:, None]
    ntype, nproc = npt.shape
    if len(vxp) != ntype * nproc:
        raise ValueError(f"{len(vxp)} particle arrays for ntype={ntype}, nproc={nproc}")
    with open(path, "wb") as f:
        _write_record(f, np.array([time], dtype="<f8"), max_sub)
        _write_record(f, np.asfortranarray(npt).T.copy().astype("<i4"), max_sub)  # column-major
        for ip in range(nproc):
            for p in range(ntype):
                a = np.asarray(vxp[ip * ntype + p], dtype="<f8")
                if a.shape != (int(npt[p, ip]), 6):
                    raise ValueError(f"species {p + 1}: array {a.shape}, np_tot {int(npt[p, ip])}")
                _write_record(f, a, max_sub)
            if flag_cex is not None:
                _write_record(f, np.asarray(flag_cex[ip], dtype="<i4"), max_sub)


def read_particles_bak(path, ntype, nproc=1, tag_neg=0):
    """(time, np_tot (ntype, nproc), [ (n, 6) per (iproc, ptype) ], flag_cex
    per iproc or None)."""
    with open(path, "rb") as f:
        time = float(_read_record(f, "<f8", 1)[0])
        npt = _read_record(f, "<i4", ntype * nproc).reshape(nproc, ntype).T.copy()
        vxp, cex = [], []
        for ip in range(nproc):
            for p in range(ntype):
                n = int(npt[p, ip])
                vxp.append(_read_record(f, "<f8", 6 * n).reshape(n, 6))
            if tag_neg > 0:
                cex.append(_read_record(f, "<i4", int(npt[tag_neg - 1, ip])))
    return time, npt, vxp, (cex if tag_neg > 0 else None)
