"""Generate the golden fixtures of the reference's default case.

Reads the reference's committed inputs (input_dir/conditions.inp,
geometry.inp, boundary.inp) and its committed output planes
(DATA/DATA_2D/*.mco, written by Src/generate_boundary.f90:398-451 and
Src/write_data.f90:322-430) and stores them in ref_default_planes.npz:

* bcnd_xy / bcnd_xz / bcnd_yz: wall-label planes of the 3D mask -> pin the
  geometry generator (Src/generate_boundary.f90).
* phi_xy, Ex_xy, Ey_xy (plane iz = n3/2+1) and phi_yz, Ey_yz, Ez_yz (plane
  ix = n1/2+1): time-averaged potential and E-field over the same samples.
  E is linear in phi, so the averaged E equals calc_Efield of the averaged
  phi; the in-plane components depend on in-plane phi values only -> pin the
  E-field stencil (Src/Efield.f90) to the printed precision (6 digits).

Run here (the reference tree is read only):
    python tests/golden/make_golden.py /path/to/reference   (or LEPIC_REFERENCE=...)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_mco(path):
    with open(path) as f:
        head = f.readline().split()
        n1, n2 = int(head[0]), int(head[1])
        vals = [float(v) for v in f.read().split()]
    a = np.array(vals, dtype=np.float64).reshape(n2 + 1, n1 + 1)
    return a[::-1, :].copy()     # row index = second coordinate, counted from 1


def first_tokens(line):
    return line.split("!")[0].replace(",", " ").split()


def main(ref):
    with open(os.path.join(ref, "input_dir", "conditions.inp")) as f:
        lines = f.readlines()
    n = [int(v) for v in first_tokens(lines[4])[:3]]
    ngrid = abs(int(first_tokens(lines[18])[0]))
    geo = []
    with open(os.path.join(ref, "input_dir", "geometry.inp")) as f:
        box = [float(v) for v in first_tokens(f.readline())[:3]]
        for ln in f:
            t = first_tokens(ln)
            if len(t) >= 7:
                geo.append([float(v) for v in t[:6]] + [int(t[6])])
    V = [0.0]
    with open(os.path.join(ref, "input_dir", "boundary.inp")) as f:
        for ln in f:
            t = first_tokens(ln)
            if t:
                V.append(float(t[0]))
    V = V[:ngrid + 1]
    D = os.path.join(ref, "DATA", "DATA_2D")
    out = dict(n=np.array(n), box_cm=np.array(box), segments=np.array(geo), V=np.array(V),
               ngrid=np.array(ngrid))
    for nm in ("bcnd_xy", "bcnd_xz", "bcnd_yz"):
        out[nm] = read_mco(os.path.join(D, nm + ".mco")).astype(np.int16)
    for nm in ("phi_xy", "Ex_xy", "Ey_xy", "phi_yz", "Ey_yz", "Ez_yz"):
        out[nm] = read_mco(os.path.join(D, nm + ".mco"))
    dst = os.path.join(HERE, "ref_default_planes.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LEPIC_REFERENCE")
    if not ref:
        sys.exit("usage: python tests/golden/make_golden.py <reference tree> (or set LEPIC_REFERENCE)")
    main(ref)
