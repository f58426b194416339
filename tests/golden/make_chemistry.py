"""Generate the chemistry fixtures of the reference's own chemistry files.

Reads the reference's input_dir/hydrogen.dat (5 charged species, 2 neutrals,
60 reactions of every type, charged targets included) and input_dir/argon.dat
(e, Ar+ and Ar: the e-Ar+ Coulomb collision with a charged target, e-Ar
elastic, excitation and ionization, Ar+-Ar elastic and charge exchange) with
the package's restatement of Src/read_reactions.f90 and stores each parsed
chemistry in hydrogen_chem.npz / argon_chem.npz: the species (name, mass in
amu, charge in e, T in eV, n/n0 as the file gives them) and every reaction
(label, col_info row, threshold, scaled E / sigma table).  The tests rebuild
a Chemistry from them with reactions.chemistry_from_arrays, so they need no
reference tree.

Run here (the reference tree is read only):
    python tests/golden/make_chemistry.py /path/to/reference   (or LEPIC_REFERENCE=...)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from essaitemporaire_lepic_module_b200 import reactions as rx  # noqa: E402
from essaitemporaire_lepic_module_b200.constants import AMU, QE  # noqa: E402


def main(ref):
    for src, dst in (("hydrogen.dat", "hydrogen_chem.npz"), ("argon.dat", "argon_chem.npz")):
        fixture(os.path.join(ref, "input_dir", src), os.path.join(HERE, dst))


def fixture(src, dst):
    chem = rx.read_dat(src, Te=1.0, ngas=1.0)
    sp = chem.species
    E = [t[0] for t in chem.tables]
    S = [t[1] for t in chem.tables]
    off = np.concatenate([[0], np.cumsum([len(e) for e in E])]).astype(np.int64)
    np.savez_compressed(
        dst,
        sp_name=np.array([s.name for s in sp]),
        sp_mass_amu=np.array([abs(s.mass) / AMU for s in sp]),
        sp_charge_e=np.array([s.charge / QE for s in sp]),
        sp_T=np.array([s.T for s in sp]),
        sp_n=np.array([s.ni0 for s in sp]),
        labels=np.array(chem.labels), col_info=chem.col_info, Eth=chem.Eth,
        tab_off=off, tab_E=np.concatenate(E), tab_S=np.concatenate(S))
    print("wrote", dst, len(chem.labels), "reactions")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LEPIC_REFERENCE")
    if not ref:
        sys.exit("usage: python tests/golden/make_chemistry.py <reference tree> (or set LEPIC_REFERENCE)")
    main(ref)
