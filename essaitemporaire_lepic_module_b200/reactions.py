"""Cross-section tables in the reference's chemistry ``.dat`` format.

* ``write_dat`` writes a chemistry file (IONS / NEUTRALS / REACTION sections
  with ``----`` separated ``E(eV) sigma(m^2)`` tables) like the reference's
  ``input_dir/argon.dat``.
* ``read_dat`` restates the parts of Src/read_reactions.f90:1-474 that the
  hot path needs (species, reaction labels -> col_info, thresholds, scaled
  tables).  Surface reactions are skipped.
* ``ordering`` restates Src/read_reactions.f90:477-661: one merged sorted
  energy grid, every table re-interpolated on it, (sigma v)_max over
  E >= 1 eV and the per-incident-species reaction lists.

col_info layout (1-based like the reference, Src/read_reactions.f90:12-24):
col_info[icol, 0] = n_re, [1] = n_by, [2:2+n_re] reactant species,
[2+n_re:2+n_re+n_by] byproduct species, [2+n_re+n_by] reaction type
(1 collision, 2 ionization, 3 excitation, 4 charge exchange, 5
dissociation), [3+n_re+n_by] number of byproduct electrons.
"""
from __future__ import annotations

import re
from dataclasses import dataclass

import numpy as np

from .constants import AMU, ME, QE

RTYPES = {"COLLISION": 1, "IONIZATION": 2, "EXCITATION": 3, "CHARGEEXCHANGE": 4, "DISSOCIATION": 5}


@dataclass
class Species:
    name: str
    mass: float        # kg, negative for neutrals (reference convention)
    charge: float      # C
    T: float           # eV
    ni0: float         # n/n0 (neutrals: multiplied by ngas)


@dataclass
class Chemistry:
    species: list          # Species, electrons first, charged before neutrals
    labels: list           # reaction labels
    col_info: np.ndarray   # int32 (ncol, 10), 1-based species indices
    Eth: np.ndarray        # threshold energies (eV) after scaling
    tables: list           # [(E ndarray, sigma ndarray)] after scaling

    @property
    def ntype(self):
        return sum(1 for s in self.species if s.charge != 0.0)

    @property
    def n_neu(self):
        return sum(1 for s in self.species if s.charge == 0.0)


def write_dat(path, ions, neutrals, reactions):
    """ions/neutrals: [(name, mass_amu, charge_e, T_eV, n_over_n0)];
    reactions: [(label, Eth, dE, scaleE, scaleS, rtype, E, sigma)]."""
    out = []
    for title, plist in (("IONS", ions), ("NEUTRALS", neutrals)):
        out.append(title)
        out.append("name   mass  charge  temp.(eV)  n/n0")
        out.append("-" * 37)
        for name, m, q, T, n in plist:
            out.append(f"{name:<6s} {m:10.4f} {q:6.1f} {T:12.6g} {n:6.3f}")
        out.append("-" * 37)
        out.append("")
    for label, Eth, dE, sE, sS, rtype, E, S in reactions:
        out.append("REACTION")
        out.append(label)
        out.append(f" {float(Eth)!r}    {float(dE)!r}")
        out.append(f" {float(sE)!r}    {float(sS)!r}")
        out.append(rtype)
        out.append("-" * 60)
        for e, s in zip(E, S):
            out.append(f" {float(e)!r}  {float(s)!r}")
        out.append("-" * 60)
        out.append("")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_dat(path, Te, ngas):
    """Parse a chemistry file (Src/read_reactions.f90:1-474, subset)."""
    species = [Species("[e]", ME, -QE, float(Te), 1.0)]
    labels, col_info, Eth, tables = [], [], [], []
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    i = 0

    def skip_to_dashes(i):
        while not lines[i].strip().startswith("----"):
            i += 1
        return i + 1

    while i < len(lines):
        tok = lines[i].split()
        name = tok[0][:4].upper() if tok else ""
        if name in ("IONS", "NEUT"):
            i = skip_to_dashes(i + 1)
            while not lines[i][:2] == "--":
                pname = lines[i][:6].strip()
                m, q, T, n = (float(v.replace("d", "e").replace("D", "e")) for v in lines[i][6:].split()[:4])
                q = q * QE
                m = m * AMU
                if q == 0.0:
                    n = n * ngas
                    m = -abs(m)
                species.append(Species(pname, m, q, T, n))
                i += 1
            i += 1
        elif name == "REAC":
            label = lines[i + 1].split()[0]
            eth, de = (float(v) for v in lines[i + 2].split()[:2])
            sE, sS = (float(v) for v in lines[i + 3].split()[:2])
            rtype = lines[i + 4].split()[0].upper()
            i = skip_to_dashes(i + 5)
            E, S = [], []
            while not lines[i].strip().startswith("----"):
                a, b = lines[i].split()[:2]
                E.append(float(a) * sE)
                S.append(float(b) * sS)
                i += 1
            i += 1
            names = [s.name for s in species]
            lhs, rhs = label.split("->")
            re_ = [names.index(t) + 1 for t in re.findall(r"\[[^\]]*\]", lhs)]
            by_ = [names.index(t) + 1 for t in re.findall(r"\[[^\]]*\]", rhs)]
            ci = np.zeros(10, dtype=np.int32)
            ci[0], ci[1] = len(re_), len(by_)
            ci[2:2 + len(re_)] = re_
            ci[2 + len(re_):2 + len(re_) + len(by_)] = by_
            ci[2 + len(re_) + len(by_)] = RTYPES[rtype]
            ci[3 + len(re_) + len(by_)] = sum(1 for b in by_ if b == 1)
            labels.append(label)
            col_info.append(ci)
            Eth.append(eth * sE)
            tables.append((np.array(E), np.array(S)))
        else:
            i += 1
    # charged species first, neutrals after (reference keeps file order; the
    # synthetic files list ions before neutrals)
    return Chemistry(species=species, labels=labels,
                     col_info=np.array(col_info, dtype=np.int32).reshape(-1, 10),
                     Eth=np.array(Eth, dtype=np.float64), tables=tables)


def chemistry_from_arrays(d, Te, ngas):
    """A Chemistry from the arrays a chemistry fixture stores (species name,
    mass in amu, charge in e, T in eV, n/n0; reaction label, col_info row,
    threshold, E / sigma table), with the electron temperature Te and the
    neutral density ngas applied as read_dat applies them."""
    species = []
    for k, name in enumerate(d["sp_name"]):
        name = str(name)
        if k == 0 and name == "[e]":
            species.append(Species("[e]", ME, -QE, float(Te), 1.0))
            continue
        m, q, T, n = (float(d["sp_mass_amu"][k]) * AMU, float(d["sp_charge_e"][k]) * QE,
                      float(d["sp_T"][k]), float(d["sp_n"][k]))
        if q == 0.0:
            n = n * ngas
            m = -abs(m)
        species.append(Species(name, m, q, T, n))
    off = d["tab_off"]
    tables = [(np.array(d["tab_E"][off[c]:off[c + 1]]), np.array(d["tab_S"][off[c]:off[c + 1]]))
              for c in range(len(off) - 1)]
    return Chemistry(species=species, labels=[str(x) for x in d["labels"]],
                     col_info=np.array(d["col_info"], dtype=np.int32).reshape(-1, 10),
                     Eth=np.array(d["Eth"], dtype=np.float64), tables=tables)


@dataclass
class Tables:
    sig_Er: np.ndarray     # merged energy grid (npt,)
    sig: np.ndarray        # (ncol, npt) sigma on the merged grid
    sigv_mx: np.ndarray    # (10, ncol) (sigma v)_max per incident species
    sig_list: np.ndarray   # (10, ncol) 1-based reaction indices per species
    p_ncol: np.ndarray     # (10,)
    Eth: np.ndarray        # (ncol,)
    col_info: np.ndarray   # (ncol, 10)


def ordering(chem: Chemistry, qe=QE):
    """Src/read_reactions.f90:477-661 restated with numpy."""
    ncol = len(chem.tables)
    allE = np.concatenate([t[0] for t in chem.tables]) if ncol else np.zeros(0)
    # stable ascending order then drop repeats (the reference keeps the first
    # of equal values; equal values are identical so the grid is the same)
    grid = []
    sav = 1.0e10
    for e in np.sort(allE, kind="stable"):
        if e != sav:
            grid.append(e)
            sav = e
    sig_Er = np.array(grid, dtype=np.float64)
    sig = np.zeros((ncol, len(sig_Er)))
    for c, (E, S) in enumerate(chem.tables):
        Ez = np.append(E, 0.0)
        Sz = np.append(S, 0.0)
        sig_p = 0.0
        for ipt, ekp in enumerate(sig_Er):
            for j in range(len(E)):
                EL, ER, sL, sR = Ez[j], Ez[j + 1], Sz[j], Sz[j + 1]
                if ekp < EL:
                    sig_p = sL
                    break
                if EL <= ekp <= ER:
                    sig_p = sL + (ekp - EL) * (sR - sL) / (ER - EL)
                    break
            sig[c, ipt] = sig_p
    sigv_mx = np.zeros((10, ncol))
    sig_list = np.zeros((10, ncol), dtype=np.int32)
    ind_col = np.zeros(10, dtype=np.int32)
    masses = [s.mass for s in chem.species]
    for c in range(ncol):
        r1, r2 = int(chem.col_info[c, 2]), int(chem.col_info[c, 3])
        ind_col[r1 - 1] += 1
        sig_list[r1 - 1, ind_col[r1 - 1] - 1] = c + 1
        m1, m2 = abs(masses[r1 - 1]), abs(masses[r2 - 1])
        mu = m1 * m2 / (m1 + m2)
        for ipt, e in enumerate(sig_Er):
            vr = np.sqrt(2.0 * e * qe / mu)
            if e >= 1.0:
                sigv_mx[r1 - 1, c] = max(sigv_mx[r1 - 1, c], vr * sig[c, ipt])
    p_ncol = ind_col.copy()
    return Tables(sig_Er=sig_Er, sig=sig, sigv_mx=sigv_mx, sig_list=sig_list, p_ncol=p_ncol,
                  Eth=chem.Eth.copy(), col_info=chem.col_info.copy())


def coulomb_table_synthetic(sigma0, E0=1.0, npts=400, emax=1000.0):
    """A synthetic e-Ar+ elastic reaction with a charged target (DSMC): sigma =
    sigma0 below E0 eV and sigma0 (E0/E)^2 above, the Coulomb-like fall of the
    reference's [e]+[Ar+]->[e]+[Ar+] table."""
    E = np.concatenate([[0.0], np.geomspace(1e-3, emax, npts)])
    S = np.full_like(E, sigma0)
    m = E > E0
    S[m] = sigma0 * (E0 / E[m]) ** 2
    return ("[e]+[Ar+]->[e]+[Ar+]", 0.0, 0.0, 1.0, 1.0, "COLLISION", E, S)


def argon_tables_synthetic(npts=400, emax=1000.0):
    """The synthetic analytic e-Ar / Ar+-Ar cross sections of the 128^3
    benchmark: elastic 1e-19 m^2, excitation 1.5e-21 m^2 above 11.5 eV,
    ionization 2.5e-20 ln(E/15.8)/(E/15.8) m^2 above 15.8 eV, charge exchange
    5e-19 m^2.  Log-spaced grid 1e-3..emax eV plus 0 and points bracketing the
    thresholds."""
    base = np.concatenate([[0.0], np.geomspace(1e-3, emax, npts)])
    def grid_with(*pts):
        return np.unique(np.concatenate([base, np.array(pts, dtype=np.float64)]))
    E_el = base
    S_el = np.full_like(E_el, 1e-19)
    E_ex = grid_with(11.5, 11.5 * (1 + 1e-6))
    S_ex = np.where(E_ex > 11.5, 1.5e-21, 0.0)
    E_io = grid_with(15.8)
    x = E_io / 15.8
    with np.errstate(divide="ignore", invalid="ignore"):
        S_io = np.where(E_io > 15.8, 2.5e-20 * np.log(x) / x, 0.0)
    E_cx = np.concatenate([[0.0], np.geomspace(1e-3, emax, npts // 4)])
    S_cx = np.full_like(E_cx, 5e-19)
    return [
        ("[e]+[Ar]->[e]+[Ar]", 0.0, 0.0, 1.0, 1.0, "COLLISION", E_el, S_el),
        ("[e]+[Ar]->[e]+[Ar]", 11.5, 0.0, 1.0, 1.0, "EXCITATION", E_ex, S_ex),
        ("[e]+[Ar]->[e]+[Ar+]+[e]", 15.8, 0.0, 1.0, 1.0, "IONIZATION", E_io, S_io),
        ("[Ar+]+[Ar]->[Ar+]+[Ar]", 0.0, 0.0, 1.0, 1.0, "CHARGEEXCHANGE", E_cx, S_cx),
    ]
