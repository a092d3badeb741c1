"""Gaussian basis sets for the RI integral entry points (rigw_eri_2center,
rigw_eri_3center_raw, rigw_eri_3center): the reference's basis-file format and
the shells of a molecule.

A basis file (src/m_basis_set.f90:155-170, 236-245) holds the number of shells,
then per shell a line "ng am" and ng lines "alpha coeff", the coefficients
multiplying normalized primitives.  Shells are listed atom by atom in input
order, the order of the reference's basis functions (src/m_basis_set.f90:90-340);
``Engine.eri_*`` turn each contraction into the reference's shell coefficients
(``rigw.shell_coefficients``)."""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

BOHR_A = 0.52917721092   # src/m_definitions.f90:43


@dataclass
class Shell:
    am: int
    alpha: np.ndarray
    coeff: np.ndarray
    center: np.ndarray = field(default_factory=lambda: np.zeros(3))   # Bohr


def parse_basis_file(text: str, center=(0.0, 0.0, 0.0)) -> list[Shell]:
    tok = text.split()
    pos = 0
    nshell = int(tok[pos])
    pos += 1
    out = []
    for _ in range(nshell):
        ng, am = int(tok[pos]), int(tok[pos + 1])
        pos += 2
        a = np.array([float(tok[pos + 2 * k]) for k in range(ng)])
        c = np.array([float(tok[pos + 2 * k + 1]) for k in range(ng)])
        pos += 2 * ng
        out.append(Shell(am, a, c, np.asarray(center, dtype=float)))
    return out


def molecule_shells(atoms, basis: dict) -> list[Shell]:
    """``atoms`` = [(Z, (x, y, z) in Angstrom), ...], ``basis`` maps Z to a basis
    file's text."""
    shells = []
    for z, xyz in atoms:
        shells += parse_basis_file(basis[int(z)], center=tuple(np.asarray(xyz, float) / BOHR_A))
    return shells


def nfunctions(shells, pure: bool = True) -> int:
    return sum((2 * s.am + 1) if pure else (s.am + 1) * (s.am + 2) // 2 for s in shells)


def water_cluster(n: int, spacing: float = 3.0) -> list:
    """n water molecules on a cubic lattice of the given spacing (Angstrom), each
    with the geometry of the H2O workload (O at its site, H at +-0.757 y, 0.587 z)."""
    side = int(np.ceil(n ** (1.0 / 3.0)))
    atoms = []
    for k in range(n):
        o = spacing * np.array([k % side, (k // side) % side, k // (side * side)], dtype=float)
        atoms += [(8, tuple(o)), (1, tuple(o + [0.0, 0.757, 0.587])), (1, tuple(o + [0.0, -0.757, 0.587]))]
    return atoms
