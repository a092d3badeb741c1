"""Reader for CC4S CoulombVertex / EigenEnergies files (real, half-grid case).

Follows MOLGW's readers:

* ``read_cc4s_coulombvertex`` (src/m_eri_ao_mo.f90:1192-1331): the vertex is a
  complex (naux, nstate, nstate) tensor, auxiliary index fastest; MOLGW splits
  it into real and imaginary halves so that nauxil = 2*naux and
  eri_3center_mo(1:naux, i, j) = Re V, eri_3center_mo(naux+1:, i, j) = Im V.
  The serial branch reads i outer, j inner.
* ``read_cc4s_eigenenergies`` (src/m_io.f90:4048-4119): energies from the
  ``.elements`` text file, occupation 2 for energy < fermiEnergy + 1e-8, C = I.
"""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np


def _yaml_values(path: Path, key: str):
    vals = []
    for line in Path(path).read_text().splitlines():
        m = re.match(rf"\s*-?\s*{key}:\s*(\S+)", line)
        if m:
            vals.append(m.group(1))
    return vals


def read_eigenenergies(root: str | Path):
    root = str(root)
    efermi = float(_yaml_values(Path(root + "_EigenEnergies.yaml"), "fermiEnergy")[0])
    energy = np.loadtxt(root + "_EigenEnergies.elements", dtype=np.float64).reshape(-1)
    occupation = np.where(energy < efermi + 1.0e-8, 2.0, 0.0)
    return energy, occupation, efermi


def read_coulomb_vertex(root: str | Path) -> np.ndarray:
    """Return eri_3center_mo as ``[nstate, nstate, 2*naux]`` with
    ``out[i, j, :] = eri_3center_mo(:, i+1, j+1)`` of the serial reader."""
    root = str(root)
    lengths = [int(v) for v in _yaml_values(Path(root + "_CoulombVertex.yaml"), "length")]
    half = _yaml_values(Path(root + "_CoulombVertex.yaml"), "halfGrid")
    if not half or int(half[0]) != 1:
        raise ValueError("read_cc4s_coulombvertex: only works for half grid (real wavefunctions)")
    naux, nstate = lengths[0], lengths[1]
    raw = np.fromfile(root + "_CoulombVertex.elements", dtype=np.complex128)
    if raw.size != naux * nstate * nstate:
        raise ValueError(f"CoulombVertex size {raw.size} != {naux}*{nstate}*{nstate}")
    v = raw.reshape(nstate, nstate, naux)           # record (i, j) read in order i outer, j inner
    return np.concatenate([v.real, v.imag], axis=2)
