"""Reader for the GW ingredients MOLGW writes with ``postscf='DUMP_GW'``.

Follows ``dump_gw_ingredients`` (src/m_gw_selfenergy_analytic.f90:799-881):

* ``energies.dat`` (formatted): the number of states n = nvirtual_G - ncore_G - 1,
  then the n energies energy(ncore_G+1 : nvirtual_G-1, spin 1) in Ha, one per line;
* ``v.dat`` (formatted): nauxil_global, n, n;
* ``v.bin`` (stream, unformatted): for each spin and each state q of the window,
  the Fortran array eri_3center_mo(:, window, q), i.e. doubles with the
  auxiliary index fastest, then p, then q, then spin.

``omegas.dat`` and ``w.bin`` (RPA poles for the analytic self-energy) are not
needed by the imaginary-axis path.  The dump holds no occupations: the caller
gives the number of doubly occupied states of the window (``nocc``).  The window
is used both for W (transitions i -> a) and for G (states p in Sigma).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .synth import GWInstance


def read_energies(path: str | Path) -> np.ndarray:
    vals = Path(path).read_text().split()
    n = int(vals[0])
    energy = np.array([float(v.replace("D", "E").replace("d", "e")) for v in vals[1:1 + n]], dtype=np.float64)
    if energy.size != n:
        raise ValueError(f"{path}: {energy.size} energies for {n} states")
    return energy


def read_vertex(root: str | Path, nspin: int = 1) -> np.ndarray:
    """``v[s, q, p, P] = eri_3center_mo(P, p, q, s)`` over the dumped window."""
    root = Path(root)
    naux, n1, n2 = (int(v) for v in (root / "v.dat").read_text().split()[:3])
    raw = np.fromfile(root / "v.bin", dtype="<f8")
    if raw.size != nspin * n1 * n2 * naux:
        raise ValueError(f"v.bin holds {raw.size} doubles, expected {nspin}*{n2}*{n1}*{naux}")
    return raw.reshape(nspin, n2, n1, naux)


def read_dump_gw(root: str | Path, nocc: int, nomega: int = 32, nsemin: int | None = None,
                 nsemax: int | None = None) -> GWInstance:
    """G0W0 problem of a DUMP_GW directory (closed shell, spin 1).

    ``nocc``: doubly occupied states of the window; Sigma states default to HOMO
    and LUMO (1-based, within the window)."""
    root = Path(root)
    energy = read_energies(root / "energies.dat")
    v = read_vertex(root)[0]                         # [q, p, P]
    n = energy.size
    if v.shape[0] != n or v.shape[1] != n:
        raise ValueError(f"energies.dat has {n} states, v.bin a {v.shape[0]} x {v.shape[1]} window")
    if not 0 < nocc < n:
        raise ValueError(f"nocc={nocc} outside (0, {n})")
    nsemin = nocc if nsemin is None else nsemin
    nsemax = nocc + 1 if nsemax is None else nsemax
    occupation = np.concatenate([np.full(nocc, 2.0), np.zeros(n - nocc)])
    # M(P, a, i) = eri_3center_mo(P, a, i): q = i (occupied), p = a (virtual)
    m_ia = np.ascontiguousarray(v[:nocc, nocc:, :])
    # M(P, p, m) for the Sigma states m: q = m, all p
    m_sigma = np.ascontiguousarray(v[nsemin - 1:nsemax, :, :])
    return GWInstance(nocc=nocc, nvirt=n - nocc, naux=v.shape[2], nomega=nomega, energy=energy,
                      occupation=occupation, m_ia=m_ia, m_sigma=m_sigma, nsemin=nsemin, nsemax=nsemax)


def write_dump_gw(root: str | Path, energy: np.ndarray, vertex: np.ndarray) -> None:
    """Write ``energies.dat``, ``v.dat`` and ``v.bin`` in the layout above
    (``vertex[q, p, P]``); used to test the reader and to export instances."""
    root = Path(root)
    root.mkdir(parents=True, exist_ok=True)
    n = energy.size
    (root / "energies.dat").write_text(f"{n}\n" + "".join(f"  {e:.17E}\n" for e in energy))
    (root / "v.dat").write_text(f"{vertex.shape[2]}\n{n}\n{n}\n")
    np.ascontiguousarray(vertex, dtype="<f8").tofile(root / "v.bin")
