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
                 nsemax: int | None = None, nocc_2: int | None = None,
                 energy_2: np.ndarray | None = None) -> GWInstance:
    """G0W0 problem of a DUMP_GW directory.

    Closed shell (default): ``nocc`` doubly occupied states of the window.  Open
    shell: give ``nocc_2`` and ``energy_2``, the occupied count and the energies
    of the second spin channel over the same window (v.bin holds both spins but
    energies.dat only spin 1, as dump_gw_ingredients writes them); ``nocc`` is
    then the first channel's singly occupied count and the instance carries the
    second channel in ``spin2``.  Sigma states default to HOMO and LUMO of the
    first channel (1-based, within the window)."""
    root = Path(root)
    energy = read_energies(root / "energies.dat")
    spin = nocc_2 is not None
    vs = read_vertex(root, nspin=2 if spin else 1)
    v = vs[0]                                        # [q, p, P]
    n = energy.size
    if v.shape[0] != n or v.shape[1] != n:
        raise ValueError(f"energies.dat has {n} states, v.bin a {v.shape[0]} x {v.shape[1]} window")
    if not 0 < nocc < n:
        raise ValueError(f"nocc={nocc} outside (0, {n})")
    nsemin = nocc if nsemin is None else nsemin
    nsemax = nocc + 1 if nsemax is None else nsemax
    full = 1.0 if spin else 2.0
    occupation = np.concatenate([np.full(nocc, full), np.zeros(n - nocc)])
    # M(P, a, i) = eri_3center_mo(P, a, i): q = i (occupied), p = a (virtual)
    m_ia = np.ascontiguousarray(v[:nocc, nocc:, :])
    # M(P, p, m) for the Sigma states m: q = m, all p
    m_sigma = np.ascontiguousarray(v[nsemin - 1:nsemax, :, :])
    inst = GWInstance(nocc=nocc, nvirt=n - nocc, naux=v.shape[2], nomega=nomega, energy=energy,
                      occupation=occupation, m_ia=m_ia, m_sigma=m_sigma, nsemin=nsemin, nsemax=nsemax,
                      spin_channel=spin)
    if spin:
        e2 = np.asarray(energy_2, dtype=np.float64)
        if e2.shape != energy.shape or not 0 < nocc_2 < n:
            raise ValueError("energy_2 must cover the window and 0 < nocc_2 < n")
        v2 = vs[1]
        ch2 = GWInstance(nocc=nocc_2, nvirt=n - nocc_2, naux=v.shape[2], nomega=nomega, energy=e2,
                         occupation=np.concatenate([np.ones(nocc_2), np.zeros(n - nocc_2)]),
                         m_ia=np.ascontiguousarray(v2[:nocc_2, nocc_2:, :]),
                         m_sigma=np.ascontiguousarray(v2[nsemin - 1:nsemax, :, :]), nsemin=nsemin, nsemax=nsemax,
                         spin_channel=True)
        inst.spin2 = ch2
    return inst


def write_dump_gw(root: str | Path, energy: np.ndarray, vertex: np.ndarray) -> None:
    """Write ``energies.dat``, ``v.dat`` and ``v.bin`` in the layout above
    (``vertex[q, p, P]``, or ``[nspin, q, p, P]`` with spin 1's energies only);
    used to test the reader and to export instances."""
    root = Path(root)
    root.mkdir(parents=True, exist_ok=True)
    n = energy.size
    (root / "energies.dat").write_text(f"{n}\n" + "".join(f"  {e:.17E}\n" for e in energy))
    (root / "v.dat").write_text(f"{vertex.shape[-1]}\n{n}\n{n}\n")
    np.ascontiguousarray(vertex, dtype="<f8").tofile(root / "v.bin")
