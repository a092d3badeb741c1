"""The ENERGY_QP file: quasiparticle energies handed from one GW run to the next.

Mirrors ``write_energy_qp`` / ``read_energy_qp`` (src/m_io.f90:3645-3733): list-
directed lines ``nspin``, ``nstate``, then ``istate e(istate, 1) [e(istate, 2)]``
in Ha.  ``read_energy_qp`` returns the energies and the reference's
reading_status: 0 read, 1 no file (ENERGY_QP or energy_qp), 2 dimensions differ,
-1 a scissor line (istate = -1).  Under ``force_energy_qp`` a run takes these as
the energies in G when the status is 0 and the mean-field energies otherwise
(src/m_selfenergy_evaluation.f90:164-181).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np


def write_energy_qp(root: str | Path, energy_qp: np.ndarray) -> Path:
    """``energy_qp``: [nstate] or [nstate, nspin] (Ha); writes ``root/ENERGY_QP``."""
    e = np.asarray(energy_qp, dtype=np.float64)
    if e.ndim == 1:
        e = e[:, None]
    nstate, nspin = e.shape
    path = Path(root) / "ENERGY_QP"
    lines = [f"{nspin:12d}", f"{nstate:12d}"]
    lines += [f"{i + 1:12d}" + "".join(f" {v:25.17E}" for v in e[i]) for i in range(nstate)]
    path.write_text("\n".join(lines) + "\n")
    return path


def read_energy_qp(root: str | Path, nstate: int, nspin: int = 1) -> tuple[np.ndarray, int]:
    """(energy_qp [nstate, nspin], reading_status) from ``root/ENERGY_QP`` or ``root/energy_qp``."""
    root = Path(root)
    energy_qp = np.zeros((nstate, nspin))
    path = next((p for p in (root / "ENERGY_QP", root / "energy_qp") if p.exists()), None)
    if path is None:
        return energy_qp, 1
    rows = [ln.replace("D", "E").replace("d", "e").split() for ln in path.read_text().splitlines() if ln.strip()]
    nspin_read, nstate_read = int(rows[0][0]), int(rows[1][0])
    if nstate_read != nstate or nspin_read != nspin:
        return energy_qp, 2
    for i in range(nstate):
        row = rows[2 + i]
        energy_qp[i, :] = [float(v) for v in row[1:1 + nspin]]
        if int(row[0]) == -1:
            return energy_qp, -1
    return energy_qp, 0
