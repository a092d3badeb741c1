"""Generate the He cc-pVDZ / PAuto fixture of the reference-pinned tests.

Run next to the MOLGW sources:

    python tests/golden/make_he_fixture.py /path/to/molgw

It reads from the MOLGW tree:

* ``basis/He_cc-pVDZ`` (the orbital basis the inputs name);
* the GW settings of ``tests/inputs/he_gw+sox_pade.in``,
  ``he_gw+sosex_pade.in``, ``he_gw+sosex2_pade.in`` and ``he_gw+g3w2_pade.in``
  (nomega_chi_imag, nomega_sigma, step_sigma, nomega_sigma_calc,
  step_sigma_calc, mu_origin; eta keeps its default 0.001 Ha,
  src/input_variables.f90:374);
* their known answers in ``tests/inputs/testsuite`` (SCF total energy at 1e-7
  Ha, HOMO energy at 1e-4 eV).

It runs the oracle's Gaussian front end (``oracle/gaussian_ri.py``: PAuto
auxiliary basis, RI integrals, RI Hartree-Fock) and writes
``he_ccpvdz_pauto.npz`` next to this script: the basis file text, the orbital
energies and occupations, the MO 3-center tensor M[p, q, P] over all five
states and the 40 auxiliary functions, the SCF energy of the front end, and
per input its settings and the reference's known answers.  The tests read only
this fixture.
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

INPUTS = ("he_gw+sox_pade.in", "he_gw+sosex_pade.in", "he_gw+sosex2_pade.in", "he_gw+g3w2_pade.in")
KEYS = ("postscf", "nomega_chi_imag", "nomega_sigma", "step_sigma", "nomega_sigma_calc", "step_sigma_calc",
        "mu_origin", "analytic_chi", "basis", "auxil_basis", "scf", "selfenergy_state_range")


def read_input(path: Path) -> dict:
    out = {}
    for line in path.read_text().splitlines():
        m = re.match(r"\s*(\w+)\s*=\s*'?([^'\s]+)'?", line)
        if m and m.group(1).lower() in KEYS:
            out[m.group(1).lower()] = m.group(2)
    return out


def read_known_answers(testsuite: Path, name: str) -> dict:
    """The block of ``name`` in tests/inputs/testsuite: 'label , value , 0 , tol' lines."""
    lines = testsuite.read_text().splitlines()
    start = next(k for k, l in enumerate(lines) if l.split(",")[0].strip() == name)
    out = {}
    for l in lines[start + 1:]:
        parts = [p.strip() for p in l.split(",")]
        if len(parts) < 4:
            break
        out[parts[0]] = (float(parts[1]), float(parts[3]))
    return out


def main(molgw: Path):
    from oracle import gaussian_ri as g
    basis_text = (molgw / "basis" / "He_cc-pVDZ").read_text()
    scf, m, det = g.atom_ri_hf(basis_text, 2)
    runs = {}
    for name in INPUTS:
        settings = read_input(molgw / "tests" / "inputs" / name)
        answers = read_known_answers(molgw / "tests" / "inputs" / "testsuite", name)
        runs[name] = {"settings": settings, "known_answers": answers}
    np.savez_compressed(
        HERE / "he_ccpvdz_pauto.npz", basis_text=np.array(basis_text), energy=scf.e_orb,
        occupation=scf.occupation, m_full=m, scf_energy=scf.energy, nauxil=det["nauxil"],
        metric_min_eigenvalue=float(scf.metric_eigenvalues.min()), runs=np.array(json.dumps(runs)))
    print("wrote", HERE / "he_ccpvdz_pauto.npz", "E_SCF =", scf.energy, "nauxil =", det["nauxil"])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_he_fixture.py <path of the MOLGW source tree>")
    main(Path(sys.argv[1]))
