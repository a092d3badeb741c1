"""Generate the H2O cc-pVDZ fixture: the G0W0@HF workload on H2O with the
cc-pVDZ-RI auxiliary basis, and two reference inputs that pin its front end.

Run next to the MOLGW sources:

    python tests/golden/make_h2o_fixture.py /path/to/molgw

It reads from the MOLGW tree:

* ``basis/{O,H}_cc-pVDZ``, ``{O,H}_cc-pVTZ``, ``{O,H}_cc-pVDZ-RI`` and
  ``{O,H}_cc-pVTZ-RI``;
* ``tests/inputs/h2o_rt_tddft_hf_PC2B.in`` (HF, cc-pVDZ / cc-pVDZ-RI) and
  ``tests/inputs/h2o_mp3.in`` (HF, cc-pVDZ / cc-pVTZ-RI, frozencore='molgw'):
  their geometries, bases and their known answers in ``tests/inputs/testsuite``
  (SCF total energy and the RI-MP2 correlation energy, 1e-7 Ha);
* ``tests/inputs/h2o_gw_contour.in`` (HF, cc-pVTZ with the Auto auxiliary basis,
  G0W0 by contour deformation, frozencore='molgw'): geometry, basis, GW settings
  and known answers (SCF total energy 1e-7 Ha, HOMO and LUMO 1e-4 eV).

The workload itself is H2O with O at (0, 0, 0) and the H atoms at
(0, +-0.757, 0.587) Angstrom, HF in cc-pVDZ (24 functions) with cc-pVDZ-RI (84
auxiliary functions), 5 doubly occupied orbitals, a 16-point Gauss-Legendre
imaginary-frequency grid and the HOMO and LUMO as Sigma states, with the Sigma
grid of tests/inputs/h2o_gw_pade.in.  No reference run exists for it: its
inputs come from the oracle's front end (oracle/gaussian_ri.py), which the two
inputs above pin.

Writes ``h2o_ccpvdz.npz`` next to this script: the basis texts, per case the
geometry and known answers, and for the workload the orbital energies and
occupations, the MO coefficients, the AO 3-center tensor B(mu nu, P) (metric
folded in; the MO tensor M[p, q, P] = sum C B C follows), the SCF energy, and the
oracle's G0W0 output (E_RPA, E_GW, QP energies); for the contour input, the
oracle's QP energies and Sigma on its real grid.  The tests read only this
fixture (and recompute the front end from its basis texts).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from tests.golden.make_he_fixture import read_known_answers  # noqa: E402

PIN_INPUTS = ("h2o_rt_tddft_hf_PC2B.in", "h2o_mp3.in", "h2o_gw_contour.in")
CONTOUR_KEYS = ("nomega_chi_imag", "nomega_chi_real", "step_sigma", "nomega_sigma", "selfenergy_state_range",
                "eta", "postscf")
WORKLOAD_ATOMS = [(8, (0.0, 0.0, 0.0)), (1, (0.0, 0.757, 0.587)), (1, (0.0, -0.757, 0.587))]
WORKLOAD_GRID = dict(nomega=16, nomega_sigma=101, step_sigma=0.025, nomega_sigma_calc=50, step_sigma_calc=0.075,
                     eta=0.01)
SYMBOL = {1: "H", 8: "O"}
ZOF = {v.upper(): k for k, v in SYMBOL.items()}


def read_case(path: Path) -> dict:
    """Namelist values (basis, auxil_basis, frozencore, natom, GW settings) and
    the atom lines (atomic number or element symbol, then x y z in Angstrom)."""
    text = path.read_text()
    head, tail = text.split("\n/", 1)
    vals = {}
    for line in head.splitlines():
        line = line.split("!")[0]
        if "=" in line:
            k, v = line.split("=", 1)
            vals[k.strip().lower()] = v.strip().strip("'\"")
    natom = int(vals["natom"])
    atoms = []
    for line in tail.strip().splitlines()[:natom]:
        z, x, y, zz = line.split()[:4]
        zn = ZOF[z.upper()] if z.upper() in ZOF else int(float(z))
        atoms.append((zn, (float(x), float(y), float(zz))))
    return {"basis": vals["basis"], "auxil_basis": vals["auxil_basis"], "frozencore": vals.get("frozencore", "no"),
            "atoms": atoms, "settings": {k: vals[k] for k in CONTOUR_KEYS if k in vals}}


def main(molgw: Path):
    from oracle import gaussian_ri as g
    from oracle import rigw_oracle as o
    basis = {}
    for name in ("cc-pVDZ", "cc-pVTZ", "cc-pVDZ-RI", "cc-pVTZ-RI"):
        basis[name] = {str(z): (molgw / "basis" / f"{s}_{name}").read_text() for z, s in SYMBOL.items()}
    cases = {}
    for name in PIN_INPUTS:
        case = read_case(molgw / "tests" / "inputs" / name)
        case["known_answers"] = read_known_answers(molgw / "tests" / "inputs" / "testsuite", name)
        cases[name] = case

    bas = {z: basis["cc-pVDZ"][str(z)] for z in SYMBOL}
    aux = {z: basis["cc-pVDZ-RI"][str(z)] for z in SYMBOL}
    scf, m, det = g.molecule_ri_hf(WORKLOAD_ATOMS, bas, aux)
    nocc = int(np.sum(scf.occupation > 0))
    nstate = scf.e_orb.size
    rng = o.selfenergy_set_state_range(nstate, scf.occupation, selfenergy_state_min=nocc,
                                       selfenergy_state_max=nocc + 1)
    grid = {k: v for k, v in WORKLOAD_GRID.items() if k != "nomega"}
    ref = o.g0w0_imag(scf.e_orb, scf.occupation, m[:nocc, nocc:], m[nocc - 1:nocc + 1], WORKLOAD_GRID["nomega"],
                      rng, **grid)
    contour = contour_run(cases["h2o_gw_contour.in"], basis)
    np.savez_compressed(
        HERE / "h2o_ccpvdz.npz", basis=np.array(json.dumps(basis)), cases=np.array(json.dumps(cases)),
        workload_atoms=np.array(json.dumps(WORKLOAD_ATOMS)), workload_grid=np.array(json.dumps(WORKLOAD_GRID)),
        energy=scf.e_orb, occupation=scf.occupation, c_matrix=scf.c, b3_ao=scf.b3,
        scf_energy=scf.energy, nauxil=det["nauxil"], oracle_erpa=ref.erpa, oracle_egw=ref.egw,
        oracle_qp=ref.energy_qp_g, oracle_sigma_calc=ref.sigma_calc,
        contour_qp=contour.energy_qp_g, contour_sigma=contour.sigma, contour_de_max=contour.de_max)
    print("wrote", HERE / "h2o_ccpvdz.npz", "E_SCF =", scf.energy, "nauxil =", det["nauxil"],
          "QP HOMO/LUMO (eV) =", ref.energy_qp_g * g.HA_EV, "contour QP (eV) =", contour.energy_qp_g * g.HA_EV)


def contour_run(case: dict, basis: dict):
    from oracle import rigw_oracle as o
    from tests.h2o_case import contour_inputs
    scf, m, rng, ncore, m_ia, m_sig, st = contour_inputs(case, basis)
    return o.g0w0_contour(scf.e_orb, scf.occupation, m_ia, m_sig, rng, ncore, st["nomega_chi_imag"],
                          st["nomega_chi_real"], nomega_sigma=st["nomega_sigma"], step_sigma=st["step_sigma"],
                          eta=st["eta"])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_h2o_fixture.py <path of the MOLGW source tree>")
    main(Path(sys.argv[1]))
