"""Generate the CO fixture of the GW density-matrix tests.

Run next to the MOLGW sources:

    python tests/golden/make_co_dm_fixture.py /path/to/molgw

It reads from the MOLGW tree ``tests/inputs/co_gw_dm_imag.in`` (HF in the
Cartesian cc-pVDZ_gaussian basis with cc-pVDZ-RI, frozencore='molgw',
pt_density_matrix='GW_IMAGINARY' with 128 imaginary frequencies for W and 16
for the density matrix, use_correlated_density_matrix='yes'), its known answers
in ``tests/inputs/testsuite`` (SCF total energy, and the kinetic, nuclear,
Hartree and exchange energies of the correlated density matrix, 1e-7 Ha), and
the four basis files.  It runs the oracle's front end and
gw_density_matrix_imag and writes ``co_dm.npz`` next to this script: the basis
texts, the case, the known answers, and the oracle's density-matrix correction
and energies (for regression).  The tests read only this fixture.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from tests.golden.make_he_fixture import read_known_answers  # noqa: E402

INPUT = "co_gw_dm_imag.in"
SYMBOL = {6: "C", 8: "O"}


def read_case(path: Path) -> dict:
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
        atoms.append((int(float(z)), (float(x), float(y), float(zz))))
    return {"basis": vals["basis"], "auxil_basis": vals["auxil_basis"], "gaussian_type": vals["gaussian_type"],
            "frozencore": vals["frozencore"], "pt_density_matrix": vals["pt_density_matrix"],
            "nomega_chi_imag": int(vals["nomega_chi_imag"]), "nomega_sigma": int(vals["nomega_sigma"]),
            "atoms": atoms}


def main(molgw: Path):
    from tests import co_case
    case = read_case(molgw / "tests" / "inputs" / INPUT)
    case["known_answers"] = read_known_answers(molgw / "tests" / "inputs" / "testsuite", INPUT)
    basis = {name: {str(z): (molgw / "basis" / f"{s}_{name}").read_text() for z, s in SYMBOL.items()}
             for name in (case["basis"], case["auxil_basis"])}
    d = {"case": case, "basis": basis}
    run = co_case.oracle_run(d)
    np.savez_compressed(HERE / "co_dm.npz", case=np.array(json.dumps(case)), basis=np.array(json.dumps(basis)),
                        p_corr=run["p_corr"], energies=np.array(json.dumps(run["energies"])))
    print("wrote", HERE / "co_dm.npz", run["energies"])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_co_dm_fixture.py <path of the MOLGW source tree>")
    main(Path(sys.argv[1]))
