"""CO, HF in the Cartesian cc-pVDZ_gaussian basis with cc-pVDZ-RI, and its GW
density matrix from the imaginary axis (tests/inputs/co_gw_dm_imag.in; known
answers at tests/inputs/testsuite:975-980), read from the committed fixture
tests/golden/co_dm.npz."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "co_dm.npz"
LABELS = {"kinetic": "Kinetic Energy", "nucleus": "Nucleus Energy", "hartree": "Hartree Energy",
          "exchange": "Exchange Energy"}


def load() -> dict:
    d = dict(np.load(GOLDEN))
    d["case"] = json.loads(str(d["case"]))
    d["basis"] = json.loads(str(d["basis"]))
    d["energies"] = json.loads(str(d["energies"]))
    return d


def front_end(d: dict):
    from oracle import gaussian_ri as g
    c = d["case"]
    bas = {int(z): t for z, t in d["basis"][c["basis"]].items()}
    aux = {int(z): t for z, t in d["basis"][c["auxil_basis"]].items()}
    return g.molecule_ri_hf([(z, tuple(x)) for z, x in c["atoms"]], bas, aux, cart=c["gaussian_type"] == "CART")


def windows(d: dict, scf, m):
    """Frozen core from frozencore='molgw', the Sigma range over every state above it."""
    from oracle import gaussian_ri as g
    from oracle import rigw_oracle as o
    ncore = sum(g.element_core(z) for z, _ in d["case"]["atoms"])
    rng = o.selfenergy_set_state_range(scf.e_orb.size, scf.occupation, ncoreg=ncore)
    return ncore, rng


def instance(d: dict, scf, m):
    """GWInstance of W (frozen core in W and G) and of the Sigma range."""
    from molgw_b200.synth import GWInstance
    ncore, rng = windows(d, scf, m)
    nocc = int(np.sum(scf.occupation > 0))
    return GWInstance(nocc=nocc - ncore, nvirt=scf.e_orb.size - nocc, naux=m.shape[2],
                      nomega=d["case"]["nomega_chi_imag"], energy=scf.e_orb.copy(),
                      occupation=scf.occupation.copy(), m_ia=np.ascontiguousarray(m[ncore:nocc, nocc:]),
                      m_sigma=np.ascontiguousarray(m[rng.nsemin - 1:rng.nsemax, ncore:]), nsemin=rng.nsemin,
                      nsemax=rng.nsemax, ncore_w=ncore, ncore_g=ncore)


def oracle_run(d: dict) -> dict:
    """The oracle's W, gw_density_matrix_imag and correlated-density energies."""
    from oracle import gaussian_ri as g
    from oracle import rigw_oracle as o
    scf, m, det = front_end(d)
    ncore, rng = windows(d, scf, m)
    e, occ = scf.e_orb, scf.occupation
    nocc = int(np.sum(occ > 0))
    om, wt = o.imaginary_quad_grid(d["case"]["nomega_chi_imag"])
    sf = o.polarizability_grid(np.ascontiguousarray(m[ncore:nocc, nocc:]), e[ncore:nocc], e[nocc:], occ[ncore:nocc],
                               occ[nocc:], om, wt)
    pc = o.gw_density_matrix_imag(e, m[ncore:, ncore:], sf, rng, d["case"]["nomega_sigma"])
    en = g.correlated_dm_energies(scf, det, pc)
    return {"p_corr": pc, "energies": {k: en[k] for k in ("kinetic", "nucleus", "hartree", "exchange", "trace_mo")},
            "scf": scf, "m": m, "details": det, "erpa": sf.erpa}
