"""The H2O cc-pVDZ workload (HF, cc-pVDZ-RI auxiliary basis, 16 imaginary
frequencies, HOMO and LUMO) and the two reference inputs that pin its front end
(tests/inputs/h2o_rt_tddft_hf_PC2B.in, h2o_mp3.in; known answers at
tests/inputs/testsuite:782-790), and the contour-deformation G0W0@HF input
tests/inputs/h2o_gw_contour.in (known answers at testsuite:777-780), read from
the committed fixture tests/golden/h2o_ccpvdz.npz."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "h2o_ccpvdz.npz"


def load() -> dict:
    d = dict(np.load(GOLDEN))
    for k in ("basis", "cases", "workload_atoms", "workload_grid"):
        d[k] = json.loads(str(d[k]))
    c, b3 = d["c_matrix"], d["b3_ao"]
    d["m_full"] = np.einsum("ip,jq,ijP->pqP", c, c, b3, optimize=True)
    return d


def bases(d: dict, name: str):
    """Basis texts per atomic number, or the name of a generated auxiliary basis."""
    if name.upper() in ("AUTO", "PAUTO"):
        return name.upper()
    return {int(z): t for z, t in d["basis"][name].items()}


def front_end(d: dict, case: str | None = None):
    """The oracle's RI-HF of the workload (case None) or of a pinning input."""
    from oracle import gaussian_ri as g
    if case is None:
        atoms, bas, aux = d["workload_atoms"], "cc-pVDZ", "cc-pVDZ-RI"
    else:
        c = d["cases"][case]
        atoms, bas, aux = c["atoms"], c["basis"], c["auxil_basis"]
    return g.molecule_ri_hf([(z, tuple(x)) for z, x in atoms], bases(d, bas), bases(d, aux))


def grid(d: dict) -> dict:
    return {k: v for k, v in d["workload_grid"].items() if k != "nomega"}


def instance(d: dict):
    """GWInstance of the workload: 5 occupied, 19 empty, HOMO and LUMO as Sigma states."""
    from molgw_b200.synth import GWInstance
    m = d["m_full"]
    nocc = int(np.sum(d["occupation"] > 0))
    return GWInstance(nocc=nocc, nvirt=m.shape[0] - nocc, naux=m.shape[2], nomega=d["workload_grid"]["nomega"],
                      energy=d["energy"].copy(), occupation=d["occupation"].copy(),
                      m_ia=np.ascontiguousarray(m[:nocc, nocc:]),
                      m_sigma=np.ascontiguousarray(m[nocc - 1:nocc + 1]), nsemin=nocc, nsemax=nocc + 1, **grid(d))


def contour_settings(case: dict) -> dict:
    """GW settings of the contour input; eta keeps its default 0.001 Ha
    (src/input_variables.f90:374)."""
    s = case["settings"]
    return dict(nomega_chi_imag=int(s["nomega_chi_imag"]), nomega_chi_real=int(s["nomega_chi_real"]),
                nomega_sigma=int(s["nomega_sigma"]), step_sigma=float(s["step_sigma"]),
                selfenergy_state_range=int(s["selfenergy_state_range"]), eta=float(s.get("eta", 0.001)))


def contour_inputs(case: dict, basis: dict):
    """RI-HF of the contour input (Auto auxiliary basis) and its windows:
    frozen core from frozencore='molgw', W from state ncore+1, Sigma states
    nhomo -+ selfenergy_state_range, p from ncore+1."""
    from oracle import gaussian_ri as g
    from oracle import rigw_oracle as o
    st = contour_settings(case)
    bas = {int(z): t for z, t in basis[case["basis"]].items()}
    scf, m, det = g.molecule_ri_hf([(z, tuple(x)) for z, x in case["atoms"]], bas, case["auxil_basis"])
    ncore = sum(g.element_core(z) for z, _ in case["atoms"]) if case["frozencore"].lower() == "molgw" else 0
    nocc = int(np.sum(scf.occupation > 0))
    rng = o.selfenergy_set_state_range(scf.e_orb.size, scf.occupation, ncoreg=ncore,
                                       selfenergy_state_range=st["selfenergy_state_range"])
    m_ia = np.ascontiguousarray(m[ncore:nocc, nocc:])
    m_sig = np.ascontiguousarray(m[rng.nsemin - 1:rng.nsemax, ncore:])
    return scf, m, rng, ncore, m_ia, m_sig, st
