"""The He cc-pVDZ / PAuto case of the reference's test suite
(tests/inputs/he_gw+sox_pade.in, he_gw+sosex_pade.in, he_gw+sosex2_pade.in,
he_gw+g3w2_pade.in; known answers at tests/inputs/testsuite:1135-1161), read
from the committed fixture tests/golden/he_ccpvdz_pauto.npz."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "he_ccpvdz_pauto.npz"
ETA = 0.001                       # default eta, src/input_variables.f90:374

# postscf -> (sox, factor_sosex, g3w2), src/m_selfenergy_evaluation.f90:494-503
VERTEX = {"gw+sox_pade": (True, None, False), "gw+sosex_pade": (True, 1.0, False),
          "gw+2sosex_pade": (True, 2.0, False), "gw+g3w2_pade": (True, 2.0, True)}


def load() -> dict:
    d = dict(np.load(GOLDEN))
    d["runs"] = json.loads(str(d["runs"]))
    d["basis_text"] = str(d["basis_text"])
    return d


def settings(run: dict) -> dict:
    s = run["settings"]
    return dict(nomega=int(s["nomega_chi_imag"]), nomega_sigma=int(s["nomega_sigma"]),
                step_sigma=float(s["step_sigma"]), nomega_sigma_calc=int(s["nomega_sigma_calc"]),
                step_sigma_calc=float(s["step_sigma_calc"]), mu_origin=float(s.get("mu_origin", -100.0)))


def homo_answer(run: dict) -> tuple[float, float]:
    return next(v for k, v in run["known_answers"].items() if k.endswith("HOMO energy"))


def instance(d: dict, run: dict):
    """GWInstance of the run: one doubly occupied state, four empty ones, the
    HOMO as the only Sigma state (selfenergy_state_range = 0), and the window
    tensor M[q, r, P] for the vertex terms."""
    from molgw_b200.synth import GWInstance
    st = settings(run)
    m = d["m_full"]
    nocc = int(np.sum(d["occupation"] > 0))
    inst = GWInstance(nocc=nocc, nvirt=m.shape[0] - nocc, naux=m.shape[2], nomega=st["nomega"],
                      energy=d["energy"].copy(), occupation=d["occupation"].copy(),
                      m_ia=np.ascontiguousarray(m[:nocc, nocc:]), m_sigma=np.ascontiguousarray(m[[nocc - 1]]),
                      nsemin=nocc, nsemax=nocc, nomega_sigma_calc=st["nomega_sigma_calc"],
                      step_sigma_calc=st["step_sigma_calc"], nomega_sigma=st["nomega_sigma"],
                      step_sigma=st["step_sigma"], eta=ETA)
    return inst, np.ascontiguousarray(m)


def oracle_run(d: dict, name: str):
    """The oracle's selfenergy_evaluation for the input ``name``."""
    from oracle import rigw_oracle as o
    run = d["runs"][name]
    inst, m = instance(d, run)
    sox, factor, g3w2 = VERTEX[run["settings"]["postscf"]]
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    return o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                       nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                       nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc,
                       eta=inst.eta, sox=sox, factor_sosex=factor, m_full=m, g3w2=g3w2,
                       mu_origin=settings(run)["mu_origin"])
