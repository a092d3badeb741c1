"""The H2O cc-pVDZ workload (HF, cc-pVDZ-RI auxiliary basis, 16 imaginary
frequencies, HOMO and LUMO) and the two reference inputs that pin its front end
(tests/inputs/h2o_rt_tddft_hf_PC2B.in, h2o_mp3.in; known answers at
tests/inputs/testsuite:782-790), read from the committed fixture
tests/golden/h2o_ccpvdz.npz."""
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


def bases(d: dict, name: str) -> dict:
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
