"""The oracle pinned on known answers of the reference's own test suite that
run the whole imaginary-axis path: He, HF in cc-pVDZ with the PAuto auxiliary
basis (tests/inputs/testsuite:1135-1161).  The oracle's Gaussian front end
(oracle/gaussian_ri.py) reproduces the SCF total energy, and its
selfenergy_evaluation (W, Sigma_c, SOX, SOSEX and G3W2 on the imaginary axis,
Thiele continuation, graphical QP equation) the HOMO energies of GW+SOX,
GW+SOSEX, GW+2SOSEX and GW+G3W2, each within the tolerance the reference's
suite states (1e-7 Ha, 1e-4 eV).  CPU only."""
import numpy as np
import pytest

from oracle import gaussian_ri as g
from tests import he_case
from tests.conftest import HA_EV


@pytest.fixture(scope="module")
def he():
    return he_case.load()


def test_front_end_reproduces_the_scf_energy_and_the_fixture(he):
    scf, m, det = g.atom_ri_hf(he["basis_text"], 2)
    ref, tol = he["runs"]["he_gw+sox_pade.in"]["known_answers"]["SCF Total Energy"]
    assert abs(scf.energy - ref) < tol
    assert det["nauxil"] == det["naux_basis"] == 40           # no metric eigenvalue below 1e-6
    assert np.allclose(scf.e_orb, he["energy"], atol=1e-12)
    # M is defined up to the sign of each MO: compare sign-fixed products
    assert np.allclose(np.einsum("pqP,rsP->pqrs", m, m), np.einsum("pqP,rsP->pqrs", he["m_full"], he["m_full"]),
                       atol=1e-11)
    # Sigma_x - V_xc of HF is <p|F|p> - e_p = 0 at convergence (src/m_selfenergy_tools.f90:787-796)
    assert np.abs(scf.fock_mo_diag - scf.e_orb).max() < 1e-10


def test_ri_matches_four_center_hartree_fock(he):
    """PAuto spans the orbital products of He: the RI SCF energy equals the
    four-center one within 1e-9 Ha."""
    scf, _, det = g.atom_ri_hf(he["basis_text"], 2)
    eri = g.coulomb_4center(det["bf"])
    S, H = det["S"], det["H"]
    w, u = np.linalg.eigh(S)
    X = u / np.sqrt(w)
    D = np.zeros_like(S)
    for _ in range(60):
        F = H + np.einsum("ijkl,kl->ij", eri, D) - 0.5 * np.einsum("ikjl,kl->ij", eri, D)
        c = X @ np.linalg.eigh(X.T @ F @ X)[1]
        D = 2.0 * c[:, :1] @ c[:, :1].T
    F = H + np.einsum("ijkl,kl->ij", eri, D) - 0.5 * np.einsum("ikjl,kl->ij", eri, D)
    assert abs(0.5 * float(np.sum(D * (H + F))) - scf.energy) < 1e-9


@pytest.mark.parametrize("name", ["he_gw+sox_pade.in", "he_gw+sosex_pade.in", "he_gw+sosex2_pade.in",
                                  "he_gw+g3w2_pade.in"])
def test_oracle_reproduces_the_known_homo(he, name):
    res = he_case.oracle_run(he, name)
    ref, tol = he_case.homo_answer(he["runs"][name])
    assert abs(res.ehomo * HA_EV - ref) < tol
