"""The GW density matrix from the imaginary axis (pt_density_matrix
'GW_IMAGINARY') pinned on the reference's CO test (tests/inputs/co_gw_dm_imag.in;
testsuite:975-980): HF in the Cartesian cc-pVDZ_gaussian basis with cc-pVDZ-RI
(2 of 132 metric eigenvalues below 1e-6 dropped), frozencore='molgw', W on 128
imaginary frequencies, the density matrix on 16.  The oracle's front end gives
the SCF energy, and its gw_density_matrix_imag + correlated-density energies
give the kinetic, nuclear, Hartree and exchange energies of the correlated
density matrix, each within the suite's 1e-7 Ha.  CPU only (a few seconds)."""
import numpy as np
import pytest

from tests import co_case


@pytest.fixture(scope="module")
def co():
    return co_case.load()


@pytest.fixture(scope="module")
def run(co):
    return co_case.oracle_run(co)


def test_front_end_reproduces_the_scf_energy(co, run):
    ref, tol = co["case"]["known_answers"]["SCF Total Energy"]
    assert abs(run["scf"].energy - ref) < tol
    assert (run["details"]["nbf"], run["details"]["naux_basis"], run["details"]["nauxil"]) == (30, 132, 130)


@pytest.mark.parametrize("key", ["kinetic", "nucleus", "hartree", "exchange"])
def test_correlated_density_energies_match_the_known_answers(co, run, key):
    ref, tol = co["case"]["known_answers"][co_case.LABELS[key]]
    assert abs(run["energies"][key] - ref) < tol


def test_correction_moves_the_energies_and_keeps_the_trace(co, run):
    """The pinned values are those of the corrected density matrix, not of HF's:
    the correction moves each energy by more than 1e-3 Ha; it conserves the
    electron number to 1e-4 (as the suite's Trace checks of the other GW
    density-matrix inputs)."""
    from oracle import gaussian_ri as g
    hf = g.correlated_dm_energies(run["scf"], run["details"], np.zeros_like(run["p_corr"]))
    for key in ("kinetic", "nucleus", "hartree", "exchange"):
        assert abs(run["energies"][key] - hf[key]) > 1e-3
    assert abs(run["energies"]["trace_mo"] - 14.0) < 1e-4
    assert np.allclose(run["p_corr"], run["p_corr"].T, atol=0)
    assert np.abs(run["p_corr"] - co["p_corr"]).max() < 1e-10
