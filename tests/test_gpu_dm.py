"""The GW density matrix from the imaginary axis on the CUDA path
(rigw_gw_density_matrix_imag after rigw_polarizability_imag): CO in the
Cartesian cc-pVDZ_gaussian basis with cc-pVDZ-RI, 128 imaginary frequencies of
W, 16 of the density matrix (tests/inputs/co_gw_dm_imag.in).  The correction
matches the oracle's to 1e-10 of its largest entry, and the energies of the
correlated density matrix match the reference suite's known answers within its
1e-7 Ha.  Device-pointer-free host path; one spin channel."""
import numpy as np
import pytest

from tests import co_case

pytestmark = pytest.mark.gpu


def test_co_density_matrix_matches_the_oracle_and_the_known_answers(engine):
    from oracle import gaussian_ri as g
    co = co_case.load()
    scf, m, det = co_case.front_end(co)
    inst = co_case.instance(co, scf, m)
    ncore = inst.ncore_g
    p_gpu, erpa = engine.gw_density_matrix_imag(inst, m[ncore:, ncore:], co["case"]["nomega_sigma"])
    ref = co["p_corr"]
    assert np.abs(p_gpu - ref).max() < 1e-10 * np.abs(ref).max()
    assert np.array_equal(p_gpu, p_gpu.T)
    en = g.correlated_dm_energies(scf, det, p_gpu)
    for key, label in co_case.LABELS.items():
        known, tol = co["case"]["known_answers"][label]
        assert abs(en[key] - known) < tol, (key, en[key], known)
