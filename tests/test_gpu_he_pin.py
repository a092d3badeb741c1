"""The CUDA path pinned on known answers of the reference's own test suite:
He, HF in cc-pVDZ with the PAuto auxiliary basis (tests/inputs/testsuite:
1135-1153).  The M tensors and orbital energies of the oracle's front end
(committed fixture) go through the C ABI as MOLGW's Fortran would pass them:
rigw_polarizability_imag -> rigw_gw_selfenergy_imag -> rigw_sox_selfenergy_imag
(and rigw_sosex_selfenergy_imag) -> rigw_qp_solve.  The HOMO energies of
GW+SOX, GW+SOSEX and GW+2SOSEX must lie within the suite's 1e-4 eV of its
known answers and within 1e-6 eV of the oracle; plain GW within 1e-6 eV of the
oracle (the suite holds no imaginary-axis GW value for He)."""
import numpy as np
import pytest

from tests import he_case
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def he():
    return he_case.load()


@pytest.mark.parametrize("name", ["he_gw+sox_pade.in", "he_gw+sosex_pade.in", "he_gw+sosex2_pade.in"])
def test_vertex_homo_matches_the_reference_known_answer(engine, he, name):
    run = he["runs"][name]
    inst, m = he_case.instance(he, run)
    sox, factor, _ = he_case.VERTEX[run["settings"]["postscf"]]
    out = engine.gw_sox_imag(inst) if factor is None else engine.gw_sosex_imag(inst, m, factor_sosex=factor)
    ref, tol = he_case.homo_answer(run)
    assert abs(out.energy_qp_g[0] * HA_EV - ref) < tol
    orc = he_case.oracle_run(he, name)
    assert abs(out.energy_qp_g[0] - orc.energy_qp_g[0]) * HA_EV < 1e-6
    assert np.abs(out.sigma_calc - orc.sigma_calc.T).max() < 1e-9 * np.abs(orc.sigma_calc).max()


def test_plain_gw_matches_the_oracle(engine, he):
    from oracle import rigw_oracle as o
    run = he["runs"]["he_gw+sox_pade.in"]
    inst, _ = he_case.instance(he, run)
    out = engine.g0w0(inst)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=1, selfenergy_state_max=1)
    ref = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                      nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                      nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc, eta=inst.eta)
    assert abs(out.erpa - ref.erpa) < 1e-10
    assert abs(out.energy_qp_g[0] - ref.energy_qp_g[0]) * HA_EV < 1e-6
