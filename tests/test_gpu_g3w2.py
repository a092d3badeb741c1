"""G3W2 on the imaginary axis on the GPU (g3w2_selfenergy_imag_grid,
src/m_g3w2_selfenergy.f90:2018-2196): Sigma^G3W2 through the C ABI from the
resident W against the oracle (itself pinned on a loop-for-loop restatement,
tests/test_g3w2.py) within 1e-10 of its largest entry, for even and odd window
widths; bitwise repeatability; and the whole GW+G3W2_PADE sequence (Sigma_c +
SOX + 2 SOSEX + G3W2, Pade, QP) on He against the reference suite's known answer
(tests/inputs/testsuite:1159-1161, -24.680279 eV at 1e-4) and the oracle
(1e-6 eV)."""
import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.rigw import efermi_of
from oracle import rigw_oracle as o
from tests import he_case
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


def _case(shape, seed):
    inst, mf = synth.with_window(synth.make_instance(*shape, seed=seed), seed=seed + 1)
    inst.nomega_sigma_calc = 9
    return inst, mf


def _points(inst):
    return efermi_of(inst) + 1j * inst.step_sigma_calc * np.arange(inst.nomega_sigma_calc)


def _oracle(inst, mf, z):
    no, e = inst.nocc, inst.energy
    omega, weight = o.imaginary_quad_grid(inst.nomega)
    sf = o.polarizability_grid(inst.m_ia, e[:no], e[no:], inst.occupation[:no], inst.occupation[no:], omega, weight)
    sig = list(range(inst.nsemin - 1, inst.nsemax))
    return o.g3w2_selfenergy_imag(e, mf, sig, sf.chi, sf.omega, sf.weight_quad, z)


def _gpu(eng, inst, mf, z):
    _, _, wpol = eng.polarizability_grid_scalapack(inst)
    try:
        return eng.g3w2_selfenergy_imag_grid(wpol, inst, mf, z)
    finally:
        wpol.release()


@pytest.mark.parametrize("shape", [(3, 12, 20, 4), (2, 7, 11, 3), (1, 4, 40, 8), (4, 25, 64, 4)])
def test_g3w2_matches_oracle(engine, shape):
    inst, mf = _case(shape, seed=sum(shape))
    z = _points(inst)
    ref = _oracle(inst, mf, z)
    out = _gpu(engine, inst, mf, z)
    assert out.shape == ref.shape
    assert np.abs(out - ref).max() <= 1e-10 * np.abs(ref).max()


def test_g3w2_is_repeatable(engine):
    inst, mf = _case((3, 12, 20, 4), seed=5)
    z = _points(inst)
    a = _gpu(engine, inst, mf, z)
    b = _gpu(engine, inst, mf, z)
    assert np.array_equal(a, b)


def test_he_gw_plus_g3w2_matches_the_reference_known_answer(engine):
    he = he_case.load()
    name = "he_gw+g3w2_pade.in"
    run = he["runs"][name]
    inst, m = he_case.instance(he, run)
    out = engine.gw_g3w2_imag(inst, m, efermi=he_case.settings(run)["mu_origin"])
    ref, tol = he_case.homo_answer(run)
    assert abs(out.energy_qp_g[0] * HA_EV - ref) < tol
    orc = he_case.oracle_run(he, name)
    assert abs(out.energy_qp_g[0] - orc.energy_qp_g[0]) * HA_EV < 1e-6
    assert np.abs(out.sigma_calc - orc.sigma_calc.T).max() < 1e-9 * np.abs(orc.sigma_calc).max()
