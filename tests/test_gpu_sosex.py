"""GW+SOSEX on the imaginary axis on the GPU against the oracle
(sosex_selfenergy_imag_grid, src/m_g3w2_selfenergy.f90:2200-2478): Sigma^SOSEX
through the C ABI from the resident W within 1e-10 of its largest entry (FP64
throughout; W itself agrees with the oracle's to ~1e-12), odd and even window
widths, chunks of Sigma states under a small HBM budget, bitwise repeatability,
and the GW+SOSEX QP energies within 1e-6 eV."""
import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.rigw import Engine, efermi_of
from oracle import rigw_oracle as o
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


def _case(shape, seed=11):
    return synth.with_window(synth.make_instance(*shape, seed=seed), seed=seed + 1)


def _points(inst):
    return efermi_of(inst) + 1j * inst.step_sigma_calc * np.arange(inst.nomega_sigma_calc)


def _oracle(inst, mf, z, factor=1.0):
    no = inst.nocc
    e = inst.energy
    omega, weight = o.imaginary_quad_grid(inst.nomega)
    sf = o.polarizability_grid(inst.m_ia, e[:no], e[no:], inst.occupation[:no], inst.occupation[no:], omega, weight)
    sig = list(range(inst.nsemin - 1, inst.nsemax))
    return o.sosex_selfenergy_imag(e, mf, no, sig, sf.chi, sf.omega, sf.weight_quad, z, factor)


def _gpu(eng, inst, mf, z, factor=1.0):
    _, _, wpol = eng.polarizability_grid_scalapack(inst)
    try:
        return eng.sosex_selfenergy_imag_grid(wpol, inst, mf, z, factor)
    finally:
        wpol.release()


@pytest.mark.parametrize("shape", [(9, 80, 200, 16), (5, 37, 51, 8), (3, 12, 20, 8), (1, 3, 5, 8)])
def test_sosex_matches_oracle(engine, shape):
    inst, mf = _case(shape)
    z = _points(inst)[:21]
    out = _gpu(engine, inst, mf, z, 2.0)
    ref = _oracle(inst, mf, z, 2.0)
    assert np.abs(out - ref).max() <= 1e-10 * np.abs(ref).max()


def test_sosex_is_repeatable(engine):
    inst, mf = _case((9, 80, 200, 16), seed=3)
    z = _points(inst)
    assert np.array_equal(_gpu(engine, inst, mf, z), _gpu(engine, inst, mf, z))


def test_sosex_chunked_under_a_small_budget():
    from dataclasses import replace
    inst, mf = _case((20, 200, 30, 4), seed=4)
    # six Sigma states at 21 MB of T, B1, B2 and R each, beside ~30 MB of W and
    # window tensor: one or two states per pass under 100 MB
    inst = replace(inst, nsemin=18, nsemax=23, m_sigma=np.ascontiguousarray(mf[17:23]))
    z = _points(inst)
    ref = _oracle(inst, mf, z)
    eng = Engine(0, hbm_budget_bytes=100 << 20)
    try:
        out = _gpu(eng, inst, mf, z)
        assert eng.last_stats()["chunks"] > 1
    finally:
        eng.close()
    assert np.abs(out - ref).max() <= 1e-10 * np.abs(ref).max()


def test_gw_plus_sosex_qp_matches_oracle(engine):
    inst, mf = _case((9, 80, 200, 16), seed=42)
    out = engine.gw_sosex_imag(inst, mf, factor_sosex=2.0)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    ref = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                      nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                      nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc,
                      eta=inst.eta, sox=True, factor_sosex=2.0, m_full=mf)
    assert np.abs(out.sigma_calc - ref.sigma_calc.T).max() <= 1e-9 * np.abs(ref.sigma_calc).max()
    assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV <= 1e-6


def test_gw_plus_sosex_builds_w_from_energy_g(engine):
    """energy_g != energy: the vertex path's W takes energy_g (src/m_gw_selfenergy_grid.f90:604)."""
    from dataclasses import replace
    inst, mf = _case((5, 37, 51, 8), seed=21)
    eg = inst.energy + np.random.default_rng(2).uniform(-0.05, 0.05, inst.nstate)
    out = engine.gw_sosex_imag(replace(inst, energy_g=eg), mf, factor_sosex=2.0)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    ref = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                      nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                      nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc,
                      eta=inst.eta, energy_g=eg, sox=True, factor_sosex=2.0, m_full=mf)
    assert np.abs(out.sigma_calc - ref.sigma_calc.T).max() <= 1e-9 * np.abs(ref.sigma_calc).max()
    assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV <= 1e-6
