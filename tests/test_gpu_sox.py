"""GW+SOX on the imaginary axis on the GPU against the oracle
(sox_selfenergy_imag_grid, src/m_g3w2_selfenergy.f90:2482-2591): Sigma^SOX
through the C ABI within 1e-11 of its largest entry (FP64 throughout), ragged
sizes (odd widths, auxiliary counts off the 16-wide k-tiles, evaluation points
off the 16-point passes), chunked products under a small HBM budget, bitwise
repeatability, and the GW+SOX QP energies within 1e-6 eV."""
import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.rigw import Engine, efermi_of
from oracle import rigw_oracle as o
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


def _points(inst):
    return efermi_of(inst) + 1j * inst.step_sigma_calc * np.arange(inst.nomega_sigma_calc)


def _oracle_sox(inst, z):
    window = inst.energy[: inst.m_sigma.shape[1]]
    return o.sox_selfenergy_imag(window, inst.m_sigma, inst.m_ia, z)


@pytest.mark.parametrize("shape", [(9, 80, 200, 16), (5, 37, 51, 8), (2, 33, 17, 8), (1, 3, 5, 8)])
def test_sox_matches_oracle(engine, shape):
    inst = synth.make_instance(*shape, seed=11)
    z = _points(inst)[:21]
    out = engine.sox_selfenergy_imag_grid(inst, z)
    ref = _oracle_sox(inst, z)
    assert out.shape == ref.shape
    assert np.abs(out - ref).max() <= 1e-11 * np.abs(ref).max()


def test_sox_is_repeatable(engine):
    inst = synth.make_instance(9, 80, 200, 16, seed=3)
    z = _points(inst)
    a = engine.sox_selfenergy_imag_grid(inst, z)
    b = engine.sox_selfenergy_imag_grid(inst, z)
    assert np.array_equal(a, b)


def test_sox_chunked_under_a_small_budget():
    from dataclasses import replace
    inst = synth.make_instance(9, 80, 200, 16, seed=4)
    # twelve Sigma states: operands ~5.7 MB, (p q|j c) 0.52 MB per state
    msig = np.random.default_rng(5).standard_normal((12, inst.nstate, inst.naux)) * 0.05
    inst = replace(inst, m_sigma=msig, nsemin=1, nsemax=12)
    z = _points(inst)
    ref = _oracle_sox(inst, z)
    eng = Engine(0, hbm_budget_bytes=10 << 20)
    try:
        out = eng.sox_selfenergy_imag_grid(inst, z)
        assert eng.last_stats()["chunks"] > 1
    finally:
        eng.close()
    assert np.abs(out - ref).max() <= 1e-11 * np.abs(ref).max()


def test_gw_plus_sox_qp_matches_oracle(engine):
    inst = synth.make_instance(9, 80, 200, 16, seed=42)
    out = engine.gw_sox_imag(inst)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    ref = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                      nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                      nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc,
                      eta=inst.eta, sox=True)
    assert np.abs(out.sigma_calc - ref.sigma_calc.T).max() <= 1e-9 * np.abs(ref.sigma_calc).max()
    assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV <= 1e-6


def test_sox_device_pointers_match_host_pointers(engine):
    import torch
    inst = synth.make_instance(5, 37, 51, 8, seed=2)
    z = _points(inst)
    host = engine.sox_selfenergy_imag_grid(inst, z)
    dev = engine.sox_selfenergy_imag_grid(inst, z, device_arrays={
        "m_ov": torch.from_numpy(np.ascontiguousarray(inst.m_ia)).cuda(),
        "m_pq": torch.from_numpy(np.ascontiguousarray(inst.m_sigma)).cuda()})
    assert np.array_equal(host, dev)


def test_gw_plus_sox_builds_w_from_energy_g(engine):
    """energy_g != energy: the vertex path's W takes energy_g (src/m_gw_selfenergy_grid.f90:604)."""
    from dataclasses import replace
    inst = synth.make_instance(5, 37, 51, 8, seed=4)
    eg = inst.energy + np.random.default_rng(1).uniform(-0.05, 0.05, inst.nstate)
    out = engine.gw_sox_imag(replace(inst, energy_g=eg))
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    ref = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                      nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                      nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc,
                      eta=inst.eta, energy_g=eg, sox=True)
    assert np.abs(out.sigma_calc - ref.sigma_calc.T).max() <= 1e-9 * np.abs(ref.sigma_calc).max()
    assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV <= 1e-6
