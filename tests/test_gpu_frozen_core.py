"""Frozen core (MOLGW's ncorew / ncoreg), Sigma_x - V_xc and the frequency split on
the GPU against the oracle or the one-GPU solve.  Frozen core: the W window and the states p of Sigma start above the core
(src/m_selfenergy_tools.f90:67-122, src/m_gw_selfenergy_grid.f90:92-93, 270-290);
the engine takes the windows as the Fortran passes them."""
from dataclasses import replace

import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.rigw import RIGW_FP64
from oracle import rigw_oracle as o
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ncore", [1, 3])
def test_frozen_core_matches_oracle(engine, ncore):
    full = synth.make_instance(9, 80, 200, 16, seed=42)
    inst = replace(full, nocc=full.nocc - ncore, m_ia=np.ascontiguousarray(full.m_ia[ncore:]),
                   m_sigma=np.ascontiguousarray(full.m_sigma[:, ncore:]), ncore_w=ncore, ncore_g=ncore)
    out = engine.g0w0(inst, RIGW_FP64)
    rng = o.selfenergy_set_state_range(full.nstate, full.occupation, ncoreg=ncore, selfenergy_state_min=full.nsemin,
                                       selfenergy_state_max=full.nsemax)
    ref = o.g0w0_imag(full.energy, full.occupation, inst.m_ia, inst.m_sigma, full.nomega, rng,
                      nomega_sigma=full.nomega_sigma, step_sigma=full.step_sigma,
                      nomega_sigma_calc=full.nomega_sigma_calc, step_sigma_calc=full.step_sigma_calc, eta=full.eta,
                      ncore_w=ncore)
    assert abs(out.erpa - ref.erpa) <= 1e-10 * abs(ref.erpa)
    assert np.abs(out.sigma_calc - ref.sigma_calc.T).max() <= 1e-9 * np.abs(ref.sigma_calc).max()
    assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV <= 1e-6
    # freezing changes the answer (the core transitions and core states in G are gone)
    assert abs(out.erpa - engine.g0w0(full, RIGW_FP64).erpa) > 1e-8


def test_exchange_minus_vxc_matches_oracle(engine):
    """Sigma_x - V_xc of the Sigma states (a DFT starting point): enters the QP
    equation only (src/m_selfenergy_tools.f90:202-363)."""
    inst = synth.make_instance(9, 80, 200, 16, seed=42)
    xc = np.array([-0.085, 0.043])
    out = engine.g0w0(replace(inst, exchange_m_vxc=xc), RIGW_FP64)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    ref = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                      nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                      nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc, eta=inst.eta,
                      exchange_m_vxc=xc)
    assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV <= 1e-6
    assert np.abs(out.energy_qp_z - ref.energy_qp_z).max() * HA_EV <= 1e-6
    assert np.abs(out.energy_qp_g - engine.g0w0(inst, RIGW_FP64).energy_qp_g).max() > 1e-3


def test_frequency_split_partials_sum_to_the_full_solve(engine):
    """MOLGW's frequency split on one GPU: two ranks' partial Sigma_c and energies
    (W on each rank's frequencies) summed, then the QP equation on the sum, equal
    the one-GPU solve (src/m_gw_selfenergy_grid.f90:325, 626, 658)."""
    from molgw_b200 import parallel
    inst = synth.make_instance(9, 80, 200, 16, seed=42)
    full = engine.g0w0(inst, RIGW_FP64)
    parts = [engine.frequency_partials(inst, parallel.frequency_shard(inst.nomega, r, 2)) for r in range(2)]
    sig = sum(p[0] for p in parts)
    en = sum(p[1] for p in parts)
    assert abs(en[0] - full.erpa) <= 1e-12 * abs(full.erpa) and abs(en[1] - full.egw) <= 1e-12 * abs(full.egw)
    assert np.abs(sig - full.sigma_calc).max() <= 1e-12 * np.abs(full.sigma_calc).max()
    qp = engine.qp_solve(inst, sig)
    assert np.abs(qp.energy_qp_g - full.energy_qp_g).max() * HA_EV <= 1e-6
