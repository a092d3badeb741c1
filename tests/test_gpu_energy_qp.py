"""G from energy_g (force_energy_qp, src/m_selfenergy_evaluation.f90:164-181) and
the ENERGY_QP round trip of successive runs on the GPU, against the oracle.
Tolerances as in the FP64 parity tests: E_RPA 1e-10 relative, sigma_calc 1e-9 of
its largest entry, QP energies 1e-6 eV."""
import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.energy_qp import read_energy_qp
from oracle import rigw_oracle as o
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


def _oracle(inst, energy_g=None):
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    return o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                       nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                       nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc,
                       eta=inst.eta, energy_g=energy_g)


def _close(out, ref):
    assert abs(out.erpa - ref.erpa) <= 1e-10 * abs(ref.erpa)
    assert np.abs(out.sigma_calc - ref.sigma_calc.T).max() <= 1e-9 * np.abs(ref.sigma_calc).max()
    assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV <= 1e-6


def test_energy_g_matches_oracle(engine):
    from dataclasses import replace
    inst = synth.make_instance(9, 80, 200, 16, seed=42)
    eg = inst.energy + np.random.default_rng(3).uniform(-0.02, 0.02, inst.nstate)
    _close(engine.g0w0(replace(inst, energy_g=eg)), _oracle(inst, eg))


def test_force_energy_qp_runs_match_oracle(engine, tmp_path):
    # 16 frequencies: an 8-frequency Pade fit amplifies 1e-14 changes of Sigma to
    # 1e-3 meV in the QP energies, in the oracle too
    inst = synth.make_instance(9, 80, 200, 16, seed=42)
    outs = engine.gw_imag_force_energy_qp(inst, nstep=3)
    eq = None
    for out in outs:
        ref = _oracle(inst, eq)
        _close(out, ref)
        eq = inst.energy.copy()
        eq[inst.nsemin - 1:inst.nsemax] = ref.energy_qp_g
    # the same runs through ENERGY_QP files: two runs, then one more from the file
    first = engine.gw_imag_force_energy_qp(inst, nstep=2, workdir=tmp_path)
    e_file, status = read_energy_qp(tmp_path, inst.nstate)
    assert status == 0
    assert np.array_equal(e_file[inst.nsemin - 1:inst.nsemax, 0], first[1].energy_qp_g)
    third = engine.gw_imag_force_energy_qp(inst, nstep=1, workdir=tmp_path)[0]
    assert np.abs(third.energy_qp_g - outs[2].energy_qp_g).max() * HA_EV <= 1e-9
