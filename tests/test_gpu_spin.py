"""Open-shell (nspin = 2) G0W0 on the GPU against the oracle: one W from both spin
channels' transitions, Sigma and QP per channel from the resident factors.
Tolerances as in the FP64 parity tests (E_RPA 1e-10 relative, sigma_calc 1e-9 of
its largest entry, QP 1e-6 eV); split precision within 1 meV of FP64."""
import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.rigw import RIGW_BF16X3, RIGW_FP64
from oracle import rigw_oracle as o
from tests.conftest import HA_EV
from tests.spin_cases import as_two_channels, open_shell_instance, oracle_channels

pytestmark = pytest.mark.gpu


def _oracle(inst):
    return o.g0w0_imag_spin(oracle_channels(inst), inst.nomega, nomega_sigma=inst.nomega_sigma,
                            step_sigma=inst.step_sigma, nomega_sigma_calc=inst.nomega_sigma_calc,
                            step_sigma_calc=inst.step_sigma_calc, eta=inst.eta)


def test_open_shell_matches_oracle(engine):
    inst = open_shell_instance()
    outs, refs = engine.g0w0_spin(inst, RIGW_FP64), _oracle(inst)
    for out, ref in zip(outs, refs):
        assert abs(out.erpa - ref.erpa) <= 1e-10 * abs(ref.erpa)
        assert abs(out.egw - ref.egw) <= 1e-10 * abs(ref.egw)
        assert np.abs(out.sigma_calc - ref.sigma_calc.T).max() <= 1e-9 * np.abs(ref.sigma_calc).max()
        assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV <= 1e-6
        assert abs(out.ehomo - ref.ehomo) * HA_EV <= 1e-6 and abs(out.elumo - ref.elumo) * HA_EV <= 1e-6


def test_two_identical_channels_reproduce_the_closed_shell(engine):
    inst = synth.make_instance(9, 80, 200, 16, seed=42)
    ref = engine.g0w0(inst, RIGW_FP64)
    for out in engine.g0w0_spin(as_two_channels(inst), RIGW_FP64):
        assert abs(out.erpa - ref.erpa) <= 1e-11 * abs(ref.erpa)
        assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV <= 1e-7
        assert abs(out.ehomo - ref.ehomo) * HA_EV <= 1e-7 and abs(out.elumo - ref.elumo) * HA_EV <= 1e-7


def test_open_shell_split_precision(engine):
    inst = open_shell_instance()
    f64, spl = engine.g0w0_spin(inst, RIGW_FP64), engine.g0w0_spin(inst, RIGW_BF16X3)
    for a, b in zip(f64, spl):
        assert np.abs(a.energy_qp_g - b.energy_qp_g).max() * HA_EV * 1e3 <= 1.0


def test_open_shell_gw_plus_sox_matches_oracle(engine):
    inst = open_shell_instance()
    outs = engine.g0w0_spin(inst, RIGW_FP64, sox=True)
    refs = o.g0w0_imag_spin(oracle_channels(inst), inst.nomega, nomega_sigma=inst.nomega_sigma,
                            step_sigma=inst.step_sigma, nomega_sigma_calc=inst.nomega_sigma_calc,
                            step_sigma_calc=inst.step_sigma_calc, eta=inst.eta, sox=True)
    for out, ref in zip(outs, refs):
        assert np.abs(out.sigma_calc - ref.sigma_calc.T).max() <= 1e-9 * np.abs(ref.sigma_calc).max()
        assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV <= 1e-6
