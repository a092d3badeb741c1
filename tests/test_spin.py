"""Open-shell (nspin = 2) restatement in the oracle: one chi0 over the transitions
of both spin channels (src/m_gw_selfenergy_grid.f90:118-149), Sigma and the QP
equation per channel (:279-319), se_init's efermi over both channels
(src/m_selfenergy_tools.f90:584-585)."""
import numpy as np

from molgw_b200 import synth
from oracle import rigw_oracle as o
from tests.spin_cases import as_two_channels, open_shell_instance, oracle_channels


def test_two_identical_channels_reproduce_the_closed_shell():
    # 16 frequencies: an 8-frequency Pade fit amplifies 1e-14 changes of Sigma to 1e-3 meV
    inst = synth.make_instance(9, 80, 200, 16, seed=42)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    kw = dict(nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma, nomega_sigma_calc=inst.nomega_sigma_calc,
              step_sigma_calc=inst.step_sigma_calc, eta=inst.eta)
    ref = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng, **kw)
    for r in o.g0w0_imag_spin(oracle_channels(as_two_channels(inst)), inst.nomega, **kw):
        assert abs(r.erpa - ref.erpa) <= 1e-12 * abs(ref.erpa)
        assert abs(r.egw - ref.egw) <= 1e-12 * abs(ref.egw)
        assert np.abs(r.sigma_calc - ref.sigma_calc).max() <= 1e-12 * np.abs(ref.sigma_calc).max()
        assert np.abs(r.energy_qp_g - ref.energy_qp_g).max() <= 1e-9
        assert abs(r.ehomo - ref.ehomo) <= 1e-9 and abs(r.elumo - ref.elumo) <= 1e-9


def test_spin_polarized_instance_runs():
    inst = open_shell_instance()
    out = o.g0w0_imag_spin(oracle_channels(inst), inst.nomega, nomega_sigma=inst.nomega_sigma,
                           step_sigma=inst.step_sigma, nomega_sigma_calc=inst.nomega_sigma_calc,
                           step_sigma_calc=inst.step_sigma_calc, eta=inst.eta)
    assert len(out) == 2 and out[0].erpa == out[1].erpa and out[0].erpa < 0.0
    for r in out:
        assert np.all(np.isfinite(r.energy_qp_g)) and r.ehomo < r.elumo


def test_host_efermi_rule():
    """molgw_b200.rigw.efermi_of follows se_init (src/m_selfenergy_tools.f90:584-585):
    half-way between the highest energy of state nhomo_G and the lowest of state
    nhomo_G + 1 over the spin channels, from the energies in G."""
    from dataclasses import replace
    from molgw_b200.rigw import efermi_of
    inst = synth.make_instance(4, 30, 70, 8, seed=41)
    e = inst.energy
    assert efermi_of(inst) == 0.5 * (e[3] + e[4])
    fc = replace(inst, nocc=3, m_ia=inst.m_ia[1:], ncore_w=1, ncore_g=1)     # frozen core keeps nhomo_G
    assert efermi_of(fc) == efermi_of(inst)
    eg = e + 0.01
    assert efermi_of(replace(inst, energy_g=eg)) == 0.5 * (eg[3] + eg[4])
    two = open_shell_instance()
    e1, e2 = two.energy, two.spin2.energy
    assert efermi_of(two) == 0.5 * (max(e1[4], e2[4]) + min(e1[5], e2[5]))


def test_gw_plus_sox_two_identical_channels_reproduce_the_closed_shell():
    """Sigma^SOX runs per spin with no spin factor (src/m_g3w2_selfenergy.f90:2530-2580),
    and W from two identical half-occupied channels is the closed-shell W, so GW+SOX
    per channel equals the closed-shell GW+SOX."""
    from tests.spin_cases import as_two_channels, oracle_channels
    # 16 frequencies: an 8-frequency Pade fit amplifies the 1e-16 differences of the
    # two chi0 summation orders to 1e-5 Ha in the QP energies, without SOX as well
    inst = synth.make_instance(9, 80, 200, 16, seed=42)
    kw = dict(nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
              nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc, eta=inst.eta)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    ref = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng, sox=True, **kw)
    for out in o.g0w0_imag_spin(oracle_channels(as_two_channels(inst)), inst.nomega, sox=True, **kw):
        assert np.abs(out.sigma_calc - ref.sigma_calc).max() <= 1e-14 * np.abs(ref.sigma_calc).max()
        assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() <= 1e-10
