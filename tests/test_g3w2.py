"""G (W-v) G (W-v) G on the imaginary axis (g3w2_selfenergy_imag_grid,
src/m_g3w2_selfenergy.f90:2018-2196) in the oracle: the separable form (the
three-energy denominators factor per state index, so each frequency pair is a
trilinear contraction) against a loop-for-loop restatement of the Fortran, and
the GW+G3W2_PADE sequence of the driver.  CPU only; the reference suite's
GW+G3W2 He values need an SCF and are not reproducible here."""
import numpy as np
import pytest

from molgw_b200 import synth
from oracle import rigw_oracle as o


def _case(no, nv, naux, nomega, seed):
    inst, mf = synth.with_window(synth.make_instance(no, nv, naux, nomega, seed=seed), seed=seed + 1)
    omega, weight = o.imaginary_quad_grid(nomega)
    e = inst.energy
    sf = o.polarizability_grid(inst.m_ia, e[:no], e[no:], inst.occupation[:no], inst.occupation[no:], omega, weight)
    z = 0.5 * (e[no - 1] + e[no]) + 1j * 0.1 * np.arange(4)
    return inst, mf, sf, z, list(range(inst.nsemin - 1, inst.nsemax))


@pytest.mark.parametrize("shape", [(2, 3, 5, 3), (2, 4, 6, 2)])
def test_separable_form_matches_loop_form(shape):
    inst, mf, sf, z, sig = _case(*shape, seed=13)
    ref = o.g3w2_selfenergy_imag_loops(inst.energy, mf, sig, sf.chi, sf.omega, sf.weight_quad, z)
    out = o.g3w2_selfenergy_imag(inst.energy, mf, sig, sf.chi, sf.omega, sf.weight_quad, z)
    assert np.abs(out - ref).max() <= 1e-13 * np.abs(ref).max()


def test_conjugate_symmetry():
    inst, mf, sf, z, sig = _case(3, 5, 8, 3, seed=17)
    a = o.g3w2_selfenergy_imag(inst.energy, mf, sig, sf.chi, sf.omega, sf.weight_quad, z)
    b = o.g3w2_selfenergy_imag(inst.energy, mf, sig, sf.chi, sf.omega, sf.weight_quad, z.conj())
    assert np.abs(b - a.conj()).max() <= 1e-14 * np.abs(a).max()


def test_gw_plus_g3w2_sequence():
    inst, mf, sf, z, sig = _case(3, 6, 10, 4, seed=19)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    kw = dict(nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma, nomega_sigma_calc=8,
              step_sigma_calc=inst.step_sigma_calc, eta=inst.eta)
    base = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng, sox=True,
                       factor_sosex=2.0, m_full=mf, **kw)
    full = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng, sox=True,
                       factor_sosex=2.0, m_full=mf, g3w2=True, **kw)
    from molgw_b200.rigw import efermi_of
    pts = efermi_of(inst) + 1j * inst.step_sigma_calc * np.arange(8)
    add = o.g3w2_selfenergy_imag(inst.energy, mf, sig, sf.chi, sf.omega, sf.weight_quad, pts)
    assert np.abs(full.sigma_calc - base.sigma_calc - add.T).max() <= 1e-12 * np.abs(full.sigma_calc).max()
