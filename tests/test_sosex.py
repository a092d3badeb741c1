"""GW+SOSEX on the imaginary axis (sosex_selfenergy_imag_grid,
src/m_g3w2_selfenergy.f90:2200-2478) in the oracle: the vectorised form used as
the GPU checker against a loop-for-loop restatement of the Fortran (bra-kets
recomputed for every frequency, sign and evaluation point), and the properties of
the sum.  CPU only.

The reference suite's GW+SOSEX values (tests/inputs/testsuite:1139-1145, He
cc-pVDZ) need an SCF with Gaussian integrals and are not reproducible here; the
loop form is the pin."""
import numpy as np
import pytest

from molgw_b200 import synth
from oracle import rigw_oracle as o


def _case(no, nv, naux, nomega, seed):
    inst, mf = synth.with_window(synth.make_instance(no, nv, naux, nomega, seed=seed), seed=seed + 1)
    omega, weight = o.imaginary_quad_grid(nomega)
    e = inst.energy
    sf = o.polarizability_grid(inst.m_ia, e[:no], e[no:], inst.occupation[:no], inst.occupation[no:], omega, weight)
    z = 0.5 * (e[no - 1] + e[no]) + 1j * 0.1 * np.arange(5)
    sig = list(range(inst.nsemin - 1, inst.nsemax))
    return inst, mf, sf, z, sig


@pytest.mark.parametrize("shape", [(2, 5, 6, 3), (3, 4, 9, 4), (4, 7, 5, 2)])
def test_vectorised_matches_loop_form(shape):
    inst, mf, sf, z, sig = _case(*shape, seed=7)
    no = shape[0]
    ref = o.sosex_selfenergy_imag_loops(inst.energy, mf, no, sig, sf.chi, sf.omega, sf.weight_quad, z, 2.0)
    vec = o.sosex_selfenergy_imag(inst.energy, mf, no, sig, sf.chi, sf.omega, sf.weight_quad, z, 2.0)
    assert np.abs(vec - ref).max() <= 1e-13 * np.abs(ref).max()


def test_conjugate_symmetry_and_factor():
    inst, mf, sf, z, sig = _case(3, 8, 10, 4, seed=9)
    a = o.sosex_selfenergy_imag(inst.energy, mf, 3, sig, sf.chi, sf.omega, sf.weight_quad, z)
    b = o.sosex_selfenergy_imag(inst.energy, mf, 3, sig, sf.chi, sf.omega, sf.weight_quad, z.conj())
    assert np.abs(b - a.conj()).max() <= 1e-14 * np.abs(a).max()
    two = o.sosex_selfenergy_imag(inst.energy, mf, 3, sig, sf.chi, sf.omega, sf.weight_quad, z, 2.0)
    assert np.abs(two - 2.0 * a).max() <= 1e-15 * np.abs(a).max()


def test_gw_plus_sosex_adds_sox_and_sosex():
    inst, mf, sf, z, sig = _case(4, 12, 20, 8, seed=3)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    kw = dict(nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
              nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc, eta=inst.eta)
    sox = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng, sox=True, **kw)
    both = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng, sox=True,
                       factor_sosex=1.0, m_full=mf, **kw)
    from molgw_b200.rigw import efermi_of
    pts = efermi_of(inst) + 1j * inst.step_sigma_calc * np.arange(inst.nomega_sigma_calc)
    add = o.sosex_selfenergy_imag(inst.energy, mf, 4, sig, sf.chi, sf.omega, sf.weight_quad, pts)
    assert np.abs(both.sigma_calc - sox.sigma_calc - add.T).max() <= 1e-12 * np.abs(both.sigma_calc).max()
    assert np.abs(both.energy_qp_g - sox.energy_qp_g).max() > 1e-6
