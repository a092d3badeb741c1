"""GW+SOX on the imaginary axis (sox_selfenergy_imag_grid,
src/m_g3w2_selfenergy.f90:2482-2591) in the oracle: the vectorised form used as
the GPU checker against a loop-for-loop restatement of the Fortran (two RI
integrals per term through evaluate_eri_mo), and the properties of the sum.
CPU only.

The reference suite's GW+SOX value (tests/inputs/testsuite:1135-1137, He
cc-pVDZ, HOMO -24.821330 eV) needs an SCF with Gaussian integrals and is not
reproducible here; the loop form is the pin."""
import numpy as np
import pytest

from molgw_b200 import synth
from oracle import rigw_oracle as o


def _window(seed, no, nv, naux):
    rng = np.random.default_rng(seed)
    ns = no + nv
    a = rng.standard_normal((ns, ns, naux)) * 0.3
    m = 0.5 * (a + a.transpose(1, 0, 2))                   # (p q|P) symmetric in p, q
    e = np.concatenate([np.sort(rng.uniform(-1.2, -0.3, no)), np.sort(rng.uniform(0.05, 2.5, nv))])
    return m, e


@pytest.mark.parametrize("no,nv,naux,sig", [(3, 5, 7, [1, 2, 3, 4]), (2, 9, 4, [0, 1, 2]), (4, 6, 11, [3, 4])])
def test_vectorised_matches_loop_form(no, nv, naux, sig):
    m, e = _window(no * 100 + nv, no, nv, naux)
    efermi = 0.5 * (e[no - 1] + e[no])
    z = efermi + 1j * 0.15 * np.arange(9)
    ref = o.sox_selfenergy_imag_loops(e, m, no, sig, z)
    vec = o.sox_selfenergy_imag(e, m[sig], m[:no, no:], z, chunk=13)
    assert np.abs(vec - ref).max() <= 1e-13 * np.abs(ref).max()


def test_conjugate_symmetry_and_decay():
    """Sigma(z*) = Sigma(z)* for real integrals and energies, and z Sigma(z) tends to
    minus the sum of the numerators as |z| grows."""
    no, nv, naux = 3, 7, 9
    m, e = _window(7, no, nv, naux)
    z = np.array([0.1 + 0.4j, -0.2 + 1.3j])
    s = o.sox_selfenergy_imag(e, m[:4], m[:no, no:], z)
    sc = o.sox_selfenergy_imag(e, m[:4], m[:no, no:], z.conj())
    assert np.abs(sc - s.conj()).max() <= 1e-14 * np.abs(s).max()
    big = np.array([1e7j])
    lim = o.sox_selfenergy_imag(e, m[:4], m[:no, no:], big)[:, 0] * big[0]
    num = o.sox_selfenergy_imag(e * 0.0, m[:4], m[:no, no:], np.array([1.0]))[:, 0]   # sum of numerators
    assert np.abs(lim - num).max() <= 1e-5 * np.abs(num).max()


def test_gw_plus_sox_moves_the_qp_energies():
    inst = synth.make_instance(3, 20, 40, 8, seed=5)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    kw = dict(nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
              nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc, eta=inst.eta)
    gw = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng, **kw)
    gws = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng, sox=True, **kw)
    window = inst.energy[: inst.m_sigma.shape[1]]
    sox = o.sox_selfenergy_imag(window, inst.m_sigma, inst.m_ia, gws_points(inst))
    assert np.abs(gws.sigma_calc - gw.sigma_calc - sox.T).max() <= 1e-12 * np.abs(gws.sigma_calc).max()
    assert np.abs(gws.energy_qp_g - gw.energy_qp_g).max() > 1e-6


def gws_points(inst):
    from molgw_b200.rigw import efermi_of
    return efermi_of(inst) + 1j * inst.step_sigma_calc * np.arange(inst.nomega_sigma_calc)


def test_vertex_path_builds_w_from_energy_g():
    """On the vertex path the reference calls gw_selfenergy_grid with energy_g
    (src/m_selfenergy_evaluation.f90:496), which builds W from that argument
    (src/m_gw_selfenergy_grid.f90:604).  With energy_g != energy, the GW+SOX
    sigma_calc equals W, Sigma_c and the SOX loop form all taken from energy_g,
    and differs from a W built from energy."""
    inst, mf = synth.with_window(synth.make_instance(3, 12, 20, 8, seed=5), seed=6)
    no = inst.nocc
    eg = inst.energy + np.random.default_rng(3).uniform(-0.05, 0.05, inst.nstate)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    kw = dict(nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
              nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc, eta=inst.eta)
    res = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                      energy_g=eg, sox=True, **kw)
    omega, weight = o.imaginary_quad_grid(inst.nomega)
    occ = inst.occupation

    def by_hand(ew):
        sf = o.polarizability_grid(inst.m_ia, ew[:no], ew[no:], occ[:no], occ[no:], omega, weight)
        se = o.se_init_imaginary_axis(eg, rng, "pade", inst.nomega_sigma, inst.step_sigma,
                                      inst.nomega_sigma_calc, inst.step_sigma_calc)
        sig = list(range(inst.nsemin - 1, inst.nsemax))
        gw = o.gw_selfenergy_imag(eg, inst.m_sigma, sf, se.omega_calc, 1)
        return gw + o.sox_selfenergy_imag_loops(eg, mf, no, sig, se.omega_calc).T

    ref = by_hand(eg)
    assert np.abs(res.sigma_calc - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.abs(by_hand(inst.energy) - ref).max() > 1e-6 * np.abs(ref).max()
