"""The oracle (CPU restatement of MOLGW's path) against the reference's own known
answers and the identities of the algorithm.  CPU only."""
import numpy as np
import pytest

from oracle import rigw_oracle as o
from tests.conftest import instance_from_golden


def test_lih_analytic_rpa_matches_reference(golden_lih):
    # tests/inputs/testsuite:1206-1207 (lih_bulk08_abinit_rpa.in): -0.1152301335 Ha, tol 1e-7
    d = golden_lih
    nocc = d["m_ia"].shape[0]
    e = d["energy"]
    ec = o.analytic_rpa_correlation(d["m_ia"], e[:nocc], e[nocc:])
    assert abs(ec - float(d["ref_rpa_analytic"])) < float(d["ref_rpa_tol"])


def test_lih_testing_integral_matches_reference(golden_lih):
    # tests/inputs/testsuite:1209-1211: 'Testing integral (11|11)' 2.92396387E-01, tol 1e-7
    v = golden_lih["vertex_11"]
    assert abs(float(v @ v) - float(golden_lih["ref_integral_11_11"])) < 1e-7


@pytest.mark.parametrize("nomega,tol", [(16, 1e-9), (32, 1e-10), (64, 1e-10)])
def test_lih_imaginary_axis_rpa_converges_to_analytic(golden_lih, nomega, tol):
    d = golden_lih
    nocc = d["m_ia"].shape[0]
    e, occ = d["energy"], d["occupation"]
    w, wt = o.imaginary_quad_grid(nomega)
    sf = o.polarizability_grid(d["m_ia"], e[:nocc], e[nocc:], occ[:nocc], occ[nocc:], w, wt, keep_chi=False)
    assert abs(sf.erpa - float(d["ref_rpa_analytic"])) < 1e-7
    assert abs(sf.erpa - float(d["rpa_analytic_oracle"])) < tol


def test_gauss_legendre_exact_for_polynomials():
    x, w = o.coeffs_gausslegint(0.0, 1.0, 16)
    for deg in range(0, 31):
        # the Newton iteration stops at 1e-13 (src/m_numerical_tools.f90:54)
        assert abs(np.sum(w * x ** deg) - 1.0 / (deg + 1)) < 1e-12


def test_imag_grid_integrates_lorentzian():
    # int_0^inf 2a/(w^2+a^2) dw = pi for any a > 0: the mapped grid handles it
    om, wt = o.imaginary_quad_grid(64)
    for a in (0.3, 1.0, 5.0):
        assert abs(np.sum(wt * 2 * a / (om ** 2 + a ** 2)) - np.pi) < 1e-6


def test_energy_identities_logdet_and_traces(golden_synth):
    d = golden_synth
    nocc = d["m_ia"].shape[0]
    e, occ = d["energy"], d["occupation"]
    w, wt = o.imaginary_quad_grid(4)
    sf = o.polarizability_grid(d["m_ia"], e[:nocc], e[nocc:], occ[:nocc], occ[nocc:], w, wt, keep_eigval=True)
    for k in range(4):
        lam = sf.eigval[k]
        eps = np.linalg.inv(np.eye(len(lam)) + sf.chi[k])    # chi = eps^-1 chi0 = eps^-1 - 1
        sign, logdet = np.linalg.slogdet(eps)
        assert sign > 0 and abs(logdet - np.sum(np.log(lam))) < 1e-10
        assert abs(np.trace(eps) - np.sum(lam)) < 1e-10
        assert abs(np.trace(np.linalg.inv(eps)) - np.sum(1 / lam)) < 1e-10
        assert lam.min() >= 1.0 - 1e-12


def test_pade_reproduces_input_points():
    rng = np.random.default_rng(0)
    z = 0.1 + 1j * np.linspace(0, 2, 9)
    f = 1.0 / (z - 0.5) + 0.3 / (z + 0.7) + 0.01 * rng.standard_normal(9)
    aa = o.calculate_pade_a(z, f)
    for zi, fi in zip(z, f):
        assert abs(o.pade_eval(aa, z, zi) - fi) < 1e-10 * max(1, abs(fi))


def test_pade_exact_for_rational_function():
    z = 1j * np.linspace(0.0, 3.0, 11) + 0.05
    f = 2.0 / (z - 1.5) - 1.0 / (z + 0.8)
    aa = o.calculate_pade_a(z, f)
    for x in (-0.3, 0.2, 0.9):
        assert abs(o.pade_eval(aa, z, x + 0.01j) - (2.0 / (x + 0.01j - 1.5) - 1.0 / (x + 0.01j + 0.8))) < 1e-8


def test_pade_continuation_sensitivity_bounds_the_parity_tolerance(golden_lih):
    """The reference's continuation (se_pade_fit on 2*50-1 points) turns 1e-15
    relative changes of sigma_calc into ~1e-6 changes of Sigma on the real grid,
    while the graphical QP energies move by < 1e-7 eV.  This fixes the tolerances
    of the GPU parity tests for the real-grid Sigma and the QP energies."""
    d = golden_lih
    e = d["energy"]
    nsemin, nsemax = int(d["nsemin"]), int(d["nsemax"])
    rng = o.selfenergy_set_state_range(len(e), d["occupation"], selfenergy_state_min=nsemin,
                                       selfenergy_state_max=nsemax)
    sc = d["sigma_calc"].T.copy()
    outs = []
    for trial in range(3):
        se = o.se_init_imaginary_axis(e, rng, "pade", 101, 0.025, 50, 0.075)
        noise = 1.0 + (1e-15 * np.random.default_rng(trial).standard_normal(sc.shape) if trial else 0.0)
        se.sigma_calc[:] = sc * noise
        o.se_pade_fit(se, 0.01)
        eqp, _, _, _ = o.find_qp_energy_graphical(se, np.zeros(2), e[nsemin - 1:nsemax])
        outs.append((se.sigma.copy(), eqp))
    dsig = max(np.abs(outs[k][0] - outs[0][0]).max() for k in (1, 2)) / np.abs(outs[0][0]).max()
    dqp = max(np.abs(outs[k][1] - outs[0][1]).max() for k in (1, 2)) * 27.21138505
    assert 1e-8 < dsig < 2e-5
    assert dqp < 1e-7


def test_find_fixed_point_linear():
    x = np.linspace(-1, 1, 21)
    fx = 0.2 + 0.5 * x           # fixed point at x = 0.4, Z = 1/(1-0.5) = 2
    efp, zw = o.find_fixed_point(x, fx)
    assert abs(efp[0] - 0.4) < 1e-12 and abs(zw[0] - 2.0) < 1e-12 and zw[1] == -1.0


def test_aomo_oracle_against_einsum():
    rng = np.random.default_rng(3)
    nbf, naux, nstate = 9, 7, 9
    pairs = np.array([(k, l) for l in range(1, nbf + 1) for k in range(1, l + 1)])
    b = rng.standard_normal((naux, nbf, nbf))
    b = b + b.transpose(0, 2, 1)
    eri3 = np.array([[b[p, k - 1, l - 1] * (0.5 if k == l else 1.0) for (k, l) in pairs] for p in range(naux)])
    c = np.linalg.qr(rng.standard_normal((nbf, nbf)))[0].T.copy()       # [nstate][nbf]
    out = o.calculate_eri_3center_mo(eri3, pairs, c, 2, 8, 1, 4)
    ref = np.einsum("mi,nj,pij->nmp", c[1:8], c[0:4], b)
    assert np.abs(out - ref).max() < 1e-12


def test_oracle_reproduces_golden_synth(golden_synth):
    d = golden_synth
    inst = instance_from_golden(d)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    res = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                      nomega_sigma=101, step_sigma=0.025, nomega_sigma_calc=50, step_sigma_calc=0.075, eta=0.01)
    assert abs(res.erpa - float(d["erpa"])) < 1e-12
    assert np.abs(res.sigma_calc.T - d["sigma_calc"]).max() < 1e-12
    assert np.abs(res.energy_qp_g - d["energy_qp_g"]).max() < 1e-12


def test_state_range_and_transition_table():
    occ = np.array([2.0] * 5 + [0.0] * 7)
    rng = o.selfenergy_set_state_range(12, occ, selfenergy_state_range=1)
    assert (rng.nhomo_g, rng.nlumo_g, rng.nsemin, rng.nsemax) == (5, 6, 4, 6)
    tt = o.transition_table(occ, ncore_w=1)
    assert len(tt) == 4 * 7 and tuple(tt[0]) == (2, 6) and tuple(tt[1]) == (2, 7)
