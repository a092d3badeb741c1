"""G0W0 by contour deformation on the CUDA path (rigw_gw_selfenergy_contour):
chi0 at imaginary and real frequencies on the DMMA engine, the low-rank W from
a Jacobi eigensolver on the device, Sigma_c on the real grid (imaginary-axis
integral + residues) and the QP equation.

* H2O, HF in cc-pVTZ with the Auto auxiliary basis, frozencore='molgw', 16
  imaginary and 6 real frequencies (tests/inputs/h2o_gw_contour.in): the HOMO
  and LUMO QP energies within the suite's 1e-4 eV of its known answers
  (tests/inputs/testsuite:777-780), Sigma_c within 1e-9 (relative to its
  largest entry) and the QP energies within 1e-6 eV of the oracle, the same
  eigenpairs kept at every frequency.
* Seeded synthetic instances against the oracle: auxiliary sizes 70, 61 and
  300 (the device pads to a multiple of 64: 2 and 5 block pairs per round of
  the eigensolver), frozen core in W and G, energy_g != energy (se%energy0 and
  the poles from energy_g, the QP equation from energy).
* Device-pointer mode equals host mode bitwise.

Sigma_c on the real grid needs no continuation, so the QP energies are well
conditioned and held to 1e-6 eV."""
import numpy as np
import pytest

from oracle import rigw_oracle as o
from tests import h2o_case
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


def _synthetic(nocc, nvirt, naux, seed):
    """Energies, occupations and a symmetric M[p, q, P] with max eig(-chi0(0)) = 0.8."""
    rng = np.random.default_rng(seed)
    e = np.concatenate([np.sort(rng.uniform(-1.2, -0.3, nocc)), np.sort(rng.uniform(0.05, 1.8, nvirt))])
    occ = np.concatenate([np.full(nocc, 2.0), np.zeros(nvirt)])
    n = nocc + nvirt
    m = rng.standard_normal((n, n, naux))
    m = 0.5 * (m + m.transpose(1, 0, 2))
    de = (e[nocc:][None, :] - e[:nocc, None]).reshape(-1)
    mt = m[:nocc, nocc:].reshape(-1, naux)
    chi0 = (mt * (4.0 / de)[:, None]).T @ mt
    m *= np.sqrt(0.8 / np.linalg.eigvalsh(chi0).max())
    return e, occ, m


def _both(engine, e, occ, m, ncore, nsemin, nsemax, nimag, nreal, nomega_sigma, step, eta, energy_g=None):
    nocc = int(np.sum(occ > 0))
    m_ia = np.ascontiguousarray(m[ncore:nocc, nocc:])
    m_sig = np.ascontiguousarray(m[nsemin - 1:nsemax, ncore:])
    rng = o.selfenergy_set_state_range(e.size, occ, ncoreg=ncore, selfenergy_state_min=nsemin,
                                       selfenergy_state_max=nsemax)
    assert (rng.nsemin, rng.nsemax) == (nsemin, nsemax)
    ref = o.g0w0_contour(e, occ, m_ia, m_sig, rng, ncore, nimag, nreal, nomega_sigma=nomega_sigma, step_sigma=step,
                         eta=eta, energy_g=energy_g)
    out = engine.g0w0_contour(e, occ, m_ia, m_sig, nsemin, nsemax, nimag, nreal, nomega_sigma, step, eta,
                              ncore_w=ncore, ncore_g=ncore, energy_g=energy_g)
    return ref, out, m_ia, m_sig


def _assert_close(ref, out):
    assert abs(out.de_max - ref.de_max) <= 1e-14 * max(1.0, abs(ref.de_max))
    assert np.allclose(out.omega_real, ref.omega_real, rtol=0, atol=1e-15)
    assert list(out.rank) == list(ref.nrank_imag) + list(ref.nrank_real)
    assert np.abs(out.sigma - ref.sigma).max() < 1e-9 * np.abs(ref.sigma).max()
    assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV < 1e-6
    assert np.abs(out.energy_qp_z - ref.energy_qp_z).max() * HA_EV < 1e-6


def test_h2o_contour_reproduces_the_known_answers(engine):
    d = h2o_case.load()
    case = d["cases"]["h2o_gw_contour.in"]
    scf, m, rng, ncore, m_ia, m_sig, st = h2o_case.contour_inputs(case, d["basis"])
    out = engine.g0w0_contour(scf.e_orb, scf.occupation, m_ia, m_sig, rng.nsemin, rng.nsemax, st["nomega_chi_imag"],
                              st["nomega_chi_real"], st["nomega_sigma"], st["step_sigma"], st["eta"],
                              ncore_w=ncore, ncore_g=ncore)
    for label, value in (("GW HOMO energy", out.ehomo), ("GW LUMO energy", out.elumo)):
        ref, tol = case["known_answers"][label]
        assert abs(value * HA_EV - ref) < tol, (label, value * HA_EV, ref)
    ref = o.g0w0_contour(scf.e_orb, scf.occupation, m_ia, m_sig, rng, ncore, st["nomega_chi_imag"],
                         st["nomega_chi_real"], nomega_sigma=st["nomega_sigma"], step_sigma=st["step_sigma"],
                         eta=st["eta"])
    _assert_close(ref, out)
    assert np.abs(out.sigma - h2o_case.load()["contour_sigma"]).max() < 1e-9 * np.abs(ref.sigma).max()


@pytest.mark.parametrize("naux", [70, 61, 300])
def test_synthetic_matches_the_oracle(engine, naux):
    e, occ, m = _synthetic(6, 40, naux, seed=naux)
    ref, out, _, _ = _both(engine, e, occ, m, ncore=1, nsemin=5, nsemax=8, nimag=12, nreal=8, nomega_sigma=21,
                           step=0.02, eta=0.001)
    _assert_close(ref, out)


def test_energy_g_splits_the_grid_from_the_qp_equation(engine):
    e, occ, m = _synthetic(5, 30, 48, seed=5)
    eg = e.copy()
    eg[5:] += 0.02          # e.g. QP energies read back under force_energy_qp
    ref, out, _, _ = _both(engine, e, occ, m, ncore=0, nsemin=4, nsemax=7, nimag=10, nreal=6, nomega_sigma=15,
                           step=0.03, eta=0.001, energy_g=eg)
    _assert_close(ref, out)
    plain = engine.g0w0_contour(e, occ, np.ascontiguousarray(m[:5, 5:]), np.ascontiguousarray(m[3:7]), 4, 7, 10, 6,
                                15, 0.03, 0.001)
    assert np.abs(plain.energy_qp_g - out.energy_qp_g).max() > 1e-4


def test_device_pointers_equal_host_mode(engine):
    import torch
    e, occ, m = _synthetic(6, 40, 70, seed=11)
    m_ia = np.ascontiguousarray(m[1:6, 6:])
    m_sig = np.ascontiguousarray(m[4:8, 1:])
    host = engine.g0w0_contour(e, occ, m_ia, m_sig, 5, 8, 12, 8, 21, 0.02, 0.001, ncore_w=1, ncore_g=1)
    dev = engine.g0w0_contour(e, occ, torch.from_numpy(m_ia).cuda(), torch.from_numpy(m_sig).cuda(), 5, 8, 12, 8, 21,
                              0.02, 0.001, ncore_w=1, ncore_g=1)
    assert np.array_equal(host.sigma, dev.sigma)
    assert np.array_equal(host.energy_qp_g, dev.energy_qp_g)
