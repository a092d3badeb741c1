"""Parity of the CUDA path (through the C ABI) with the oracle and the golden
fixtures.  Tolerances (FP64 path):
  E_RPA, E_GW           |d| < 1e-10 * max(1, |E|) Ha
  sigma_calc            |d| < 1e-9 * max|Sigma|
  Sigma on real grid    |d| < 2e-5 * max|Sigma|   (the 99-point Thiele recursion amplifies
                                                   1e-15 input differences to ~5e-6 in the
                                                   oracle itself: tests/test_oracle.py)
  QP energies           |d| < 1e-6 eV
"""
import numpy as np
import pytest

from molgw_b200 import synth
from oracle import rigw_oracle as o
from tests.conftest import HA_EV, instance_from_golden

pytestmark = pytest.mark.gpu

SIGMA_GRID = dict(nomega_sigma=101, step_sigma=0.025, nomega_sigma_calc=50, step_sigma_calc=0.075, eta=0.01)


def assert_matches(out, ref, qp_tol_ev=1e-6):
    assert abs(out.erpa - float(ref["erpa"])) < 1e-10 * max(1.0, abs(float(ref["erpa"])))
    assert abs(out.egw - float(ref["egw"])) < 1e-10 * max(1.0, abs(float(ref["egw"])))
    sc = np.asarray(ref["sigma_calc"])
    assert np.abs(out.sigma_calc - sc).max() < 1e-9 * np.abs(sc).max()
    sg = np.asarray(ref["sigma"])
    assert np.abs(out.sigma - sg).max() < 2e-5 * np.abs(sg).max()
    assert np.abs(out.energy_qp_g - ref["energy_qp_g"]).max() * HA_EV < qp_tol_ev
    assert np.abs(out.energy_qp_z - ref["energy_qp_z"]).max() * HA_EV < qp_tol_ev
    assert np.abs(out.zz - ref["zz"]).max() < 1e-6
    assert abs(out.ehomo - float(ref["ehomo"])) * HA_EV < qp_tol_ev
    assert abs(out.elumo - float(ref["elumo"])) * HA_EV < qp_tol_ev


def oracle_outputs(inst):
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    res = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng, **SIGMA_GRID)
    return dict(erpa=res.erpa, egw=res.egw, sigma_calc=res.sigma_calc.T, sigma=res.sigma.T,
                energy_qp_g=res.energy_qp_g, energy_qp_z=res.energy_qp_z, zz=res.zz, ehomo=res.ehomo,
                elumo=res.elumo)


def test_g0w0_synthetic_matches_golden(engine, golden_synth):
    out = engine.g0w0(instance_from_golden(golden_synth))
    assert_matches(out, golden_synth)


def test_g0w0_lih_cc4s_matches_golden(engine, golden_lih):
    out = engine.g0w0(instance_from_golden(golden_lih))
    assert_matches(out, golden_lih)
    # the imaginary-axis RPA of the real LiH tensor is the reference's analytic value
    assert abs(out.erpa - float(golden_lih["ref_rpa_analytic"])) < 1e-7


def test_dropin_call_sequence_matches_golden(engine, golden_synth):
    """polarizability_grid -> wpol%chi -> gw_selfenergy_imag -> pade + QP, as
    selfenergy_evaluation calls them."""
    inst = instance_from_golden(golden_synth)
    erpa, egw, wpol = engine.polarizability_grid_scalapack(inst)
    assert abs(erpa - float(golden_synth["erpa"])) < 1e-10
    assert abs(egw - float(golden_synth["egw"])) < 1e-10
    chi = wpol.chi()
    ref = golden_synth["chi_first"]
    assert np.abs(chi[0] - ref).max() < 1e-11 * max(1.0, np.abs(ref).max())
    sc = engine.gw_selfenergy_imag_scalapack(wpol, inst)
    ref_sc = golden_synth["sigma_calc"]
    assert np.abs(sc - ref_sc).max() < 1e-9 * np.abs(ref_sc).max()
    qp = engine.qp_solve(inst, sc)
    assert np.abs(qp.energy_qp_g - golden_synth["energy_qp_g"]).max() * HA_EV < 1e-6
    wpol.release()


def test_qp_solve_polynomial_technique(engine, golden_synth):
    """imaginary_axis_homolumo: quadratic fit on real points inside the gap."""
    inst = instance_from_golden(golden_synth)
    nc = 21
    eh, el = inst.energy[inst.nsemin - 1], inst.energy[inst.nsemin]
    zc = (eh + 0.01 + np.arange(nc) / (nc - 1.0) * (el - eh - 0.02)).astype(np.complex128)
    rng = np.random.default_rng(5)
    sc = (rng.standard_normal((inst.nsig, nc)) * 0.01).astype(np.complex128)
    inst.nomega_sigma_calc = nc
    out = engine.qp_solve(inst, sc, technique=1, omega_calc=zc)
    se = o.SelfEnergyGrid(omega=0.5 * (eh + el) + 0.025 * np.arange(-50, 51), omega_calc=zc,
                          energy0=np.zeros(inst.nsig), sigma=np.zeros((101, inst.nsig), complex),
                          sigma_calc=sc.T.copy())
    o.self_energy_polynomial(se)
    assert np.abs(out.sigma - se.sigma.T).max() < 1e-12
    eqp, zz, _, _ = o.find_qp_energy_graphical(se, np.zeros(inst.nsig), inst.energy[inst.nsemin - 1:inst.nsemax])
    assert np.abs(out.energy_qp_g - eqp).max() * HA_EV < 1e-9


@pytest.mark.parametrize("nocc,nvirt,naux,nomega", [(5, 37, 85, 8), (3, 29, 129, 6), (7, 64, 256, 4)])
def test_edge_shapes_match_oracle(engine, nocc, nvirt, naux, nomega):
    """Odd auxiliary count, one past a 128-panel, exactly two panels.  With so few
    frequencies the reference's 99-point Thiele continuation is ill-conditioned
    (in the oracle itself 1e-15 noise on sigma_calc moves the real-axis Sigma by
    O(1) and the QP energies by up to tens of meV), so these shapes check the
    well-conditioned outputs of the kernels: energies and sigma_calc."""
    inst = synth.make_instance(nocc, nvirt, naux, nomega, seed=naux)
    out, ref = engine.g0w0(inst), oracle_outputs(inst)
    assert abs(out.erpa - ref["erpa"]) < 1e-10 * max(1.0, abs(ref["erpa"]))
    assert abs(out.egw - ref["egw"]) < 1e-10 * max(1.0, abs(ref["egw"]))
    assert np.abs(out.sigma_calc - ref["sigma_calc"]).max() < 1e-9 * np.abs(ref["sigma_calc"]).max()


def test_ragged_batch_equals_single_solves(engine):
    insts = [synth.make_instance(4, 30, 70, 8, seed=21), synth.make_instance(7, 60, 150, 12, seed=22),
             synth.make_instance(5, 41, 130, 16, seed=23)]
    batch = engine.g0w0_batch(insts)
    for inst, b in zip(insts, batch):
        s = engine.g0w0(inst)
        assert abs(b.erpa - s.erpa) < 1e-13
        assert np.abs(b.sigma_calc - s.sigma_calc).max() < 1e-13
        assert np.abs(b.energy_qp_g - s.energy_qp_g).max() < 1e-13


def test_qp_only_mode_gives_the_same_qp_energies(engine, golden_synth):
    """RIGW_PROBLEM_QP_ONLY skips the tr eps^-1 solve (E_GW); every other output is unchanged."""
    inst = instance_from_golden(golden_synth)
    full = engine.g0w0(inst)
    lean = engine.g0w0(inst, qp_only=True)
    assert np.isnan(lean.egw) and lean.erpa == full.erpa
    assert np.array_equal(lean.sigma_calc, full.sigma_calc)
    assert np.array_equal(lean.energy_qp_g, full.energy_qp_g)


def test_repeat_runs_are_bitwise_identical(engine, golden_synth):
    inst = instance_from_golden(golden_synth)
    a = engine.g0w0(inst)
    b = engine.g0w0(inst)
    assert a.erpa == b.erpa and a.egw == b.egw
    assert np.array_equal(a.sigma_calc, b.sigma_calc)
    assert np.array_equal(a.energy_qp_g, b.energy_qp_g)


def test_device_resident_inputs(engine, golden_synth):
    import torch
    inst = instance_from_golden(golden_synth)
    host = engine.g0w0(inst)
    nocc = inst.nocc
    e = inst.energy
    occ = inst.occupation
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in {
        "m_ia": inst.m_ia, "e_occ": e[:nocc], "e_virt": e[nocc:], "occ_occ": occ[:nocc],
        "occ_virt": occ[nocc:], "m_pm": inst.m_sigma, "e_p": e, "e_sig": e[inst.nsemin - 1:inst.nsemax],
        "occ_sig": occ[inst.nsemin - 1:inst.nsemax]}.items()}
    out = engine.g0w0(inst, device_arrays=dev)
    assert out.erpa == host.erpa
    assert np.array_equal(out.energy_qp_g, host.energy_qp_g)


def test_indefinite_eps_is_reported(engine):
    """A host-built input whose eps(iw) is indefinite (inverted occupations make
    chi0 positive) must come back as RIGW_ERR_NOT_SPD, not as a fault."""
    from molgw_b200.rigw import RigwError
    inst = synth.make_instance(4, 30, 64, 4, seed=31)
    inst.m_ia = inst.m_ia * 30.0
    inst.occupation = np.concatenate([np.zeros(4), np.full(30, 2.0)])
    with pytest.raises(RigwError) as ei:
        engine.g0w0(inst)
    assert ei.value.code == 4
    # the context stays usable
    out = engine.g0w0(synth.make_instance(4, 30, 64, 4, seed=32))
    assert np.isfinite(out.erpa)


def test_single_instance_840_matches_oracle(engine):
    """The 21/207/840/32 workload at full size against the oracle."""
    inst = synth.single_instance_840()
    out = engine.g0w0(inst)
    ref = oracle_outputs(inst)
    assert_matches(out, ref)


def test_aomo_matches_oracle(engine):
    rng = np.random.default_rng(7)
    nbf, naux = 37, 61
    pairs = np.array([(k, l) for l in range(1, nbf + 1) for k in range(1, l + 1)])
    keep = rng.random(len(pairs)) > 0.1                    # screened pairs are absent
    pairs = pairs[keep]
    eri3 = rng.standard_normal((naux, len(pairs)))
    c = np.linalg.qr(rng.standard_normal((nbf, nbf)))[0].T.copy()
    for (m0, m1, n0, n1) in [(6, 37, 1, 5), (1, 37, 4, 5), (3, 3, 2, 9)]:
        out = engine.calculate_eri_3center_mo(eri3, pairs, c, m0, m1, n0, n1)
        ref = o.calculate_eri_3center_mo(eri3, pairs, c, m0, m1, n0, n1)
        assert np.abs(out - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("nocc,nvirt,naux,nomega", [(1, 3, 1, 1), (1, 1, 7, 2), (2, 5, 130, 1), (3, 40, 64, 3)])
def test_tiny_shapes_all_precisions(engine, nocc, nvirt, naux, nomega):
    """One transition, one auxiliary function, one frequency: everything is padded
    (64- or 128-wide transition tiles, 128-wide auxiliary panels).  FP64 against
    the oracle; the tensor-core chi0 paths against FP64."""
    from molgw_b200.rigw import RIGW_BF16X3, RIGW_OZAKI
    inst = synth.make_instance(nocc, nvirt, naux, nomega, seed=100 + naux)
    out, ref = engine.g0w0(inst), oracle_outputs(inst)
    assert abs(out.erpa - ref["erpa"]) < 1e-10 * max(1.0, abs(ref["erpa"]))
    assert np.abs(out.sigma_calc - ref["sigma_calc"]).max() < 1e-9 * np.abs(ref["sigma_calc"]).max()
    for prec in (RIGW_BF16X3, RIGW_OZAKI(4)):
        sp = engine.g0w0(inst, prec)
        assert abs(sp.erpa - out.erpa) <= 1e-4 * max(1e-12, abs(out.erpa)) + 1e-14
        assert np.abs(sp.sigma_calc - out.sigma_calc).max() <= 1e-4 * np.abs(out.sigma_calc).max()
