"""Split-precision chi0 (bf16 hi/lo products on tcgen05, fp32 accumulation) against
the FP64 path and the oracle.  The eps factorization, Sigma and the QP solve stay
FP64.  Tolerances:
  HOMO/LUMO QP energies   |d| <= 1 meV against FP64 (the stated accuracy bar)
  E_RPA                   |d| <= 1e-4 * |E_RPA|
  chi(iw)                 |d| <= 1e-4 * max|chi|
"""
import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.rigw import RIGW_BF16X3, RIGW_FP64
from tests.conftest import HA_EV, instance_from_golden

pytestmark = pytest.mark.gpu


def compare(engine, inst):
    a = engine.g0w0(inst, RIGW_FP64)
    b = engine.g0w0(inst, RIGW_BF16X3)
    dqp = np.abs(a.energy_qp_g - b.energy_qp_g).max() * HA_EV * 1e3
    assert dqp <= 1.0, dqp
    assert abs(a.erpa - b.erpa) <= 1e-4 * abs(a.erpa)
    return dqp


def test_split_precision_synthetic_small(engine, golden_synth):
    compare(engine, instance_from_golden(golden_synth))


def test_split_precision_lih_cc4s(engine, golden_lih):
    compare(engine, instance_from_golden(golden_lih))


def test_split_precision_single_instance_840(engine):
    dqp = compare(engine, synth.single_instance_840())
    assert dqp > 0.0      # the split path is a different arithmetic, not a copy of the FP64 one


def test_split_precision_chi_matches_fp64(engine, golden_synth):
    inst = instance_from_golden(golden_synth)
    _, _, w64 = engine.polarizability_grid_scalapack(inst, RIGW_FP64)
    _, _, w16 = engine.polarizability_grid_scalapack(inst, RIGW_BF16X3)
    c64, c16 = w64.chi(), w16.chi()
    assert np.abs(c64 - c16).max() <= 1e-4 * np.abs(c64).max()
    w64.release()
    w16.release()


def test_split_precision_ragged_batch(engine):
    insts = [synth.make_instance(4, 30, 70, 8, seed=41), synth.make_instance(9, 80, 200, 16, seed=42),
             synth.make_instance(6, 50, 130, 12, seed=43)]
    outs = engine.g0w0_batch(insts, RIGW_BF16X3)
    for inst, o in zip(insts, outs):
        ref = engine.g0w0(inst, RIGW_FP64)
        assert np.abs(o.energy_qp_g - ref.energy_qp_g).max() * HA_EV * 1e3 <= 1.0


@pytest.mark.parametrize("nbf,naux,ranges", [(37, 61, [(6, 37, 1, 5), (3, 3, 2, 9)]),
                                              (300, 700, [(41, 300, 1, 40), (1, 300, 39, 42)])])
def test_split_precision_aomo_matches_fp64(engine, nbf, naux, ranges):
    """AO->MO with both products split (bf16 hi/lo on tcgen05, FP64 results):
    within 2e-5 of the largest entry of the FP64 transform, and not identical to it."""
    from oracle import rigw_oracle as o
    rng = np.random.default_rng(nbf)
    pairs = np.array([(k, l) for l in range(1, nbf + 1) for k in range(1, l + 1)])
    pairs = pairs[rng.random(len(pairs)) > 0.1]
    eri3 = rng.standard_normal((naux, len(pairs)))
    c = np.linalg.qr(rng.standard_normal((nbf, nbf)))[0].T.copy()
    for (m0, m1, n0, n1) in ranges:
        f64 = engine.calculate_eri_3center_mo(eri3, pairs, c, m0, m1, n0, n1)
        spl = engine.calculate_eri_3center_mo(eri3, pairs, c, m0, m1, n0, n1, precision=RIGW_BF16X3)
        err = np.abs(spl - f64).max() / np.abs(f64).max()
        assert 0.0 < err <= 2e-5, err
        if nbf < 100:
            ref = o.calculate_eri_3center_mo(eri3, pairs, c, m0, m1, n0, n1)
            assert np.abs(spl - ref).max() <= 2e-5 * np.abs(ref).max()
