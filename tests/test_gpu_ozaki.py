"""Ozaki-sliced INT8 chi0 (s signed 7-bit slices per row, exact INT32 products on
tcgen05, FP64 recombination) against the FP64 path.  The eps factorization,
Sigma and the QP solve stay FP64.

Each slice adds 7 bits, so the chi0 error falls by about 2^-7 per slice.
Tolerances, with tol(s) = c * 128^-(s-3) floored at 1e-12:
  E_RPA        |d| <= tol(s) |E_RPA|,           c = 2e-3
  sigma_calc   |d| <= tol(s) max|sigma_calc|,   c = 1e-3
  chi(iw)      |d| <= tol(s) max|chi|,          c = 1e-3
  HOMO/LUMO QP |d| <= 1 meV for every s (the accuracy bar), <= 0.01 meV from s = 5
  on the 32- and 16-frequency instances (the 8-frequency Pade fit amplifies
  1e-14 input changes to 1e-3 meV, in the oracle too).
"""
import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.rigw import RIGW_FP64, RIGW_OZAKI
from tests.conftest import HA_EV, instance_from_golden

pytestmark = pytest.mark.gpu

SLICES = [3, 4, 5, 6, 7]


def tol(s, c):
    return max(c * 128.0 ** (-(s - 3)), 1e-12)


def errors(engine, inst, ref, s):
    b = engine.g0w0(inst, RIGW_OZAKI(s))
    dqp = np.abs(ref.energy_qp_g - b.energy_qp_g).max() * HA_EV * 1e3
    de = abs(ref.erpa - b.erpa) / abs(ref.erpa)
    ds = np.abs(ref.sigma_calc - b.sigma_calc).max() / np.abs(ref.sigma_calc).max()
    return dqp, de, ds


@pytest.mark.parametrize("which", ["synth", "lih"])
def test_ozaki_golden_instances_converge_with_slices(engine, golden_synth, golden_lih, which):
    inst = instance_from_golden(golden_synth if which == "synth" else golden_lih)
    ref = engine.g0w0(inst, RIGW_FP64)
    prev = None
    for s in SLICES:
        dqp, de, ds = errors(engine, inst, ref, s)
        assert dqp <= 1.0, (s, dqp)
        if s >= 5:
            assert dqp <= 0.01, (s, dqp)
        assert de <= tol(s, 2e-3), (s, de)
        assert ds <= tol(s, 1e-3), (s, ds)
        if prev is not None and prev > 1e-11:
            assert ds < 0.1 * prev, (s, ds, prev)    # each slice buys ~7 bits
        prev = ds


def test_ozaki_single_instance_840(engine):
    inst = synth.single_instance_840()
    ref = engine.g0w0(inst, RIGW_FP64)
    for s in (3, 5, 7):
        dqp, de, ds = errors(engine, inst, ref, s)
        assert dqp <= (1.0 if s < 5 else 0.01), (s, dqp)
        assert de <= tol(s, 2e-3) and ds <= tol(s, 1e-3), (s, de, ds)
        if s == 3:
            assert dqp > 0.0    # a different arithmetic, not a copy of the FP64 path


def test_ozaki_chi_matches_fp64(engine, golden_synth):
    inst = instance_from_golden(golden_synth)
    _, _, w64 = engine.polarizability_grid_scalapack(inst, RIGW_FP64)
    c64 = w64.chi()
    for s in SLICES:
        _, _, wz = engine.polarizability_grid_scalapack(inst, RIGW_OZAKI(s))
        assert np.abs(c64 - wz.chi()).max() <= tol(s, 1e-3) * np.abs(c64).max(), s
        wz.release()
    w64.release()


def test_ozaki_bitwise_repeatable(engine, golden_synth):
    inst = instance_from_golden(golden_synth)
    a = engine.g0w0(inst, RIGW_OZAKI(4))
    b = engine.g0w0(inst, RIGW_OZAKI(4))
    assert a.erpa == b.erpa and np.array_equal(a.sigma_calc, b.sigma_calc)


def test_ozaki_ragged_batch_and_mixed_precisions(engine):
    insts = [synth.make_instance(4, 30, 70, 8, seed=41), synth.make_instance(9, 80, 200, 16, seed=42),
             synth.make_instance(6, 50, 130, 12, seed=43)]
    refs = [engine.g0w0(i, RIGW_FP64) for i in insts]
    outs = engine.g0w0_batch(insts, RIGW_OZAKI(3))
    for r, o in zip(refs, outs):
        assert np.abs(o.energy_qp_g - r.energy_qp_g).max() * HA_EV * 1e3 <= 1.0
    # one batch whose problems use different slice counts
    alone = [engine.g0w0(i, RIGW_OZAKI(s)) for i, s in zip(insts, (3, 5, 7))]
    mixed = engine.g0w0_batch(insts, [RIGW_OZAKI(s) for s in (3, 5, 7)])
    for a, m in zip(alone, mixed):
        assert a.erpa == m.erpa and np.array_equal(a.sigma_calc, m.sigma_calc)


def test_ozaki_rejects_bad_slice_counts():
    with pytest.raises(ValueError):
        RIGW_OZAKI(2)
    with pytest.raises(ValueError):
        RIGW_OZAKI(8)


@pytest.mark.parametrize("nbf,naux,ranges", [(37, 61, [(6, 37, 1, 5), (3, 3, 2, 9)]),
                                              (300, 700, [(41, 300, 1, 40), (1, 300, 39, 42)])])
def test_ozaki_aomo_matches_fp64(engine, nbf, naux, ranges):
    """AO->MO with both products Ozaki-sliced (rows of each operand scaled to their
    own maximum, s int8 digits, exact INT32 products, FP64 recombination).  The
    truncation error of one product is about sqrt(nbf) 2^-7s of its largest entry;
    the bound allows 64 times that, floored at 1e-13, and the error must fall with s."""
    rng = np.random.default_rng(nbf + 1)
    pairs = np.array([(k, l) for l in range(1, nbf + 1) for k in range(1, l + 1)])
    pairs = pairs[rng.random(len(pairs)) > 0.1]
    eri3 = rng.standard_normal((naux, len(pairs)))
    c = np.linalg.qr(rng.standard_normal((nbf, nbf)))[0].T.copy()
    for (m0, m1, n0, n1) in ranges:
        f64 = engine.calculate_eri_3center_mo(eri3, pairs, c, m0, m1, n0, n1)
        scale = np.abs(f64).max()
        errs = []
        for s in (3, 5, 7):
            oz = engine.calculate_eri_3center_mo(eri3, pairs, c, m0, m1, n0, n1, precision=RIGW_OZAKI(s))
            err = np.abs(oz - f64).max() / scale
            assert err <= max(64.0 * np.sqrt(nbf) * 2.0 ** (-7 * s), 1e-13), (s, err)
            errs.append(err)
        assert 0.0 < errs[0] and errs[1] < errs[0] and errs[2] <= errs[1]
