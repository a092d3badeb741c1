"""Autotuner: candidates are timed on the caller's batch, the chosen launch
shapes are kept for later batches of the same precision class, and results do
not change beyond summation order.  Tolerances: E_RPA 1e-12 relative,
sigma_calc 1e-11 relative, QP energies 1e-8 eV (FP64); QP energies 1e-6 eV
(split precision)."""
import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.rigw import RIGW_BF16X3, RIGW_FP64, RIGW_OZAKI, Engine
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


def _batch():
    return [synth.make_instance(no, nv, na, nw, sd) for (no, nv, na, nw, sd) in
            [(4, 30, 70, 8, 71), (9, 80, 200, 16, 72), (6, 44, 300, 16, 73)]]


@pytest.mark.parametrize("precision", [RIGW_FP64, RIGW_BF16X3, RIGW_OZAKI(4)])
def test_autotune_keeps_results_and_reports_candidates(precision):
    eng = Engine(0)
    insts = _batch()
    before = eng.g0w0_batch(insts, precision)
    rep = eng.autotune(insts, precision)
    after = eng.g0w0_batch(insts, precision)
    eng.close()
    assert rep["chi0_rows"] in (64, 128) and rep["update_rows"] in (64, 128)
    # split classes also time an L2-resident frequency group and a group of 8
    assert rep["chains"] in (0, 1, 2, 4, 8)
    assert rep["split_group"] == 0 if precision == RIGW_FP64 else rep["split_group"] >= 0
    assert rep["precision_class"] == (0 if precision == RIGW_FP64 else (1 if precision == RIGW_BF16X3 else 2))
    assert len(rep["candidates"]) >= 3
    assert all(c["total_ms"] > 0 for c in rep["candidates"])
    chosen = [c for c in rep["candidates"]
              if (c["chi0_rows"], c["update_rows"], c["split_group"], c["chains"]) ==
              (rep["chi0_rows"], rep["update_rows"], rep["split_group"], rep["chains"])]
    assert chosen, "the chosen shapes are one of the timed candidates"
    for a, b in zip(before, after):
        assert np.abs(a.energy_qp_g - b.energy_qp_g).max() * HA_EV <= (1e-8 if precision == RIGW_FP64 else 1e-6)
        if precision == RIGW_FP64:
            assert abs(a.erpa - b.erpa) <= 1e-12 * abs(a.erpa)
            assert np.abs(a.sigma_calc - b.sigma_calc).max() <= 1e-11 * np.abs(a.sigma_calc).max()


def test_tuning_applies_to_other_batches_of_the_class():
    eng = Engine(0)
    sample = _batch()[:2]
    rep = eng.autotune(sample, RIGW_FP64)
    other = [synth.make_instance(5, 41, 130, 12, 74)]
    ref = Engine(0)
    a = eng.g0w0_batch(other, RIGW_FP64)[0]
    b = ref.g0w0_batch(other, RIGW_FP64)[0]
    eng.close()
    ref.close()
    assert rep["tuned_ms"] > 0
    assert abs(a.erpa - b.erpa) <= 1e-12 * abs(a.erpa)
    assert np.abs(a.energy_qp_g - b.energy_qp_g).max() * HA_EV <= 1e-8
