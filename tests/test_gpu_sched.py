"""Memory-bounded batches: frequency chunks and waves give the same results as one
fused plan (Sigma_c and the energies are sums over frequencies; only the
summation order differs).  Tolerances: energies and sigma_calc 1e-12 relative,
QP energies 1e-6 eV."""
import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.rigw import RIGW_BF16X3, RIGW_FP64, Engine, lib
from tests.conftest import HA_EV, instance_from_golden

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert abs(a.erpa - b.erpa) <= 1e-12 * max(1.0, abs(a.erpa))
    assert abs(a.egw - b.egw) <= 1e-12 * max(1.0, abs(a.egw))
    assert np.abs(a.sigma_calc - b.sigma_calc).max() <= 1e-12 * np.abs(a.sigma_calc).max()
    assert np.abs(a.energy_qp_g - b.energy_qp_g).max() * HA_EV < 1e-6


def test_chunked_single_problem_equals_fused(engine, golden_synth):
    inst = instance_from_golden(golden_synth)
    ref = engine.g0w0(inst)
    fused = lib().rigw_footprint_bytes(inst.naux, inst.nocc, inst.nvirt, inst.nomega, inst.nstate, 2, 0)
    small = Engine(0, hbm_budget_bytes=int(fused * 0.45))
    out = small.g0w0(inst)
    st = small.last_stats()
    assert st["chunks"] >= 3 and st["waves"] >= 2
    _same(ref, out)
    small.close()


@pytest.mark.parametrize("precision", [RIGW_FP64, RIGW_BF16X3])
def test_chunked_ragged_batch_equals_single_solves(engine, precision):
    insts = [synth.make_instance(4, 30, 70, 8, seed=51), synth.make_instance(8, 70, 190, 12, seed=52),
             synth.make_instance(6, 44, 100, 16, seed=53)]
    refs = [engine.g0w0(i, precision) for i in insts]
    total = sum(lib().rigw_footprint_bytes(i.naux, i.nocc, i.nvirt, i.nomega, i.nstate, 2, precision)
                for i in insts)
    small = Engine(0, hbm_budget_bytes=int(total * 0.4))
    outs = small.g0w0_batch(insts, precision)
    assert small.last_stats()["waves"] >= 2
    for r, o in zip(refs, outs):
        if precision == RIGW_FP64:
            _same(r, o)
        else:   # chunked split precision: the same arithmetic per frequency, summed in another order
            assert np.abs(r.energy_qp_g - o.energy_qp_g).max() * HA_EV < 1e-6
    small.close()


def test_budget_too_small_is_reported(engine):
    from molgw_b200.rigw import RigwError
    tiny = Engine(0, hbm_budget_bytes=1 << 16)
    with pytest.raises(RigwError) as ei:
        tiny.g0w0(synth.make_instance(4, 30, 70, 8, seed=54))
    assert ei.value.code == 3
    tiny.close()
