"""Request loop (continuous batching): every result is the same alone and in the
mix.  FP64: energies, sigma_calc and QP energies within 1e-12 relative / 1e-6
eV (batch composition changes only which problems share a launch); split
precision: QP energies within 1e-6 eV."""
import threading

import numpy as np
import pytest

from molgw_b200 import synth
from molgw_b200.rigw import RIGW_BF16X3, RIGW_FP64, Server
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


def _mix():
    return [synth.make_instance(no, nv, na, nw, sd) for (no, nv, na, nw, sd) in
            [(4, 30, 70, 8, 61), (9, 80, 200, 16, 62), (6, 44, 100, 16, 63), (5, 41, 130, 12, 64),
             (7, 64, 256, 8, 65), (3, 29, 96, 8, 66)]]


def _close(a, b, tight=True):
    assert np.abs(a.energy_qp_g - b.energy_qp_g).max() * HA_EV < 1e-6
    if tight:
        assert abs(a.erpa - b.erpa) <= 1e-12 * max(1.0, abs(a.erpa))
        assert np.abs(a.sigma_calc - b.sigma_calc).max() <= 1e-12 * np.abs(a.sigma_calc).max()


@pytest.mark.parametrize("precision", [RIGW_FP64, RIGW_BF16X3])
def test_same_result_alone_and_in_the_mix(precision):
    insts = _mix()
    srv = Server(0, workers=2, max_batch=8)
    alone = []
    for inst in insts:
        alone.append(srv.wait(srv.submit(inst, precision)))
    tickets = [srv.submit(inst, precision) for inst in insts]     # arrive together
    mixed = [srv.wait(t) for t in tickets]
    c = srv.counters()
    srv.close()
    assert c["completed"] == 2 * len(insts)
    assert c["batches"] < 2 * len(insts)                          # the mix was batched
    for a, b in zip(alone, mixed):
        _close(a, b, tight=(precision == RIGW_FP64))


def test_concurrent_submitters_and_small_budget(engine):
    """Four host threads submit; each worker has a budget below the largest
    problem, which is then split into frequency chunks; results match the
    single-context solve."""
    insts = _mix()
    refs = [engine.g0w0(i) for i in insts]
    from molgw_b200.rigw import lib
    big = max(lib().rigw_footprint_bytes(i.naux, i.nocc, i.nvirt, i.nomega, i.nstate, 2, 0) for i in insts)
    srv = Server(0, hbm_budget_bytes=int(big * 1.2), workers=2, max_batch=4)
    outs = [None] * len(insts)

    def client(k0):
        for k in range(k0, len(insts), 4):
            outs[k] = srv.wait(srv.submit(insts[k]))

    th = [threading.Thread(target=client, args=(k,)) for k in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    srv.close()
    for r, o in zip(refs, outs):
        _close(r, o, tight=False)
        assert abs(r.erpa - o.erpa) <= 1e-12 * max(1.0, abs(r.erpa))


def test_completion_stamps_and_cancel_on_close():
    """The loop stamps submission and completion on the monotonic clock; closing
    it with requests still queued cancels them instead of running them all."""
    import time
    insts = _mix()
    srv = Server(0, workers=1, max_batch=1)
    t_before = time.monotonic_ns()
    tickets = [srv.submit(inst) for inst in insts * 4]        # 24 requests, one per batch
    while not srv.info(tickets[0])[0]:
        time.sleep(0.001)
    done, sub, fin = srv.info(tickets[0])
    assert done and t_before <= sub <= fin <= time.monotonic_ns()
    queued = srv.counters()["queued"]
    th = threading.Thread(target=srv.close)
    th.start()
    th.join(timeout=120)
    assert not th.is_alive()
    assert queued > 0
