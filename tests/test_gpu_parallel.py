"""The frequency-sharded data path on the GPU: two ranks (processes) on cuda:0,
each computing W and Sigma_c on its share of the Gauss-Legendre frequencies
through the C ABI (Engine.frequency_partials), one all-reduce of the partial
Sigma_c and energies over gloo, then the QP equation on the sum
(parallel.g0w0_frequency_sharded).  The result equals the one-GPU solve:
sigma_calc and the energies within 1e-12 relative, the QP energies within 1e-6
eV.  The ranks exchange data on the host only; none of their kernels waits on
the other rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from molgw_b200 import parallel, synth
    from molgw_b200.rigw import Engine
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    eng = Engine(0)
    try:
        inst = synth.make_instance(9, 80, 200, 16, seed=42)
        out = parallel.g0w0_frequency_sharded(eng, inst)
        q.put((rank, out.sigma_calc, out.erpa, out.egw, out.energy_qp_g))
    finally:
        eng.close()
        dist.destroy_process_group()


def test_two_ranks_frequency_sharded_equals_one_gpu(engine):
    from molgw_b200 import synth
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    inst = synth.make_instance(9, 80, 200, 16, seed=42)
    ref = engine.g0w0(inst)
    for _, sig, erpa, egw, eqp in res:
        assert np.abs(sig - ref.sigma_calc).max() < 1e-12 * np.abs(ref.sigma_calc).max()
        assert abs(erpa - ref.erpa) < 1e-12 * abs(ref.erpa)
        assert abs(egw - ref.egw) < 1e-12 * abs(ref.egw)
        assert np.abs(eqp - ref.energy_qp_g).max() * HA_EV < 1e-6
