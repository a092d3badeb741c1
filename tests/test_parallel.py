"""Multi-rank host logic on CPU (gloo, world size 2): frequency sharding of one
molecule with one all-reduce of the partial Sigma_c and energies, and the
molecule sharding of a ragged batch."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from molgw_b200 import parallel, synth
from oracle import rigw_oracle as o


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _partial(inst, idx):
    """Oracle partial Sigma and energies over the frequencies ``idx``."""
    om, wt = o.imaginary_quad_grid(inst.nomega)
    nocc = inst.nocc
    e, occ = inst.energy, inst.occupation
    sf = o.polarizability_grid(inst.m_ia, e[:nocc], e[nocc:], occ[:nocc], occ[nocc:], om[idx], wt[idx])
    rng = o.selfenergy_set_state_range(inst.nstate, occ, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    se = o.se_init_imaginary_axis(e, rng, "pade", 101, 0.025, 20, 0.075)
    sig = o.gw_selfenergy_imag(e, inst.m_sigma, sf, se.omega_calc, 1)
    return sig.T.copy(), np.array([sf.erpa, sf.egw])


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        inst = synth.make_instance(4, 24, 40, 8, seed=99)
        idx = parallel.frequency_shard(inst.nomega, rank, world)
        sig, en = _partial(inst, idx)
        sig_sum, en_sum = parallel.allreduce_partials(sig, en)
        q.put((rank, sig_sum, en_sum))
    finally:
        dist.destroy_process_group()


def test_frequency_sharding_allreduce_equals_full_sum():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    inst = synth.make_instance(4, 24, 40, 8, seed=99)
    full_sig, full_en = _partial(inst, np.arange(inst.nomega))
    for _, sig, en in res:
        assert np.abs(sig - full_sig).max() < 1e-13 * np.abs(full_sig).max()
        assert np.abs(en - full_en).max() < 1e-12


def test_frequency_shard_partitions_like_poorman():
    parts = [parallel.frequency_shard(32, r, 3) for r in range(3)]
    allidx = np.sort(np.concatenate(parts))
    assert np.array_equal(allidx, np.arange(32))
    assert list(parts[1][:3]) == [1, 4, 7]


def test_shard_molecules_balances_a_ragged_batch():
    sizes = [s[:4] for s in synth.batch_sizes(64)]
    shards = parallel.shard_molecules(sizes, 4)
    assert sorted(i for s in shards for i in s) == list(range(64))
    loads = [sum(parallel.solve_cost(*sizes[i]) for i in s) for s in shards]
    assert max(loads) / min(loads) < 1.1


class _OracleEngine:
    """Stand-in for the library context on CPU: the oracle's partial W / Sigma_c
    and its Pade + QP, so that the host logic of the sharded path runs on gloo."""

    def frequency_partials(self, inst, idx, precision=0):
        return _partial(inst, np.asarray(idx))

    def qp_solve(self, inst, sigma):
        from types import SimpleNamespace
        rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                           selfenergy_state_max=inst.nsemax)
        se = o.se_init_imaginary_axis(inst.energy, rng, "pade", 101, 0.025, 20, 0.075)
        se.sigma_calc[:] = sigma.T
        o.se_pade_fit(se, 0.01)
        eqp, _, _, _ = o.find_qp_energy_graphical(se, np.zeros(inst.nsig), inst.energy[inst.nsemin - 1:inst.nsemax])
        return SimpleNamespace(sigma_calc=sigma, energy_qp_g=eqp, erpa=None, egw=None)


def _sharded_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        inst = synth.make_instance(4, 24, 40, 3, seed=98)   # 3 frequencies over 4 ranks: one rank has none
        inst.nomega_sigma_calc = 20
        out = parallel.g0w0_frequency_sharded(_OracleEngine(), inst)
        q.put((rank, out.sigma_calc, out.erpa, out.egw, out.energy_qp_g))
    finally:
        dist.destroy_process_group()


def test_sharded_g0w0_host_logic_on_four_ranks():
    """parallel.g0w0_frequency_sharded on 4 gloo ranks for 3 frequencies (one rank
    owns none and contributes zeros): every rank ends with the full Sigma_c, the
    full energies and the QP energies of the one-rank solve."""
    world = 4
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_sharded_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    inst = synth.make_instance(4, 24, 40, 3, seed=98)
    inst.nomega_sigma_calc = 20
    full_sig, full_en = _partial(inst, np.arange(inst.nomega))
    ref = _OracleEngine().qp_solve(inst, full_sig)
    for _, sig, erpa, egw, eqp in res:
        assert np.abs(sig - full_sig).max() < 1e-13 * np.abs(full_sig).max()
        assert abs(erpa - full_en[0]) < 1e-12 and abs(egw - full_en[1]) < 1e-12
        assert np.abs(eqp - ref.energy_qp_g).max() * 27.21138505 < 1e-6   # eV; three frequencies: Pade amplifies 1e-13 noise
