"""Work distribution over ranks (one process per GPU, torch.distributed).

Two ways the imaginary-axis G0W0 path shards:

* molecules (replicas): every molecule is an independent solve, so a batch is
  split over ranks with no data-path collective (``shard_molecules``);
* frequencies of one molecule: chi0(iw), eps(iw) and the omega' term of Sigma
  are independent per frequency, as in MOLGW's "poorman" split
  (src/m_gw_selfenergy_grid.f90:626,658: a frequency belongs to rank
  MODULO(iomega-1, nproc)).  The only exchange is one sum of the partial
  Sigma_c(z_k) and of the partial E_RPA/E_GW (src/m_gw_selfenergy_grid.f90:325
  world%sum), done here with one all-reduce (``allreduce_partials``); the QP
  solve then runs on the summed Sigma.
"""
from __future__ import annotations

import numpy as np


def frequency_shard(nomega: int, rank: int, world: int) -> np.ndarray:
    """0-based frequency indices owned by ``rank`` (round robin, like the poorman split)."""
    return np.arange(nomega)[np.arange(nomega) % world == rank]


def solve_cost(nocc: int, nvirt: int, naux: int, nomega: int) -> float:
    """FLOP estimate of one solve: chi0 + Cholesky + triangular solves."""
    n = float(naux)
    return nomega * (n * n * nocc * nvirt + 2.0 * n ** 3 / 3.0)


def shard_molecules(sizes, world: int):
    """Longest-processing-time assignment of molecules to ranks.

    ``sizes`` is a list of (nocc, nvirt, naux, nomega); returns ``world`` lists of
    molecule indices with near-equal estimated cost."""
    order = sorted(range(len(sizes)), key=lambda i: -solve_cost(*sizes[i][:4]))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        out[r].append(i)
        load[r] += solve_cost(*sizes[i][:4])
    for lst in out:
        lst.sort()
    return out


def allreduce_partials(sigma_calc: np.ndarray, energies: np.ndarray, group=None):
    """Sum the per-rank partial Sigma_c (complex [nsig, nc]) and energy partials
    ([erpa, egw]) over the process group with one all-reduce."""
    import torch
    import torch.distributed as dist
    flat = np.concatenate([sigma_calc.real.ravel(), sigma_calc.imag.ravel(), energies.ravel()])
    t = torch.from_numpy(flat.copy())
    backend = dist.get_backend(group)
    if backend == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    flat = t.cpu().numpy()
    n = sigma_calc.size
    sig = flat[:n].reshape(sigma_calc.shape) + 1j * flat[n:2 * n].reshape(sigma_calc.shape)
    return sig, flat[2 * n:]


def g0w0_frequency_sharded(engine, inst, precision: int = 0, group=None):
    """One molecule's G0W0 over the ranks of ``group``: this rank's share of the
    Gauss-Legendre frequencies (``frequency_shard``) through W and Sigma_c on its
    GPU (``Engine.frequency_partials``), one all-reduce of the partial Sigma_c and
    energies, then the Pade continuation and the QP equation on the sum (every
    rank holds the same result).  The sequence of gw_selfenergy_grid under the
    poorman split (src/m_gw_selfenergy_grid.f90:626, 658, 325)."""
    import torch.distributed as dist
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    idx = frequency_shard(inst.nomega, rank, world)
    if idx.size:
        sigma, energies = engine.frequency_partials(inst, idx, precision)
    else:                               # more ranks than frequencies: this rank adds zeros
        sigma = np.zeros((inst.nsig, inst.nomega_sigma_calc), dtype=np.complex128)
        energies = np.zeros(2)
    if world > 1:
        sigma, energies = allreduce_partials(sigma, energies, group)
    out = engine.qp_solve(inst, sigma)
    out.erpa, out.egw = float(energies[0]), float(energies[1])
    return out
