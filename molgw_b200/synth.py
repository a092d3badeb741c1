"""Seeded synthetic RI-GW instances with the shapes and value distributions of the
benchmark workloads (no public dataset exists for this path).

One instance is a closed-shell (nspin=1) G0W0@HF problem on the imaginary axis (an
open-shell one carries its second spin channel in ``spin2``):

* occupied energies ~ U[-30, -8] eV, virtual energies ~ U[0.5, 40] eV, sorted,
  stored in Hartree (eV / 27.21138505, src/m_definitions.f90:43);
* occupation 2 for occupied states, 0 for virtual ones;
* the W-window tensor M[P, a, i] ~ N(0, s^2), where s = sqrt(0.8 / lmax) and
  lmax is the largest eigenvalue of -chi0(i0) = sum_t 4/de_t M_t M_t^T built
  with the unscaled N(0,1) draw, so that eig(eps(i0)) lies in [1, 1.8];
* the Sigma tensor M[P, p, m] for p over all states and m in {HOMO, LUMO}
  (S = 2): its occupied-virtual entries coincide with the W tensor (M is
  symmetric in its two state indices), the other entries are fresh draws from
  the same N(0, s^2);
* Sigma_x - V_xc = 0 (G0W0@HF), Sigma grid of tests/inputs/h2o_gw_pade.in:
  nomega_sigma_calc=50, step_sigma_calc=0.075, nomega_sigma=101,
  step_sigma=0.025, eta=0.01 Ha.

State indices follow MOLGW: states 1..nocc are occupied, HOMO = nocc,
LUMO = nocc+1; the Sigma range is nsemin..nsemax = HOMO..LUMO.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np

HA_EV = 27.21138505


@dataclass
class GWInstance:
    """One G0W0 problem in the library's host layout (C order, float64)."""
    nocc: int
    nvirt: int
    naux: int
    nomega: int
    energy: np.ndarray        # [nstate] Ha, sorted occupied then virtual
    occupation: np.ndarray    # [nstate]
    m_ia: np.ndarray          # [nocc, nvirt, naux]   (Fortran eri_3center_mo(P, a, i))
    m_sigma: np.ndarray       # [nsig, nstate, naux]  (Fortran eri_3center_mo(P, p, m))
    nsemin: int = 0           # 1-based Sigma state range
    nsemax: int = 0
    nomega_sigma_calc: int = 50
    step_sigma_calc: float = 0.075
    nomega_sigma: int = 101
    step_sigma: float = 0.025
    eta: float = 0.01
    seed: int = 0
    # Energies of the states in G (energy_g of selfenergy_evaluation); None: ``energy``.
    # W and the QP equation keep ``energy`` (src/m_selfenergy_evaluation.f90:164-181).
    energy_g: np.ndarray | None = None
    # Second spin channel (nspin = 2): its own window, energies, occupations (1 or 0)
    # and M tensors over the same states and auxiliary basis; None: closed shell.
    spin2: "GWInstance | None" = None
    spin_channel: bool = False        # occupations per spin channel (1 or 0), not 2 or 0
    # Frozen core (MOLGW's ncorew / ncoreg): the W window starts at state ncore_w + 1
    # (m_ia covers occupied states ncore_w+1 .. ncore_w+nocc), the states p of Sigma
    # at ncore_g + 1 (m_sigma is [nsig, nstate - ncore_g, naux]).
    ncore_w: int = 0
    ncore_g: int = 0
    # Sigma_x - V_xc of the Sigma states (setup_exchange_m_vxc diagonal, [nsig] Ha);
    # None: zero (G0W0@HF)
    exchange_m_vxc: np.ndarray | None = None

    @property
    def nstate(self) -> int:
        return self.nocc + self.nvirt

    @property
    def nsig(self) -> int:
        return self.nsemax - self.nsemin + 1


def _energies(rng: np.random.Generator, nocc: int, nvirt: int) -> np.ndarray:
    e_occ = np.sort(rng.uniform(-30.0, -8.0, nocc))
    e_virt = np.sort(rng.uniform(0.5, 40.0, nvirt))
    return np.concatenate([e_occ, e_virt]) / HA_EV


def _lambda_max(m_t: np.ndarray, de: np.ndarray) -> float:
    """Largest eigenvalue of sum_t (4/de_t) m_t m_t^T, m_t rows of ``m_t``."""
    w = np.sqrt(4.0 / de)
    a = m_t * w[:, None]                    # [Nia, naux]
    if a.shape[1] <= 2500:
        g = a.T @ a
        return float(np.linalg.eigvalsh(g)[-1])
    # large instances: power iteration on a^T a (converges to ~1e-10 quickly
    # because the top of the spectrum of a Wishart-like matrix is separated)
    v = np.ones(a.shape[1]) / np.sqrt(a.shape[1])
    lam = 0.0
    for _ in range(300):
        u = a.T @ (a @ v)
        lam_new = float(np.linalg.norm(u))
        v = u / lam_new
        if abs(lam_new - lam) < 1e-12 * lam_new:
            break
        lam = lam_new
    return lam_new


def make_instance(nocc: int, nvirt: int, naux: int, nomega: int, seed: int,
                  with_sigma: bool = True, lambda_max=None) -> GWInstance:
    """Build one seeded instance (numpy Generator(PCG64(seed))).

    ``lambda_max(m_t, de)`` may replace the host eigenvalue computation of the
    scaling (same quantity, e.g. evaluated on a GPU for large batches)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    energy = _energies(rng, nocc, nvirt)
    occupation = np.concatenate([np.full(nocc, 2.0), np.zeros(nvirt)])
    m_raw = rng.standard_normal((nocc, nvirt, naux))
    de = (energy[nocc:][None, :] - energy[:nocc][:, None]).reshape(-1)
    lmax = (lambda_max or _lambda_max)(m_raw.reshape(-1, naux), de)
    s = np.sqrt(0.8 / lmax)
    m_ia = m_raw * s
    nstate = nocc + nvirt
    homo, lumo = nocc, nocc + 1                    # 1-based
    if with_sigma:
        m_sigma = np.empty((2, nstate, naux))
        # column m = HOMO: p occupied -> fresh, p virtual -> M[P, a, HOMO]
        m_sigma[0, :nocc] = rng.standard_normal((nocc, naux)) * s
        m_sigma[0, nocc:] = m_ia[homo - 1]
        # column m = LUMO: p occupied -> M[P, LUMO, i], p virtual -> fresh
        m_sigma[1, :nocc] = m_ia[:, lumo - nocc - 1]
        m_sigma[1, nocc:] = rng.standard_normal((nvirt, naux)) * s
    else:
        m_sigma = np.zeros((0, nstate, naux))
    return GWInstance(nocc=nocc, nvirt=nvirt, naux=naux, nomega=nomega, energy=energy,
                      occupation=occupation, m_ia=m_ia, m_sigma=m_sigma,
                      nsemin=homo, nsemax=lumo, seed=seed)


def with_window(inst: GWInstance, seed: int = 0) -> tuple[GWInstance, np.ndarray]:
    """The full 3-center tensor of the window, [nstate, nstate, naux] symmetric
    in its first two indices (eri_3center_mo(:, q, r) over ncore_G+1 ..
    nvirtual_G-1), for the vertex corrections that need the occupied-occupied
    and empty-empty blocks.  The occupied-empty block is ``inst.m_ia``; the
    other blocks are seeded N(0, 1) scaled like it; ``m_ia`` and ``m_sigma`` of
    the returned instance are re-read from the tensor so that every input agrees."""
    rng = np.random.Generator(np.random.PCG64(seed))
    no, nv, naux = inst.m_ia.shape
    s = float(inst.m_ia.std())
    m = np.empty((no + nv, no + nv, naux))
    oo = rng.standard_normal((no, no, naux)) * s
    vv = rng.standard_normal((nv, nv, naux)) * s
    m[:no, :no] = 0.5 * (oo + oo.transpose(1, 0, 2))
    m[no:, no:] = 0.5 * (vv + vv.transpose(1, 0, 2))
    m[:no, no:] = inst.m_ia
    m[no:, :no] = inst.m_ia.transpose(1, 0, 2)
    sig = np.arange(inst.nsemin - 1, inst.nsemax)
    return replace(inst, m_ia=np.ascontiguousarray(m[:no, no:]), m_sigma=np.ascontiguousarray(m[sig])), m


# Workloads of the benchmark table --------------------------------------------
def single_instance_840(seed: int = 2) -> GWInstance:
    """Nocc=21, Nvirt=207, Naux=840, 32 imaginary frequencies."""
    return make_instance(21, 207, 840, 32, seed)


def large_instance_4000(seed: int = 3) -> GWInstance:
    """Nocc=100, Nvirt=1100, Naux=4000, 48 imaginary frequencies."""
    return make_instance(100, 1100, 4000, 48, seed)


def batch_sizes(count: int = 256, base_seed: int = 4):
    """Ragged molecule sizes: Nocc ~ U{5..60}, Nvirt = round(Nocc*U[8,10]),
    Naux = 4*(Nocc+Nvirt), 32 frequencies; molecule k uses seed base_seed+k."""
    out = []
    for k in range(count):
        rng = np.random.Generator(np.random.PCG64(base_seed + k))
        nocc = int(rng.integers(5, 61))
        nvirt = int(round(nocc * rng.uniform(8.0, 10.0)))
        out.append((nocc, nvirt, 4 * (nocc + nvirt), 32, base_seed + k))
    return out


def batch_instances(count: int = 256, base_seed: int = 4, lambda_max=None):
    return [make_instance(no, nv, na, nw, sd, lambda_max=lambda_max)
            for (no, nv, na, nw, sd) in batch_sizes(count, base_seed)]


def serving_sizes(rate: float = 200.0, duration: float = 60.0, seed: int = 5, large_fraction: float = 0.05):
    """Poisson arrivals and request sizes: 95% drawn like the ragged batch, 5%
    large (Nocc=150, Nvirt=1500, Naux=6000, 48 frequencies).  Returns a list of
    (arrival_time_s, (nocc, nvirt, naux, nomega, seed))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    t = 0.0
    k = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        if rng.random() < large_fraction:
            size = (150, 1500, 6000, 48, 100000 + k)
        else:
            r2 = np.random.Generator(np.random.PCG64(1000 + k))
            nocc = int(r2.integers(5, 61))
            nvirt = int(round(nocc * r2.uniform(8.0, 10.0)))
            size = (nocc, nvirt, 4 * (nocc + nvirt), 32, 1000 + k)
        out.append((t, size))
        k += 1
    return out


def make_instance_device(nocc: int, nvirt: int, naux: int, nomega: int, seed: int, device: str = "cuda"):
    """The same distributions generated directly in device memory (torch, float64,
    seeded torch.Generator), for batches too large to draw on the host.

    Returns (GWInstance with m_ia = m_sigma = None, dict of device tensors in the
    layout of ``Engine.make_problem``'s ``device_arrays``)."""
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    energy = _energies(rng, nocc, nvirt)
    occupation = np.concatenate([np.full(nocc, 2.0), np.zeros(nvirt)])
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    m = torch.randn((nocc, nvirt, naux), generator=g, dtype=torch.float64, device=device)
    de = torch.from_numpy((energy[nocc:][None, :] - energy[:nocc][:, None]).reshape(-1)).to(device)
    a = m.reshape(-1, naux) * torch.sqrt(4.0 / de)[:, None]
    lmax = float(torch.linalg.eigvalsh(a.T @ a)[-1].item())
    del a
    s = float(np.sqrt(0.8 / lmax))
    m.mul_(s)
    nstate = nocc + nvirt
    ms = torch.empty((2, nstate, naux), dtype=torch.float64, device=device)
    ms[0, :nocc] = torch.randn((nocc, naux), generator=g, dtype=torch.float64, device=device) * s
    ms[0, nocc:] = m[nocc - 1]
    ms[1, :nocc] = m[:, 0]
    ms[1, nocc:] = torch.randn((nvirt, naux), generator=g, dtype=torch.float64, device=device) * s
    inst = GWInstance(nocc=nocc, nvirt=nvirt, naux=naux, nomega=nomega, energy=energy, occupation=occupation,
                      m_ia=None, m_sigma=None, nsemin=nocc, nsemax=nocc + 1, seed=seed)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(device)
    dev = {"m_ia": m, "m_pm": ms, "e_occ": t(energy[:nocc]), "e_virt": t(energy[nocc:]),
           "occ_occ": t(occupation[:nocc]), "occ_virt": t(occupation[nocc:]), "e_p": t(energy),
           "e_sig": t(energy[nocc - 1:nocc + 1]), "occ_sig": t(occupation[nocc - 1:nocc + 1])}
    return inst, dev


def torch_lambda_max(device: str = "cuda"):
    """lambda_max hook evaluating max eig of sum_t (4/de_t) m_t m_t^T with torch
    (float64) on ``device``; used to generate large batches quickly."""
    import torch

    def f(m_t: np.ndarray, de: np.ndarray) -> float:
        a = torch.from_numpy(m_t).to(device) * torch.from_numpy(np.sqrt(4.0 / de)).to(device)[:, None]
        g = a.T @ a
        return float(torch.linalg.eigvalsh(g)[-1].item())
    return f
