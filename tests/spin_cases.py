"""Synthetic open-shell (nspin = 2) instances for the spin tests: two channels over
the same 35 states and 70 auxiliary functions, occupations 1 or 0 per channel."""
from dataclasses import replace

import numpy as np

from molgw_b200 import synth


def open_shell_instance(nomega: int = 16):
    """Channel 1: 5 occupied; channel 2: 4 occupied, energies of channel 1 moved by
    N(0, 0.01 Ha) and re-sorted, its own M tensors."""
    c1 = synth.make_instance(5, 30, 70, nomega, seed=51)
    c2 = synth.make_instance(4, 31, 70, nomega, seed=52)
    rng = np.random.default_rng(53)
    e2 = np.sort(c1.energy + rng.normal(0.0, 0.01, c1.energy.size))
    c1 = replace(c1, occupation=np.concatenate([np.ones(5), np.zeros(30)]))
    c2 = replace(c2, energy=e2, occupation=np.concatenate([np.ones(4), np.zeros(31)]))
    return replace(c1, spin2=c2)


def as_two_channels(inst):
    """A closed-shell instance as two identical spin channels (occupations halved)."""
    half = replace(inst, occupation=inst.occupation / 2.0)
    return replace(half, spin2=half)


def oracle_channels(inst):
    return [dict(energy=c.energy, occupation=c.occupation, m_ia=c.m_ia, m_sigma=c.m_sigma, nsemin=c.nsemin,
                 nsemax=c.nsemax) for c in (inst, inst.spin2)]
