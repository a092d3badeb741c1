"""The FP64 path at the shapes of the precision-sweep workload (Nocc=100,
Nvirt=1100, Naux=4000: 32 Cholesky panels, chi0 over 110 000 transitions,
multi-GB item budgets) against the oracle, on three of the 48 Gauss-Legendre
frequencies passed as the caller's omega and weights: the lowest, a middle and
the highest node, so that D(iw) spans its whole range.  The oracle finishes
them in under a minute on the host cores.

Checked: E_RPA, E_GW and sigma_calc with the tolerances of
tests/test_gpu_parity.py plus the rounding that the quadrature weights carry:
at a node of weight w the integrand is a difference of two sums of N terms of
size one (ln det eps against tr eps - N, |U^-T M|^2 against |M|^2), each term
rounded once, so it carries about N u w / (2 pi) (u = 2^-53).  The highest of
the 48 nodes has w = 8351, which makes that 5.9e-10 Ha at N = 4000 (6e-11 at
the 840-function instance of the parity tests, inside their 1e-10).  The QP energies and the
real-axis Sigma of a three-frequency Sigma_c are not a well-conditioned output:
in the oracle itself a relative perturbation of 1e-13 on sigma_calc moves the
99-point Thiele continuation by O(1) and the QP energies by up to 5 meV, so they
are left to the full-grid parity tests."""
import os

import numpy as np
import pytest

from molgw_b200 import synth
from oracle import rigw_oracle as o
from tests.test_gpu_parity import SIGMA_GRID

pytestmark = pytest.mark.gpu

FREQ_INDEX = [0, 23, 47]


@pytest.fixture(scope="module")
def large_case():
    from threadpoolctl import threadpool_limits
    inst = synth.large_instance_4000()
    om, wt = o.imaginary_quad_grid(inst.nomega)
    freq = (om[FREQ_INDEX].copy(), wt[FREQ_INDEX].copy())
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    with threadpool_limits(limits=os.cpu_count() or 1):
        res = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng, freq=freq,
                          **SIGMA_GRID)
    return inst, freq, res


U = 2.0 ** -53


def _weight_rounding(inst, freq):
    return inst.naux * U * float(np.sum(freq[1])) / (2.0 * np.pi)


def _check(inst, freq, res, erpa, egw, sigma):
    wr = _weight_rounding(inst, freq)
    sc = res.sigma_calc.T
    d = {"erpa": abs(erpa - res.erpa), "egw": abs(egw - res.egw), "sigma": float(np.abs(sigma - sc).max()),
         "weight_rounding": wr}
    assert d["erpa"] < 1e-10 * max(1.0, abs(res.erpa)) + 4.0 * wr, d
    assert d["egw"] < 1e-10 * max(1.0, abs(res.egw)) + 4.0 * wr, d
    msig = float(np.abs(sc).max())
    assert d["sigma"] < 1e-9 * msig + 4.0 * wr * float(np.max(np.sum(inst.m_sigma ** 2, axis=2))), d


def test_fp64_fused_solve_at_sweep_shapes(engine, large_case):
    inst, freq, res = large_case
    out = engine.g0w0(inst, freq=freq)
    _check(inst, freq, res, out.erpa, out.egw, out.sigma_calc)


def test_fp64_drop_in_calls_at_sweep_shapes(engine, large_case):
    """polarizability_grid -> gw_selfenergy_imag through the separate calls, with
    the frequencies passed as one rank of the frequency split passes them."""
    inst, freq, res = large_case
    sigma, energies = engine.frequency_partials(inst, FREQ_INDEX)
    _check(inst, freq, res, energies[0], energies[1], sigma)
