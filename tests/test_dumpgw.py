"""DUMP_GW ingestion: files in the layout of MOLGW's dump_gw_ingredients
(src/m_gw_selfenergy_analytic.f90:799-881) read back into a G0W0 problem."""
import numpy as np
import pytest

from molgw_b200 import dumpgw
from oracle import rigw_oracle as o
from tests.conftest import HA_EV


def _vertex(n, naux, seed):
    rng = np.random.default_rng(seed)
    r = rng.standard_normal((n, n, naux)) * 0.05
    return (r + r.transpose(1, 0, 2)) / 2.0          # (pq|P) = (qp|P)


def _energies(n, nocc):
    e = np.sort(np.concatenate([np.linspace(-1.2, -0.35, nocc), np.linspace(0.05, 2.0, n - nocc)]))
    return e


def test_round_trip_layout(tmp_path):
    n, nocc, naux = 23, 5, 31
    v, e = _vertex(n, naux, 1), _energies(n, nocc)
    dumpgw.write_dump_gw(tmp_path, e, v)
    raw = np.fromfile(tmp_path / "v.bin", dtype="<f8")
    # Fortran order of eri_3center_mo(:, window, q): P fastest, then p, then q
    assert raw[naux * n * 3 + naux * 7 + 11] == v[3, 7, 11]
    inst = dumpgw.read_dump_gw(tmp_path, nocc, nomega=8)
    assert np.array_equal(inst.energy, e)
    assert inst.nocc == nocc and inst.nvirt == n - nocc and inst.naux == naux
    assert np.array_equal(inst.m_ia, v[:nocc, nocc:, :])
    assert np.array_equal(inst.m_sigma, v[nocc - 1:nocc + 1])
    assert (inst.nsemin, inst.nsemax) == (nocc, nocc + 1)


def test_reader_rejects_inconsistent_files(tmp_path):
    n, nocc, naux = 9, 3, 7
    dumpgw.write_dump_gw(tmp_path, _energies(n, nocc), _vertex(n, naux, 2))
    (tmp_path / "v.dat").write_text(f"{naux}\n{n + 1}\n{n + 1}\n")
    with pytest.raises(ValueError):
        dumpgw.read_dump_gw(tmp_path, nocc)


def test_dumped_problem_runs_through_the_oracle(tmp_path):
    n, nocc, naux = 20, 4, 26
    dumpgw.write_dump_gw(tmp_path, _energies(n, nocc), _vertex(n, naux, 3))
    inst = dumpgw.read_dump_gw(tmp_path, nocc, nomega=8)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    res = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng)
    assert np.isfinite(res.erpa) and res.erpa < 0.0
    assert np.all(np.isfinite(res.energy_qp_g))


@pytest.mark.gpu
def test_dumped_problem_on_the_gpu_matches_the_oracle(tmp_path, engine):
    n, nocc, naux = 60, 8, 150
    dumpgw.write_dump_gw(tmp_path, _energies(n, nocc), _vertex(n, naux, 4))
    inst = dumpgw.read_dump_gw(tmp_path, nocc, nomega=16)
    out = engine.g0w0(inst)
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    ref = o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                      nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                      nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc, eta=inst.eta)
    assert abs(out.erpa - ref.erpa) < 1e-10 * max(1.0, abs(ref.erpa))
    assert np.abs(out.sigma_calc - ref.sigma_calc.T).max() < 1e-9 * np.abs(ref.sigma_calc).max()
    assert np.abs(out.energy_qp_g - ref.energy_qp_g).max() * HA_EV < 1e-6


def test_open_shell_dump_round_trip(tmp_path):
    """nspin = 2: v.bin holds both spins, energies.dat spin 1; the second channel's
    occupied count and energies come from the caller."""
    n, naux = 21, 27
    v = np.stack([_vertex(n, naux, 5), _vertex(n, naux, 6)])
    e1 = _energies(n, 5)
    e2 = np.sort(e1 + np.random.default_rng(7).normal(0.0, 0.01, n))
    dumpgw.write_dump_gw(tmp_path, e1, v)
    inst = dumpgw.read_dump_gw(tmp_path, 5, nomega=8, nocc_2=4, energy_2=e2)
    assert inst.spin2 is not None and inst.spin_channel and inst.spin2.spin_channel
    assert np.array_equal(inst.m_ia, v[0, :5, 5:]) and np.array_equal(inst.spin2.m_ia, v[1, :4, 4:])
    assert np.array_equal(inst.occupation[:5], np.ones(5)) and inst.occupation[5] == 0.0
    assert np.array_equal(inst.spin2.energy, e2) and inst.spin2.nocc == 4
    assert np.array_equal(inst.spin2.m_sigma, v[1, 4:6])
    out = o.g0w0_imag_spin([dict(energy=c.energy, occupation=c.occupation, m_ia=c.m_ia, m_sigma=c.m_sigma,
                                 nsemin=c.nsemin, nsemax=c.nsemax) for c in (inst, inst.spin2)], inst.nomega)
    assert all(np.all(np.isfinite(r.energy_qp_g)) for r in out)
