"""ENERGY_QP round trip (src/m_io.f90:3645-3733) and G built from energy_g under
force_energy_qp (src/m_selfenergy_evaluation.f90:164-181), on the CPU."""
import numpy as np

from molgw_b200 import synth
from molgw_b200.energy_qp import read_energy_qp, write_energy_qp
from oracle import rigw_oracle as o


def test_write_read_round_trip(tmp_path):
    e = np.linspace(-1.3, 2.1, 11) + 1e-13
    write_energy_qp(tmp_path, e)
    back, status = read_energy_qp(tmp_path, 11)
    assert status == 0 and np.array_equal(back[:, 0], e)
    e2 = np.stack([e, e + 0.5], -1)
    write_energy_qp(tmp_path, e2)
    back, status = read_energy_qp(tmp_path, 11, nspin=2)
    assert status == 0 and np.array_equal(back, e2)


def test_read_statuses(tmp_path):
    assert read_energy_qp(tmp_path, 5)[1] == 1                      # no file
    write_energy_qp(tmp_path, np.zeros(6))
    assert read_energy_qp(tmp_path, 5)[1] == 2                      # other nstate
    assert read_energy_qp(tmp_path, 6, nspin=2)[1] == 2             # other nspin
    (tmp_path / "ENERGY_QP").unlink()
    (tmp_path / "energy_qp").write_text("1\n3\n1 -0.5D0\n-1 0.1D0\n3 0.7D0\n")
    e, status = read_energy_qp(tmp_path, 3)                         # lower-case name, scissor line
    assert status == -1 and e[0, 0] == -0.5


def _run(inst, energy_g=None):
    rng = o.selfenergy_set_state_range(inst.nstate, inst.occupation, selfenergy_state_min=inst.nsemin,
                                       selfenergy_state_max=inst.nsemax)
    return o.g0w0_imag(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nomega, rng,
                       nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                       nomega_sigma_calc=inst.nomega_sigma_calc, step_sigma_calc=inst.step_sigma_calc,
                       eta=inst.eta, energy_g=energy_g)


def test_energy_g_defaults_to_energy():
    inst = synth.make_instance(4, 30, 70, 8, seed=41)
    a, b = _run(inst), _run(inst, inst.energy.copy())
    assert np.array_equal(a.sigma_calc, b.sigma_calc) and np.array_equal(a.energy_qp_g, b.energy_qp_g)


def test_uniform_shift_of_energy_g_moves_only_the_qp_equation():
    """Sigma depends on z - e_p and se_init's points move with efermi(energy_g), so
    a uniform shift of energy_g leaves sigma_calc unchanged; W and the energy0 of
    the QP equation do not move, so the QP energies do."""
    inst = synth.make_instance(4, 30, 70, 8, seed=41)
    a, b = _run(inst), _run(inst, inst.energy + 0.01)
    assert np.abs(a.sigma_calc - b.sigma_calc).max() <= 1e-12 * np.abs(a.sigma_calc).max()
    assert a.erpa == b.erpa
    assert np.abs(a.energy_qp_g - b.energy_qp_g).max() > 1e-4
