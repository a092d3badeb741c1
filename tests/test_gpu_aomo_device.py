"""The AO->MO transform with its tensors in device memory
(rigw_eri_3center_mo_ex with RIGW_PROBLEM_DEVICE_POINTERS) and the drop-in path
from the AO tensor to the QP energies with one upload (Engine.g0w0_from_ao, as
polarizability_grid_scalapack calls calculate_eri_3center_mo itself,
src/m_gw_selfenergy_grid.f90:92).  Device mode equals host mode bitwise; the
He cc-pVDZ/PAuto AO tensor of the oracle's front end goes through the whole path
and matches the oracle (E_RPA 1e-10, QP 1e-6 eV)."""
import numpy as np
import pytest

from oracle import gaussian_ri as g
from oracle import rigw_oracle as o
from tests import he_case
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


def _pairs(nbf):
    return np.array([(k, l) for l in range(1, nbf + 1) for k in range(1, l + 1)], dtype=np.int32)


@pytest.mark.parametrize("precision", [0, 1])   # RIGW_FP64, RIGW_BF16X3
def test_device_mode_equals_host_mode(engine, precision):
    import torch
    rng = np.random.default_rng(17)
    nbf, naux = 60, 150
    pairs = _pairs(nbf)
    pairs = pairs[rng.random(len(pairs)) > 0.1]            # screened pairs are absent
    eri3 = rng.standard_normal((naux, len(pairs)))
    c = np.linalg.qr(rng.standard_normal((nbf, nbf)))[0].T.copy()
    d_eri3 = torch.from_numpy(eri3).cuda()
    for (m0, m1, n0, n1) in [(9, 60, 1, 8), (1, 60, 8, 9)]:
        host = engine.calculate_eri_3center_mo(eri3, pairs, c, m0, m1, n0, n1, precision)
        dev = engine.calculate_eri_3center_mo(d_eri3, pairs, c, m0, m1, n0, n1, precision)
        assert np.array_equal(host, dev.cpu().numpy())


def test_ao_tensor_to_qp_energies_he(engine):
    """The He AO tensor B(mu nu, P) (pair-packed, diagonal x0.5 as the reference
    stores it, src/m_eri_calculate.f90:1841) and the HF orbitals through both
    transforms and the solve on the device, against the oracle on the MO tensor."""
    he = he_case.load()
    scf, m, _ = g.atom_ri_hf(he["basis_text"], 2)
    nbf = scf.c.shape[0]
    pairs = _pairs(nbf)
    eri3 = np.stack([scf.b3[k - 1, l - 1] * (0.5 if k == l else 1.0) for k, l in pairs], axis=1)   # [naux, npair]
    grid = dict(nomega_sigma=31, step_sigma=0.1, nomega_sigma_calc=21, step_sigma_calc=0.1, eta=0.001)
    out = engine.g0w0_from_ao(eri3, pairs, scf.c.T.copy(), scf.e_orb, scf.occupation, nomega=16, nsemin=1,
                              nsemax=1, **grid)
    rng = o.selfenergy_set_state_range(5, scf.occupation, selfenergy_state_min=1, selfenergy_state_max=1)
    ref = o.g0w0_imag(scf.e_orb, scf.occupation, m[:1, 1:], m[[0]], 16, rng, **grid)
    assert abs(out.erpa - ref.erpa) < 1e-10
    assert np.abs(out.sigma_calc - ref.sigma_calc.T).max() < 1e-9 * np.abs(ref.sigma_calc).max()
    assert abs(out.energy_qp_g[0] - ref.energy_qp_g[0]) * HA_EV < 1e-6
