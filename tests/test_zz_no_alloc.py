"""The allocation-free continuation + QP entry point (rigw_qp_solve_noalloc), for
callers that may not allocate device memory, against the allocating entry point
(rigw_qp_solve) on the same sigma_calc.  Same tolerances as the parity tests:
QP energies and Z within 1e-6 eV / 1e-6, the real-grid Sigma within 2e-5 of its
largest value.  Two calls in a row, since the calls share the library's fixed
scratch array."""
import numpy as np
import pytest

from tests.conftest import HA_EV, instance_from_golden

pytestmark = pytest.mark.gpu


def _run(golden_synth, torch, qp_solve_noalloc, nsig, nc, nreal, efermi):
    sc = golden_synth["sigma_calc"]
    inst = instance_from_golden(golden_synth)
    d_sc = torch.from_numpy(np.ascontiguousarray(np.stack([sc.real, sc.imag], -1))).cuda()
    d_e = torch.from_numpy(inst.energy[inst.nsemin - 1:inst.nsemax].copy()).cuda()
    outs = [torch.full((nsig,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
    d_sigma = torch.full((nsig, nreal, 2), float("nan"), dtype=torch.float64, device="cuda")
    qp_solve_noalloc(d_sc, d_e, outs[0], outs[1], outs[2], d_sigma, device=0, nomega_sigma=inst.nomega_sigma,
                     step_sigma=inst.step_sigma, step_sigma_calc=inst.step_sigma_calc, eta=inst.eta, efermi=efermi)
    torch.cuda.synchronize()
    s = d_sigma.cpu().numpy()
    return [o.cpu().numpy() for o in outs], s[..., 0] + 1j * s[..., 1]


def test_noalloc_qp_matches_allocating_entry(engine, golden_synth):
    import torch
    from molgw_b200.rigw import qp_solve_noalloc
    inst = instance_from_golden(golden_synth)
    sc = golden_synth["sigma_calc"]
    ref = engine.qp_solve(inst, sc)
    nsig, nc = sc.shape
    nreal = 2 * (inst.nomega_sigma // 2) + 1
    e = inst.energy
    efermi = 0.5 * (e[inst.nocc - 1] + e[inst.nocc])
    for _ in range(2):
        (g, z, zz), sigma = _run(golden_synth, torch, qp_solve_noalloc, nsig, nc, nreal, efermi)
        assert np.abs(g - ref.energy_qp_g).max() * HA_EV < 1e-6
        assert np.abs(z - ref.energy_qp_z).max() * HA_EV < 1e-6
        assert np.abs(zz - ref.zz).max() < 1e-6
        assert np.abs(sigma - ref.sigma).max() < 2e-5 * np.abs(ref.sigma).max()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from molgw_b200.rigw import RigwError, qp_solve_noalloc
    sc = torch.zeros((65, 50, 2), dtype=torch.float64, device="cuda")
    e = torch.zeros(65, dtype=torch.float64, device="cuda")
    out = torch.zeros(65, dtype=torch.float64, device="cuda")
    with pytest.raises(RigwError) as ei:
        qp_solve_noalloc(sc, e, out)
    assert ei.value.code == 1 and "exceed the fixed scratch" in str(ei.value)
