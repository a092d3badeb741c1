"""The allocation-free continuation + QP entry point (rigw_qp_solve_noalloc), for
callers that may not allocate device memory, against the allocating entry point
(rigw_qp_solve) on the same sigma_calc, and against the oracle's QP energies of
the golden fixture.  Same tolerances as the parity tests: QP energies and Z
within 1e-6 eV / 1e-6, the real-grid Sigma within 2e-5 of its largest value.
Every case runs two calls in a row, since the calls share the library's fixed
scratch array.  Cases: the Pade technique with the library's evaluation points
or the caller's, the polynomial technique (imaginary_axis_homolumo, which needs
the caller's real points), and the real-grid Sigma written to the caller's
array or left in the scratch array (sigma = NULL)."""
import numpy as np
import pytest

from tests.conftest import HA_EV, instance_from_golden

pytestmark = pytest.mark.gpu

RIGW_PADE, RIGW_HOMOLUMO = 0, 1


def _homolumo_points(inst, nc=21):
    """Real evaluation points inside the gap, as se_init sets them for
    imaginary_axis_homolumo (src/m_selfenergy_tools.f90:616-633)."""
    eh, el = inst.energy[inst.nocc - 1], inst.energy[inst.nocc]
    return (eh + 0.01 + np.arange(nc) / (nc - 1.0) * (el - eh - 0.02)).astype(np.complex128)


def _noalloc(torch, inst, sc, technique, oc, want_sigma, efermi):
    from molgw_b200.rigw import qp_solve_noalloc
    nsig = sc.shape[0]
    nreal = 2 * (inst.nomega_sigma // 2) + 1
    d_sc = torch.from_numpy(np.ascontiguousarray(np.stack([sc.real, sc.imag], -1))).cuda()
    d_e = torch.from_numpy(inst.energy[inst.nsemin - 1:inst.nsemax].copy()).cuda()
    d_oc = None if oc is None else torch.from_numpy(np.ascontiguousarray(np.stack([oc.real, oc.imag], -1))).cuda()
    outs = [torch.full((nsig,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
    d_sigma = torch.full((nsig, nreal, 2), float("nan"), dtype=torch.float64, device="cuda") if want_sigma else None
    qp_solve_noalloc(d_sc, d_e, outs[0], outs[1], outs[2], d_sigma, device=0, omega_calc=d_oc,
                     technique=technique, nomega_sigma=inst.nomega_sigma, step_sigma=inst.step_sigma,
                     step_sigma_calc=inst.step_sigma_calc, eta=inst.eta, efermi=efermi)
    torch.cuda.synchronize()
    sigma = None
    if want_sigma:
        s = d_sigma.cpu().numpy()
        sigma = s[..., 0] + 1j * s[..., 1]
    return [o.cpu().numpy() for o in outs], sigma


@pytest.mark.parametrize("technique,given_points", [(RIGW_PADE, False), (RIGW_PADE, True), (RIGW_HOMOLUMO, True)])
@pytest.mark.parametrize("want_sigma", [True, False])
def test_noalloc_qp_matches_allocating_entry(engine, golden_synth, technique, given_points, want_sigma):
    import torch
    from molgw_b200.rigw import efermi_of
    inst = instance_from_golden(golden_synth)
    efermi = efermi_of(inst)
    if technique == RIGW_HOMOLUMO:
        oc = _homolumo_points(inst)
        inst.nomega_sigma_calc = oc.size
        _, _, wpol = engine.polarizability_grid_scalapack(inst)
        try:
            sc = engine.gw_selfenergy_imag_scalapack(wpol, inst, omega_calc=oc)
        finally:
            wpol.release()
    else:
        sc = golden_synth["sigma_calc"]
        oc = efermi + 1j * inst.step_sigma_calc * np.arange(sc.shape[1]) if given_points else None
    ref = engine.qp_solve(inst, sc, technique, omega_calc=oc, efermi=efermi)
    for _ in range(2):
        (g, z, zz), sigma = _noalloc(torch, inst, sc, technique, oc, want_sigma, efermi)
        assert np.abs(g - ref.energy_qp_g).max() * HA_EV < 1e-6
        assert np.abs(z - ref.energy_qp_z).max() * HA_EV < 1e-6
        assert np.abs(zz - ref.zz).max() < 1e-6
        if want_sigma:
            assert np.abs(sigma - ref.sigma).max() < 2e-5 * np.abs(ref.sigma).max()
        if technique == RIGW_PADE:
            # the oracle's QP energies of the golden fixture (same sigma_calc and grid)
            assert np.abs(g - golden_synth["energy_qp_g"]).max() * HA_EV < 1e-6
            assert np.abs(zz - golden_synth["zz"]).max() < 1e-6


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from molgw_b200.rigw import RigwError, qp_solve_noalloc
    sc = torch.zeros((65, 50, 2), dtype=torch.float64, device="cuda")
    e = torch.zeros(65, dtype=torch.float64, device="cuda")
    out = torch.zeros(65, dtype=torch.float64, device="cuda")
    with pytest.raises(RigwError) as ei:
        qp_solve_noalloc(sc, e, out)
    assert ei.value.code == 1 and "exceed the fixed scratch" in str(ei.value)
