"""RI Coulomb integrals on the device (rigw_eri_2center, rigw_eri_3center_raw,
rigw_eri_3center) against the oracle's McMurchie-Davidson restatement, whose
front end reproduces the reference suite's SCF energies in the same bases:

* H2O cc-pVDZ / cc-pVDZ-RI (pure functions, up to d / f);
* H2O cc-pVTZ with the Auto auxiliary basis (f orbital shells, g auxiliary);
* CO in the Cartesian cc-pVDZ_gaussian basis with Cartesian cc-pVDZ-RI.

(P|Q) and (mu nu|P) match elementwise to 1e-12 of the largest entry.  The
metric-contracted tensor is defined up to an orthogonal transformation of the
auxiliary index (the eigenvectors of (P|Q)), so it is compared through the RI
four-center integrals sum_P B(ij,P) B(kl,P) (1e-11), and the number of kept
auxiliary functions must equal the oracle's.  Then the H2O workload goes from
the device integrals through both AO->MO transforms and the solve to the QP
energies of the fixture (1e-4 eV, the suite's QP tolerance)."""
import numpy as np
import pytest

from tests import co_case, h2o_case
from tests.conftest import HA_EV

pytestmark = pytest.mark.gpu


def _pairs(nbf):
    return np.array([(k, l) for l in range(1, nbf + 1) for k in range(1, l + 1)], dtype=np.int32)


def _cases():
    from oracle import gaussian_ri as g
    d = h2o_case.load()
    yield "h2o_dz", h2o_case.front_end(d), True
    c = d["cases"]["h2o_gw_contour.in"]
    bas = {int(z): t for z, t in d["basis"][c["basis"]].items()}
    yield "h2o_tz_auto", g.molecule_ri_hf([(z, tuple(x)) for z, x in c["atoms"]], bas, "AUTO"), True
    co = co_case.load()
    yield "co_cart", co_case.front_end(co), False


@pytest.mark.parametrize("which", ["h2o_dz", "h2o_tz_auto", "co_cart"])
def test_integrals_match_the_oracle(engine, which):
    from oracle import gaussian_ri as g
    (scf, m, det), pure = next((v, p) for k, v, p in _cases() if k == which)
    bf, aux = det["bf"], det["aux"]
    v2_ref = g.coulomb_2center(aux)
    v2 = engine.eri_2center(aux.shells, pure_aux=pure)
    assert np.abs(v2 - v2_ref).max() < 1e-12 * np.abs(v2_ref).max()
    nbf = det["nbf"]
    pairs = _pairs(nbf)
    raw = engine.eri_3center_raw(bf.shells, aux.shells, pairs, pure=pure, pure_aux=pure)
    ref3 = g.coulomb_3center(bf, aux)
    ref_raw = np.stack([ref3[k - 1, l - 1] for k, l in pairs], axis=1)
    assert np.abs(raw - ref_raw).max() < 1e-12 * np.abs(ref_raw).max()
    eri3 = engine.eri_3center(bf.shells, aux.shells, pairs, pure=pure, pure_aux=pure)
    assert eri3.shape[0] == det["nauxil"]
    ref_b = np.stack([scf.b3[k - 1, l - 1] * (0.5 if k == l else 1.0) for k, l in pairs], axis=1)
    four = eri3.T @ eri3
    four_ref = ref_b.T @ ref_b
    assert np.abs(four - four_ref).max() < 1e-11 * np.abs(four_ref).max()


def test_h2o_workload_from_device_integrals(engine):
    d = h2o_case.load()
    scf, m, det = h2o_case.front_end(d)
    pairs = _pairs(det["nbf"])
    eri3 = engine.eri_3center(det["bf"].shells, det["aux"].shells, pairs)
    out = engine.g0w0_from_ao(eri3, pairs, scf.c.T.copy(), scf.e_orb, scf.occupation, nomega=16, nsemin=5, nsemax=6,
                              **h2o_case.grid(d))
    assert abs(out.erpa - float(d["oracle_erpa"])) < 1e-10
    ref_sig = d["oracle_sigma_calc"]
    assert np.abs(out.sigma_calc - ref_sig.T).max() < 1e-9 * np.abs(ref_sig).max()
    assert np.abs(out.energy_qp_g - d["oracle_qp"]).max() * HA_EV < 1e-4


def test_device_output_equals_host_output(engine):
    import torch
    d = h2o_case.load()
    scf, m, det = h2o_case.front_end(d)
    pairs = _pairs(det["nbf"])
    bf, aux = det["bf"].shells, det["aux"].shells
    host = engine.eri_3center_raw(bf, aux, pairs)
    dev = torch.empty(host.shape, dtype=torch.float64, device="cuda")
    assert engine.eri_3center_raw(bf, aux, pairs, out=dev) is dev
    assert np.array_equal(dev.cpu().numpy(), host)
    host_b = engine.eri_3center(bf, aux, pairs)
    dev_b = engine.eri_3center(bf, aux, pairs, out=torch.empty(host.shape, dtype=torch.float64, device="cuda"))
    assert np.array_equal(dev_b.cpu().numpy(), host_b)
