"""Generate the golden fixtures of the parity tests.

Run in a checkout next to the MOLGW sources:

    python tests/golden/make_golden.py /path/to/molgw

It writes, next to this script:

* ``lih_bulk08.npz`` - the W-window and Sigma tensors of MOLGW's bulk-LiH CC4S
  test data (tests/data_for_tests/lih_bulk08_*, read as src/m_eri_ao_mo.f90:
  1192-1331 and src/m_io.f90:4048-4119 do), with the reference's own known
  answers (tests/inputs/testsuite:1206-1207 analytic RPA correlation
  -0.1152301335 Ha; :1209-1211 '(11|11)' = 2.92396387E-01) and the oracle's
  imaginary-axis G0W0 outputs for 16 frequencies;
* ``synth_small.npz`` - a seeded synthetic instance (Nocc=6, Nvirt=44,
  Naux=100, 16 frequencies) with the oracle's outputs.

The oracle outputs are produced by ``oracle/rigw_oracle.py``.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from molgw_b200 import cc4s, synth  # noqa: E402
from oracle import rigw_oracle as o  # noqa: E402

NOMEGA = 16
SIGMA_GRID = dict(nomega_sigma=101, step_sigma=0.025, nomega_sigma_calc=50, step_sigma_calc=0.075, eta=0.01)


def run_oracle(energy, occupation, m_ia, m_sigma, nsemin, nsemax, nomega):
    rng = o.selfenergy_set_state_range(len(energy), occupation, selfenergy_state_min=nsemin,
                                       selfenergy_state_max=nsemax)
    assert (rng.nsemin, rng.nsemax) == (nsemin, nsemax)
    res = o.g0w0_imag(energy, occupation, m_ia, m_sigma, nomega, rng, **SIGMA_GRID)
    w, wt = o.imaginary_quad_grid(nomega)
    nocc = m_ia.shape[0]
    sf = o.polarizability_grid(m_ia, energy[:nocc], energy[nocc:nocc + m_ia.shape[1]], occupation[:nocc],
                               occupation[nocc:nocc + m_ia.shape[1]], w, wt, keep_chi=True)
    return dict(erpa=res.erpa, egw=res.egw, sigma_calc=res.sigma_calc.T.copy(), sigma=res.sigma.T.copy(),
                energy_qp_g=res.energy_qp_g, energy_qp_z=res.energy_qp_z, zz=res.zz, ehomo=res.ehomo,
                elumo=res.elumo, chi=sf.chi, omega=w, weight=wt)


def main(ref: Path):
    root = ref / "tests" / "data_for_tests" / "lih_bulk08"
    e, occ, efermi = cc4s.read_eigenenergies(root)
    v = cc4s.read_coulomb_vertex(root)                  # [i, j, P] = eri_3center_mo(P, i+1, j+1)
    nocc = int(np.count_nonzero(occ > 0))
    m_ia = np.ascontiguousarray(np.transpose(v[nocc:, :nocc, :], (1, 0, 2)))   # M(P, a, i) -> [i][a][P]
    nsemin, nsemax = nocc, nocc + 1
    m_sigma = np.ascontiguousarray(np.stack([v[:, nsemin - 1, :], v[:, nsemax - 1, :]]))  # M(P, p, m) -> [m][p][P]
    out = run_oracle(e, occ, m_ia, m_sigma, nsemin, nsemax, NOMEGA)
    np.savez_compressed(
        HERE / "lih_bulk08.npz", energy=e, occupation=occ, m_ia=m_ia, m_sigma=m_sigma, nsemin=nsemin,
        nsemax=nsemax, nomega=NOMEGA, ref_rpa_analytic=-0.1152301335, ref_rpa_tol=1e-7,
        ref_integral_11_11=2.92396387e-01, ref_integral_tol=1e-7,
        integral_11_11=float(np.dot(v[0, 0], v[0, 0])), vertex_11=v[0, 0].copy(),
        rpa_analytic_oracle=o.analytic_rpa_correlation(m_ia, e[:nocc], e[nocc:]),
        **{k: v for k, v in out.items() if k != "chi"}, chi_first=out["chi"][0])

    inst = synth.make_instance(6, 44, 100, NOMEGA, seed=11)
    out = run_oracle(inst.energy, inst.occupation, inst.m_ia, inst.m_sigma, inst.nsemin, inst.nsemax, NOMEGA)
    np.savez_compressed(
        HERE / "synth_small.npz", energy=inst.energy, occupation=inst.occupation, m_ia=inst.m_ia,
        m_sigma=inst.m_sigma, nsemin=inst.nsemin, nsemax=inst.nsemax, nomega=NOMEGA, seed=11,
        **{k: v for k, v in out.items() if k != "chi"}, chi_first=out["chi"][0])
    print("wrote", HERE / "lih_bulk08.npz", HERE / "synth_small.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the MOLGW source tree>")
    main(Path(sys.argv[1]))
