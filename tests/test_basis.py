"""Basis-file helpers of the RI integral entry points (molgw_b200/basis.py) and
the shell coefficients the library takes (molgw_b200.rigw.shell_coefficients),
on the basis texts of the committed H2O fixture: the product parser reads what
the oracle's does, centres go to Bohr, function counts, and the coefficient
convention (contraction normalized so that its x^l component has norm (2l-1)!!,
the factor the pure or Cartesian transform divides out)."""
import json

import numpy as np
import pytest

from molgw_b200 import basis as B
from molgw_b200.rigw import shell_coefficients
from oracle import gaussian_ri as g
from tests import h2o_case


@pytest.fixture(scope="module")
def texts():
    d = h2o_case.load()
    return d["basis"] if isinstance(d["basis"], dict) else json.loads(str(d["basis"]))


@pytest.mark.parametrize("name", ["cc-pVDZ", "cc-pVTZ", "cc-pVDZ-RI", "cc-pVTZ-RI"])
def test_parser_reads_what_the_oracle_reads(texts, name):
    for z, text in texts[name].items():
        mine, ref = B.parse_basis_file(text), g.parse_basis_file(text)
        assert len(mine) == len(ref) > 0
        for a, b in zip(mine, ref):
            assert a.am == b.am
            assert np.array_equal(a.alpha, np.asarray(b.alpha)) and np.array_equal(a.coeff, np.asarray(b.coeff))


def test_molecule_shells_centres_and_counts(texts):
    atoms = [(8, (0.0, 0.0, 0.0)), (1, (0.0, 0.757, 0.587)), (1, (0.0, -0.757, 0.587))]
    sh = B.molecule_shells(atoms, {int(z): t for z, t in texts["cc-pVDZ"].items()})
    assert B.nfunctions(sh) == 24 and B.nfunctions(sh, pure=False) == 25
    h = [s for s in sh if np.allclose(s.center, np.array([0.0, 0.757, 0.587]) / B.BOHR_A, rtol=0, atol=1e-15)]
    assert len(h) == len(B.parse_basis_file(texts["cc-pVDZ"]["1"]))


def test_water_cluster_lattice():
    atoms = B.water_cluster(8, spacing=3.0)
    assert len(atoms) == 24 and [z for z, _ in atoms[:3]] == [8, 1, 1]
    oxy = np.array([xyz for z, xyz in atoms if z == 8])
    assert {tuple(x) for x in oxy} == {(3.0 * i, 3.0 * j, 3.0 * k) for i in (0, 1) for j in (0, 1) for k in (0, 1)}
    o, h1, h2 = (np.array(atoms[k][1]) for k in range(3))
    assert np.allclose(h1 - o, [0.0, 0.757, 0.587]) and np.allclose(h2 - o, [0.0, -0.757, 0.587])


@pytest.mark.parametrize("name", ["cc-pVTZ", "cc-pVTZ-RI"])
def test_shell_coefficients_normalize_the_xl_component(texts, name):
    for text in texts[name].values():
        for s in B.parse_basis_file(text):
            d = shell_coefficients(s.am, s.alpha, s.coeff)
            p = s.alpha[:, None] + s.alpha[None, :]
            # <sum_k d_k x^l e^{-a_k r^2} | same> / (2l-1)!! = sum_jk d_j d_k (pi/p)^{3/2} / (2p)^l
            norm = float(np.sum(np.outer(d, d) * (np.pi / p) ** 1.5 / (2.0 * p) ** s.am))
            assert abs(norm - 1.0) < 1e-13
