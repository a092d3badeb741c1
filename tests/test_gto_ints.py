"""oracle/gto_ints.c (the shell-blocked C McMurchie-Davidson integrals of the
oracle's front end) against the Python restatement in oracle/gaussian_ri.py
on several centers and shells up to g, and over the branches of its Boys
function (small, mid and large arguments).  CPU only."""
import numpy as np
import pytest

from oracle import gaussian_ri as g

S = g.Shell
A, B, C = np.zeros(3), np.array([0.3, -0.5, 1.2]), np.array([-0.7, 0.4, -0.9])


@pytest.fixture(scope="module")
def lib():
    assert g._c_available()


def _basis():
    sh = [S(2, np.array([1.3, 0.4]), np.array([0.6, 0.5]), A.copy()), S(1, np.array([0.9]), np.array([1.0]), B.copy()),
          S(0, np.array([3.0, 0.5]), np.array([0.3, 0.8]), C.copy()), S(3, np.array([0.8]), np.array([1.0]), C.copy())]
    ax = [S(3, np.array([1.1]), np.array([1.0]), A.copy()), S(4, np.array([0.7]), np.array([1.0]), B.copy()),
          S(0, np.array([2.0]), np.array([1.0]), C.copy()), S(2, np.array([0.5]), np.array([1.0]), B.copy())]
    return g.build_functions(sh), g.build_functions(ax)


def test_one_body_matches_python(lib):
    bf, _ = _basis()
    nuc = [(8, A), (1, B), (3, C)]
    for c, p in zip(g.one_body(bf, nuc), g.one_body_py(bf, nuc)):
        assert np.abs(c - p).max() < 1e-13 * max(1.0, np.abs(p).max())


def test_two_and_three_center_match_python(lib):
    bf, aux = _basis()
    p2 = g.coulomb_2center_py(aux)
    assert np.abs(g.coulomb_2center(aux) - p2).max() < 1e-13 * np.abs(p2).max()
    p3 = g.coulomb_3center_py(bf, aux)
    assert np.abs(g.coulomb_3center(bf, aux) - p3).max() < 1e-13 * np.abs(p3).max()


@pytest.mark.parametrize("dist", [0.0, 0.5, 3.0, 9.0, 20.0])
def test_boys_branches_over_distance(lib, dist):
    ax = [S(4, np.array([2.3]), np.array([1.0]), np.zeros(3)),
          S(4, np.array([1.7]), np.array([1.0]), np.array([dist * 0.6, dist * 0.8, 0.0])),
          S(3, np.array([9.0]), np.array([1.0]), np.array([0.0, 0.0, dist]))]
    aux = g.build_functions(ax)
    p = g.coulomb_2center_py(aux)
    assert np.abs(g.coulomb_2center(aux) - p).max() < 1e-13 * np.abs(p).max()
