"""Gaussian-basis front end of the oracle: RI integrals and an RI Hartree-Fock
SCF, enough to run MOLGW's He test inputs end to end on the host.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; it
produces the M tensors and orbital energies that the parity tests hand to the
CUDA path, so that Sigma_c, the Pade continuation and the QP equation can be
checked against known answers held by the reference's own test suite
(tests/inputs/testsuite:1131-1153, He cc-pVDZ with the PAuto auxiliary basis).

What it restates, and from where:

* basis files: MOLGW's format (first line: number of shells; per shell
  "ng am" then ng lines "alpha coeff"), contraction coefficients on
  normalized primitives, each contracted Cartesian function normalized to one
  (src/m_basis_set.f90:90-340, src/m_gaussian.f90:58-81); pure (real solid
  harmonic) functions for both bases, the default gaussian_type
  (src/input_variables.f90:285);
* the PAuto auxiliary basis: every sum of two primitive exponents and
  angular momenta on a center is a candidate; candidates are taken from the
  largest exponent down in groups whose exponents lie within a ratio
  auto_auxil_fsam = 1.5 of the largest, each group gives one shell per
  angular momentum 0 .. l at the geometric mean of its distinct exponents,
  with l = max(l of the group, l of the previous group) capped at
  lmax_obs + auto_auxil_lmaxinc (= 1) or 2 l_val (src/m_basis_set.f90:638-952);
* the RI metric: (P|Q) diagonalized, eigenvalues below TOO_LOW_EIGENVAL =
  1e-6 dropped, (P|Q)^-1/2 = eigvec[:, kept] / sqrt(eigval[kept])
  (src/m_eri_calculate.f90:1049-1262, src/m_eri.f90:27), and the 3-center
  integrals B(mu nu, P) = sum_Q (mu nu|Q) (Q|P)^-1/2
  (src/m_eri_calculate.f90:1584-1950);
* the integrals themselves: MOLGW takes them from LIBCINT (a third-party
  library, absent here).  They are restated with the McMurchie-Davidson
  scheme (Hermite expansion coefficients and Hermite Coulomb integrals over
  the Boys function; Helgaker, Jorgensen, Olsen, "Molecular Electronic-
  Structure Theory", ch. 9), a published algorithm;
* restricted Hartree-Fock with RI Coulomb and exchange, converged to a tight
  density threshold (the converged state does not depend on MOLGW's mixing
  scheme); E = 1/2 sum D (h + F) + E_nn.
"""
from __future__ import annotations

import ctypes
import subprocess
from dataclasses import dataclass, field
from math import comb, factorial, sqrt, pi
from pathlib import Path

import numpy as np
from scipy import special

TOO_LOW_EIGENVAL = 1.0e-6         # src/m_eri.f90:27
AUTO_AUXIL_FSAM = 1.5             # src/input_variables.f90:262
AUTO_AUXIL_LMAXINC = 1            # src/input_variables.f90:263


# ----------------------------------------------------------------------------- basis sets
@dataclass
class Shell:
    am: int
    alpha: np.ndarray
    coeff: np.ndarray              # on normalized primitives
    center: np.ndarray = field(default_factory=lambda: np.zeros(3))


def parse_basis_file(text: str, center=(0.0, 0.0, 0.0)) -> list[Shell]:
    """MOLGW basis file (src/m_basis_set.f90:155-170, 236-245)."""
    tok = text.split()
    pos = 0
    nshell = int(tok[pos]); pos += 1
    shells = []
    for _ in range(nshell):
        ng, am = int(tok[pos]), int(tok[pos + 1]); pos += 2
        a = np.array([float(tok[pos + 2 * k]) for k in range(ng)])
        c = np.array([float(tok[pos + 2 * k + 1]) for k in range(ng)])
        pos += 2 * ng
        shells.append(Shell(am, a, c, np.asarray(center, dtype=float)))
    return shells


def lmax_abs(lmax_obs: int, z: int) -> int:
    """get_lmax_abs (src/m_basis_set.f90:933-950)."""
    lval = 0 if z <= 2 else 1 if z <= 18 else 2 if z <= 54 else 3
    return max(lmax_obs + AUTO_AUXIL_LMAXINC, 2 * lval)


def pauto_auxiliary(shells: list[Shell], z: int, pauto: bool = True) -> list[Shell]:
    """PAuto (or, with ``pauto`` False, Auto) auxiliary basis of one center
    (init_auxil_basis_set_auto, src/m_basis_set.f90:638-831): one uncontracted
    shell per (exponent, am).  PAuto takes every sum of two primitive exponents
    and angular momenta of the center as a candidate, Auto every primitive
    exponent and angular momentum doubled (:733-758)."""
    cand_e, cand_l = [], []
    lmax_obs = 0
    for si in shells:
        lmax_obs = max(lmax_obs, si.am)
        if not pauto:
            for ai in si.alpha:
                cand_e.append(2.0 * ai)
                cand_l.append(2 * si.am)
            continue
        for sj in shells:
            for ai in si.alpha:
                for aj in sj.alpha:
                    cand_e.append(ai + aj)
                    cand_l.append(si.am + sj.am)
    cand_e, cand_l = np.array(cand_e), np.array(cand_l)
    lmax = lmax_abs(lmax_obs, z)
    remaining = np.ones(cand_e.size, dtype=bool)
    out = []
    am_current = 0
    while remaining.any():
        idx = np.where(remaining)[0]
        cur = idx[np.argmax(cand_e[idx])]            # MAXLOC: first of the largest
        e_cur = cand_e[cur]
        trial_e, trial_l = [e_cur], [cand_l[cur]]
        remaining[cur] = False
        for k in range(cand_e.size):
            if remaining[k] and e_cur / cand_e[k] < AUTO_AUXIL_FSAM:
                trial_e.append(cand_e[k])
                trial_l.append(cand_l[k])
                remaining[k] = False
        prod, n = 1.0, 0
        for i in range(len(trial_e)):
            new = all(not (trial_l[i] == trial_l[j] and abs(trial_e[i] - trial_e[j]) < 1.0e-6) for j in range(i))
            if new:
                n += 1
                prod *= trial_e[i]
        e_sel = prod ** (1.0 / n)
        am_sel = min(max(max(trial_l), am_current), lmax)
        am_current = am_sel
        for am in range(am_sel + 1):
            out.append(Shell(am, np.array([e_sel]), np.array([1.0]), shells[0].center.copy()))
    return out


def cart_exponents(l: int) -> list[tuple[int, int, int]]:
    """Cartesian components of a shell in the order of the reference (libint:
    x first, src/m_basis_set.f90:281-315)."""
    out = []
    for nx in range(l, -1, -1):
        for nz in range(0, l - nx + 1):
            out.append((nx, l - nx - nz, nz))
    return out


def _dfact(n: int) -> float:
    return 1.0 if n <= 0 else float(np.prod(np.arange(n, 0, -2, dtype=float)))


def primitive_norm(a: float, l: tuple[int, int, int]) -> float:
    """Normalization of x^i y^j z^k exp(-a r^2)."""
    i, j, k = l
    L = i + j + k
    return sqrt((2 * a / pi) ** 1.5 * (4 * a) ** L / (_dfact(2 * i - 1) * _dfact(2 * j - 1) * _dfact(2 * k - 1)))


def solid_harmonic_coeffs(l: int) -> np.ndarray:
    """Real solid harmonics S_lm (m = -l..l) as combinations of the Cartesian
    monomials of cart_exponents(l) (Helgaker et al. eq. 6.4.73); rows are m."""
    carts = cart_exponents(l)
    index = {c: k for k, c in enumerate(carts)}
    T = np.zeros((2 * l + 1, len(carts)))
    for row, m in enumerate(range(-l, l + 1)):
        am = abs(m)
        vm = 0.0 if m >= 0 else 0.5
        nlm = 1.0 / (2 ** am * factorial(l)) * sqrt(2.0 * factorial(l + am) * factorial(l - am) / (2.0 if m == 0 else 1.0))
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                v = vm
                vtop = int(np.floor(am / 2.0 - vm)) + vm
                while v <= vtop + 1e-9:
                    c = ((-1) ** (t + v - vm)) * (0.25 ** t) * comb(l, t) * comb(l - t, am + t) * comb(t, u) \
                        * comb(am, int(round(2 * v)))
                    ex = (int(round(2 * t + am - 2 * (u + v))), int(round(2 * (u + v))), l - 2 * t - am)
                    T[row, index[ex]] += nlm * c
                    v += 1.0
    return T


@dataclass
class BasisFunctions:
    """Contracted Cartesian functions and the pure combinations built on them."""
    prims: list                    # per Cartesian function: (center, exps, coefs incl. primitive norms, (i,j,k))
    cart_to_pure: np.ndarray       # [nbf_pure, nbf_cart]
    shell_of: list                 # pure function -> shell index
    shells: list = field(default_factory=list)


def build_functions(shells: list[Shell], pure: bool = True) -> BasisFunctions:
    """Contracted functions of the shells: pure (real solid harmonics) or, with
    ``pure`` False (gaussian_type='CART'), the Cartesian monomials themselves,
    each normalized on its own (the (nx, ny, nz) part of the normalization,
    src/m_cart_to_pure.f90:262-279)."""
    prims, blocks, shell_of = [], [], []
    ncart = 0
    for si, sh in enumerate(shells):
        carts = cart_exponents(sh.am)
        start = ncart
        for c in carts:
            # one normalization for every component (the reference's common_norm_factor,
            # src/m_gaussian.f90:74-75): the solid-harmonic coefficients act on monomials
            coef = np.array([ck * primitive_norm(a, (sh.am, 0, 0)) for a, ck in zip(sh.alpha, sh.coeff)])
            prims.append((sh.center, sh.alpha.copy(), coef, c))
            ncart += 1
        blocks.append((start, solid_harmonic_coeffs(sh.am) if pure else np.eye(len(carts))))
        shell_of += [si] * ((2 * sh.am + 1) if pure else len(carts))
    T = np.zeros((len(shell_of), ncart))
    r = 0
    for start, tb in blocks:
        T[r:r + tb.shape[0], start:start + tb.shape[1]] = tb
        r += tb.shape[0]
    bf = BasisFunctions(prims, T, shell_of, list(shells))
    # every function normalized to one (the contraction then too)
    s = bf.cart_to_pure @ (_c_one_body(bf, [])[0] if _c_available() else overlap_cart(bf)) @ bf.cart_to_pure.T
    bf.cart_to_pure = bf.cart_to_pure / np.sqrt(np.diag(s))[:, None]
    return bf


# ----------------------------------------------------------------------------- McMurchie-Davidson
def hermite_e(i: int, j: int, a: float, b: float, qx: float) -> np.ndarray:
    """E^{ij}_t, t = 0..i+j, of exp(-a x_A^2) x_A^i exp(-b x_B^2) x_B^j, Q = A - B."""
    p = a + b
    E = np.zeros((i + 1, j + 1, i + j + 2))
    E[0, 0, 0] = np.exp(-a * b / p * qx * qx)
    xpa, xpb = -b / p * qx, a / p * qx
    for ii in range(i + 1):
        for jj in range(j + 1):
            if ii == 0 and jj == 0:
                continue
            for t in range(ii + jj + 1):
                if ii > 0:
                    v = xpa * E[ii - 1, jj, t] + (t + 1) * E[ii - 1, jj, t + 1]
                    if t > 0:
                        v += E[ii - 1, jj, t - 1] / (2 * p)
                else:
                    v = xpb * E[ii, jj - 1, t] + (t + 1) * E[ii, jj - 1, t + 1]
                    if t > 0:
                        v += E[ii, jj - 1, t - 1] / (2 * p)
                E[ii, jj, t] = v
    return E[i, j, : i + j + 1]


def boys(nmax: int, T: float) -> np.ndarray:
    """F_n(T), n = 0..nmax."""
    n = np.arange(nmax + 1, dtype=float)
    if T < 1.0e-12:
        return 1.0 / (2 * n + 1) - T / (2 * n + 3)
    return 0.5 * T ** (-(n + 0.5)) * special.gamma(n + 0.5) * special.gammainc(n + 0.5, T)


def hermite_r(tmax: int, umax: int, vmax: int, p: float, rpc: np.ndarray) -> np.ndarray:
    """Hermite Coulomb integrals R_tuv (order 0) for exponent p and P - C = rpc."""
    nmax = tmax + umax + vmax
    F = boys(nmax, p * float(rpc @ rpc))
    R = np.zeros((nmax + 1, tmax + 1, umax + 1, vmax + 1))
    for n in range(nmax + 1):
        R[n, 0, 0, 0] = (-2 * p) ** n * F[n]
    X, Y, Z = rpc
    for n in range(nmax - 1, -1, -1):
        for t in range(tmax + 1):
            for u in range(umax + 1):
                for v in range(vmax + 1):
                    if t + u + v == 0 or t + u + v > nmax - n:
                        continue
                    if t > 0:
                        val = X * R[n + 1, t - 1, u, v] + ((t - 1) * R[n + 1, t - 2, u, v] if t > 1 else 0.0)
                    elif u > 0:
                        val = Y * R[n + 1, t, u - 1, v] + ((u - 1) * R[n + 1, t, u - 2, v] if u > 1 else 0.0)
                    else:
                        val = Z * R[n + 1, t, u, v - 1] + ((v - 1) * R[n + 1, t, u, v - 2] if v > 1 else 0.0)
                    R[n, t, u, v] = val
    return R[0]


def _pair(pa, pb):
    """Hermite expansion of the product of two primitives: (p, P, E[t,u,v])."""
    (A, a, la), (B, b, lb) = pa, pb
    p = a + b
    P = (a * A + b * B) / p
    ex = [hermite_e(la[k], lb[k], a, b, A[k] - B[k]) for k in range(3)]
    E = ex[0][:, None, None] * ex[1][None, :, None] * ex[2][None, None, :]
    return p, P, E


def _overlap_prim(pa, pb):
    p, _, E = _pair(pa, pb)
    return E[0, 0, 0] * (pi / p) ** 1.5


def _kinetic_prim(pa, pb):
    (A, a, la), (B, b, lb) = pa, pb
    i, j, k = lb

    def s(lb2):
        if min(lb2) < 0:
            return 0.0
        return _overlap_prim(pa, (B, b, lb2))
    t = b * (2 * (i + j + k) + 3) * s(lb)
    t -= 2 * b * b * (s((i + 2, j, k)) + s((i, j + 2, k)) + s((i, j, k + 2)))
    t -= 0.5 * (i * (i - 1) * s((i - 2, j, k)) + j * (j - 1) * s((i, j - 2, k)) + k * (k - 1) * s((i, j, k - 2)))
    return t


def _nuclear_prim(pa, pb, C):
    p, P, E = _pair(pa, pb)
    R = hermite_r(E.shape[0] - 1, E.shape[1] - 1, E.shape[2] - 1, p, P - C)
    return 2 * pi / p * float(np.sum(E * R))


def _eri_pairs(p1, P1, E1, p2, P2, E2):
    alpha = p1 * p2 / (p1 + p2)
    T1, U1, V1 = (d - 1 for d in E1.shape)
    T2, U2, V2 = (d - 1 for d in E2.shape)
    R = hermite_r(T1 + T2, U1 + U2, V1 + V2, alpha, P1 - P2)
    sign2 = ((-1.0) ** np.arange(T2 + 1))[:, None, None] * ((-1.0) ** np.arange(U2 + 1))[None, :, None] \
        * ((-1.0) ** np.arange(V2 + 1))[None, None, :]
    E2s = E2 * sign2
    tot = 0.0
    for t in range(T1 + 1):
        for u in range(U1 + 1):
            for v in range(V1 + 1):
                if E1[t, u, v] == 0.0:
                    continue
                tot += E1[t, u, v] * float(np.sum(E2s * R[t:t + T2 + 1, u:u + U2 + 1, v:v + V2 + 1]))
    return 2 * pi ** 2.5 / (p1 * p2 * sqrt(p1 + p2)) * tot


def _contracted(f):
    center, exps, coefs, l = f
    return [((np.asarray(center, float)), a, l, c) for a, c in zip(exps, coefs)]


def overlap_cart(bf: BasisFunctions) -> np.ndarray:
    n = len(bf.prims)
    S = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1):
            v = 0.0
            for (A, a, la, ca) in _contracted(bf.prims[i]):
                for (B, b, lb, cb) in _contracted(bf.prims[j]):
                    v += ca * cb * _overlap_prim((A, a, la), (B, b, lb))
            S[i, j] = S[j, i] = v
    return S


def one_body_py(bf: BasisFunctions, nuclei) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Overlap, kinetic and nuclear-attraction matrices over the pure functions;
    ``nuclei`` = [(Z, (x, y, z)), ...]."""
    n = len(bf.prims)
    S, T, V = (np.zeros((n, n)) for _ in range(3))
    for i in range(n):
        for j in range(i + 1):
            s = t = v = 0.0
            for (A, a, la, ca) in _contracted(bf.prims[i]):
                for (B, b, lb, cb) in _contracted(bf.prims[j]):
                    pa, pb = (A, a, la), (B, b, lb)
                    s += ca * cb * _overlap_prim(pa, pb)
                    t += ca * cb * _kinetic_prim(pa, pb)
                    for z, c in nuclei:
                        v -= z * ca * cb * _nuclear_prim(pa, pb, np.asarray(c, float))
            S[i, j] = S[j, i] = s
            T[i, j] = T[j, i] = t
            V[i, j] = V[j, i] = v
    X = bf.cart_to_pure
    return X @ S @ X.T, X @ T @ X.T, X @ V @ X.T


def _pair_list(bf: BasisFunctions, i: int, j: int):
    out = []
    for (A, a, la, ca) in _contracted(bf.prims[i]):
        for (B, b, lb, cb) in _contracted(bf.prims[j]):
            p, P, E = _pair((A, a, la), (B, b, lb))
            out.append((ca * cb, p, P, E))
    return out


def _single_list(bf: BasisFunctions, i: int):
    """A single function as a pair with an s function of exponent 0 at its center."""
    out = []
    for (A, a, la, ca) in _contracted(bf.prims[i]):
        p, P, E = _pair((A, a, la), (A, 0.0, (0, 0, 0)))
        out.append((ca, p, P, E))
    return out


def coulomb_2center_py(aux: BasisFunctions) -> np.ndarray:
    """(P|Q) over the pure auxiliary functions."""
    n = len(aux.prims)
    L = [_single_list(aux, i) for i in range(n)]
    V = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1):
            v = sum(c1 * c2 * _eri_pairs(p1, P1, E1, p2, P2, E2) for (c1, p1, P1, E1) in L[i] for (c2, p2, P2, E2) in L[j])
            V[i, j] = V[j, i] = v
    X = aux.cart_to_pure
    return X @ V @ X.T


def coulomb_3center_py(bf: BasisFunctions, aux: BasisFunctions) -> np.ndarray:
    """(mu nu|P) over pure functions, [nbf, nbf, naux]."""
    n, na = len(bf.prims), len(aux.prims)
    LA = [_single_list(aux, k) for k in range(na)]
    out = np.zeros((n, n, na))
    for i in range(n):
        for j in range(i + 1):
            pl = _pair_list(bf, i, j)
            for k in range(na):
                v = sum(c1 * c2 * _eri_pairs(p1, P1, E1, p2, P2, E2) for (c1, p1, P1, E1) in pl for (c2, p2, P2, E2) in LA[k])
                out[i, j, k] = out[j, i, k] = v
    X, Y = bf.cart_to_pure, aux.cart_to_pure
    return np.einsum("ai,bj,ijk,ck->abc", X, X, out, Y, optimize=True)


def coulomb_4center(bf: BasisFunctions) -> np.ndarray:
    """(mu nu|la si) over pure functions (small bases only: a cross-check of RI)."""
    n = len(bf.prims)
    pl = {(i, j): _pair_list(bf, i, j) for i in range(n) for j in range(i + 1)}
    out = np.zeros((n, n, n, n))
    keys = list(pl)
    for x, (i, j) in enumerate(keys):
        for (k, l) in keys[: x + 1]:
            v = sum(c1 * c2 * _eri_pairs(p1, P1, E1, p2, P2, E2) for (c1, p1, P1, E1) in pl[(i, j)]
                    for (c2, p2, P2, E2) in pl[(k, l)])
            for a, b in ((i, j), (j, i)):
                for c, d in ((k, l), (l, k)):
                    out[a, b, c, d] = out[c, d, a, b] = v
    X = bf.cart_to_pure
    return np.einsum("ai,bj,ck,dl,ijkl->abcd", X, X, X, X, out, optimize=True)


# ----------------------------------------------------------------------------- the same integrals in C
# gto_ints.c restates the scheme above over whole shells (one Boys evaluation
# per primitive combination); the Python functions stay as its cross-check.
_LIB_PATH = Path(__file__).with_name("libgto_ints.so")
_SRC_PATH = Path(__file__).with_name("gto_ints.c")
_lib = None


class _CShell(ctypes.Structure):
    _fields_ = [("x", ctypes.c_double), ("y", ctypes.c_double), ("z", ctypes.c_double),
                ("l", ctypes.c_int), ("nprim", ctypes.c_int),
                ("a", ctypes.POINTER(ctypes.c_double)), ("c", ctypes.POINTER(ctypes.c_double))]


def build_library(force: bool = False) -> Path:
    """Compile gto_ints.c next to it (gcc -O2); a no-op when the library is newer."""
    if force or not _LIB_PATH.exists() or _LIB_PATH.stat().st_mtime < _SRC_PATH.stat().st_mtime:
        subprocess.run(["gcc", "-O2", "-shared", "-fPIC", str(_SRC_PATH), "-o", str(_LIB_PATH), "-lm"], check=True)
    return _LIB_PATH


def _c_available() -> bool:
    global _lib
    if _lib is None:
        try:
            build_library()
            _lib = ctypes.CDLL(str(_LIB_PATH))
        except (OSError, subprocess.CalledProcessError, FileNotFoundError):
            _lib = False
    return bool(_lib)


def _c_shells(shells: list[Shell]):
    """ctypes shell array; coefficients carry the common primitive norm of each shell."""
    arr = (_CShell * len(shells))()
    keep = []
    for k, sh in enumerate(shells):
        a = np.ascontiguousarray(sh.alpha, dtype=float)
        c = np.ascontiguousarray([ck * primitive_norm(ak, (sh.am, 0, 0)) for ak, ck in zip(sh.alpha, sh.coeff)],
                                 dtype=float)
        keep += [a, c]
        x, y, z = (float(v) for v in sh.center)
        arr[k] = _CShell(x, y, z, sh.am, len(a), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                         c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return arr, keep


def _ptr(x: np.ndarray):
    return x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c_one_body(bf: BasisFunctions, nuclei):
    """Cartesian S, T, V from the C library."""
    arr, keep = _c_shells(bf.shells)
    n = len(bf.prims)
    S, T, V = (np.zeros((n, n)) for _ in range(3))
    zc = np.array([float(z) for z, _ in nuclei] or [0.0])
    xyz = np.array([list(map(float, c)) for _, c in nuclei] or [[0.0, 0.0, 0.0]]).ravel()
    _lib.gto_one_body(len(bf.shells), arr, len(nuclei), _ptr(zc), _ptr(xyz), _ptr(S), _ptr(T), _ptr(V))
    return S, T, V


def one_body(bf: BasisFunctions, nuclei) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Overlap, kinetic and nuclear-attraction matrices over the pure functions;
    ``nuclei`` = [(Z, (x, y, z)), ...] in Bohr."""
    if not _c_available():
        return one_body_py(bf, nuclei)
    S, T, V = _c_one_body(bf, nuclei)
    X = bf.cart_to_pure
    return X @ S @ X.T, X @ T @ X.T, X @ V @ X.T


def coulomb_2center(aux: BasisFunctions) -> np.ndarray:
    """(P|Q) over the pure auxiliary functions."""
    if not _c_available():
        return coulomb_2center_py(aux)
    arr, keep = _c_shells(aux.shells)
    n = len(aux.prims)
    V = np.zeros((n, n))
    _lib.gto_coulomb2(len(aux.shells), arr, _ptr(V))
    X = aux.cart_to_pure
    return X @ V @ X.T


def coulomb_3center(bf: BasisFunctions, aux: BasisFunctions) -> np.ndarray:
    """(mu nu|P) over pure functions, [nbf, nbf, naux]."""
    if not _c_available():
        return coulomb_3center_py(bf, aux)
    arr, keep = _c_shells(bf.shells)
    arra, keepa = _c_shells(aux.shells)
    n, na = len(bf.prims), len(aux.prims)
    out = np.zeros((n, n, na))
    _lib.gto_coulomb3(len(bf.shells), arr, len(aux.shells), arra, _ptr(out))
    X, Y = bf.cart_to_pure, aux.cart_to_pure
    return np.einsum("ai,bj,ijk,ck->abc", X, X, out, Y, optimize=True)


# ----------------------------------------------------------------------------- RI and SCF
def inverse_sqrt_metric(v2: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(P|Q)^-1/2 as the reference forms it: eigenvectors of the kept
    eigenvalues (> TOO_LOW_EIGENVAL) over the square roots of the eigenvalues,
    [naux_basis, nauxil_kept] (src/m_eri_calculate.f90:1093-1190)."""
    w, q = np.linalg.eigh(v2)
    keep = w > TOO_LOW_EIGENVAL
    return q[:, keep] / np.sqrt(w[keep]), w


@dataclass
class SCFResult:
    energy: float                  # total energy (Ha)
    e_orb: np.ndarray              # orbital energies (Ha)
    c: np.ndarray                  # [nbf, nstate] MO coefficients
    occupation: np.ndarray
    b3: np.ndarray                 # [nbf, nbf, nauxil] RI 3-center integrals
    fock_mo_diag: np.ndarray       # <p|F|p> of the final Fock matrix
    iterations: int
    metric_eigenvalues: np.ndarray


def rhf_ri(S, H, b3, nelec: int, e_nn: float = 0.0, tol: float = 1e-12, maxiter: int = 200) -> SCFResult:
    """Restricted HF with RI Coulomb and exchange; DIIS on the commutator FDS - SDF."""
    nocc = nelec // 2
    w, u = np.linalg.eigh(S)
    X = u / np.sqrt(w)
    D = np.zeros_like(S)
    fs, es = [], []
    e_old = 0.0

    def fock(D):
        J = np.einsum("ijP,P->ij", b3, np.einsum("klP,kl->P", b3, D))
        K = np.einsum("ikP,kl,ljP->ij", b3, D, b3, optimize=True)
        return H + J - 0.5 * K

    F = H.copy()
    for it in range(1, maxiter + 1):
        if fs:
            n = len(fs)
            B = -np.ones((n + 1, n + 1))
            B[n, n] = 0.0
            for a in range(n):
                for b in range(n):
                    B[a, b] = float(np.sum(es[a] * es[b]))
            rhs = np.zeros(n + 1)
            rhs[n] = -1.0
            coef = np.linalg.lstsq(B, rhs, rcond=None)[0][:n]
            Fx = sum(c * f for c, f in zip(coef, fs))
        else:
            Fx = F
        e, cp = np.linalg.eigh(X.T @ Fx @ X)
        C = X @ cp
        Dn = 2.0 * C[:, :nocc] @ C[:, :nocc].T
        F = fock(Dn)
        energy = 0.5 * float(np.sum(Dn * (H + F))) + e_nn
        err = F @ Dn @ S - S @ Dn @ F
        fs.append(F)
        es.append(err)
        if len(fs) > 8:
            fs.pop(0)
            es.pop(0)
        dd = np.abs(Dn - D).max()
        D = Dn
        if it > 2 and dd < tol and abs(energy - e_old) < tol:
            break
        e_old = energy
    # final orbitals from the Fock matrix of the converged density
    e, cp = np.linalg.eigh(X.T @ F @ X)
    C = X @ cp
    occ = np.zeros(C.shape[1])
    occ[:nocc] = 2.0
    fmo = np.einsum("ip,ij,jp->p", C, F, C)
    return SCFResult(energy, e, C, occ, b3, fmo, it, np.array([]))


def mo_3center(scf: SCFResult) -> np.ndarray:
    """eri_3center_mo(P, p, q) as [p, q, P] (calculate_eri_3center_mo, src/m_eri_ao_mo.f90:416-582)."""
    return np.einsum("ip,jq,ijP->pqP", scf.c, scf.c, scf.b3, optimize=True)


def atom_ri_hf(basis_text: str, z: int, nelec: int | None = None):
    """One atom at the origin: PAuto auxiliary basis, RI integrals, RI-RHF.
    Returns (SCFResult, M [nstate, nstate, nauxil] over the MOs, details)."""
    shells = parse_basis_file(basis_text)
    aux_shells = pauto_auxiliary(shells, z)
    bf = build_functions(shells)
    aux = build_functions(aux_shells)
    S, T, V = one_body(bf, [(z, (0.0, 0.0, 0.0))])
    v2 = coulomb_2center(aux)
    sqrtinv, eig = inverse_sqrt_metric(v2)
    b3 = np.einsum("ijQ,QP->ijP", coulomb_3center(bf, aux), sqrtinv)
    scf = rhf_ri(S, T + V, b3, z if nelec is None else nelec)
    scf.metric_eigenvalues = eig
    details = {"nbf": S.shape[0], "naux_basis": v2.shape[0], "nauxil": b3.shape[2],
               "aux_shells": [(s.am, float(s.alpha[0])) for s in aux_shells], "bf": bf, "aux": aux,
               "S": S, "H": T + V}
    return scf, mo_3center(scf), details


BOHR_A = 0.52917721092             # src/m_definitions.f90:43
HA_EV = 27.21138505                # src/m_definitions.f90:44


def nuclear_repulsion(nuclei) -> float:
    e = 0.0
    for i, (zi, ci) in enumerate(nuclei):
        for zj, cj in nuclei[:i]:
            e += zi * zj / float(np.linalg.norm(np.asarray(ci, float) - np.asarray(cj, float)))
    return e


def molecule_ri_hf(atoms, basis: dict, auxil: dict | str | None = None, charge: int = 0, tol: float = 1e-12,
                   cart: bool = False):
    """RI-RHF of a molecule.  ``atoms`` = [(Z, (x, y, z) in Angstrom), ...]
    (the reference's default length_unit, src/input_variables.f90:502);
    ``basis`` / ``auxil`` map Z to the text of a basis file in the reference's
    format; ``auxil`` None (or "PAUTO") builds the PAuto auxiliary basis per
    atom, "AUTO" the Auto one.  ``cart``: Cartesian functions for both bases
    (gaussian_type='CART'), else pure ones.  Shells
    are listed atom by atom in input order, as the reference does
    (src/m_basis_set.f90:90-340).  Returns (SCFResult, M [nstate, nstate,
    nauxil] over the MOs, details)."""
    nuclei = [(int(z), np.asarray(xyz, float) / BOHR_A) for z, xyz in atoms]
    shells, aux_shells = [], []
    for z, c in nuclei:
        sh = parse_basis_file(basis[z], center=tuple(c))
        shells += sh
        if isinstance(auxil, dict):
            aux_shells += parse_basis_file(auxil[z], center=tuple(c))
        else:
            aux_shells += pauto_auxiliary(sh, z, pauto=(auxil or "PAUTO").upper() == "PAUTO")
    bf = build_functions(shells, pure=not cart)
    aux = build_functions(aux_shells, pure=not cart)
    S, T, V = one_body(bf, nuclei)
    v2 = coulomb_2center(aux)
    sqrtinv, eig = inverse_sqrt_metric(v2)
    b3 = np.einsum("ijQ,QP->ijP", coulomb_3center(bf, aux), sqrtinv, optimize=True)
    nelec = sum(z for z, _ in nuclei) - charge
    e_nn = nuclear_repulsion(nuclei)
    scf = rhf_ri(S, T + V, b3, nelec, e_nn=e_nn, tol=tol)
    scf.metric_eigenvalues = eig
    details = {"nbf": S.shape[0], "naux_basis": v2.shape[0], "nauxil": b3.shape[2], "e_nn": e_nn,
               "bf": bf, "aux": aux, "S": S, "H": T + V, "T": T, "V": V}
    return scf, mo_3center(scf), details


def element_core(z: int) -> int:
    """Frozen core states per all-electron atom, frozencore='molgw'
    (element_core, src/m_elements.f90:40-68)."""
    return 0 if z <= 4 else 1 if z <= 12 else 5 if z <= 30 else 9 if z <= 48 else 18


def rimp2_energy(energy: np.ndarray, m: np.ndarray, nocc: int, ncore: int = 0) -> float:
    """Closed-shell RI-MP2 correlation energy from the MO 3-center tensor
    M[p, q, P] (mp2_energy_ri, src/m_mp2_energy.f90:25-143): the ring term
    2 sum (ia|jb)^2 / D and the exchange term -sum (ia|jb)(ib|ja) / D over
    i, j in ncore..nocc-1 and a, b >= nocc, D = e_i + e_j - e_a - e_b."""
    e = np.asarray(energy, float)
    mia = m[ncore:nocc, nocc:, :]
    iajb = np.einsum("iaP,jbP->iajb", mia, mia, optimize=True)
    eo, ev = e[ncore:nocc], e[nocc:]
    d = eo[:, None, None, None] + eo[None, None, :, None] - ev[None, :, None, None] - ev[None, None, None, :]
    return float(np.sum(iajb * (2.0 * iajb - iajb.transpose(0, 3, 2, 1)) / d))


def correlated_dm_energies(scf: SCFResult, details: dict, p_corr_mo: np.ndarray, spin_fact: float = 2.0) -> dict:
    """Energies of the correlated density matrix (get_dm_mbpt,
    src/m_dm_mbpt_driver.f90:228-249): P_AO = C (P_corr + diag(occupation)) C^T
    (update_density_matrix, src/m_mbpt_density_matrix.f90:840-880), kinetic and
    nuclear energies as traces, the RI Hartree energy 1/2 sum J P, and the RI
    exchange energy 1/2 sum K P with K built from the eigenvectors of P_AO whose
    eigenvalues are >= 1e-5 (get_c_matrix_from_p_matrix,
    src/m_hamiltonian_tools.f90:1356-1412; setup_exchange_ri,
    src/m_hamiltonian_twobodies.f90:707-784)."""
    c = scf.c
    p_mo = p_corr_mo + np.diag(scf.occupation)
    p_ao = c @ p_mo @ c.T
    b3 = scf.b3
    jmat = np.einsum("ijP,P->ij", b3, np.einsum("klP,kl->P", b3, p_ao))
    w, u = np.linalg.eigh(-p_ao)
    w = -w
    nocc = int(np.max(np.nonzero(w >= 1.0e-5)[0])) + 1 if np.any(w >= 1.0e-5) else 0
    ct = u[:, :nocc] * np.sqrt(np.maximum(w[:nocc], 0.0) / spin_fact)
    tmp = np.einsum("mnP,ni->imP", b3, ct, optimize=True)
    kmat = -np.einsum("imP,inP->mn", tmp, tmp, optimize=True)
    return {"kinetic": float(np.sum(details["T"] * p_ao)), "nucleus": float(np.sum(details["V"] * p_ao)),
            "hartree": 0.5 * float(np.sum(jmat * p_ao)), "exchange": 0.5 * float(np.sum(kmat * p_ao)),
            "trace_mo": float(np.trace(p_mo)), "p_ao": p_ao}
