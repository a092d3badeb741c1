"""CPU restatement of MOLGW's imaginary-frequency RI-GW path (test infrastructure).

This module is the ORACLE: only the test suite, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` import it, and
only as the checker or as the timed CPU baseline.  The product path (the CUDA
library under ``molgw_b200/csrc``) never calls into it.

Every function follows a routine of MOLGW 3.4 statement by statement and issues
the same BLAS/LAPACK call sequence (through SciPy's bundled OpenBLAS):

* ``coeffs_gausslegint``      src/m_numerical_tools.f90:35-82
* ``imaginary_quad_grid``     src/m_spectral_function.f90:286-306 (alpha=1, beta=2)
* ``transition_table``        src/m_spectral_function.f90:239-266, 359-378
* ``calculate_eri_3center_mo`` src/m_eri_ao_mo.f90:416-582
* ``polarizability_grid``     src/m_gw_selfenergy_grid.f90:33-209
                              (DSYRK('L','N') -> negate -> symmetrize -> 1-chi0 ->
                               DSYEV('N') -> LU inverse -> DGEMM)
* ``gw_selfenergy_imag``      src/m_gw_selfenergy_grid.f90:213-338
* ``selfenergy_set_state_range`` src/m_selfenergy_tools.f90:67-122
* ``se_init_imaginary_axis``  src/m_selfenergy_tools.f90:557-699
* ``pade`` / ``calculate_pade_a`` src/m_numerical_tools.f90:86-146
* ``se_pade_fit``             src/m_selfenergy_tools.f90:965-999
* ``self_energy_polynomial``  src/m_selfenergy_tools.f90:1005-1033
* ``find_qp_energy_linearization`` src/m_selfenergy_tools.f90:202-249
* ``find_qp_energy_graphical`` / ``find_fixed_point`` src/m_selfenergy_tools.f90:253-420
* ``output_homolumo``         src/m_hamiltonian_tools.f90:564-612
* ``sox_selfenergy_imag``     src/m_g3w2_selfenergy.f90:2482-2591 (GW+SOX on the
                              imaginary axis, added before the Pade fit,
                              src/m_selfenergy_evaluation.f90:494-503)
* ``sosex_selfenergy_imag``   src/m_g3w2_selfenergy.f90:2200-2478 (GW+SOSEX on the
                              imaginary axis, after SOX, :498-500)
* ``g3w2_selfenergy_imag``    src/m_g3w2_selfenergy.f90:2018-2196 (GW+G3W2 on the
                              imaginary axis, after SOSEX, :501-503)

Pinning: the reference's own known answer that needs no Gaussian integrals is
the analytic RPA correlation energy of bulk LiH from the shipped CC4S tensor
(tests/inputs/testsuite:1206-1207, -0.1152301335 Ha, tol 1e-7).  The analytic
RPA of this module reproduces it to 1e-7, and the imaginary-axis RPA of
``polarizability_grid`` converges to it with the number of frequencies (see
tests/test_oracle.py).  The H2O GW values of the reference suite need an SCF with
Gaussian integrals and are not reproducible here.

Units: Hartree.  Arrays are numpy, with the Fortran index order kept in the
shapes (``m_ia`` is ``[nocc, nvirt, naux]`` in C order, i.e. the Fortran
``eri_3center_mo(naux, a, i)`` column-major array).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla
from scipy.linalg import blas as sblas
from scipy.linalg import lapack as slapack

HA_EV = 27.21138505            # src/m_definitions.f90:43
PI = 3.14159265358979323       # src/m_definitions.f90:50
COMPLETELY_EMPTY = 1.0e-5      # src/m_definitions.f90:66


# ---------------------------------------------------------------------------
# Frequency grids
# ---------------------------------------------------------------------------
def coeffs_gausslegint(xmin: float, xmax: float, n: int):
    """Gauss-Legendre nodes/weights by Newton iteration, tol 1e-13.

    Follows src/m_numerical_tools.f90:35-82 (Rybicki's routine) literally.
    """
    x = np.zeros(n)
    w = np.zeros(n)
    tol = 1.0e-13
    xl = (xmax - xmin) * 0.5
    xmean = (xmax + xmin) * 0.5
    for i in range(1, (n + 1) // 2 + 1):
        z = math.cos(PI * (i - 0.25) / (n + 0.5))
        while True:
            p1 = 1.0
            p2 = 0.0
            for j in range(1, n + 1):
                p3 = p2
                p2 = p1
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j
            pp = n * (p2 - z * p1) / (1.0 - z * z)
            z1 = z
            z = z1 - p1 / pp
            if abs(z - z1) < tol:
                break
        x[i - 1] = xmean - xl * z
        x[n - i] = xmean + xl * z
        w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp)
        w[n - i] = w[i - 1]
    return x, w


def imaginary_quad_grid(nomega: int):
    """Imaginary-frequency grid of sf_init(IMAGINARY_QUAD).

    src/m_spectral_function.f90:286-306 with alpha=1, beta=2 (:155-156):
    w_k <- w_k/(2^a-1)*a*(1-x_k)^(-a-1)*b ;  omega_k = 1/(2^a-1)*((1-x_k)^-a - 1)*b.
    Returns (omega_imag, weight); the frequencies are i*omega_imag.
    """
    alpha, beta = 1.0, 2.0
    x, w = coeffs_gausslegint(0.0, 1.0, nomega)
    weight = w / (2.0 ** alpha - 1.0) * alpha * (1.0 - x) ** (-alpha - 1.0) * beta
    omega = 1.0 / (2.0 ** alpha - 1.0) * (1.0 / (1.0 - x) ** alpha - 1.0) * beta
    return omega, weight


# ---------------------------------------------------------------------------
# Transition space
# ---------------------------------------------------------------------------
def transition_table(occupation: np.ndarray, ncore_w: int = 0, nvirtual_w: int | None = None,
                     spin_fact: float = 2.0):
    """Resonant transitions (i, a), i outer / a inner, 1-based state indices.

    src/m_spectral_function.f90:239-266 with skip_transition :359-378 (nspin=1).
    """
    nstate = occupation.shape[0]
    if nvirtual_w is None:
        nvirtual_w = nstate + 1
    table = []
    for istate in range(1, nstate + 1):
        for jstate in range(1, nstate + 1):
            o1 = occupation[jstate - 1]
            o2 = occupation[istate - 1]
            skip = False
            if jstate <= ncore_w or istate <= ncore_w:
                skip = True
            if jstate >= nvirtual_w or istate >= nvirtual_w:
                skip = True
            if o1 < COMPLETELY_EMPTY and o2 < COMPLETELY_EMPTY:
                skip = True
            if o1 > spin_fact - COMPLETELY_EMPTY and o2 > spin_fact - COMPLETELY_EMPTY:
                skip = True
            if skip:
                continue
            if o1 - o2 > 0.0:
                continue
            table.append((istate, jstate))
    return np.array(table, dtype=np.int64).reshape(-1, 2)


# ---------------------------------------------------------------------------
# AO -> MO transform of the RI 3-center integrals
# ---------------------------------------------------------------------------
def calculate_eri_3center_mo(eri3: np.ndarray, index_basis: np.ndarray, c: np.ndarray,
                             m_min: int, m_max: int, n_min: int, n_max: int) -> np.ndarray:
    """M(P, m, n) = sum_{mu nu} C_{mu m} C_{nu n} B(mu nu, P).

    src/m_eri_ao_mo.f90:416-582.  ``eri3`` is ``[naux, npair]`` (the Fortran
    ``eri_3center(npair, naux)`` column-major array), ``index_basis`` is
    ``[npair, 2]`` 1-based basis indices (src/m_eri.f90:252-320), diagonal pairs
    carry the x0.5 convention of src/m_eri_calculate.f90:1841,1854.  ``c`` is
    ``[nstate, nbf]`` (Fortran ``c_matrix(nbf, nstate)``).  State ranges are
    1-based inclusive.  Returns ``[n_count, m_count, naux]`` (Fortran
    ``eri_3center_mo(naux, m, n)``).
    """
    naux, npair = eri3.shape
    nbf = c.shape[1]
    ms = slice(m_min - 1, m_max)
    ns = slice(n_min - 1, n_max)
    c_t = c[ns, :]                       # c_t(n, nbf) = TRANSPOSE(c_matrix(:, n))
    kbf = index_basis[:, 0] - 1
    lbf = index_basis[:, 1] - 1
    out = np.zeros((n_max - n_min + 1, m_max - m_min + 1, naux))
    for p in range(naux):
        # pair loop (OpenMP reduction in the reference), :515-524
        tmp1 = np.zeros((c_t.shape[0], nbf))
        b = eri3[p]
        np.add.at(tmp1.T, kbf, (c_t[:, lbf] * b).T)
        np.add.at(tmp1.T, lbf, (c_t[:, kbf] * b).T)
        # DGEMM('T','T') :527-530 -> tmp2(m, n) = C(:,m)^T tmp1(n,:)^T
        tmp2 = c[ms, :] @ tmp1.T
        out[:, :, p] = tmp2.T
    return out


# ---------------------------------------------------------------------------
# chi0 / epsilon / chi on the imaginary axis
# ---------------------------------------------------------------------------
@dataclass
class SpectralFunction:
    """Container of src/m_spectral_function.f90:48-91 (the fields the path uses)."""
    omega: np.ndarray            # imaginary parts
    weight_quad: np.ndarray
    chi: np.ndarray | None = None   # [nomega, naux, naux]
    erpa: float = 0.0
    egw: float = 0.0
    eigval: list = field(default_factory=list)


def polarizability_grid(m_ia: np.ndarray, e_occ: np.ndarray, e_virt: np.ndarray,
                        occ_occ: np.ndarray, occ_virt: np.ndarray,
                        omega: np.ndarray, weight: np.ndarray, keep_chi: bool = True,
                        keep_eigval: bool = False, spin2: tuple | None = None) -> SpectralFunction:
    """RPA polarizability on the imaginary grid, src/m_gw_selfenergy_grid.f90:33-209.

    ``m_ia`` is ``[nocc, nvirt, naux]`` (transition t = (i, a), a fastest, as the
    transition table orders them).  Per frequency: scale M by
    sqrt(2*docc*de/(w^2+de^2)) (:126-137), DSYRK('L','N') (:145-149), chi0 = -chi0,
    symmetrize lower->upper (src/m_scalapack.f90:2461-2551 serial branch), 1-chi0,
    DSYEV('N') eigenvalues -> E_RPA, E_GW (:171-173), DGETRF/DGETRI inverse
    (src/m_linear_algebra.f90:179-205), DGEMM chi = (1-chi0)^-1 chi0 (:179-188).

    ``spin2`` = (m_ia, e_occ, e_virt, occ_occ, occ_virt) of the second spin channel:
    its transitions follow those of the first, as the spin index of the transition
    table orders them (src/m_spectral_function.f90:239-266), in the same DSYRK.
    """
    nocc, nvirt, naux = m_ia.shape
    docc = (occ_occ[:, None] - occ_virt[None, :]).reshape(-1)
    de = (e_virt[None, :] - e_occ[:, None]).reshape(-1)
    m_t = np.ascontiguousarray(m_ia.reshape(nocc * nvirt, naux).T)   # eri3(naux, t), Fortran order
    if spin2 is not None:
        m2, eo2, ev2, oo2, ov2 = spin2
        docc = np.concatenate([docc, (oo2[:, None] - ov2[None, :]).reshape(-1)])
        de = np.concatenate([de, (ev2[None, :] - eo2[:, None]).reshape(-1)])
        m_t = np.ascontiguousarray(np.concatenate([m_t, m2.reshape(-1, naux).T], axis=1))
    sf = SpectralFunction(omega=omega.copy(), weight_quad=weight.copy())
    if keep_chi:
        sf.chi = np.zeros((len(omega), naux, naux))
    erpa = 0.0
    egw = 0.0
    for iw, w in enumerate(omega):
        factor_sqrt = np.sqrt(2.0 * docc * de / (w * w + de * de))
        eri3_t = np.asfortranarray(m_t * factor_sqrt[None, :])
        chi0 = sblas.dsyrk(1.0, eri3_t, lower=1, trans=0)          # lower triangle
        chi0 = -chi0
        il = np.tril_indices(naux, -1)
        chi0 = np.tril(chi0)
        chi0[il[1], il[0]] = chi0[il]                              # symmetrize_matrix_sca('L')
        one_m_chi0 = -chi0
        one_m_chi0[np.diag_indices(naux)] += 1.0
        eigval = sla.eigvalsh(one_m_chi0, driver="ev")             # DSYEV('N')
        if keep_eigval:
            sf.eigval.append(eigval)
        erpa += np.sum(np.log(eigval) + 1.0 - eigval) / (2.0 * PI) * weight[iw]
        egw += np.sum(-(1.0 - eigval) / eigval + 1.0 - eigval) / (2.0 * PI) * weight[iw]
        if keep_chi:
            lu, piv, info = slapack.dgetrf(one_m_chi0)
            if info != 0:
                raise ArithmeticError(f"dgetrf info={info}")
            inv, info = slapack.dgetri(lu, piv)
            if info != 0:
                raise ArithmeticError(f"dgetri info={info}")
            sf.chi[iw] = sblas.dgemm(1.0, inv, chi0)
    sf.erpa = erpa
    sf.egw = egw
    return sf


def analytic_rpa_correlation(m_ia: np.ndarray, e_occ: np.ndarray, e_virt: np.ndarray) -> float:
    """Closed-shell direct-RPA correlation energy from the Casida problem.

    MOLGW's analytic RPA (postscf='RPA', src/m_acfd.f90:104-107 ->
    src/m_linear_response.f90 polarizability, get_rpa_correlation
    src/m_build_bse.f90:287-314) is E_c = 1/2 sum_n Omega_n - 1/4 tr(A+B) - 1/4 tr(A-B)
    with A+B = de + 4K, A-B = de (singlet), K_{ia,jb} = sum_P M_Pia M_Pjb.
    Omega^2 are the eigenvalues of (A-B)^1/2 (A+B) (A-B)^1/2.
    """
    nocc, nvirt, naux = m_ia.shape
    de = (e_virt[None, :] - e_occ[:, None]).reshape(-1)
    m = m_ia.reshape(nocc * nvirt, naux)
    k = m @ m.T
    apb = np.diag(de) + 4.0 * k
    amb = np.diag(de)
    sq = np.sqrt(de)
    c = sq[:, None] * apb * sq[None, :]
    omega2 = sla.eigvalsh(c)
    omega_n = np.sqrt(omega2)
    return 0.5 * np.sum(omega_n) - 0.25 * np.trace(apb) - 0.25 * np.trace(amb)


# ---------------------------------------------------------------------------
# Self-energy on the imaginary axis
# ---------------------------------------------------------------------------
@dataclass
class StateRange:
    """Module variables set by selfenergy_set_state_range (1-based)."""
    ncore_g: int
    nvirtual_g: int
    nhomo_g: int
    nlumo_g: int
    nsemin: int
    nsemax: int


def selfenergy_set_state_range(nstate: int, occupation: np.ndarray, ncoreg: int = 0,
                               nvirtualg: int = 100000, selfenergy_state_min: int = 1,
                               selfenergy_state_max: int = 100000,
                               selfenergy_state_range: int = 100000) -> StateRange:
    """src/m_selfenergy_tools.f90:67-122 (no frozen-core atom tables: ncoreg given)."""
    ncore_g = ncoreg
    nvirtual_g = min(nvirtualg, nstate + 1)
    nhomo_g = 1
    for p in range(1, nstate + 1):
        if not occupation[p - 1] < COMPLETELY_EMPTY:
            nhomo_g = max(nhomo_g, p)
    nlumo_g = 100000
    for p in range(1, nstate + 1):
        if not occupation[p - 1] > COMPLETELY_EMPTY:
            nlumo_g = min(nlumo_g, p)
    nsemin = max(ncore_g + 1, selfenergy_state_min, 1, nhomo_g - selfenergy_state_range)
    nsemax = min(nvirtual_g - 1, selfenergy_state_max, nstate, nhomo_g + selfenergy_state_range)
    return StateRange(ncore_g, nvirtual_g, nhomo_g, nlumo_g, nsemin, nsemax)


@dataclass
class SelfEnergyGrid:
    """selfenergy_grid type, src/m_selfenergy_tools.f90:45-60 (one spin)."""
    omega: np.ndarray            # real grid, index -nomega..nomega -> [0..2*nomega]
    omega_calc: np.ndarray       # complex evaluation points
    energy0: np.ndarray          # per state of the range
    sigma: np.ndarray | None = None        # [2*nomega+1, nstate_range] complex
    sigma_calc: np.ndarray | None = None   # [nomega_calc, nstate_range] complex

    @property
    def nomega(self) -> int:
        return (len(self.omega) - 1) // 2


def fermi_level(energy0: np.ndarray, nhomo_g: int, mu_origin: float = -100.0) -> float:
    """efermi of se_init, src/m_selfenergy_tools.f90:573-596."""
    if mu_origin > -99.0:
        if mu_origin < energy0[nhomo_g - 1] or mu_origin > energy0[nhomo_g]:
            raise ValueError("se_init: efermi needs to be in the HOMO-LUMO gap")
        return mu_origin
    return 0.5 * (energy0[nhomo_g - 1] + energy0[nhomo_g])


def se_init_imaginary_axis(energy0: np.ndarray, rng: StateRange, technique: str = "pade",
                           nomega_sigma: int = 51, step_sigma: float = 0.01,
                           nomega_sigma_calc: int = 1, step_sigma_calc: float = 0.03,
                           mu_origin: float = -100.0, efermi: float | None = None) -> SelfEnergyGrid:
    """se_init for imaginary_axis_pade / imaginary_axis_homolumo, :557-699.
    ``efermi``: the value over both spin channels (nspin = 2), else from energy0."""
    if efermi is None:
        efermi = fermi_level(energy0, rng.nhomo_g, mu_origin)
    nom = nomega_sigma // 2
    omega = efermi + step_sigma * np.arange(-nom, nom + 1, dtype=np.float64)
    if technique == "pade":
        omega_calc = efermi + step_sigma_calc * np.arange(nomega_sigma_calc) * 1j
    elif technique == "homolumo":
        eh = energy0[rng.nhomo_g - 1]
        el = energy0[rng.nhomo_g]
        omega_calc = (eh + 0.01 + np.arange(nomega_sigma_calc) / (nomega_sigma_calc - 1.0)
                      * (el - eh - 0.02)).astype(np.complex128)
    else:
        raise ValueError(technique)
    ns = rng.nsemax - rng.nsemin + 1
    return SelfEnergyGrid(omega=omega, omega_calc=omega_calc, energy0=np.zeros(ns),
                          sigma=np.zeros((2 * nom + 1, ns), dtype=np.complex128),
                          sigma_calc=np.zeros((nomega_sigma_calc, ns), dtype=np.complex128))


def gw_selfenergy_imag(energy: np.ndarray, m_sigma: np.ndarray, sf: SpectralFunction,
                       omega_calc: np.ndarray, pstate_first: int) -> np.ndarray:
    """Sigma_c on the evaluation points, src/m_gw_selfenergy_grid.f90:213-338.

    ``m_sigma`` is ``[nsig, prange, naux]`` (Fortran ``eri_3center_mo(naux, p, m)``
    for p = ncore_G+1..nvirtual_G-1, m = nsemin..nsemax).  ``pstate_first`` is
    ncore_G+1 (1-based).  Returns sigma_calc ``[nomega_calc, nsig]``.
    """
    nsig, prange, naux = m_sigma.shape
    sig = np.zeros((len(omega_calc), nsig), dtype=np.complex128)
    e_p = energy[pstate_first - 1: pstate_first - 1 + prange]
    for m in range(nsig):
        eri3 = np.asfortranarray(m_sigma[m].T)                  # (naux, prange)
        for iw in range(len(sf.omega)):
            chi_eri3 = sblas.dgemm(1.0, sf.chi[iw], eri3)       # DGEMM('N','N') :297-300
            v_chi_v = np.einsum("ij,ij->j", eri3, chi_eri3)     # DOT_PRODUCT per p :307
            om = 1j * sf.omega[iw]
            a = omega_calc[:, None] - e_p[None, :]
            fac = 1.0 / (a + om) + 1.0 / (a - om)
            sig[:, m] -= sf.weight_quad[iw] * (fac * v_chi_v[None, :]).sum(axis=1) / (2.0 * PI)
    return sig


# ---------------------------------------------------------------------------
# Analytic continuation
# ---------------------------------------------------------------------------
def calculate_pade_a(z_in: np.ndarray, f_in: np.ndarray) -> np.ndarray:
    """Thiele continued-fraction coefficients, src/m_numerical_tools.f90:120-146."""
    n = len(z_in)
    g = np.zeros((n, n), dtype=np.complex128)
    g[0, :] = f_in
    for ip in range(1, n):
        for jp in range(ip, n):
            g[ip, jp] = (g[ip - 1, ip - 1] - g[ip - 1, jp]) / ((z_in[jp] - z_in[ip - 1]) * g[ip - 1, jp])
    return np.diag(g).copy()


def pade_eval(aa: np.ndarray, z_in: np.ndarray, z_out: complex) -> complex:
    """Continued-fraction evaluation of src/m_numerical_tools.f90:86-116."""
    n = len(z_in)
    az_m1, az = 0.0 + 0.0j, aa[0]
    bz_m1, bz = 1.0 + 0.0j, 1.0 + 0.0j
    for ip in range(1, n):
        az_new = az + (z_out - z_in[ip - 1]) * aa[ip] * az_m1
        bz_new = bz + (z_out - z_in[ip - 1]) * aa[ip] * bz_m1
        az_m1, az = az, az_new
        bz_m1, bz = bz, bz_new
    return az / bz


def pade(z_in: np.ndarray, f_in: np.ndarray, z_out: complex) -> complex:
    """pade(), src/m_numerical_tools.f90:86-116 (coefficients are recomputed per call,
    exactly as the reference does; they depend on z_in, f_in only)."""
    return pade_eval(calculate_pade_a(z_in, f_in), z_in, z_out)


def se_pade_fit(se: SelfEnergyGrid, eta: float) -> None:
    """src/m_selfenergy_tools.f90:965-999: symmetric data on 2*Nc-1 points, then
    Thiele continuation to omega_j + i*eta*sign with sign = -sgn(omega_j - Re z_1)."""
    nc = len(se.omega_calc)
    for s in range(se.sigma_calc.shape[1]):
        omega_sym = np.zeros(2 * nc - 1, dtype=np.complex128)
        sigma_sym = np.zeros(2 * nc - 1, dtype=np.complex128)
        omega_sym[nc - 1] = se.omega_calc[0]
        sigma_sym[nc - 1] = se.sigma_calc[0, s]
        for k in range(2, nc + 1):
            omega_sym[nc + k - 2] = se.omega_calc[k - 1]
            sigma_sym[nc + k - 2] = se.sigma_calc[k - 1, s]
            omega_sym[nc - k] = np.conj(se.omega_calc[k - 1])
            sigma_sym[nc - k] = np.conj(se.sigma_calc[k - 1, s])
        aa = calculate_pade_a(omega_sym, sigma_sym)
        for j, w in enumerate(se.omega):
            sign_eta = -math.copysign(1.0, w - se.omega_calc[0].real)
            se.sigma[j, s] = pade_eval(aa, omega_sym, w + 1j * eta * sign_eta)


def self_energy_polynomial(se: SelfEnergyGrid) -> None:
    """Quadratic fit for imaginary_axis_homolumo, src/m_selfenergy_tools.f90:1005-1033."""
    nc = len(se.omega_calc)
    mid = nc // 2          # Fortran nomega_calc/2+1, 1-based
    for s in range(se.sigma_calc.shape[1]):
        sc = se.sigma_calc[:, s]
        a0 = sc[mid].real
        a1 = (sc[nc - 1].real - sc[0].real) / (se.omega_calc[nc - 1].real - se.omega_calc[0].real)
        a2 = (sc[nc - 1].real + sc[0].real - 2.0 * sc[mid].real) \
            / (se.omega_calc[nc - 1].real - se.omega_calc[0].real) ** 2 * 2.0
        d = se.omega - se.omega_calc[mid]
        se.sigma[:, s] = a0 + a1 * d + a2 * d * d


# ---------------------------------------------------------------------------
# Quasiparticle equation
# ---------------------------------------------------------------------------
def find_fixed_point(xx: np.ndarray, fx: np.ndarray, nfpmx: int = 4):
    """Sign changes of f(x)-x with Z weights, src/m_selfenergy_tools.f90:367-420."""
    z_weight = -np.ones(nfpmx)
    efp = np.zeros(nfpmx)
    gx = fx - xx
    for ix in range(len(xx) - 1):
        if gx[ix] * gx[ix + 1] < 0.0:
            z_zero = 1.0 / (1.0 - (fx[ix + 1] - fx[ix]) / (xx[ix + 1] - xx[ix]))
            if z_zero < 0.00001:
                continue
            if z_zero > z_weight[nfpmx - 1]:
                cand = [k for k in range(nfpmx) if z_zero > z_weight[k]]
                jf = min(cand)
                z_weight[jf + 1:] = z_weight[jf:nfpmx - 1].copy()
                efp[jf + 1:] = efp[jf:nfpmx - 1].copy()
                z_weight[jf] = z_zero
                gpxi = (gx[ix + 1] - gx[ix]) / (xx[ix + 1] - xx[ix])
                efp[jf] = xx[ix] - gx[ix] / gpxi
    return efp, z_weight


def find_qp_energy_linearization(se: SelfEnergyGrid, exchange_m_vxc: np.ndarray,
                                 energy0: np.ndarray):
    """src/m_selfenergy_tools.f90:202-249 (range states; zz present)."""
    nom = se.nomega
    if nom > 0:
        zz = (se.sigma[nom + 1].real - se.sigma[nom - 1].real) / (se.omega[nom + 1] - se.omega[nom - 1]).real
        zz = 1.0 / (1.0 - zz)
        zz = np.minimum(np.maximum(zz, 0.0), 1.0)
        eqp = se.energy0 + zz * (energy0 - se.energy0 + se.sigma[nom].real + exchange_m_vxc)
    else:
        zz = np.ones_like(energy0)
        eqp = energy0 + se.sigma[nom].real + exchange_m_vxc
    return eqp, zz


def find_qp_energy_graphical(se: SelfEnergyGrid, exchange_m_vxc: np.ndarray, energy0: np.ndarray):
    """src/m_selfenergy_tools.f90:253-363 for the states of the range.

    Returns (energy_qp_g, zz, fixed_points, z_weights).
    """
    ns = len(energy0)
    nom = se.nomega
    eqp = np.zeros(ns)
    zz = np.zeros(ns)
    efps = np.zeros((ns, 4))
    zws = np.zeros((ns, 4))
    if nom > 0:
        for s in range(ns):
            lhs = se.omega.real + se.energy0[s]
            rhs = se.sigma[:, s].real + exchange_m_vxc[s] + energy0[s]
            efp, zw = find_fixed_point(lhs, rhs)
            efps[s], zws[s] = efp, zw
            if zw.max() > 1.0e-6:
                iqp = int(np.argmax(zw))
                eqp[s] = efp[iqp]
                zz[s] = zw[iqp]
            else:
                eqp[s] = energy0[s]
                zz[s] = 1.0
            if np.count_nonzero(zw > 0.0) == 0:
                eqp[s] = energy0[s] + se.sigma[nom, s].real + exchange_m_vxc[s]
    else:
        eqp = energy0 + se.sigma[nom].real + exchange_m_vxc
        zz[:] = 1.0
    return eqp, zz, efps, zws


def output_homolumo(occupation: np.ndarray, energy: np.ndarray, istate_min: int, istate_max: int,
                    spin_fact: float = 2.0):
    """HOMO/LUMO over a state range for one spin channel, src/m_hamiltonian_tools.f90:564-612
    (spin_fact 2 for nspin = 1, 1 for a channel of nspin = 2)."""
    ehomo, elumo = -np.inf, np.inf
    for s in range(istate_min, istate_max + 1):
        if occupation[s - 1] / spin_fact > COMPLETELY_EMPTY:
            ehomo = max(ehomo, energy[s - 1])
        if occupation[s - 1] / spin_fact < 1.0 - COMPLETELY_EMPTY:
            elumo = min(elumo, energy[s - 1])
    return ehomo, elumo


# ---------------------------------------------------------------------------
# One-shot G0W0 on the imaginary axis (the path of selfenergy_evaluation)
# ---------------------------------------------------------------------------
@dataclass
class G0W0Result:
    erpa: float
    egw: float
    sigma_calc: np.ndarray       # [Nc, nsig] complex
    sigma: np.ndarray            # [Nsigma, nsig] complex (real grid)
    energy_qp_g: np.ndarray      # graphical, per range state
    energy_qp_z: np.ndarray      # linearized
    zz: np.ndarray
    ehomo: float
    elumo: float
    nsemin: int
    nsemax: int


def g0w0_imag(energy: np.ndarray, occupation: np.ndarray, m_ia: np.ndarray, m_sigma: np.ndarray,
              nomega_chi_imag: int, rng: StateRange, nomega_sigma: int = 51,
              step_sigma: float = 0.01, nomega_sigma_calc: int = 50,
              step_sigma_calc: float = 0.075, eta: float = 0.01,
              exchange_m_vxc: np.ndarray | None = None, technique: str = "pade",
              ncore_w: int = 0, energy_g: np.ndarray | None = None, sox: bool = False,
              m_ov_g: np.ndarray | None = None, factor_sosex: float | None = None,
              m_full: np.ndarray | None = None, g3w2: bool = False,
              freq: tuple | None = None, mu_origin: float = -100.0) -> G0W0Result:
    """Path of selfenergy_evaluation for imaginary_axis_pade / _homolumo
    (src/m_selfenergy_evaluation.f90:214-246, 587-611).

    ``m_ia`` is the W-window tensor ``[nocc_w, nvirt_w, naux]``; ``m_sigma`` is
    ``[nsig, prange, naux]`` with p = ncore_G+1.. nvirtual_G-1.

    ``energy_g`` (default ``energy``) are the energies in G, as read from
    ENERGY_QP under force_energy_qp (:164-181): se%init and the Sigma sum take
    them, W (energy_w = energy for GW) and the energy0 of the QP equation
    (find_qp_energy_*(se, ..., energy, ...), :587-590) keep ``energy``.  On the
    vertex path (``sox``, ``factor_sosex`` or ``g3w2``) the reference calls
    gw_selfenergy_grid with energy_g (:496), which builds its own W from that
    argument (src/m_gw_selfenergy_grid.f90:604), so W there takes ``energy_g``.

    ``sox``: GW+SOX_PADE, Sigma^SOX from energy_g added to sigma_calc before the
    fit (:494-503); ``m_ov_g`` is the occupied x empty block of the G window
    (default ``m_ia``, the W window, when both windows start at the same state).
    ``factor_sosex``: GW+SOSEX_PADE (GW+2SOSEX_PADE with 2), SOX and then
    factor_sosex x SOSEX added (:496-500); ``m_full`` is the G-window tensor
    [nstate_G, nstate_G, naux].  ``g3w2``: the G3W2 term added last (:501-503);
    GW+G3W2_PADE is sox=True, factor_sosex=2, g3w2=True.
    ``freq`` = (omega, weight) replaces the Gauss-Legendre grid of W (wpol%omega,
    wpol%weight_quad), e.g. a subset of it for one rank of the frequency split.
    ``mu_origin``: the input variable of that name, the origin of the imaginary
    axis of the evaluation points when > -99 (src/m_selfenergy_tools.f90:573-585).
    """
    eg = energy if energy_g is None else energy_g
    ew = eg if (sox or factor_sosex is not None or g3w2) else energy
    occ_w = occupation[ncore_w:ncore_w + m_ia.shape[0]]
    e_occ = ew[ncore_w:ncore_w + m_ia.shape[0]]
    nlumo = ncore_w + m_ia.shape[0]
    e_virt = ew[nlumo:nlumo + m_ia.shape[1]]
    occ_v = occupation[nlumo:nlumo + m_ia.shape[1]]
    omega, weight = imaginary_quad_grid(nomega_chi_imag) if freq is None else freq
    sf = polarizability_grid(m_ia, e_occ, e_virt, occ_w, occ_v, omega, weight)
    se = se_init_imaginary_axis(eg, rng, technique, nomega_sigma, step_sigma,
                                nomega_sigma_calc, step_sigma_calc, mu_origin=mu_origin)
    se.sigma_calc[:] = gw_selfenergy_imag(eg, m_sigma, sf, se.omega_calc, rng.ncore_g + 1)
    if sox:
        mov = m_ia if m_ov_g is None else m_ov_g
        if m_ov_g is None and ncore_w != rng.ncore_g:
            raise ValueError("sox: pass m_ov_g when the W and G windows differ")
        window = eg[rng.ncore_g: rng.ncore_g + m_sigma.shape[1]]
        se.sigma_calc += sox_selfenergy_imag(window, m_sigma, mov, se.omega_calc).T
    if factor_sosex is not None:
        window = eg[rng.ncore_g: rng.ncore_g + m_sigma.shape[1]]
        sig = list(range(rng.nsemin - 1 - rng.ncore_g, rng.nsemax - rng.ncore_g))
        se.sigma_calc += sosex_selfenergy_imag(window, m_full, rng.nhomo_g - rng.ncore_g, sig, sf.chi, sf.omega,
                                               sf.weight_quad, se.omega_calc, factor_sosex).T
    if g3w2:
        window = eg[rng.ncore_g: rng.ncore_g + m_sigma.shape[1]]
        sig = list(range(rng.nsemin - 1 - rng.ncore_g, rng.nsemax - rng.ncore_g))
        se.sigma_calc += g3w2_selfenergy_imag(window, m_full, sig, sf.chi, sf.omega, sf.weight_quad,
                                              se.omega_calc).T
    if technique == "pade":
        se_pade_fit(se, eta)
    else:
        self_energy_polynomial(se)
    e0 = energy[rng.nsemin - 1: rng.nsemax]
    xc = np.zeros_like(e0) if exchange_m_vxc is None else exchange_m_vxc
    eqp_z, zz = find_qp_energy_linearization(se, xc, e0)
    eqp_g, zz_g, _, _ = find_qp_energy_graphical(se, xc, e0)
    full = energy.copy()
    full[rng.nsemin - 1: rng.nsemax] = eqp_g
    ehomo, elumo = output_homolumo(occupation, full, rng.nsemin, rng.nsemax)
    return G0W0Result(sf.erpa, sf.egw, se.sigma_calc.copy(), se.sigma.copy(), eqp_g, eqp_z, zz_g,
                      ehomo, elumo, rng.nsemin, rng.nsemax)


def fermi_level_spin(energy0_spins: list, nhomo_g: int) -> float:
    """efermi of se_init over spin channels, src/m_selfenergy_tools.f90:584-585:
    0.5 (max over spins of energy0(nhomo_G) + min over spins of energy0(nhomo_G+1))."""
    return 0.5 * (max(e[nhomo_g - 1] for e in energy0_spins) + min(e[nhomo_g] for e in energy0_spins))


def g0w0_imag_spin(channels: list, nomega_chi_imag: int, nomega_sigma: int = 51, step_sigma: float = 0.01,
                   nomega_sigma_calc: int = 50, step_sigma_calc: float = 0.075, eta: float = 0.01,
                   technique: str = "pade", sox: bool = False) -> list:
    """Open-shell (nspin = 2) selfenergy_evaluation for imaginary_axis_pade /
    _homolumo: one W from the transitions of both channels
    (src/m_gw_selfenergy_grid.f90:118-149), Sigma per spin (:279-319), the QP
    equation per spin, se_init's efermi over both spins.

    ``channels``: two dicts with energy, occupation (1 or 0), m_ia [nocc, nvirt,
    naux], m_sigma [nsig, nstate, naux], nsemin, nsemax (1-based).  Returns one
    G0W0Result per channel (E_RPA and E_GW of the whole W in each)."""
    c1, c2 = channels
    no1, no2 = c1["m_ia"].shape[0], c2["m_ia"].shape[0]
    omega, weight = imaginary_quad_grid(nomega_chi_imag)
    blk = lambda c, no: (c["m_ia"], c["energy"][:no], c["energy"][no:no + c["m_ia"].shape[1]],
                         c["occupation"][:no], c["occupation"][no:no + c["m_ia"].shape[1]])
    sf = polarizability_grid(*blk(c1, no1), omega, weight, spin2=blk(c2, no2))
    nhomo = max(no1, no2)
    efermi = fermi_level_spin([c1["energy"], c2["energy"]], nhomo)
    out = []
    for c in channels:
        nstate = c["energy"].size
        rng = StateRange(0, nstate + 1, nhomo, nhomo + 1, c["nsemin"], c["nsemax"])
        se = se_init_imaginary_axis(c["energy"], rng, technique, nomega_sigma, step_sigma, nomega_sigma_calc,
                                    step_sigma_calc, efermi=efermi)
        if technique == "homolumo":
            eh = max(ch["energy"][nhomo - 1] for ch in channels)
            el = min(ch["energy"][nhomo] for ch in channels)
            se.omega_calc = (eh + 0.01 + np.arange(nomega_sigma_calc) / (nomega_sigma_calc - 1.0)
                             * (el - eh - 0.02)).astype(np.complex128)
        se.sigma_calc[:] = gw_selfenergy_imag(c["energy"], c["m_sigma"], sf, se.omega_calc, 1)
        if sox:   # per spin, the channel's own integrals and energies (src/m_g3w2_selfenergy.f90:2530-2580)
            se.sigma_calc += sox_selfenergy_imag(c["energy"][:c["m_sigma"].shape[1]], c["m_sigma"], c["m_ia"],
                                                 se.omega_calc).T
        if technique == "pade":
            se_pade_fit(se, eta)
        else:
            self_energy_polynomial(se)
        e0 = c["energy"][c["nsemin"] - 1: c["nsemax"]]
        xc = np.zeros_like(e0)
        eqp_z, zz = find_qp_energy_linearization(se, xc, e0)
        eqp_g, zz_g, _, _ = find_qp_energy_graphical(se, xc, e0)
        full = c["energy"].copy()
        full[c["nsemin"] - 1: c["nsemax"]] = eqp_g
        ehomo, elumo = output_homolumo(c["occupation"], full, c["nsemin"], c["nsemax"], spin_fact=1.0)
        out.append(G0W0Result(sf.erpa, sf.egw, se.sigma_calc.copy(), se.sigma.copy(), eqp_g, eqp_z, zz_g,
                              ehomo, elumo, c["nsemin"], c["nsemax"]))
    return out


def sox_selfenergy_imag(energy_g: np.ndarray, m_sigma: np.ndarray, m_ov: np.ndarray,
                        omega_calc: np.ndarray, chunk: int = 1 << 17) -> np.ndarray:
    """Second-order screened exchange on the evaluation points of the imaginary
    axis, sox_selfenergy_imag_grid (src/m_g3w2_selfenergy.f90:2482-2591), one spin.

    ``energy_g`` are the G energies over the window ncore_G+1 .. nvirtual_G-1
    (occupied first: ``nocc = m_ov.shape[0]`` of them), ``m_sigma`` is
    ``[nsig, nocc + nvirt, naux]`` = eri_3center_mo(:, q, p) for the Sigma states
    p, ``m_ov`` is ``[nocc, nvirt, naux]`` = eri_3center_mo(:, b, k) over the
    same window.  With C_p[q][(j, c)] = (p q | j c) the two sums of :2534-2577 are

      - sum_{b,i,k} C_p[i][(k,b)] C_p[k][(i,b)] / (z - e_i - e_k + e_b)
      - sum_{c,j,a} C_p[a][(j,c)] C_p[c][(j,a)] / (z - e_a - e_c + e_j)

    (vcoul1 = (p i|b k), vcoul2 = (i b|k p); vcoul1 = (p a|j c), vcoul2 =
    (a j|c p)).  Returns Sigma^SOX [nsig, nomega_calc] complex; the reference adds
    it to sigma_calc (:2584-2585) before the Pade fit."""
    no, nv, naux = m_ov.shape
    e_o, e_v = energy_g[:no], energy_g[no:no + nv]
    z = np.asarray(omega_calc, dtype=np.complex128)
    mov = m_ov.reshape(no * nv, naux)
    d1 = (e_o[:, None, None] + e_o[None, :, None] - e_v[None, None, :]).ravel()
    d2 = (e_v[:, None, None] + e_v[None, None, :] - e_o[None, :, None]).ravel()
    out = np.zeros((m_sigma.shape[0], z.size), dtype=np.complex128)

    def contract(prod, delta):
        s = np.zeros(z.size, dtype=np.complex128)
        for a in range(0, prod.size, chunk):
            s += (1.0 / (z[:, None] - delta[None, a:a + chunk])) @ prod[a:a + chunk]
        return s

    for p in range(m_sigma.shape[0]):
        cp = (m_sigma[p, :no + nv] @ mov.T).reshape(no + nv, no, nv)
        occ = cp[:no]                                   # [i][k][b] = (p i|b k)
        prod1 = (occ * occ.transpose(1, 0, 2)).ravel()  # (p i|b k) (i b|k p)
        vir = cp[no:]                                   # [a][j][c] = (p a|j c)
        prod2 = (vir * vir.transpose(2, 1, 0)).ravel()  # (p a|j c) (a j|c p)
        out[p] = -contract(prod1, d1) - contract(prod2, d2)
    return out


def sox_selfenergy_imag_loops(energy_g: np.ndarray, m_full: np.ndarray, nocc: int, sig_states,
                              omega_calc: np.ndarray) -> np.ndarray:
    """Loop-for-loop restatement of sox_selfenergy_imag_grid
    (src/m_g3w2_selfenergy.f90:2532-2578) for small cases: evaluate_eri_mo(p, q,
    r, s) = sum_P M(p,q)_P M(r,s)_P over the full window tensor ``m_full``
    [nstate, nstate, naux] (symmetric in its first two indices), occupied states
    0 .. nocc-1, empty ones nocc .. nstate-1; ``sig_states`` are 0-based window
    indices of the Sigma states."""
    nstate = m_full.shape[0]
    z = np.asarray(omega_calc, dtype=np.complex128)
    eri = lambda p, q, r, s: float(m_full[p, q] @ m_full[r, s])
    out = np.zeros((len(sig_states), z.size), dtype=np.complex128)
    for b in range(nocc, nstate):
        for i in range(nocc):
            for k in range(nocc):
                for ip, p in enumerate(sig_states):
                    v1 = eri(p, i, b, k)
                    v2 = eri(i, b, k, p)
                    out[ip] -= v1 * v2 / (z - energy_g[i] - energy_g[k] + energy_g[b])
    for c in range(nocc, nstate):
        for j in range(nocc):
            for a in range(nocc, nstate):
                for ip, p in enumerate(sig_states):
                    v1 = eri(p, a, j, c)
                    v2 = eri(a, j, c, p)
                    out[ip] -= v1 * v2 / (z - energy_g[a] - energy_g[c] + energy_g[j])
    return out


def sosex_selfenergy_imag(energy_g: np.ndarray, m_full: np.ndarray, nocc: int, sig_states,
                          chi: np.ndarray, omega_p: np.ndarray, weight_p: np.ndarray,
                          omega_calc: np.ndarray, factor_sosex: float = 1.0) -> np.ndarray:
    """SOSEX without its SOX part on the evaluation points of the imaginary axis,
    sosex_selfenergy_imag_grid (src/m_g3w2_selfenergy.f90:2200-2478), one spin,
    with W - v = v^1/2 chi v^1/2 = ``chi`` [nomega', naux, naux] on the grid
    (omega'_k, w_k) of wpol_imag.

    ``m_full`` [nstate, nstate, naux] is eri_3center_mo over the G window
    (occupied states 0 .. nocc-1 first), ``sig_states`` the 0-based window indices
    of the Sigma states.  With T(r; i, a) = (r m|W-v|i a), B1 = (r a|i m),
    B2 = (r i|a m) and D = e_a - e_i, the sums of :2316-2453 are

      Sigma_m(z) = f/(2 pi) sum_k w_k sum_{s=+-1} sum_{r,i,a}
                   T / (z + s i w_k - e_r) [B1 / (s i w_k - D) - B2 / (s i w_k + D)]

    (the bra-ket of W(i w +- i w') is the bare v, chi_wwp = 1 at :2283-2286).
    The z-independent inner sums K_k(r) are formed once per frequency; the
    s = -1 term is the complex conjugate of the s = +1 one for real integrals."""
    no = nocc
    nv = m_full.shape[0] - no
    e_o, e_v = energy_g[:no], energy_g[no:no + nv]
    z = np.asarray(omega_calc, dtype=np.complex128)
    dlt = e_v[None, :] - e_o[:, None]                                  # [i, a]
    m_ov = m_full[:no, no:]                                            # [i, a, P]
    out = np.zeros((len(sig_states), z.size), dtype=np.complex128)
    nst = no + nv
    m_ov2 = m_ov.reshape(no * nv, -1)
    for ip, m in enumerate(sig_states):
        b1 = (m_full[:, no:] @ m_full[:no, m].T).transpose(0, 2, 1)   # (r a|i m) as [r, i, a]
        b2 = m_full[:, :no] @ m_full[no:, m].T                          # (r i|a m) as [r, i, a]
        for k, (wk, om) in enumerate(zip(weight_p, omega_p)):
            t = ((m_full[:, m] @ chi[k]) @ m_ov2.T).reshape(nst, no, nv)   # (r m|W-v|i a)
            g = b1 / (1j * om - dlt)[None] - b2 / (1j * om + dlt)[None]
            kr = (t * g).sum(axis=(1, 2))                             # K_k(r), s = +1
            den_p = z[:, None] + 1j * om - energy_g[None, :no + nv]
            den_m = z[:, None] - 1j * om - energy_g[None, :no + nv]
            out[ip] += wk * ((kr[None] / den_p).sum(axis=1) + (kr.conj()[None] / den_m).sum(axis=1))
    return factor_sosex * out / (2.0 * PI)


def sosex_selfenergy_imag_loops(energy_g: np.ndarray, m_full: np.ndarray, nocc: int, sig_states,
                                chi: np.ndarray, omega_p: np.ndarray, weight_p: np.ndarray,
                                omega_calc: np.ndarray, factor_sosex: float = 1.0) -> np.ndarray:
    """Loop-for-loop restatement of sosex_selfenergy_imag_grid
    (src/m_g3w2_selfenergy.f90:2262-2466) for small cases: for every omega',
    sign and evaluation point, the bra-kets of :2316-2336 and :2385-2408 as
    matrix products for each empty (resp. occupied) state, then the double loops
    over (r, i) and (a, r)."""
    no = nocc
    nst = m_full.shape[0]
    z = np.asarray(omega_calc, dtype=np.complex128)
    out = np.zeros((len(sig_states), z.size), dtype=np.complex128)
    for ip, m in enumerate(sig_states):
        for k in range(len(omega_p)):
            chi_wp = chi[k]
            for isignp in (1, -1):
                for iz in range(z.size):
                    s = 0.0 + 0.0j
                    eri3_r_m = m_full[:, m].T                              # (naux, r)
                    eri3_i_m = m_full[:no, m].T                            # (naux, i)
                    for a in range(no, nst):
                        eri3_i_a = m_full[:no, a].T                        # (naux, i)
                        eri3_r_a = m_full[:, a].T                          # (naux, r)
                        braket1_ri = eri3_r_m.T @ (chi_wp @ eri3_i_a)      # (r, i)
                        braket2_ri = eri3_r_a.T @ eri3_i_m                 # (r, i), chi_wwp = 1
                        for r in range(nst):
                            for i in range(no):
                                d1 = z[iz] + isignp * 1j * omega_p[k] - energy_g[r]
                                d2 = isignp * 1j * omega_p[k] + energy_g[i] - energy_g[a]
                                s += weight_p[k] * braket1_ri[r, i] / d1 * braket2_ri[r, i] / d2 / (2.0 * PI)
                    eri3_a_m = m_full[no:, m].T                            # (naux, a)
                    for i in range(no):
                        eri3_a_i = m_full[no:, i].T                        # (naux, a)
                        eri3_r_i = m_full[:, i].T                          # (naux, r)
                        braket1_ra = eri3_r_m.T @ (chi_wp @ eri3_a_i)      # (r, a)
                        braket2_ra = eri3_r_i.T @ eri3_a_m                 # (r, a)
                        for a in range(no, nst):
                            for r in range(nst):
                                d1 = z[iz] + isignp * 1j * omega_p[k] - energy_g[r]
                                d2 = isignp * 1j * omega_p[k] + energy_g[a] - energy_g[i]
                                s -= (weight_p[k] * braket1_ra[r, a - no] / d1 * braket2_ra[r, a - no] / d2
                                      / (2.0 * PI))
                    out[ip, iz] += s
    return factor_sosex * out


def g3w2_selfenergy_imag(energy_g: np.ndarray, m_full: np.ndarray, sig_states, chi: np.ndarray,
                         omega_p: np.ndarray, weight_p: np.ndarray, omega_calc: np.ndarray) -> np.ndarray:
    """G (W-v) G (W-v) G on the evaluation points of the imaginary axis,
    g3w2_selfenergy_imag_grid (src/m_g3w2_selfenergy.f90:2018-2196), one spin,
    diagonal (q = p), with W - v = ``chi`` [nomega', naux, naux] on wpol_imag's grid.

    braket1(u,v,w) = (v w|W(i w')-v|u p), braket2(u,v,w) = (u v|W(i w'')-v|w p)
    (:2100-2110), and the four sign pairs (s', s'') of :2113-2146 sum
    1 / [(z + s' i w' - e_u)(z + s' i w' + s'' i w'' - e_v)(z + s'' i w'' - e_w)].
    Each term is a product of one factor per state index, so the sum over
    (u, v, w) is a trilinear contraction of braket1 * braket2 with three vectors;
    braket1 depends on w' only and braket2 on w'' only.  Returns
    w' w'' (-1/(2 pi))^2 sum (...) as [nsig, nomega_calc] complex."""
    ng = m_full.shape[0]
    e = energy_g[:ng]
    z = np.asarray(omega_calc, dtype=np.complex128)
    mflat = m_full.reshape(ng * ng, -1)
    out = np.zeros((len(sig_states), z.size), dtype=np.complex128)
    for ip, p in enumerate(sig_states):
        # (v w|chi_k|u p) and (u v|chi_k|w p) for every frequency k, [k][u][v][w]
        x = np.stack([m_full[:, p] @ chi[k].T for k in range(len(omega_p))])      # [k][u][P]
        b1 = np.stack([(mflat @ x[k].T).reshape(ng, ng, ng).transpose(2, 0, 1) for k in range(len(omega_p))])
        b2 = np.stack([(mflat @ x[k].T).reshape(ng, ng, ng) for k in range(len(omega_p))])
        for k1, (w1, o1) in enumerate(zip(weight_p, omega_p)):
            for k2, (w2, o2) in enumerate(zip(weight_p, omega_p)):
                bb = b1[k1] * b2[k2]
                for iz, zz in enumerate(z):
                    acc = 0.0 + 0.0j
                    for s1 in (1.0, -1.0):
                        a = 1.0 / (zz + s1 * 1j * o1 - e)
                        for s2 in (1.0, -1.0):
                            b = 1.0 / (zz + s1 * 1j * o1 + s2 * 1j * o2 - e)
                            c = 1.0 / (zz + s2 * 1j * o2 - e)
                            acc += np.einsum("uvw,u,v,w->", bb, a, b, c)
                    out[ip, iz] += w1 * w2 * acc
    return out / (2.0 * PI) ** 2


def g3w2_selfenergy_imag_loops(energy_g: np.ndarray, m_full: np.ndarray, sig_states, chi: np.ndarray,
                               omega_p: np.ndarray, weight_p: np.ndarray, omega_calc: np.ndarray) -> np.ndarray:
    """Loop-for-loop restatement of g3w2_selfenergy_imag_grid
    (src/m_g3w2_selfenergy.f90:2082-2158) for small cases."""
    ng = m_full.shape[0]
    e = energy_g[:ng]
    z = np.asarray(omega_calc, dtype=np.complex128)
    out = np.zeros((len(sig_states), z.size), dtype=np.complex128)
    for ip, p in enumerate(sig_states):
        q = p
        for k1 in range(len(omega_p)):
            for k2 in range(len(omega_p)):
                chi_omegap_up = chi[k1] @ m_full[:, p].T          # (naux, u)
                chi_omegapp_wq = chi[k2] @ m_full[:, q].T         # (naux, w)
                wp, wpp = 1j * omega_p[k1], 1j * omega_p[k2]
                for u in range(ng):
                    for v in range(ng):
                        for w in range(ng):
                            braket1 = m_full[v, w] @ chi_omegap_up[:, u]
                            braket2 = m_full[u, v] @ chi_omegapp_wq[:, w]
                            for iz in range(z.size):
                                zz = z[iz]
                                d = 1.0 / ((zz + wp - e[u]) * (zz + wp + wpp - e[v]) * (zz + wpp - e[w]))
                                d += 1.0 / ((zz - wp - e[u]) * (zz - wp + wpp - e[v]) * (zz + wpp - e[w]))
                                d += 1.0 / ((zz + wp - e[u]) * (zz + wp - wpp - e[v]) * (zz - wpp - e[w]))
                                d += 1.0 / ((zz - wp - e[u]) * (zz - wp - wpp - e[v]) * (zz - wpp - e[w]))
                                out[ip, iz] += (weight_p[k1] * weight_p[k2] * braket1 * braket2 * d
                                                * (-1.0 / (2.0 * PI)) ** 2)
    return out


# ---------------------------------------------------------------------------
# Contour deformation (postscf G0W0_CONTOUR)
# ---------------------------------------------------------------------------
TOL_LOW_EIGVAL = 1.0e-3        # src/m_spectral_function.f90:783


def vsqrt_chi_vsqrt_lowrank(m_ia: np.ndarray, e_occ: np.ndarray, e_virt: np.ndarray, occ_occ: np.ndarray,
                            occ_virt: np.ndarray, omega: np.ndarray) -> list:
    """sf_vsqrt_chi_vsqrt_rpa with low_rank (src/m_spectral_function.f90:779-921)
    at the complex frequencies ``omega``: chi0 = M F M^T with F =
    REAL(2 docc de / (omega^2 - de^2)) (:861-872, DGEMM('N','T') :880-881),
    diagonalized (:895), eigenvalues turned into lambda / (1 - lambda) (:898) and
    those with |.| <= 1e-3 dropped (:899-913).  Returns per frequency
    (eigvec [naux, neig], eigval [neig]) of v^1/2 chi v^1/2."""
    nocc, nvirt, naux = m_ia.shape
    docc = (occ_occ[:, None] - occ_virt[None, :]).reshape(-1)
    de = (e_virt[None, :] - e_occ[:, None]).reshape(-1)
    m_t = np.asfortranarray(m_ia.reshape(nocc * nvirt, naux).T)
    out = []
    for w in omega:
        factor = np.real(2.0 * docc * de / (w * w - de * de))
        chi0 = sblas.dgemm(1.0, np.asfortranarray(m_t * factor[None, :]), m_t, trans_b=1)
        eigval, eigvec = sla.eigh(chi0, driver="ev")                   # DSYEV('V')
        eigval = eigval / (1.0 - eigval)
        keep = np.abs(eigval) > TOL_LOW_EIGVAL
        out.append((eigvec[:, keep].copy(), eigval[keep].copy()))
    return out


def real_linear_grid(nomega: int, omega_max: float) -> np.ndarray:
    """sf_init(REAL_LINEAR) frequencies (src/m_spectral_function.f90:308-316)."""
    return np.array([k / (nomega - 1) * omega_max for k in range(nomega)])


def nearest_real_frequency(omega_real: np.ndarray, omega: float) -> int:
    """sf_interpolate_vsqrt_chi_vsqrt (src/m_spectral_function.f90:925-950): no
    interpolation, the first closest grid point (MINLOC)."""
    if omega > omega_real.max() or omega < omega_real.min():
        raise ValueError("requested frequency out of range")
    return int(np.argmin(np.abs(omega_real - omega)))


@dataclass
class ContourResult:
    sigma: np.ndarray            # [2*nomega+1, nsig] complex, real grid around energy0
    omega: np.ndarray            # se%omega (real)
    omega_real: np.ndarray       # the real frequencies of W
    de_max: float
    nrank_imag: list             # kept eigenpairs per imaginary frequency
    nrank_real: list
    energy_qp_g: np.ndarray
    energy_qp_z: np.ndarray
    zz: np.ndarray
    ehomo: float
    elumo: float
    nsemin: int
    nsemax: int


def gw_selfenergy_contour(energy: np.ndarray, occupation: np.ndarray, m_ia: np.ndarray, m_sigma: np.ndarray,
                          rng: StateRange, ncore_w: int, nomega_chi_imag: int, nomega_chi_real: int,
                          nomega_sigma: int, step_sigma: float, eta: float):
    """gw_selfenergy_contour (src/m_gw_selfenergy_grid.f90:342-551) for one spin.

    ``m_ia`` is the W window [nocc_w, nvirt_w, naux] from state ncore_w+1;
    ``m_sigma`` is [nsig, prange, naux] over p = ncore_G+1 .. nvirtual_G-1.
    The self-energy is evaluated on se%omega = step_sigma * (-n..n) around
    energy0 = energy of the Sigma states (src/m_selfenergy_tools.f90:658-663, 679-680).
    Returns (sigma [2n+1, nsig], se_omega, omega_real, de_max, w_imag, w_real)."""
    nom = nomega_sigma // 2
    se_omega = step_sigma * np.arange(-nom, nom + 1)
    energy0 = energy[rng.nsemin - 1: rng.nsemax]
    nocc_w, nvirt_w = m_ia.shape[:2]
    occ_w, e_occ = occupation[ncore_w:ncore_w + nocc_w], energy[ncore_w:ncore_w + nocc_w]
    e_virt = energy[ncore_w + nocc_w: ncore_w + nocc_w + nvirt_w]
    occ_v = occupation[ncore_w + nocc_w: ncore_w + nocc_w + nvirt_w]
    wimag, wquad = imaginary_quad_grid(nomega_chi_imag)
    w_imag = vsqrt_chi_vsqrt_lowrank(m_ia, e_occ, e_virt, occ_w, occ_v, 1j * wimag)
    # largest real frequency needed (:390-414)
    de_max = 0.0
    for s in range(len(energy0)):
        for p in range(rng.ncore_g + 1, rng.nhomo_g + 1):
            for om in se_omega:
                de = energy[p - 1] - (energy0[s] + om)
                if de < -eta:
                    continue
                de_max = max(de_max, de)
        for p in range(rng.nlumo_g, rng.nvirtual_g):
            for om in se_omega:
                de = energy0[s] + om - energy[p - 1]
                if de < -eta:
                    continue
                de_max = max(de_max, de)
    omega_real = real_linear_grid(nomega_chi_real, de_max)
    w_real = vsqrt_chi_vsqrt_lowrank(m_ia, e_occ, e_virt, occ_w, occ_v, omega_real.astype(complex))
    prange = rng.nvirtual_g - rng.ncore_g - 1
    sigma = np.zeros((2 * nom + 1, len(energy0)), dtype=complex)
    for s in range(len(energy0)):
        eri3 = np.asfortranarray(m_sigma[s, :prange].T)                 # [naux, prange]
        # imaginary-axis integral (:440-478)
        for iw in range(nomega_chi_imag):
            vec, val = w_imag[iw]
            if val.size == 0:
                continue
            tmp2 = sblas.dgemm(1.0, vec, eri3, trans_a=1)                # DGEMM('T','N')
            vchiv = np.sum(tmp2 ** 2 * val[:, None], axis=0)
            for pl in range(prange):
                p = pl + rng.ncore_g + 1
                x = energy0[s] + se_omega - energy[p - 1]
                mask = np.abs(x) > eta
                term = (1.0 / (x + 1j * wimag[iw]) + 1.0 / (x - 1j * wimag[iw])) * vchiv[pl] / (2.0 * PI)
                sigma[mask, s] -= wquad[iw] * term[mask]
        # residues of the occupied states (:481-508) and of the empty states (:511-538)
        for pl in range(prange):
            p = pl + rng.ncore_g + 1
            occupied = p < rng.nlumo_g
            empty = p > rng.nhomo_g
            for io, om in enumerate(se_omega):
                for kind, on in ((-1.0, occupied), (1.0, empty)):
                    if not on:
                        continue
                    de = energy[p - 1] - (energy0[s] + om) if kind < 0 else energy0[s] + om - energy[p - 1]
                    if de < -eta:
                        continue
                    vec, val = w_real[nearest_real_frequency(omega_real, abs(de))]
                    tmp = eri3[:, pl] @ vec
                    factor = 0.5 if abs(de) < eta else 1.0
                    sigma[io, s] += kind * np.sum(tmp ** 2 * val) * factor
    return sigma, se_omega, omega_real, de_max, w_imag, w_real


def g0w0_contour(energy: np.ndarray, occupation: np.ndarray, m_ia: np.ndarray, m_sigma: np.ndarray,
                 rng: StateRange, ncore_w: int, nomega_chi_imag: int, nomega_chi_real: int,
                 nomega_sigma: int = 51, step_sigma: float = 0.01, eta: float = 0.001,
                 exchange_m_vxc: np.ndarray | None = None, energy_g: np.ndarray | None = None) -> ContourResult:
    """selfenergy_evaluation for contour_deformation (src/m_selfenergy_evaluation.f90:239-240):
    Sigma on the real grid, then the linearized and graphical QP energies and
    HOMO/LUMO over the Sigma states (:587-611).  ``energy_g`` (default
    ``energy``) seeds se%energy0 (se%init with energy_g, :185) and goes into
    gw_selfenergy_contour (W and the poles); the QP equation keeps ``energy``."""
    eg = energy if energy_g is None else energy_g
    sigma, se_omega, omega_real, de_max, w_imag, w_real = gw_selfenergy_contour(
        eg, occupation, m_ia, m_sigma, rng, ncore_w, nomega_chi_imag, nomega_chi_real, nomega_sigma,
        step_sigma, eta)
    e0 = energy[rng.nsemin - 1: rng.nsemax]
    se = SelfEnergyGrid(omega=se_omega.astype(complex), omega_calc=np.zeros(0, complex),
                        energy0=eg[rng.nsemin - 1: rng.nsemax].copy(), sigma=sigma)
    xc = np.zeros_like(e0) if exchange_m_vxc is None else exchange_m_vxc
    eqp_z, _ = find_qp_energy_linearization(se, xc, e0)
    eqp_g, zz_g, _, _ = find_qp_energy_graphical(se, xc, e0)
    full = energy.copy()
    full[rng.nsemin - 1: rng.nsemax] = eqp_g
    ehomo, elumo = output_homolumo(occupation, full, rng.nsemin, rng.nsemax)
    return ContourResult(sigma, se_omega, omega_real, de_max, [v.size for _, v in w_imag],
                         [v.size for _, v in w_real], eqp_g, eqp_z, zz_g, ehomo, elumo, rng.nsemin, rng.nsemax)


# ---------------------------------------------------------------------------
# GW density matrix from the imaginary axis (pt_density_matrix GW_IMAGINARY)
# ---------------------------------------------------------------------------
def gw_density_matrix_imag(energy: np.ndarray, m_window: np.ndarray, sf: SpectralFunction, rng: StateRange,
                           nomega_sigma: int, spin_fact: float = 2.0) -> np.ndarray:
    """gw_density_matrix_imag (src/m_mbpt_density_matrix.f90:491-640), one spin.

    ``m_window`` is M[p, q, P] over the states ncore_G+1 .. nvirtual_G-1 (the
    rows and columns of eri_3center_mo); ``sf`` holds chi = v^1/2 chi v^1/2 on
    the imaginary grid of W (wpol%chi, wpol%omega, wpol%weight_quad).  The
    frequency integral of the density matrix runs on a second Gauss-Legendre
    grid of nomega_sigma points mapped with alpha = beta = 1 (:555-567), around
    mu, the centre of the HOMO-LUMO gap (:571).  Returns the correction to the
    MO density matrix, [nstate, nstate], symmetric, zero outside the Sigma range."""
    nstate = energy.size
    x, ws = coeffs_gausslegint(0.0, 1.0, nomega_sigma)
    ws = ws / (2.0 ** 1.0 - 1.0) * 1.0 * (1.0 - x) ** (-2.0) * 1.0
    om_s = 1.0 / (2.0 ** 1.0 - 1.0) * (1.0 / (1.0 - x) - 1.0) * 1.0
    mu = 0.5 * (energy[rng.nhomo_g] + energy[rng.nhomo_g - 1])
    c0 = rng.ncore_g
    mrange = rng.nvirtual_g - rng.ncore_g - 1
    em = energy[c0:c0 + mrange] - mu
    p = np.zeros((nstate, nstate))
    zs = 1j * om_s
    for q in range(rng.nsemin, rng.nsemax + 1):
        eri3_q = m_window[:mrange, q - 1 - c0, :].T                       # [naux, mrange]
        for iw in range(len(sf.omega)):
            chi_eri3_q = sf.chi[iw] @ eri3_q                              # DGEMM('N','N')
            yw = 1j * sf.omega[iw]
            g = (1.0 / (zs[:, None] - em[None, :] + yw) + 1.0 / (zs[:, None] - em[None, :] - yw))   # [s, m]
            for pp in range(q, rng.nsemax + 1):
                eri3_p = m_window[:mrange, pp - 1 - c0, :].T
                v = np.sum(eri3_p * chi_eri3_q, axis=0)                   # [m]
                k = g / (zs[:, None] - (energy[pp - 1] - mu)) / (zs[:, None] - (energy[q - 1] - mu))
                p[pp - 1, q - 1] -= spin_fact * 2.0 / (2.0 * PI) ** 2 * np.sum(
                    sf.weight_quad[iw] * ws[:, None] * v[None, :] * k.real)
    iu = np.triu_indices(nstate, 1)
    p[iu] = p.T[iu]
    return p
