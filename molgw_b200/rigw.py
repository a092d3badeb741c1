"""Python host mirror of MOLGW's imaginary-axis GW interface over librigw (ctypes).

The names follow the reference routines the library replaces:

* ``polarizability_grid_scalapack``  src/m_gw_selfenergy_grid.f90:33-209
* ``gw_selfenergy_imag_scalapack``   src/m_gw_selfenergy_grid.f90:213-338
* ``calculate_eri_3center_mo``       src/m_eri_ao_mo.f90:416-582
* ``qp_solve`` (se_pade_fit + find_qp_energy_linearization/graphical)
                                     src/m_selfenergy_tools.f90:202-420, 965-1033
* ``g0w0`` / ``g0w0_batch``          selfenergy_evaluation for imaginary_axis_pade,
                                     src/m_selfenergy_evaluation.f90:214-246, 587-611

Errors: the library returns a status and never aborts; this module raises
``RigwError`` with the library's message, the analogue of MOLGW's ``die()``
(src/m_warning.f90:78-89).  There is no CPU fallback: importing this module
without the built library, or calling it without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "librigw.so"

RIGW_FP64 = 0
RIGW_BF16X3 = 1
RIGW_OZAKI_INT8 = 16


def RIGW_OZAKI(slices: int) -> int:
    """Precision code of the Ozaki-sliced INT8 chi0 with ``slices`` 7-bit slices (3..7)."""
    if not 3 <= slices <= 7:
        raise ValueError(f"Ozaki slices must be in [3, 7], got {slices}")
    return RIGW_OZAKI_INT8 + slices


RIGW_PADE = 0
RIGW_HOMOLUMO = 1
RIGW_PROBLEM_DEVICE_POINTERS = 1
RIGW_PROBLEM_QP_ONLY = 2
RIGW_PROBLEM_SPIN_CHANNEL = 4
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_NOMEM", 4: "ERR_NOT_SPD", 5: "ERR_NUMERIC",
                6: "ERR_TIMEOUT", 7: "ERR_UNSUPPORTED"}

_dp = C.POINTER(C.c_double)


class RigwError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rigw: {STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class Problem(C.Structure):
    _fields_ = [
        ("naux", C.c_int), ("nocc", C.c_int), ("nvirt", C.c_int), ("nomega", C.c_int),
        ("omega", _dp), ("weight", _dp), ("m_ia", _dp), ("e_occ", _dp), ("e_virt", _dp),
        ("occ_occ", _dp), ("occ_virt", _dp),
        ("nstate_p", C.c_int), ("nsig", C.c_int),
        ("m_pm", _dp), ("e_p", _dp), ("e_sig", _dp), ("occ_sig", _dp), ("exchange_m_vxc", _dp),
        ("technique", C.c_int), ("nomega_sigma_calc", C.c_int), ("step_sigma_calc", C.c_double),
        ("omega_calc", _dp), ("nomega_sigma", C.c_int), ("step_sigma", C.c_double), ("eta", C.c_double),
        ("efermi", C.c_double), ("precision", C.c_int), ("flags", C.c_int),
        ("nocc_2", C.c_int), ("nvirt_2", C.c_int), ("m_ia_2", _dp), ("e_occ_2", _dp), ("e_virt_2", _dp),
        ("occ_occ_2", _dp), ("occ_virt_2", _dp),
    ]


class SoxProblem(C.Structure):
    _fields_ = [
        ("naux", C.c_int), ("nocc", C.c_int), ("nvirt", C.c_int), ("m_ov", _dp), ("nsig", C.c_int),
        ("m_pq", _dp), ("energy", _dp), ("nomega_calc", C.c_int), ("omega_calc", _dp), ("flags", C.c_int),
    ]


class SosexProblem(C.Structure):
    _fields_ = [
        ("naux", C.c_int), ("nocc", C.c_int), ("nvirt", C.c_int), ("m_full", _dp), ("nsig", C.c_int),
        ("sig_first", C.c_int), ("energy", _dp), ("nomega_calc", C.c_int), ("omega_calc", _dp),
        ("factor_sosex", C.c_double), ("flags", C.c_int),
    ]


class G3w2Problem(C.Structure):
    _fields_ = [
        ("naux", C.c_int), ("nstate", C.c_int), ("m_full", _dp), ("nsig", C.c_int), ("sig_first", C.c_int),
        ("energy", _dp), ("nomega_calc", C.c_int), ("omega_calc", _dp), ("flags", C.c_int),
    ]


class RiShell(C.Structure):
    _fields_ = [("center", C.c_double * 3), ("am", C.c_int), ("nprim", C.c_int), ("alpha", _dp), ("coeff", _dp)]


class RiProblem(C.Structure):
    _fields_ = [
        ("nshell", C.c_int), ("shells", C.POINTER(RiShell)), ("pure", C.c_int), ("nshell_aux", C.c_int),
        ("aux_shells", C.POINTER(RiShell)), ("pure_aux", C.c_int), ("npair", C.c_int),
        ("index_basis", C.POINTER(C.c_int)), ("flags", C.c_int),
    ]


def shell_coefficients(am: int, alpha, coeff) -> np.ndarray:
    """The reference's shell coefficients (src/m_basis_set.f90:332-333) from a
    basis file's contraction (coefficients of normalized primitives): the
    contraction normalized so that its x^l component has unit norm, each
    coefficient times (2/pi)^{3/4} 2^l alpha^{(2l+3)/4}."""
    a = np.asarray(alpha, dtype=np.float64)
    c = np.asarray(coeff, dtype=np.float64)
    dfact = float(np.prod(np.arange(2 * am - 1, 0, -2))) if am > 0 else 1.0
    norm = np.sqrt((2.0 * a / np.pi) ** 1.5 * (4.0 * a) ** am / dfact)           # primitive norm of x^l
    ab = a[:, None] + a[None, :]
    ovl = dfact / (2.0 * ab) ** am * (np.pi / ab) ** 1.5                         # <x^l g_a | x^l g_b>
    s = 1.0 / np.sqrt(float(np.sum(np.outer(c * norm, c * norm) * ovl)))
    return c * s * (2.0 / np.pi) ** 0.75 * 2.0 ** am * a ** ((2 * am + 3) / 4.0)


def _ri_shells(shells, keep):
    arr = (RiShell * len(shells))()
    for k, sh in enumerate(shells):
        a = np.ascontiguousarray(sh.alpha, dtype=np.float64)
        c = np.ascontiguousarray(shell_coefficients(sh.am, sh.alpha, sh.coeff))
        keep += [a, c]
        arr[k] = RiShell((C.c_double * 3)(*[float(x) for x in sh.center]), sh.am, len(a), _ptr(a), _ptr(c))
    return arr


class DmProblem(C.Structure):
    _fields_ = [
        ("naux", C.c_int), ("nstate", C.c_int), ("m_full", _dp), ("nsig", C.c_int), ("sig_first", C.c_int),
        ("energy", _dp), ("mu", C.c_double), ("nomega_sigma", C.c_int), ("spin_fact", C.c_double),
        ("flags", C.c_int),
    ]


class ContourProblem(C.Structure):
    _fields_ = [
        ("naux", C.c_int), ("nocc_w", C.c_int), ("nvirt_w", C.c_int), ("m_ia", _dp), ("e_occ_w", _dp),
        ("e_virt_w", _dp), ("occ_occ_w", _dp), ("occ_virt_w", _dp), ("nomega_imag", C.c_int),
        ("nomega_real", C.c_int), ("nstate_p", C.c_int), ("p_occ_end", C.c_int), ("p_empty_begin", C.c_int),
        ("energy_p", _dp), ("nsig", C.c_int), ("m_pm", _dp), ("energy0", _dp), ("energy_qp0", _dp),
        ("exchange_m_vxc", _dp), ("nomega_sigma", C.c_int), ("step_sigma", C.c_double), ("eta", C.c_double),
        ("flags", C.c_int),
    ]


class ContourResult(C.Structure):
    _fields_ = [
        ("sigma", _dp), ("energy_qp_g", _dp), ("energy_qp_z", _dp), ("zz", _dp), ("rank", C.POINTER(C.c_int)),
        ("omega_real", _dp), ("de_max", C.c_double),
    ]


@dataclass
class ContourOutput:
    """Result of Engine.g0w0_contour (fields as in the oracle's ContourResult)."""
    sigma: np.ndarray            # [2n+1, nsig] complex, Sigma_c on se%omega around energy0
    omega: np.ndarray            # se%omega
    omega_real: np.ndarray       # the real frequencies of W
    de_max: float
    rank: np.ndarray             # kept eigenpairs per frequency (imaginary, then real)
    energy_qp_g: np.ndarray
    energy_qp_z: np.ndarray
    zz: np.ndarray
    ehomo: float
    elumo: float
    device_ms: float


def _vertex_w_inst(inst):
    """The instance whose W window the vertex path factors: on that path the
    reference calls gw_selfenergy_grid with energy_g (src/m_selfenergy_evaluation.f90:496),
    and that routine builds W from the energies it is given
    (src/m_gw_selfenergy_grid.f90:604), so the W energies are energy_g."""
    eg = getattr(inst, "energy_g", None)
    return inst if eg is None else replace(inst, energy=np.asarray(eg, dtype=np.float64))


def efermi_of(inst) -> float:
    """se_init's efermi from the energies in G: half-way between the highest
    energy of state nhomo_G and the lowest of state nhomo_G + 1 over the spin
    channels, nhomo_G the highest state occupied in any channel
    (src/m_selfenergy_tools.f90:584-585)."""
    chans = [inst] + ([inst.spin2] if getattr(inst, "spin2", None) is not None else [])
    eg = [np.asarray(c.energy if getattr(c, "energy_g", None) is None else c.energy_g, dtype=np.float64)
          for c in chans]
    nhomo = max(getattr(c, "ncore_w", 0) + c.nocc for c in chans)
    return 0.5 * (max(e[nhomo - 1] for e in eg) + min(e[nhomo] for e in eg))


class Result(C.Structure):
    _fields_ = [
        ("erpa", C.c_double), ("egw", C.c_double),
        ("sigma_calc", _dp), ("sigma", _dp), ("energy_qp_g", _dp), ("energy_qp_z", _dp), ("zz", _dp),
        ("ehomo", C.c_double), ("elumo", C.c_double), ("device_ms", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("stage_ms", C.c_double * 4), ("total_ms", C.c_double), ("kernel_launches", C.c_int),
        ("graph_replayed", C.c_int), ("device_bytes_in_use", C.c_size_t), ("device_bytes_peak", C.c_size_t),
        ("chunks", C.c_int), ("waves", C.c_int),
    ]


RIGW_TUNE_MAX_CANDIDATES = 16
RIGW_SERVER_MAX_WORKERS = 16


class ServerStats(C.Structure):
    _fields_ = [
        ("batches", C.c_longlong * 2), ("completed", C.c_longlong * 2), ("queued", C.c_longlong * 2),
        ("requeued", C.c_longlong * 2), ("failed", C.c_longlong), ("hold_ns", C.c_longlong),
        ("device_ms", C.c_double * 2), ("build_ms", C.c_double * 2), ("capture_ms", C.c_double * 2),
        ("alloc_ms", C.c_double * 2),
        ("busy_ns", C.c_longlong * RIGW_SERVER_MAX_WORKERS), ("workers", C.c_int),
    ]


class TuneReport(C.Structure):
    _fields_ = [
        ("chi0_rows", C.c_int), ("update_rows", C.c_int), ("split_group", C.c_int), ("chains", C.c_int),
        ("panel_group", C.c_int), ("precision_class", C.c_int), ("ncandidates", C.c_int),
        ("candidate", (C.c_int * 5) * RIGW_TUNE_MAX_CANDIDATES),
        ("candidate_ms", (C.c_float * 3) * RIGW_TUNE_MAX_CANDIDATES),
        ("default_ms", C.c_float), ("tuned_ms", C.c_float),
    ]


def load_library(path: Path | str = LIB_PATH) -> C.CDLL:
    path = Path(path)
    if not path.exists():
        raise RigwError(7, f"{path} is not built (run python -m molgw_b200.build)")
    lib = C.CDLL(str(path))
    lib.rigw_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_size_t]
    lib.rigw_destroy.argtypes = [C.c_void_p]
    lib.rigw_last_error.argtypes = [C.c_void_p]
    lib.rigw_last_error.restype = C.c_char_p
    lib.rigw_version.restype = C.c_int
    lib.rigw_last_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
    lib.rigw_footprint_bytes.argtypes = [C.c_int] * 7
    lib.rigw_footprint_bytes.restype = C.c_size_t
    lib.rigw_imag_grid.argtypes = [C.c_int, _dp, _dp]
    lib.rigw_eri_3center_mo.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                        _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, _dp]
    lib.rigw_eri_3center_mo_ex.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                           _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, _dp, C.c_int, C.c_int]
    lib.rigw_eri_3center_mo_precision.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                  C.POINTER(C.c_int), _dp, _dp, C.c_int, C.c_int, C.c_int,
                                                  C.c_int, _dp, C.c_int]
    lib.rigw_polarizability_imag.argtypes = [C.c_void_p, C.POINTER(Problem), _dp, _dp, C.POINTER(C.c_void_p)]
    lib.rigw_wpol_chi.argtypes = [C.c_void_p, C.c_void_p, _dp]
    lib.rigw_gw_selfenergy_imag.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Problem), C.POINTER(Result)]
    lib.rigw_wpol_release.argtypes = [C.c_void_p, C.c_void_p]
    lib.rigw_qp_solve.argtypes = [C.c_void_p, C.POINTER(Problem), _dp, C.POINTER(Result)]
    lib.rigw_sox_selfenergy_imag.argtypes = [C.c_void_p, C.POINTER(SoxProblem), _dp]
    lib.rigw_sosex_selfenergy_imag.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(SosexProblem), _dp]
    lib.rigw_g3w2_selfenergy_imag.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(G3w2Problem), _dp]
    lib.rigw_gw_selfenergy_contour.argtypes = [C.c_void_p, C.POINTER(ContourProblem), C.POINTER(ContourResult)]
    lib.rigw_gw_density_matrix_imag.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(DmProblem), _dp]
    lib.rigw_eri_2center.argtypes = [C.c_void_p, C.POINTER(RiProblem), _dp]
    lib.rigw_eri_3center_raw.argtypes = [C.c_void_p, C.POINTER(RiProblem), _dp]
    lib.rigw_eri_3center.argtypes = [C.c_void_p, C.POINTER(RiProblem), _dp, C.POINTER(C.c_int)]
    lib.rigw_g0w0.argtypes = [C.c_void_p, C.POINTER(Problem), C.POINTER(Result)]
    lib.rigw_g0w0_batch.argtypes = [C.c_void_p, C.c_int, C.POINTER(Problem), C.POINTER(Result)]
    lib.rigw_autotune.argtypes = [C.c_void_p, C.c_int, C.POINTER(Problem), C.POINTER(TuneReport)]
    lib.rigw_qp_solve_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_int, C.c_int,
                                          C.c_double, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp, _dp,
                                          C.c_void_p, C.c_char_p, C.c_size_t]
    return lib


def qp_solve_noalloc(sigma_calc, e_sig, energy_qp_g, energy_qp_z=None, zz=None, sigma=None, *, device=0,
                     omega_calc=None, exchange_m_vxc=None, technique=RIGW_PADE, nomega_sigma=101,
                     step_sigma=0.025, step_sigma_calc=0.075, eta=0.01, efermi=0.0, stream=0):
    """Continuation + QP equation on caller-owned CUDA tensors, with no device
    allocation inside the library (``rigw_qp_solve_noalloc``).  ``sigma_calc`` is a
    [nsig, nc, 2] float64 CUDA tensor; outputs are written in place."""
    nsig, nc = int(sigma_calc.shape[0]), int(sigma_calc.shape[1])
    buf = C.create_string_buffer(512)
    rc = lib().rigw_qp_solve_noalloc(device, nsig, nc, _ptr(omega_calc), _ptr(sigma_calc), _ptr(e_sig),
                                     _ptr(exchange_m_vxc), technique, nomega_sigma, step_sigma, step_sigma_calc,
                                     eta, efermi, _ptr(energy_qp_g), _ptr(energy_qp_z), _ptr(zz), _ptr(sigma),
                                     C.c_void_p(stream), buf, 512)
    if rc:
        raise RigwError(rc, buf.value.decode())


_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load_library()
    return _LIB


def _ptr(a) -> _dp:
    """Pointer to a C-contiguous float64 numpy array, or to a CUDA tensor (data_ptr)."""
    if a is None:
        return _dp()
    if hasattr(a, "data_ptr"):
        return C.cast(C.c_void_p(a.data_ptr()), _dp)
    if not (a.flags["C_CONTIGUOUS"] and a.dtype == np.float64):
        raise ValueError("arrays passed to librigw must be C-contiguous float64")
    return a.ctypes.data_as(_dp)


def imag_grid(nomega: int):
    """sf_init IMAGINARY_QUAD grid (omega_k imaginary parts, weights)."""
    om = np.zeros(nomega)
    wt = np.zeros(nomega)
    rc = lib().rigw_imag_grid(nomega, _ptr(om), _ptr(wt))
    if rc:
        raise RigwError(rc, "rigw_imag_grid")
    return om, wt


@dataclass
class G0W0Output:
    erpa: float
    egw: float
    sigma_calc: np.ndarray      # [nsig, nc] complex
    sigma: np.ndarray           # [nsig, nreal] complex
    energy_qp_g: np.ndarray
    energy_qp_z: np.ndarray
    zz: np.ndarray
    ehomo: float
    elumo: float
    device_ms: float


class Engine:
    """One library context on one CUDA device."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self._lib = lib()
        h = C.c_void_p()
        rc = self._lib.rigw_create(C.byref(h), device, hbm_budget_bytes)
        if rc:
            raise RigwError(rc, f"rigw_create(device={device})")
        self._h = h
        self._keep = []
        self.device = device

    def close(self):
        if self._h:
            self._lib.rigw_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_stats(self) -> dict:
        st = Stats()
        self._check(self._lib.rigw_last_stats(self._h, C.byref(st)), "rigw_last_stats")
        return dict(stage_ms=list(st.stage_ms), total_ms=st.total_ms, kernel_launches=st.kernel_launches,
                    graph_replayed=bool(st.graph_replayed), device_bytes_in_use=st.device_bytes_in_use,
                    device_bytes_peak=st.device_bytes_peak, chunks=st.chunks, waves=st.waves)

    def _check(self, rc: int, what: str):
        if rc:
            raise RigwError(rc, f"{what}: {self._lib.rigw_last_error(self._h).decode()}")

    # ---------------------------------------------------------------- problems
    def make_problem(self, inst, precision: int = RIGW_FP64, device_arrays: dict | None = None,
                     technique: int = RIGW_PADE, qp_only: bool = False,
                     efermi: float | None = None, freq: tuple | None = None) -> tuple[Problem, list]:
        """Problem descriptor for a ``molgw_b200.synth.GWInstance``-like object.

        ``device_arrays`` maps field names to CUDA tensors that replace the host
        arrays (all W/Sigma inputs must then be device tensors)."""
        nocc, nvirt = inst.nocc, inst.nvirt
        e = np.ascontiguousarray(inst.energy, dtype=np.float64)
        # G is built from energy_g (the Sigma sum over p and se_init's efermi); W and
        # the energy0 of the QP equation from the mean-field energies
        eg = e if getattr(inst, "energy_g", None) is None else np.ascontiguousarray(inst.energy_g, dtype=np.float64)
        occ = np.ascontiguousarray(inst.occupation, dtype=np.float64)
        nsemin, nsemax = inst.nsemin, inst.nsemax
        cw, cg = getattr(inst, "ncore_w", 0), getattr(inst, "ncore_g", 0)   # frozen core of W and of G
        host = {
            "e_occ": e[cw:cw + nocc].copy(), "e_virt": e[cw + nocc:cw + nocc + nvirt].copy(),
            "occ_occ": occ[cw:cw + nocc].copy(), "occ_virt": occ[cw + nocc:cw + nocc + nvirt].copy(),
            "e_p": eg[cg:].copy(), "e_sig": e[nsemin - 1:nsemax].copy(),
        }
        if inst.m_ia is not None:
            host["m_ia"] = np.ascontiguousarray(inst.m_ia)
            host["m_pm"] = np.ascontiguousarray(inst.m_sigma)
        occ_sig = occ[nsemin - 1:nsemax].copy()
        if getattr(inst, "exchange_m_vxc", None) is not None:
            host["exchange_m_vxc"] = np.ascontiguousarray(inst.exchange_m_vxc, dtype=np.float64)
        arrs = dict(host)
        flags = 0
        if device_arrays:
            arrs.update(device_arrays)
            flags = RIGW_PROBLEM_DEVICE_POINTERS
            occ_sig = device_arrays.get("occ_sig", occ_sig)
        if efermi is None:
            efermi = efermi_of(inst)
        p = Problem()
        p.naux = inst.naux
        p.nocc, p.nvirt = nocc, nvirt
        p.nomega = inst.nomega
        if freq is not None:
            # a subset of the imaginary grid (omega, weight): the frequencies of one rank
            om, wt = (np.ascontiguousarray(a, dtype=np.float64) for a in freq)
            p.nomega = om.size
            p.omega, p.weight = _ptr(om), _ptr(wt)
            arrs["omega"], arrs["weight"] = om, wt
        for k in ("m_ia", "e_occ", "e_virt", "occ_occ", "occ_virt", "m_pm", "e_p", "e_sig"):
            setattr(p, k, _ptr(arrs[k]))
        p.occ_sig = _ptr(occ_sig)
        if "exchange_m_vxc" in arrs:
            p.exchange_m_vxc = _ptr(arrs["exchange_m_vxc"])
        p.nstate_p = e.shape[0] - cg
        p.nsig = nsemax - nsemin + 1
        p.technique = technique
        p.nomega_sigma_calc = inst.nomega_sigma_calc
        p.step_sigma_calc = inst.step_sigma_calc
        p.nomega_sigma = inst.nomega_sigma
        p.step_sigma = inst.step_sigma
        p.eta = inst.eta
        p.efermi = efermi
        p.precision = precision
        p.flags = flags | (RIGW_PROBLEM_QP_ONLY if qp_only else 0)
        if getattr(inst, "spin_channel", False) or getattr(inst, "spin2", None) is not None:
            p.flags |= RIGW_PROBLEM_SPIN_CHANNEL
        keep = [arrs, occ_sig]
        s2 = getattr(inst, "spin2", None)
        if s2 is not None:
            # second spin channel of the W window (its own energies and occupations)
            e2 = np.ascontiguousarray(s2.energy, dtype=np.float64)
            o2 = np.ascontiguousarray(s2.occupation, dtype=np.float64)
            c2 = s2.ncore_w
            w2 = {"m_ia_2": np.ascontiguousarray(s2.m_ia), "e_occ_2": e2[c2:c2 + s2.nocc].copy(),
                  "e_virt_2": e2[c2 + s2.nocc:c2 + s2.nocc + s2.nvirt].copy(),
                  "occ_occ_2": o2[c2:c2 + s2.nocc].copy(),
                  "occ_virt_2": o2[c2 + s2.nocc:c2 + s2.nocc + s2.nvirt].copy()}
            if device_arrays:
                w2.update({k: v for k, v in device_arrays.items() if k.endswith("_2")})
            p.nocc_2, p.nvirt_2 = s2.nocc, s2.nvirt
            for k, v in w2.items():
                setattr(p, k, _ptr(v))
            keep.append(w2)
        return p, keep

    def _alloc_result(self, p: Problem):
        nreal = 2 * (p.nomega_sigma // 2) + 1
        bufs = {
            "sigma_calc": np.zeros((p.nsig, p.nomega_sigma_calc, 2)),
            "sigma": np.zeros((p.nsig, nreal, 2)),
            "energy_qp_g": np.zeros(p.nsig), "energy_qp_z": np.zeros(p.nsig), "zz": np.zeros(p.nsig),
        }
        r = Result()
        for k, v in bufs.items():
            setattr(r, k, _ptr(v))
        return r, bufs

    @staticmethod
    def _output(r: Result, bufs) -> G0W0Output:
        sc = bufs["sigma_calc"]
        sg = bufs["sigma"]
        return G0W0Output(r.erpa, r.egw, sc[..., 0] + 1j * sc[..., 1], sg[..., 0] + 1j * sg[..., 1],
                          bufs["energy_qp_g"].copy(), bufs["energy_qp_z"].copy(), bufs["zz"].copy(),
                          r.ehomo, r.elumo, r.device_ms)

    # ---------------------------------------------------------------- fused
    def g0w0_batch(self, insts, precision=RIGW_FP64, device_arrays=None,
                   qp_only: bool = False, freq: tuple | None = None) -> list[G0W0Output]:
        """One call for many molecules; ``precision`` is one code for all or one per molecule.
        ``freq`` = (omega, weight): the imaginary frequencies and quadrature weights
        of W in place of the Gauss-Legendre grid (wpol%omega, wpol%weight_quad)."""
        n = len(insts)
        precs = list(precision) if isinstance(precision, (list, tuple)) else [precision] * n
        probs = (Problem * n)()
        ress = (Result * n)()
        keep, bufs = [], []
        for i, inst in enumerate(insts):
            p, k = self.make_problem(inst, precs[i], device_arrays[i] if device_arrays else None,
                                     qp_only=qp_only, freq=freq)
            probs[i] = p
            keep.append(k)
            r, b = self._alloc_result(p)
            ress[i] = r
            bufs.append(b)
        self._check(self._lib.rigw_g0w0_batch(self._h, n, probs, ress), "rigw_g0w0_batch")
        return [self._output(ress[i], bufs[i]) for i in range(n)]

    def autotune(self, insts, precision=RIGW_FP64, device_arrays=None, qp_only: bool = False) -> dict:
        """Time launch-shape candidates on this batch; the context keeps the fastest
        for later batches of the same precision class.  Returns the report."""
        n = len(insts)
        precs = list(precision) if isinstance(precision, (list, tuple)) else [precision] * n
        probs = (Problem * n)()
        keep = []
        for i, inst in enumerate(insts):
            p, k = self.make_problem(inst, precs[i], device_arrays[i] if device_arrays else None,
                                     qp_only=qp_only)
            probs[i] = p
            keep.append(k)
        rep = TuneReport()
        self._check(self._lib.rigw_autotune(self._h, n, probs, C.byref(rep)), "rigw_autotune")
        cands = [{"chi0_rows": rep.candidate[k][0], "update_rows": rep.candidate[k][1],
                  "split_group": rep.candidate[k][2], "chains": rep.candidate[k][3],
                  "panel_group": rep.candidate[k][4],
                  "chi0_ms": rep.candidate_ms[k][0], "factor_ms": rep.candidate_ms[k][1],
                  "total_ms": rep.candidate_ms[k][2]} for k in range(rep.ncandidates)]
        return {"chi0_rows": rep.chi0_rows, "update_rows": rep.update_rows, "split_group": rep.split_group,
                "chains": rep.chains, "panel_group": rep.panel_group, "precision_class": rep.precision_class,
                "default_ms": rep.default_ms,
                "tuned_ms": rep.tuned_ms, "candidates": cands}

    def g0w0(self, inst, precision: int = RIGW_FP64, device_arrays=None, qp_only: bool = False,
             freq: tuple | None = None) -> G0W0Output:
        return self.g0w0_batch([inst], precision, [device_arrays] if device_arrays else None, qp_only, freq)[0]

    # ---------------------------------------------------------------- drop-in pieces
    def polarizability_grid_scalapack(self, inst, precision: int = RIGW_FP64):
        """Returns (erpa, egw, wpol handle) for the W window of ``inst``."""
        p, keep = self.make_problem(inst, precision)
        erpa, egw = C.c_double(), C.c_double()
        w = C.c_void_p()
        self._check(self._lib.rigw_polarizability_imag(self._h, C.byref(p), C.byref(erpa), C.byref(egw),
                                                       C.byref(w)), "rigw_polarizability_imag")
        return erpa.value, egw.value, WPol(self, w, inst.naux, inst.nomega)

    def gw_selfenergy_imag_scalapack(self, wpol: "WPol", inst, omega_calc=None, efermi=None) -> np.ndarray:
        p, keep = self.make_problem(inst, efermi=efermi)
        if omega_calc is not None:
            oc = np.ascontiguousarray(np.stack([omega_calc.real, omega_calc.imag], -1))
            p.omega_calc = _ptr(oc)
            keep.append(oc)
        r, bufs = self._alloc_result(p)
        self._check(self._lib.rigw_gw_selfenergy_imag(self._h, wpol.handle, C.byref(p), C.byref(r)),
                    "rigw_gw_selfenergy_imag")
        sc = bufs["sigma_calc"]
        return sc[..., 0] + 1j * sc[..., 1]

    def qp_solve(self, inst, sigma_calc: np.ndarray, technique: int = RIGW_PADE, omega_calc=None,
                 efermi=None) -> G0W0Output:
        p, keep = self.make_problem(inst, technique=technique, efermi=efermi)
        if omega_calc is not None:
            oc = np.ascontiguousarray(np.stack([omega_calc.real, omega_calc.imag], -1))
            p.omega_calc = _ptr(oc)
            keep.append(oc)
        sc = np.ascontiguousarray(np.stack([sigma_calc.real, sigma_calc.imag], -1))
        r, bufs = self._alloc_result(p)
        self._check(self._lib.rigw_qp_solve(self._h, C.byref(p), _ptr(sc), C.byref(r)), "rigw_qp_solve")
        out = self._output(r, bufs)
        out.sigma_calc = sigma_calc
        return out

    def sox_selfenergy_imag_grid(self, inst, omega_calc, m_ov=None, device_arrays: dict | None = None) -> np.ndarray:
        """Sigma^SOX on the evaluation points ``omega_calc`` for the Sigma states
        of ``inst`` (sox_selfenergy_imag_grid, src/m_g3w2_selfenergy.f90:2482-2591),
        [nsig, nomega_calc] complex, from energy_g over the G window.  ``m_ov`` is
        the occupied x empty block [nocc_G, nvirt_G, naux] of the G window; the
        default ``inst.m_ia`` is that block when the W and G windows coincide.
        ``device_arrays`` {"m_ov", "m_pq"}: CUDA tensors used in place
        (RIGW_PROBLEM_DEVICE_POINTERS; the result is then written on the device)."""
        cg = getattr(inst, "ncore_g", 0)
        if device_arrays:
            import torch
            dov, dpq = device_arrays["m_ov"], device_arrays["m_pq"]
            e = inst.energy if getattr(inst, "energy_g", None) is None else inst.energy_g
            ew = np.ascontiguousarray(np.asarray(e, dtype=np.float64)[cg:cg + dpq.shape[1]])
            oc = np.ascontiguousarray(np.stack([np.real(omega_calc), np.imag(omega_calc)], -1), dtype=np.float64)
            sp = SoxProblem()
            sp.naux = inst.naux
            sp.nocc, sp.nvirt = dov.shape[0], dov.shape[1]
            sp.m_ov, sp.m_pq = C.cast(dov.data_ptr(), _dp), C.cast(dpq.data_ptr(), _dp)
            sp.energy, sp.omega_calc = _ptr(ew), _ptr(oc)
            sp.nsig, sp.nomega_calc = dpq.shape[0], oc.shape[0]
            sp.flags = RIGW_PROBLEM_DEVICE_POINTERS
            out = torch.empty((sp.nsig, sp.nomega_calc, 2), dtype=torch.float64, device=dov.device)
            self._check(self._lib.rigw_sox_selfenergy_imag(self._h, C.byref(sp), C.cast(out.data_ptr(), _dp)),
                        "rigw_sox_selfenergy_imag")
            o = out.cpu().numpy()
            return o[..., 0] + 1j * o[..., 1]
        if m_ov is None:
            if getattr(inst, "ncore_w", 0) != cg:
                raise ValueError("sox_selfenergy_imag_grid: pass m_ov when the W and G windows differ")
            m_ov = inst.m_ia
        m_ov = np.ascontiguousarray(m_ov, dtype=np.float64)
        mpq = np.ascontiguousarray(inst.m_sigma, dtype=np.float64)
        e = inst.energy if getattr(inst, "energy_g", None) is None else inst.energy_g
        ew = np.ascontiguousarray(np.asarray(e, dtype=np.float64)[cg:cg + mpq.shape[1]])
        oc = np.ascontiguousarray(np.stack([np.real(omega_calc), np.imag(omega_calc)], -1), dtype=np.float64)
        sp = SoxProblem()
        sp.naux = inst.naux
        sp.nocc, sp.nvirt = m_ov.shape[0], m_ov.shape[1]
        if sp.nocc + sp.nvirt != mpq.shape[1]:
            raise ValueError("sox_selfenergy_imag_grid: m_ov does not span the window of m_sigma")
        sp.m_ov, sp.m_pq, sp.energy, sp.omega_calc = _ptr(m_ov), _ptr(mpq), _ptr(ew), _ptr(oc)
        sp.nsig = mpq.shape[0]
        sp.nomega_calc = oc.shape[0]
        out = np.zeros((sp.nsig, sp.nomega_calc, 2))
        self._check(self._lib.rigw_sox_selfenergy_imag(self._h, C.byref(sp), _ptr(out)),
                    "rigw_sox_selfenergy_imag")
        return out[..., 0] + 1j * out[..., 1]

    def gw_sox_imag(self, inst, precision: int = RIGW_FP64, m_ov=None, efermi: float | None = None) -> G0W0Output:
        """GW+SOX on the imaginary axis (postscf 'GW+SOX_PADE'): W and Sigma_c on
        the evaluation points, Sigma^SOX added to sigma_calc, then the
        Pade continuation and the QP equation (src/m_selfenergy_evaluation.f90:494-503,
        587-611; the imaginary-axis vertex path exists for imaginary_axis_pade only).
        W is built from energy_g when it is set, as gw_selfenergy_grid does with the
        energies it is given (src/m_gw_selfenergy_grid.f90:604)."""
        ef = efermi_of(inst) if efermi is None else efermi
        erpa, egw, wpol = self.polarizability_grid_scalapack(_vertex_w_inst(inst), precision)
        oc = ef + 1j * inst.step_sigma_calc * np.arange(inst.nomega_sigma_calc)
        try:
            sigma = self.gw_selfenergy_imag_scalapack(wpol, inst, omega_calc=oc)
        finally:
            wpol.release()
        sigma = sigma + self.sox_selfenergy_imag_grid(inst, oc, m_ov)
        out = self.qp_solve(inst, sigma, RIGW_PADE, omega_calc=oc, efermi=ef)
        out.erpa, out.egw = erpa, egw
        return out

    def sosex_selfenergy_imag_grid(self, wpol: "WPol", inst, m_full, omega_calc,
                                   factor_sosex: float = 1.0) -> np.ndarray:
        """SOSEX (without its SOX part) on the evaluation points ``omega_calc`` for
        the Sigma states of ``inst`` (sosex_selfenergy_imag_grid,
        src/m_g3w2_selfenergy.f90:2200-2478), [nsig, nomega_calc] complex, with
        W from the resident factors of ``wpol``.  ``m_full`` is the window tensor
        [nstate_G, nstate_G, naux] (``synth.with_window``)."""
        cg = getattr(inst, "ncore_g", 0)
        mf = np.ascontiguousarray(m_full, dtype=np.float64)
        ng = mf.shape[0]
        e = inst.energy if getattr(inst, "energy_g", None) is None else inst.energy_g
        ew = np.ascontiguousarray(np.asarray(e, dtype=np.float64)[cg:cg + ng])
        oc = np.ascontiguousarray(np.stack([np.real(omega_calc), np.imag(omega_calc)], -1), dtype=np.float64)
        sp = SosexProblem()
        sp.naux = inst.naux
        sp.nocc = getattr(inst, "ncore_w", 0) + inst.nocc - cg
        sp.nvirt = ng - sp.nocc
        sp.m_full, sp.energy, sp.omega_calc = _ptr(mf), _ptr(ew), _ptr(oc)
        sp.nsig = inst.nsemax - inst.nsemin + 1
        sp.sig_first = inst.nsemin - 1 - cg
        sp.nomega_calc = oc.shape[0]
        sp.factor_sosex = factor_sosex
        out = np.zeros((sp.nsig, sp.nomega_calc, 2))
        self._check(self._lib.rigw_sosex_selfenergy_imag(self._h, wpol.handle, C.byref(sp), _ptr(out)),
                    "rigw_sosex_selfenergy_imag")
        return out[..., 0] + 1j * out[..., 1]

    def gw_sosex_imag(self, inst, m_full, precision: int = RIGW_FP64, factor_sosex: float = 1.0,
                      efermi: float | None = None, g3w2: bool = False) -> G0W0Output:
        """GW+SOSEX on the imaginary axis (postscf 'GW+SOSEX_PADE'; factor_sosex = 2
        for 'GW+2SOSEX_PADE'): W, then Sigma_c + Sigma^SOX + factor_sosex Sigma^SOSEX
        on the evaluation points, then the Pade continuation and the QP equation
        (src/m_selfenergy_evaluation.f90:494-503).  W is built from energy_g when it
        is set (src/m_gw_selfenergy_grid.f90:604)."""
        ef = efermi_of(inst) if efermi is None else efermi
        erpa, egw, wpol = self.polarizability_grid_scalapack(_vertex_w_inst(inst), precision)
        oc = ef + 1j * inst.step_sigma_calc * np.arange(inst.nomega_sigma_calc)
        cg = getattr(inst, "ncore_g", 0)
        no = getattr(inst, "ncore_w", 0) + inst.nocc - cg
        try:
            sigma = self.gw_selfenergy_imag_scalapack(wpol, inst, omega_calc=oc)
            sigma = sigma + self.sosex_selfenergy_imag_grid(wpol, inst, m_full, oc, factor_sosex)
            if g3w2:
                sigma = sigma + self.g3w2_selfenergy_imag_grid(wpol, inst, m_full, oc)
        finally:
            wpol.release()
        sigma = sigma + self.sox_selfenergy_imag_grid(inst, oc, m_full[:no, no:])
        out = self.qp_solve(inst, sigma, RIGW_PADE, omega_calc=oc, efermi=ef)
        out.erpa, out.egw = erpa, egw
        return out

    def g3w2_selfenergy_imag_grid(self, wpol: "WPol", inst, m_full, omega_calc) -> np.ndarray:
        """G (W-v) G (W-v) G on the evaluation points ``omega_calc`` for the Sigma
        states of ``inst`` (g3w2_selfenergy_imag_grid, src/m_g3w2_selfenergy.f90:2018-2196),
        [nsig, nomega_calc] complex, with W from the resident factors of ``wpol``.
        ``m_full`` is the window tensor [nstate_G, nstate_G, naux]."""
        cg = getattr(inst, "ncore_g", 0)
        mf = np.ascontiguousarray(m_full, dtype=np.float64)
        ng = mf.shape[0]
        e = inst.energy if getattr(inst, "energy_g", None) is None else inst.energy_g
        ew = np.ascontiguousarray(np.asarray(e, dtype=np.float64)[cg:cg + ng])
        oc = np.ascontiguousarray(np.stack([np.real(omega_calc), np.imag(omega_calc)], -1), dtype=np.float64)
        gp = G3w2Problem()
        gp.naux, gp.nstate = inst.naux, ng
        gp.m_full, gp.energy, gp.omega_calc = _ptr(mf), _ptr(ew), _ptr(oc)
        gp.nsig = inst.nsemax - inst.nsemin + 1
        gp.sig_first = inst.nsemin - 1 - cg
        gp.nomega_calc = oc.shape[0]
        out = np.zeros((gp.nsig, gp.nomega_calc, 2))
        self._check(self._lib.rigw_g3w2_selfenergy_imag(self._h, wpol.handle, C.byref(gp), _ptr(out)),
                    "rigw_g3w2_selfenergy_imag")
        return out[..., 0] + 1j * out[..., 1]

    # ---------------------------------------------------------------- RI integrals
    def _ri_problem(self, shells, aux_shells, pure: bool, pure_aux: bool, pairs, keep):
        rp = RiProblem()
        if shells is not None:
            rp.nshell, rp.shells = len(shells), _ri_shells(shells, keep)
        rp.nshell_aux, rp.aux_shells = len(aux_shells), _ri_shells(aux_shells, keep)
        rp.pure, rp.pure_aux = int(pure), int(pure_aux)
        if pairs is not None:
            pr = np.ascontiguousarray(pairs, dtype=np.int32)
            keep.append(pr)
            rp.npair, rp.index_basis = pr.shape[0], pr.ctypes.data_as(C.POINTER(C.c_int))
        keep.append(rp.shells)
        keep.append(rp.aux_shells)
        return rp

    def eri_2center(self, aux_shells, pure_aux: bool = True) -> np.ndarray:
        """(P|Q) over the auxiliary basis on the device (rigw_eri_2center).
        Shells: objects with am, alpha, coeff (basis-file contraction on normalized
        primitives) and center (Bohr), e.g. oracle or basis-file parsers' shells."""
        keep = []
        rp = self._ri_problem(None, aux_shells, True, pure_aux, None, keep)
        n = sum((2 * s.am + 1) if pure_aux else (s.am + 1) * (s.am + 2) // 2 for s in aux_shells)
        out = np.zeros((n, n))
        self._check(self._lib.rigw_eri_2center(self._h, C.byref(rp), _ptr(out)), "rigw_eri_2center")
        return out

    @staticmethod
    def _ri_out(rp, out, n):
        """Host result array, or the caller's CUDA tensor [n, npair] (float64,
        contiguous) with RIGW_PROBLEM_DEVICE_POINTERS set."""
        if out is None:
            return np.zeros((n, rp.npair))
        if tuple(out.shape) != (n, rp.npair) or not out.is_cuda or not out.is_contiguous() or \
                str(out.dtype) != "torch.float64":
            raise ValueError(f"out must be a contiguous float64 CUDA tensor of shape {(n, rp.npair)}")
        rp.flags = RIGW_PROBLEM_DEVICE_POINTERS
        return out

    def eri_3center_raw(self, shells, aux_shells, pairs, pure: bool = True, pure_aux: bool = True, out=None):
        """(mu nu|P) [naux_basis, npair] on the device, no metric (rigw_eri_3center_raw);
        ``pairs`` [npair, 2] 1-based basis-function indices.  With ``out`` (a CUDA
        tensor) the result stays in device memory."""
        keep = []
        rp = self._ri_problem(shells, aux_shells, pure, pure_aux, pairs, keep)
        n = sum((2 * s.am + 1) if pure_aux else (s.am + 1) * (s.am + 2) // 2 for s in aux_shells)
        out = self._ri_out(rp, out, n)
        self._check(self._lib.rigw_eri_3center_raw(self._h, C.byref(rp), _ptr(out)), "rigw_eri_3center_raw")
        return out

    def eri_3center(self, shells, aux_shells, pairs, pure: bool = True, pure_aux: bool = True, out=None):
        """eri_3center as the reference stores it (rigw_eri_3center): the metric
        (P|Q)^-1/2 with eigenvalues <= 1e-6 dropped, diagonal pairs halved;
        [nauxil_kept, npair], the rigw_eri_3center_mo input.  With ``out`` (a CUDA
        tensor [naux_basis, npair]) the result stays in device memory and the
        first nauxil_kept rows are returned."""
        keep = []
        rp = self._ri_problem(shells, aux_shells, pure, pure_aux, pairs, keep)
        n = sum((2 * s.am + 1) if pure_aux else (s.am + 1) * (s.am + 2) // 2 for s in aux_shells)
        dev = out is not None
        out = self._ri_out(rp, out, n)
        nk = C.c_int()
        self._check(self._lib.rigw_eri_3center(self._h, C.byref(rp), _ptr(out), C.byref(nk)), "rigw_eri_3center")
        return out[:nk.value] if dev else out[:nk.value].copy()

    def gw_density_matrix_imag(self, inst, m_full, nomega_sigma: int, precision: int = RIGW_FP64,
                               spin_fact: float = 2.0):
        """pt_density_matrix='GW_IMAGINARY' (src/m_dm_mbpt_driver.f90:117-122): W on
        the imaginary grid of ``inst`` (rigw_polarizability_imag), then the
        correction to the MO density matrix (rigw_gw_density_matrix_imag) for the
        Sigma range of ``inst``.  ``m_full`` is the window tensor [nstate_G,
        nstate_G, naux] over the states ncore_g+1 ..; mu is the centre of the
        HOMO-LUMO gap (src/m_mbpt_density_matrix.f90:571).  Returns the
        correction [nstate, nstate] (zero on the core rows and columns) and E_RPA."""
        cg = getattr(inst, "ncore_g", 0)
        mf = np.ascontiguousarray(m_full, dtype=np.float64)
        ng = mf.shape[0]
        e = np.asarray(inst.energy, dtype=np.float64)
        occ = np.asarray(inst.occupation, dtype=np.float64)
        nhomo = max([1] + [p + 1 for p in range(e.size) if not occ[p] < 1.0e-5])
        mu = 0.5 * (e[nhomo] + e[nhomo - 1])
        erpa, _, wpol = self.polarizability_grid_scalapack(inst, precision)
        try:
            ew = np.ascontiguousarray(e[cg:cg + ng])
            dp = DmProblem()
            dp.naux, dp.nstate = inst.naux, ng
            dp.m_full, dp.energy = _ptr(mf), _ptr(ew)
            dp.nsig = inst.nsemax - inst.nsemin + 1
            dp.sig_first = inst.nsemin - 1 - cg
            dp.mu, dp.nomega_sigma, dp.spin_fact = mu, nomega_sigma, spin_fact
            pw = np.zeros((ng, ng))
            self._check(self._lib.rigw_gw_density_matrix_imag(self._h, wpol.handle, C.byref(dp), _ptr(pw)),
                        "rigw_gw_density_matrix_imag")
        finally:
            wpol.release()
        out = np.zeros((e.size, e.size))
        out[cg:cg + ng, cg:cg + ng] = pw
        return out, erpa

    def gw_g3w2_imag(self, inst, m_full, precision: int = RIGW_FP64, efermi: float | None = None) -> G0W0Output:
        """GW+G3W2 on the imaginary axis (postscf 'GW+G3W2_PADE'): Sigma_c, SOX,
        2 SOSEX and G3W2 added to sigma_calc before the Pade fit
        (src/m_selfenergy_evaluation.f90:494-503)."""
        return self.gw_sosex_imag(inst, m_full, precision, factor_sosex=2.0, efermi=efermi, g3w2=True)

    def frequency_partials(self, inst, freq_index, precision: int = RIGW_FP64):
        """The share of one rank in MOLGW's frequency split ("poorman",
        src/m_gw_selfenergy_grid.f90:626,658): W and Sigma_c(z_k) on the imaginary
        frequencies ``freq_index`` (0-based, of the inst.nomega Gauss-Legendre grid).
        Returns (sigma_calc [nsig, nc] complex, [erpa, egw]) partial sums; summed
        over ranks (``parallel.allreduce_partials``) they are the full quantities,
        and ``qp_solve`` on the sum finishes the run."""
        idx = np.asarray(freq_index, dtype=np.int64)
        om, wt = imag_grid(inst.nomega)
        freq = (om[idx], wt[idx])
        p, keep = self.make_problem(inst, precision, freq=freq)
        erpa, egw = C.c_double(), C.c_double()
        w = C.c_void_p()
        self._check(self._lib.rigw_polarizability_imag(self._h, C.byref(p), C.byref(erpa), C.byref(egw),
                                                       C.byref(w)), "rigw_polarizability_imag")
        wpol = WPol(self, w, inst.naux, idx.size)
        try:
            r, bufs = self._alloc_result(p)
            self._check(self._lib.rigw_gw_selfenergy_imag(self._h, wpol.handle, C.byref(p), C.byref(r)),
                        "rigw_gw_selfenergy_imag")
            sc = bufs["sigma_calc"]
            sigma = sc[..., 0] + 1j * sc[..., 1]
        finally:
            wpol.release()
        return sigma, np.array([erpa.value, egw.value])

    def g0w0_spin(self, inst, precision: int = RIGW_FP64, technique: int = RIGW_PADE,
                  sox: bool = False) -> list[G0W0Output]:
        """Open-shell (nspin = 2) G0W0 on the imaginary axis: one W from the
        transitions of both spin channels (``inst`` and ``inst.spin2``), then Sigma
        and the QP equation per channel with the factors resident, on the
        evaluation points of the common efermi (src/m_gw_selfenergy_grid.f90:118-149,
        279-319; src/m_selfenergy_tools.f90:584-585).  Returns one output per
        channel, each carrying E_RPA and E_GW of the whole W.  ``sox``: GW+SOX_PADE,
        Sigma^SOX of each channel (its own integrals and energies,
        src/m_g3w2_selfenergy.f90:2532-2580) added to its sigma_calc before the fit."""
        if getattr(inst, "spin2", None) is None:
            raise ValueError("g0w0_spin needs inst.spin2 (the second spin channel)")
        if sox and technique != RIGW_PADE:
            raise ValueError("g0w0_spin: SOX runs with the Pade continuation (imaginary_axis_pade) only")
        ef = efermi_of(inst)
        erpa, egw, wpol = self.polarizability_grid_scalapack(inst, precision)
        outs = []
        try:
            for ch in (replace(inst, spin2=None, spin_channel=True), replace(inst.spin2, spin_channel=True)):
                zc = None
                if technique == RIGW_HOMOLUMO:   # se_init: real points inside the gap, over both channels
                    nc = ch.nomega_sigma_calc
                    nh = max(inst.ncore_w + inst.nocc, inst.spin2.ncore_w + inst.spin2.nocc)
                    eh = max(inst.energy[nh - 1], inst.spin2.energy[nh - 1])
                    el = min(inst.energy[nh], inst.spin2.energy[nh])
                    zc = (eh + 0.01 + np.arange(nc) / (nc - 1.0) * (el - eh - 0.02)).astype(np.complex128)
                if sox:
                    zc = ef + 1j * ch.step_sigma_calc * np.arange(ch.nomega_sigma_calc)
                sc = self.gw_selfenergy_imag_scalapack(wpol, ch, zc, efermi=ef)
                if sox:
                    sc = sc + self.sox_selfenergy_imag_grid(ch, zc)
                out = self.qp_solve(ch, sc, technique, zc, efermi=ef)
                out.erpa, out.egw = erpa, egw
                outs.append(out)
        finally:
            wpol.release()
        return outs

    def gw_imag_force_energy_qp(self, inst, nstep: int = 1, precision: int = RIGW_FP64, workdir=None,
                                technique: int = RIGW_PADE) -> list[G0W0Output]:
        """``nstep`` successive imaginary-axis GW runs under force_energy_qp: run k
        takes the QP energies of run k-1 as the energies in G (the first run: the
        ENERGY_QP file of ``workdir`` when it reads with status 0, else the mean-field
        energies), keeps the mean-field energies for W and for the energy0 of the QP
        equation, and hands on the mean-field energies with the Sigma range replaced
        by its graphical QP energies (src/m_selfenergy_evaluation.f90:164-181,
        241-245, 587-611; src/m_selfenergy_tools.f90:358-359).  With ``workdir``
        every run reads and writes ``workdir/ENERGY_QP`` as the reference does.

        W does not depend on energy_g, so it is factored once and stays resident;
        each run evaluates Sigma from the resident factors and solves the QP
        equation.  Each output carries the run's E_RPA and E_GW."""
        from .energy_qp import read_energy_qp, write_energy_qp
        ns = inst.nsemin - 1
        energy = np.asarray(inst.energy, dtype=np.float64)
        eq = None
        if workdir is not None:
            e_read, status = read_energy_qp(workdir, energy.size)
            eq = e_read[:, 0] if status == 0 else None
        erpa, egw, wpol = self.polarizability_grid_scalapack(inst, precision)
        outs = []
        try:
            for _ in range(nstep):
                g = replace(inst, energy_g=energy if eq is None else eq)
                zc = None
                if technique == RIGW_HOMOLUMO:   # se_init: real points inside the gap of energy_g
                    nc = inst.nomega_sigma_calc
                    nh = inst.ncore_w + inst.nocc
                    eh, el = g.energy_g[nh - 1], g.energy_g[nh]
                    zc = (eh + 0.01 + np.arange(nc) / (nc - 1.0) * (el - eh - 0.02)).astype(np.complex128)
                sc = self.gw_selfenergy_imag_scalapack(wpol, g, zc)
                out = self.qp_solve(g, sc, technique, zc)
                out.erpa, out.egw = erpa, egw
                outs.append(out)
                eq = energy.copy()
                eq[ns:ns + out.energy_qp_g.size] = out.energy_qp_g
                if workdir is not None:
                    write_energy_qp(workdir, eq)
        finally:
            wpol.release()
        return outs

    def calculate_eri_3center_mo(self, eri3, index_basis: np.ndarray, c_matrix: np.ndarray,
                                 m_min: int, m_max: int, n_min: int, n_max: int,
                                 precision: int = RIGW_FP64):
        """calculate_eri_3center_mo (src/m_eri_ao_mo.f90:416-582): eri3 [naux, npair]
        (pair-packed, diagonal x0.5), c_matrix [nstate, nbf]; returns [n, m, naux].
        When ``eri3`` is a CUDA tensor the transform reads it in place and returns a
        CUDA tensor (RIGW_PROBLEM_DEVICE_POINTERS): nothing crosses PCIe."""
        naux, npair = int(eri3.shape[0]), int(eri3.shape[1])
        nstate, nbf = c_matrix.shape
        idx = np.ascontiguousarray(index_basis, dtype=np.int32)
        cm = np.ascontiguousarray(c_matrix, dtype=np.float64)
        shape = (n_max - n_min + 1, m_max - m_min + 1, naux)
        if hasattr(eri3, "is_cuda") and eri3.is_cuda:
            import torch
            out = torch.empty(shape, dtype=torch.float64, device=eri3.device)
            self._check(self._lib.rigw_eri_3center_mo_ex(
                self._h, nbf, nstate, npair, naux, idx.ctypes.data_as(C.POINTER(C.c_int)), _ptr(eri3), _ptr(cm),
                m_min, m_max, n_min, n_max, _ptr(out), precision, RIGW_PROBLEM_DEVICE_POINTERS),
                "rigw_eri_3center_mo_ex")
            return out
        out = np.zeros(shape)
        self._check(self._lib.rigw_eri_3center_mo_precision(
            self._h, nbf, nstate, npair, naux, idx.ctypes.data_as(C.POINTER(C.c_int)),
            _ptr(np.ascontiguousarray(eri3)), _ptr(cm), m_min, m_max, n_min, n_max,
            _ptr(out), precision), "rigw_eri_3center_mo_precision")
        return out

    def g0w0_contour(self, energy: np.ndarray, occupation: np.ndarray, m_ia, m_sigma, nsemin: int, nsemax: int,
                     nomega_imag: int, nomega_real: int, nomega_sigma: int, step_sigma: float, eta: float = 0.001,
                     ncore_w: int = 0, ncore_g: int = 0, energy_g: np.ndarray | None = None,
                     exchange_m_vxc: np.ndarray | None = None) -> ContourOutput:
        """G0W0 by contour deformation for one spin channel (postscf G0W0_CONTOUR:
        gw_selfenergy_contour, src/m_gw_selfenergy_grid.f90:342-551, then the QP
        equation, src/m_selfenergy_evaluation.f90:587-611) through
        rigw_gw_selfenergy_contour.

        ``m_ia`` is the W window [nocc_w, nvirt_w, naux] from state ncore_w+1;
        ``m_sigma`` is [nsig, nstate - ncore_g, naux] over the states p =
        ncore_g+1 .. nstate for the Sigma states nsemin..nsemax (1-based).  Both
        may be CUDA tensors (RIGW_PROBLEM_DEVICE_POINTERS).  ``energy_g`` (default
        ``energy``) is the energy of G and W and se%energy0; the QP equation
        keeps ``energy``."""
        e = np.ascontiguousarray(energy, dtype=np.float64)
        occ = np.ascontiguousarray(occupation, dtype=np.float64)
        eg = e if energy_g is None else np.ascontiguousarray(energy_g, dtype=np.float64)
        nstate = e.size
        on_dev = hasattr(m_ia, "is_cuda") and m_ia.is_cuda
        if not on_dev:
            m_ia = np.ascontiguousarray(m_ia, dtype=np.float64)
            m_sigma = np.ascontiguousarray(m_sigma, dtype=np.float64)
        nocc_w, nvirt_w, naux = (int(x) for x in m_ia.shape)
        nsig = nsemax - nsemin + 1
        nstate_p = nstate - ncore_g
        if tuple(int(x) for x in m_sigma.shape) != (nsig, nstate_p, naux):
            raise ValueError("g0w0_contour: m_sigma must be [nsig, nstate - ncore_g, naux]")
        # HOMO / LUMO of G (selfenergy_set_state_range, src/m_selfenergy_tools.f90:96-109)
        empty = 1.0e-5
        nhomo = max([1] + [p + 1 for p in range(nstate) if not occ[p] < empty])
        nlumo = min([100000] + [p + 1 for p in range(nstate) if not occ[p] > empty])
        keep = []
        cp = ContourProblem()
        cp.naux, cp.nocc_w, cp.nvirt_w = naux, nocc_w, nvirt_w
        arrays = {
            "e_occ_w": eg[ncore_w:ncore_w + nocc_w], "e_virt_w": eg[ncore_w + nocc_w:ncore_w + nocc_w + nvirt_w],
            "occ_occ_w": occ[ncore_w:ncore_w + nocc_w],
            "occ_virt_w": occ[ncore_w + nocc_w:ncore_w + nocc_w + nvirt_w],
            "energy_p": eg[ncore_g:], "energy0": eg[nsemin - 1:nsemax], "energy_qp0": e[nsemin - 1:nsemax]}
        if exchange_m_vxc is not None:
            arrays["exchange_m_vxc"] = np.asarray(exchange_m_vxc, dtype=np.float64)
        for k, v in arrays.items():
            v = np.ascontiguousarray(v, dtype=np.float64)
            keep.append(v)
            setattr(cp, k, _ptr(v))
        if on_dev:
            cp.m_ia, cp.m_pm = C.cast(m_ia.data_ptr(), _dp), C.cast(m_sigma.data_ptr(), _dp)
            cp.flags = RIGW_PROBLEM_DEVICE_POINTERS
        else:
            cp.m_ia, cp.m_pm = _ptr(m_ia), _ptr(m_sigma)
        cp.nomega_imag, cp.nomega_real = nomega_imag, nomega_real
        cp.nstate_p = nstate_p
        cp.p_occ_end = max(0, min(nstate_p, nlumo - ncore_g - 1))
        cp.p_empty_begin = max(0, min(nstate_p, nhomo - ncore_g))
        cp.nsig = nsig
        cp.nomega_sigma, cp.step_sigma, cp.eta = nomega_sigma, step_sigma, eta
        h = nomega_sigma // 2
        sig = np.zeros((nsig, 2 * h + 1, 2))
        eqp_g, eqp_z, zz = np.zeros(nsig), np.zeros(nsig), np.zeros(nsig)
        rank = np.zeros(nomega_imag + nomega_real, dtype=np.int32)
        omr = np.zeros(nomega_real)
        cr = ContourResult()
        cr.sigma, cr.energy_qp_g, cr.energy_qp_z, cr.zz = _ptr(sig), _ptr(eqp_g), _ptr(eqp_z), _ptr(zz)
        cr.rank = rank.ctypes.data_as(C.POINTER(C.c_int))
        cr.omega_real = _ptr(omr)
        self._check(self._lib.rigw_gw_selfenergy_contour(self._h, C.byref(cp), C.byref(cr)),
                    "rigw_gw_selfenergy_contour")
        full = e.copy()
        full[nsemin - 1:nsemax] = eqp_g
        ehomo, elumo = -np.inf, np.inf
        for st in range(nsemin, nsemax + 1):
            if occ[st - 1] / 2.0 > empty:
                ehomo = max(ehomo, full[st - 1])
            if occ[st - 1] / 2.0 < 1.0 - empty:
                elumo = min(elumo, full[st - 1])
        return ContourOutput(sig[..., 0].T + 1j * sig[..., 1].T, step_sigma * np.arange(-h, h + 1), omr,
                             cr.de_max, rank, eqp_g, eqp_z, zz, ehomo, elumo, self.last_stats()["total_ms"])

    def g0w0_from_ao(self, eri3, index_basis: np.ndarray, c_matrix: np.ndarray, energy: np.ndarray,
                     occupation: np.ndarray, nomega: int, nsemin: int, nsemax: int, precision: int = RIGW_FP64,
                     aomo_precision: int = RIGW_FP64, **grid) -> G0W0Output:
        """The drop-in path from the AO tensor: the W-window transform (m empty, n
        occupied) and the Sigma transform (m all states, n the Sigma states) on the
        device, then the solve in device-pointer mode, as
        polarizability_grid_scalapack / gw_selfenergy_imag_scalapack call
        calculate_eri_3center_mo themselves (src/m_gw_selfenergy_grid.f90:92, 270).
        ``eri3`` is [naux, npair], host memory (uploaded once) or a CUDA tensor."""
        import torch
        from .synth import GWInstance
        dev = eri3 if (hasattr(eri3, "is_cuda") and eri3.is_cuda) else \
            torch.from_numpy(np.ascontiguousarray(eri3, dtype=np.float64)).to(f"cuda:{self.device}")
        e = np.ascontiguousarray(energy, dtype=np.float64)
        occ = np.ascontiguousarray(occupation, dtype=np.float64)
        nstate = e.size
        nocc = int(np.sum(occ > 0))
        m_ia = self.calculate_eri_3center_mo(dev, index_basis, c_matrix, nocc + 1, nstate, 1, nocc, aomo_precision)
        m_pm = self.calculate_eri_3center_mo(dev, index_basis, c_matrix, 1, nstate, nsemin, nsemax, aomo_precision)
        inst = GWInstance(nocc=nocc, nvirt=nstate - nocc, naux=int(dev.shape[0]), nomega=nomega, energy=e,
                          occupation=occ, m_ia=None, m_sigma=None, nsemin=nsemin, nsemax=nsemax, **grid)
        small = {"e_occ": e[:nocc], "e_virt": e[nocc:], "occ_occ": occ[:nocc], "occ_virt": occ[nocc:], "e_p": e,
                 "e_sig": e[nsemin - 1:nsemax], "occ_sig": occ[nsemin - 1:nsemax]}
        arrays = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev.device) for k, v in small.items()}
        arrays.update(m_ia=m_ia, m_pm=m_pm)
        return self.g0w0(inst, precision, device_arrays=arrays)


class WPol:
    """Resident screened interaction (the device-side wpol of the reference)."""

    def __init__(self, eng: Engine, handle: C.c_void_p, naux: int, nomega: int):
        self.eng = eng
        self.handle = handle
        self.naux = naux
        self.nomega = nomega

    def chi(self) -> np.ndarray:
        out = np.zeros((self.nomega, self.naux, self.naux))
        self.eng._check(self.eng._lib.rigw_wpol_chi(self.eng._h, self.handle, _ptr(out)), "rigw_wpol_chi")
        return out

    def release(self):
        if self.handle:
            self.eng._lib.rigw_wpol_release(self.eng._h, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop (rigw_server_*): submit G0W0 problems from
    any thread, wait for their results by ticket."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, workers: int = 2, max_batch: int = 64):
        self._lib = lib()
        L = self._lib
        L.rigw_server_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_size_t, C.c_int, C.c_int]
        L.rigw_server_submit.argtypes = [C.c_void_p, C.POINTER(Problem), C.POINTER(Result), C.POINTER(C.c_uint64)]
        L.rigw_server_poll.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_int)]
        L.rigw_server_wait.argtypes = [C.c_void_p, C.c_uint64, C.c_int64, C.c_char_p, C.c_size_t]
        L.rigw_server_counters.argtypes = [C.c_void_p] + [C.POINTER(C.c_longlong)] * 3
        L.rigw_server_destroy.argtypes = [C.c_void_p]
        L.rigw_server_info.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_int), C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int64)]
        L.rigw_server_stats_get.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        h = C.c_void_p()
        rc = L.rigw_server_create(C.byref(h), device, hbm_budget_bytes, workers, max_batch)
        if rc:
            raise RigwError(rc, "rigw_server_create")
        self._h = h
        self._helper = Engine.__new__(Engine)      # problem/result builders only (no context)
        self._pending = {}

    def submit(self, inst, precision: int = RIGW_FP64, device_arrays=None, qp_only: bool = False) -> int:
        p, keep = Engine.make_problem(self._helper, inst, precision, device_arrays, qp_only=qp_only)
        r, bufs = Engine._alloc_result(self._helper, p)
        pp = Problem()
        C.pointer(pp)[0] = p
        t = C.c_uint64()
        rc = self._lib.rigw_server_submit(self._h, C.byref(pp), C.byref(r), C.byref(t))
        if rc:
            raise RigwError(rc, "rigw_server_submit")
        self._pending[t.value] = (pp, r, bufs, keep)
        return t.value

    def done(self, ticket: int) -> bool:
        d = C.c_int()
        self._lib.rigw_server_poll(self._h, ticket, C.byref(d))
        return bool(d.value)

    def info(self, ticket: int) -> tuple[bool, int, int]:
        """(done, submit time, completion time); times in ns of time.monotonic_ns's clock."""
        d, a, b = C.c_int(), C.c_int64(), C.c_int64()
        rc = self._lib.rigw_server_info(self._h, ticket, C.byref(d), C.byref(a), C.byref(b))
        if rc:
            raise RigwError(rc, "rigw_server_info")
        return bool(d.value), a.value, b.value

    def wait(self, ticket: int, timeout_s: float = 600.0) -> G0W0Output:
        buf = C.create_string_buffer(512)
        rc = self._lib.rigw_server_wait(self._h, ticket, int(timeout_s * 1e9), buf, 512)
        if rc == 6:
            raise RigwError(rc, f"ticket {ticket} not done after {timeout_s} s")
        pp, r, bufs, keep = self._pending.pop(ticket)
        if rc:
            raise RigwError(rc, buf.value.decode())
        return Engine._output(r, bufs)

    def stats(self) -> dict:
        st = ServerStats()
        self._lib.rigw_server_stats_get(self._h, C.byref(st))
        return {"batches": list(st.batches), "completed": list(st.completed), "queued": list(st.queued),
                "requeued": list(st.requeued), "failed": st.failed, "hold_s": st.hold_ns * 1e-9,
                "device_s": [st.device_ms[0] * 1e-3, st.device_ms[1] * 1e-3],
                "build_s": [st.build_ms[0] * 1e-3, st.build_ms[1] * 1e-3],
                "capture_s": [st.capture_ms[0] * 1e-3, st.capture_ms[1] * 1e-3],
                "alloc_s": [st.alloc_ms[0] * 1e-3, st.alloc_ms[1] * 1e-3],
                "busy_s": [st.busy_ns[k] * 1e-9 for k in range(st.workers)]}

    def counters(self) -> dict:
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        self._lib.rigw_server_counters(self._h, C.byref(a), C.byref(b), C.byref(c))
        return {"completed": a.value, "batches": b.value, "queued": c.value}

    def close(self):
        if self._h:
            self._lib.rigw_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
