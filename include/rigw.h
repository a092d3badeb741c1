/*
 * rigw.h - C ABI of the B200 RI-GW engine (imaginary-frequency G0W0 hot path of MOLGW).
 *
 * Every entry point returns an int status: RIGW_OK (0) or a positive error
 * code; none aborts the caller.  rigw_last_error(ctx) gives the message of the
 * last failure on that context.  Arrays are plain pointers in C (row-major)
 * order, which is the memory order of the Fortran column-major arrays named in
 * each comment; the ``_dev`` flag of a problem says that its pointers are CUDA
 * device pointers instead of host pointers.
 *
 * Reference interfaces replaced (MOLGW 3.4, paths within its source tree):
 *   rigw_imag_grid              sf_init IMAGINARY_QUAD grid   src/m_spectral_function.f90:286-306
 *                               + coeffs_gausslegint           src/m_numerical_tools.f90:35-82
 *   rigw_eri_3center_mo         calculate_eri_3center_mo      src/m_eri_ao_mo.f90:416-582
 *   rigw_polarizability_imag    polarizability_grid_scalapack src/m_gw_selfenergy_grid.f90:33-209
 *   rigw_wpol_chi               wpol%chi(:,:,iomega) (the DGEMM at src/m_gw_selfenergy_grid.f90:179-188)
 *   rigw_gw_selfenergy_imag     gw_selfenergy_imag_scalapack  src/m_gw_selfenergy_grid.f90:213-338
 *   rigw_qp_solve               se_pade_fit / self_energy_polynomial  src/m_selfenergy_tools.f90:965-1033
 *                               find_qp_energy_linearization  src/m_selfenergy_tools.f90:202-249
 *                               find_qp_energy_graphical      src/m_selfenergy_tools.f90:253-420
 *   rigw_g0w0, rigw_g0w0_batch  the sequence of selfenergy_evaluation for
 *                               imaginary_axis_pade / _homolumo, src/m_selfenergy_evaluation.f90:214-246,587-611
 *   rigw_sox_selfenergy_imag    sox_selfenergy_imag_grid      src/m_g3w2_selfenergy.f90:2482-2591
 *                               (GW+SOX_PADE: added to sigma_calc before the Pade fit,
 *                               src/m_selfenergy_evaluation.f90:494-503)
 *   rigw_sosex_selfenergy_imag  sosex_selfenergy_imag_grid    src/m_g3w2_selfenergy.f90:2200-2478
 *   rigw_g3w2_selfenergy_imag   g3w2_selfenergy_imag_grid     src/m_g3w2_selfenergy.f90:2018-2196
 *                               (GW+SOSEX_PADE: added after SOX, src/m_selfenergy_evaluation.f90:498-500)
 *   rigw_eri_2center            calculate_eri_2center (LIBCINT int2c2e) src/m_eri_calculate.f90:1049-1262
 *   rigw_eri_3center_raw        the 3-center shell loop of calculate_eri_3center_scalapack
 *                               (LIBCINT int3c2e)              src/m_eri_calculate.f90:1584-1850
 *   rigw_eri_3center            calculate_eri_3center_scalapack with the metric and the
 *                               x0.5 diagonal convention       src/m_eri_calculate.f90:1584-1950
 *   rigw_gw_density_matrix_imag gw_density_matrix_imag        src/m_mbpt_density_matrix.f90:491-640
 *                               (pt_density_matrix GW_IMAGINARY, src/m_dm_mbpt_driver.f90:117-122)
 *   rigw_gw_selfenergy_contour  gw_selfenergy_contour         src/m_gw_selfenergy_grid.f90:342-551
 *                               + sf_vsqrt_chi_vsqrt_rpa(low_rank) src/m_spectral_function.f90:779-921
 *                               + the QP equation of G0W0_CONTOUR, src/m_selfenergy_evaluation.f90:239-240,587-611
 */
#ifndef RIGW_H
#define RIGW_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RIGW_API __attribute__((visibility("default")))
#else
#define RIGW_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define RIGW_VERSION 1

enum rigw_status {
  RIGW_OK = 0,
  RIGW_ERR_ARG = 1,        /* invalid argument (shape, null pointer, range)            */
  RIGW_ERR_CUDA = 2,       /* CUDA runtime error                                        */
  RIGW_ERR_NOMEM = 3,      /* device allocation failed or HBM budget exceeded           */
  RIGW_ERR_NOT_SPD = 4,    /* eps(iw) not positive definite (a Cholesky pivot <= 0)     */
  RIGW_ERR_NUMERIC = 5,    /* non-finite QP energy or singular Pade recursion           */
  RIGW_ERR_TIMEOUT = 6,    /* a bounded wait expired                                    */
  RIGW_ERR_UNSUPPORTED = 7, /* precision or option not available in this build          */
  RIGW_ERR_CANCELLED = 8   /* request loop destroyed before the request ran               */
};

/* Arithmetic of the chi0 = M D M^T contraction (the eps factorization, Sigma and
 * the QP solve are FP64 in every mode). */
enum rigw_precision {
  RIGW_FP64 = 0,           /* FP64 DMMA tensor cores end to end (the drop-in)            */
  RIGW_BF16X3 = 1,         /* split BF16 hi/lo products on tcgen05, FP32 accumulation    */
  RIGW_OZAKI_INT8 = 16     /* + s (3 <= s <= 7): Ozaki-sliced INT8 products on tcgen05,
                              s signed 7-bit slices per row, exact INT32 accumulation,
                              FP64 recombination; use RIGW_OZAKI(s)                      */
};
#define RIGW_OZAKI(s) (RIGW_OZAKI_INT8 + (s))
#define RIGW_OZAKI_MIN_SLICES 3
#define RIGW_OZAKI_MAX_SLICES 7

enum rigw_technique {
  RIGW_PADE = 0,           /* imaginary_axis_pade: Thiele continuation                    */
  RIGW_HOMOLUMO = 1        /* imaginary_axis_homolumo: quadratic fit in the gap          */
};

#define RIGW_PROBLEM_DEVICE_POINTERS 1
/* Compute only what the QP energies need: skips the tr eps^-1 solve behind
 * 'GW  correlation energy' (egw is returned as NaN); E_RPA is still computed. */
#define RIGW_PROBLEM_QP_ONLY 2
/* Occupations are per spin channel (nspin = 2): output_homolumo then uses
 * spin_fact = 1 instead of 2.  Implied when the second channel is present. */
#define RIGW_PROBLEM_SPIN_CHANNEL 4

typedef struct rigw_ctx rigw_ctx;
typedef struct rigw_wpol rigw_wpol;

/* One G0W0 problem on the imaginary axis: closed shell (nspin = 1), or the W
 * window of an open-shell system with its second spin channel below (nspin = 2). */
typedef struct rigw_problem {
  int naux;                  /* auxiliary functions kept (nauxil_global)                  */
  int nocc, nvirt;           /* W window: occupied ncore_W+1..nhomo_W, virtual nlumo_W..nvirtual_W-1 */
  int nomega;                /* nomega_chi_imag                                           */
  const double* omega;       /* [nomega] imaginary parts of wpol%omega; NULL: built here   */
  const double* weight;      /* [nomega] wpol%weight_quad; NULL: built here               */
  const double* m_ia;        /* [nocc][nvirt][naux] = eri_3center_mo(naux, a, i)           */
  const double* e_occ;       /* [nocc]  energy(i)  (Ha)                                   */
  const double* e_virt;      /* [nvirt] energy(a)                                         */
  const double* occ_occ;     /* [nocc]  occupation(i)                                     */
  const double* occ_virt;    /* [nvirt] occupation(a)                                     */
  int nstate_p;              /* p = ncore_G+1 .. nvirtual_G-1                              */
  int nsig;                  /* Sigma states nsemin..nsemax                               */
  const double* m_pm;        /* [nsig][nstate_p][naux] = eri_3center_mo(naux, p, m)        */
  const double* e_p;         /* [nstate_p] energy(p) in G (energy_g under force_energy_qp)  */
  const double* e_sig;       /* [nsig] energy0 of the QP equation (mean-field energies)   */
  const double* occ_sig;     /* [nsig] occupation of the Sigma states (HOMO/LUMO output)   */
  const double* exchange_m_vxc; /* [nsig] Sigma_x - V_xc; NULL: zero (G0W0@HF)             */
  int technique;             /* rigw_technique                                            */
  int nomega_sigma_calc;     /* Sigma evaluation points (<= 128)                          */
  double step_sigma_calc;
  const double* omega_calc;  /* [nomega_sigma_calc][2] complex points; NULL: efermi + i*step*k, k from 0 */
  int nomega_sigma;          /* real grid has 2*(nomega_sigma/2)+1 points                 */
  double step_sigma;
  double eta;
  double efermi;             /* se_init efermi (mid-gap of the G energies, or mu_origin)   */
  int precision;             /* rigw_precision                                            */
  int flags;                 /* RIGW_PROBLEM_DEVICE_POINTERS                               */
  /* Second spin channel of the W window (nspin = 2; nocc_2 = 0 for a closed shell):
   * its transitions join those of the first channel in one chi0, as the spin index
   * of MOLGW's transition table does (src/m_gw_selfenergy_grid.f90:118-149), with
   * per-spin occupations (1 or 0).  Sigma and the QP equation then run per spin
   * (rigw_gw_selfenergy_imag + rigw_qp_solve with the resident factors); the fused
   * rigw_g0w0* calls take the first channel's Sigma states. */
  int nocc_2, nvirt_2;
  const double* m_ia_2;      /* [nocc_2][nvirt_2][naux] = eri_3center_mo(naux, a, i, 2)     */
  const double* e_occ_2;     /* [nocc_2]  energy(i, 2)                                     */
  const double* e_virt_2;    /* [nvirt_2] energy(a, 2)                                     */
  const double* occ_occ_2;   /* [nocc_2]  occupation(i, 2)                                 */
  const double* occ_virt_2;  /* [nvirt_2] occupation(a, 2)                                 */
} rigw_problem;

/* Outputs of one problem; every array is caller-owned host memory (or device
 * memory under RIGW_PROBLEM_DEVICE_POINTERS) and may be NULL when not wanted. */
typedef struct rigw_result {
  double erpa, egw;          /* 'RPA correlation energy (Ha)', 'GW  correlation energy (Ha)' */
  double* sigma_calc;        /* [nsig][nomega_sigma_calc][2] se%sigma_calc                 */
  double* sigma;             /* [nsig][2*(nomega_sigma/2)+1][2] se%sigma on the real grid   */
  double* energy_qp_g;       /* [nsig] graphical QP energies (the reported ones)           */
  double* energy_qp_z;       /* [nsig] linearized QP energies                              */
  double* zz;                /* [nsig] Z of the graphical solution                         */
  double ehomo, elumo;       /* output_homolumo over the Sigma range (Ha)                   */
  double device_ms;          /* GPU time of the solve (CUDA events)                        */
} rigw_result;

/* Per-call statistics of the last solve on a context (the device-side analogue of
 * MOLGW's stage timers timer_rpa_dynamic / timer_gw_self, src/m_timing.f90:268-284).
 * After rigw_eri_3center_mo*: stage_ms = upload + unpack of the AO tensor, the two
 * products with their operand splits, download of the result; chunks = auxiliary
 * chunks (timer_aomo_gw).  After rigw_sox_selfenergy_imag: stage_ms[0] = uploads,
 * operand transposes and download, [1] = the (p q|j c) products, [3] = the
 * frequency sums; chunks = Sigma-state chunks (timer_vertex_selfenergy). */
typedef struct rigw_stats {
  double stage_ms[4];        /* CUDA-event times: input packing, chi0 contraction,
                                eps factorization + triangular solves, energies + Sigma + QP */
  double total_ms;
  int kernel_launches;       /* kernels launched by the last solve                        */
  int graph_replayed;        /* 1 when the launch sequence was a CUDA-graph replay        */
  size_t device_bytes_in_use, device_bytes_peak;
  int chunks;                /* problem-frequency chunks the batch was split into      */
  int waves;                 /* plans run one after the other under the memory budget  */
} rigw_stats;

/* ---- context ---------------------------------------------------------------- */
RIGW_API int rigw_create(rigw_ctx** ctx, int device, size_t hbm_budget_bytes);
RIGW_API int rigw_destroy(rigw_ctx* ctx);
RIGW_API const char* rigw_last_error(const rigw_ctx* ctx);
RIGW_API int rigw_version(void);
RIGW_API int rigw_last_stats(const rigw_ctx* ctx, rigw_stats* stats);
/* Bytes of device memory a problem of these sizes needs (admission by footprint). */
RIGW_API size_t rigw_footprint_bytes(int naux, int nocc, int nvirt, int nomega, int nstate_p, int nsig,
                            int precision);

/* ---- building blocks -------------------------------------------------------- */
/* Gauss-Legendre imaginary grid: omega_k = 2x/(1-x), weight_k = 2w/(1-x)^2. */
RIGW_API int rigw_imag_grid(int nomega, double* omega, double* weight);

/* AO->MO: out[n][m][P] = sum_{mu,nu} C[m][mu] C[n][nu] B(mu nu, P) for
 * m in [mstate_min, mstate_max], n in [nstate_min, nstate_max] (1-based).
 * eri3 is [naux][npair] (eri_3center(npair, naux)), index_basis [npair][2]
 * 1-based, diagonal pairs stored x0.5; c_matrix is [nstate][nbf]
 * (c_matrix(nbf, nstate)); out is [n_count][m_count][naux]. Host pointers. */
RIGW_API int rigw_eri_3center_mo(rigw_ctx* ctx, int nbf, int nstate, int npair, int naux,
                        const int* index_basis, const double* eri3, const double* c_matrix,
                        int mstate_min, int mstate_max, int nstate_min, int nstate_max,
                        double* out);
/* The same transform with its two products in `precision`: RIGW_FP64;
 * RIGW_BF16X3 (bf16 hi/lo split of both operands, three products on the tensor
 * cores with fp32 accumulation over at most 512 basis functions, FP64 results);
 * or RIGW_OZAKI(s), 3 <= s <= 7 (each operand row scaled by a power of two to its
 * largest entry and cut into s int8 base-128 digits, exact INT32 products of the
 * digit levels i + j <= s + 1, FP64 recombination). */
RIGW_API int rigw_eri_3center_mo_precision(rigw_ctx* ctx, int nbf, int nstate, int npair, int naux,
                                           const int* index_basis, const double* eri3, const double* c_matrix,
                                           int mstate_min, int mstate_max, int nstate_min, int nstate_max,
                                           double* out, int precision);
/* The same with ``flags``: RIGW_PROBLEM_DEVICE_POINTERS reads eri3 and writes out
 * in device memory (index_basis and c_matrix stay host arrays), so that the MO
 * tensor can go straight into rigw_g0w0 / rigw_polarizability_imag in device-
 * pointer mode, as polarizability_grid_scalapack calls the transform itself
 * (src/m_gw_selfenergy_grid.f90:92): the AO tensor crosses PCIe once. */
RIGW_API int rigw_eri_3center_mo_ex(rigw_ctx* ctx, int nbf, int nstate, int npair, int naux,
                                    const int* index_basis, const double* eri3, const double* c_matrix,
                                    int mstate_min, int mstate_max, int nstate_min, int nstate_max, double* out,
                                    int precision, int flags);

/* chi0, eps(iw) = 1 - chi0 and its factorization for every frequency; keeps the
 * factors resident on the device in *wpol.  Uses the W-window fields of
 * ``prob`` (naux..occ_virt, nomega, omega, weight, precision, flags). */
RIGW_API int rigw_polarizability_imag(rigw_ctx* ctx, const rigw_problem* prob, double* erpa, double* egw,
                             rigw_wpol** wpol);
/* wpol%chi(:,:,iomega) = (1-chi0)^-1 chi0 for all frequencies, [nomega][naux][naux]. */
RIGW_API int rigw_wpol_chi(rigw_ctx* ctx, const rigw_wpol* wpol, double* chi);
/* Sigma_c on the evaluation points from resident factors; uses the Sigma fields
 * of ``prob``; writes result->sigma_calc. */
RIGW_API int rigw_gw_selfenergy_imag(rigw_ctx* ctx, const rigw_wpol* wpol, const rigw_problem* prob,
                            rigw_result* result);
RIGW_API int rigw_wpol_release(rigw_ctx* ctx, rigw_wpol* wpol);
/* Continuation + QP equation from sigma_calc (host arrays of ``result``). */
RIGW_API int rigw_qp_solve(rigw_ctx* ctx, const rigw_problem* prob, const double* sigma_calc,
                  rigw_result* result);

/* Second-order screened exchange on the evaluation points, one spin channel
 * (sox_selfenergy_imag_grid).  With C_p[q][(j,c)] = (p q|j c) over the G window,
 *   Sigma^SOX_p(z) = - sum_{i,k occ; b empty} C_p[i][(k,b)] C_p[k][(i,b)] / (z - e_i - e_k + e_b)
 *                    - sum_{a,c empty; j occ} C_p[a][(j,c)] C_p[c][(j,a)] / (z - e_a - e_c + e_j).
 * GW+SOX adds it to sigma_calc of rigw_gw_selfenergy_imag / rigw_g0w0 and then
 * calls rigw_qp_solve. */
typedef struct rigw_sox_problem {
  int naux;
  int nocc, nvirt;           /* G window: occupied ncore_G+1..nhomo_G, empty nhomo_G+1..nvirtual_G-1 */
  const double* m_ov;        /* [nocc][nvirt][naux] = eri_3center_mo(naux, b, k) over the G window */
  int nsig;                  /* Sigma states nsemin..nsemax                                */
  const double* m_pq;        /* [nsig][nocc+nvirt][naux] = eri_3center_mo(naux, q, p)       */
  const double* energy;      /* [nocc+nvirt] energy_g over the G window (Ha)               */
  int nomega_calc;           /* evaluation points (se%omega_calc)                          */
  const double* omega_calc;  /* [nomega_calc][2] complex points                            */
  int flags;                 /* RIGW_PROBLEM_DEVICE_POINTERS                               */
} rigw_sox_problem;
/* sigma_sox: [nsig][nomega_calc][2], overwritten (host memory, or device memory
 * under RIGW_PROBLEM_DEVICE_POINTERS). */
RIGW_API int rigw_sox_selfenergy_imag(rigw_ctx* ctx, const rigw_sox_problem* prob, double* sigma_sox);

/* SOSEX without its SOX part on the evaluation points, one spin channel
 * (sosex_selfenergy_imag_grid), with W - v = v^1/2 chi v^1/2 from the resident
 * factors of ``wpol`` (its frequency grid and weights are wpol_imag's).  With
 * T_k(r; i,a) = (r m|W(i w_k) - v|i a), B1 = (r a|i m), B2 = (r i|a m), D = e_a - e_i:
 *   Sigma_m(z) = f/(2 pi) sum_k w_k sum_{s=+-1} sum_{r,i,a}
 *                T_k / (z + s i w_k - e_r) [B1 / (s i w_k - D) - B2 / (s i w_k + D)].
 * The wpol must hold the identity part of the solve (not RIGW_PROBLEM_QP_ONLY). */
typedef struct rigw_sosex_problem {
  int naux;
  int nocc, nvirt;           /* G window: occupied ncore_G+1..nhomo_G, empty nhomo_G+1..nvirtual_G-1 */
  const double* m_full;      /* [nocc+nvirt][nocc+nvirt][naux] = eri_3center_mo(naux, q, r) over the window */
  int nsig;                  /* Sigma states nsemin..nsemax                                */
  int sig_first;             /* window index (0-based) of nsemin: nsemin - ncore_G - 1     */
  const double* energy;      /* [nocc+nvirt] energy_g over the window (Ha)                 */
  int nomega_calc;
  const double* omega_calc;  /* [nomega_calc][2] complex points                            */
  double factor_sosex;       /* factor_sosex: 1, or 2 for the 2SOSEX variants              */
  int flags;                 /* RIGW_PROBLEM_DEVICE_POINTERS (m_full, sigma_sosex on the device) */
} rigw_sosex_problem;
/* sigma_sosex: [nsig][nomega_calc][2], overwritten. */
RIGW_API int rigw_sosex_selfenergy_imag(rigw_ctx* ctx, const rigw_wpol* wpol, const rigw_sosex_problem* prob,
                                        double* sigma_sosex);

/* G (W-v) G (W-v) G on the evaluation points, one spin channel, diagonal
 * (g3w2_selfenergy_imag_grid), with W - v from the resident factors of ``wpol``
 * (its frequency grid and weights are wpol_imag's).  Over the states u, v, w
 * of the G window:
 *   Sigma_p(z) = (2 pi)^-2 sum_{k', k''} w_k' w_k'' (v w|W_k'-v|u p) (u v|W_k''-v|w p)
 *      sum_{s', s'' = +-1} 1 / [(z + s' i w_k' - e_u)(z + s' i w_k' + s'' i w_k'' - e_v)(z + s'' i w_k'' - e_w)].
 * m_full must be symmetric in its two state indices (real orbitals).  The wpol
 * must hold the identity part of the solve (not RIGW_PROBLEM_QP_ONLY). */
typedef struct rigw_g3w2_problem {
  int naux;
  int nstate;                /* states of the G window, ncore_G+1 .. nvirtual_G-1          */
  const double* m_full;      /* [nstate][nstate][naux] = eri_3center_mo(naux, q, r) over the window */
  int nsig;                  /* Sigma states nsemin..nsemax                                */
  int sig_first;             /* window index (0-based) of nsemin: nsemin - ncore_G - 1     */
  const double* energy;      /* [nstate] energy_g over the window (Ha)                     */
  int nomega_calc;
  const double* omega_calc;  /* [nomega_calc][2] complex points                            */
  int flags;                 /* RIGW_PROBLEM_DEVICE_POINTERS (m_full, sigma_g3w2 on the device) */
} rigw_g3w2_problem;
/* sigma_g3w2: [nsig][nomega_calc][2], overwritten. */
RIGW_API int rigw_g3w2_selfenergy_imag(rigw_ctx* ctx, const rigw_wpol* wpol, const rigw_g3w2_problem* prob,
                                       double* sigma_g3w2);

/* ---- RI Coulomb integrals --------------------------------------------------------
 * Gaussian shells of the orbital and auxiliary bases (angular momentum <= 4).  The
 * coefficients are the reference's shell coefficients: the normalized contraction
 * coefficient of each primitive times (2/pi)^{3/4} 2^l alpha^{(2l+3)/4}, i.e. the
 * x^l component normalized up to the (nx, ny, nz) factor, which the library
 * applies with the pure (real solid harmonics, m = -l..l) or Cartesian (x^l
 * first, nx from l down and nz from 0 up) transform of each shell. */
typedef struct rigw_shell {
  double center[3];          /* Bohr                                                       */
  int am;
  int nprim;
  const double* alpha;       /* [nprim] exponents                                          */
  const double* coeff;       /* [nprim] shell coefficients as above                        */
} rigw_shell;
typedef struct rigw_ri_problem {
  int nshell;                /* orbital basis (ignored by rigw_eri_2center)                */
  const rigw_shell* shells;
  int pure;                  /* 1: pure functions, 0: Cartesian                            */
  int nshell_aux;            /* auxiliary basis                                            */
  const rigw_shell* aux_shells;
  int pure_aux;
  int npair;                 /* basis-function pairs kept (screening is the caller's)      */
  const int* index_basis;    /* [npair][2] 1-based (index_basis of src/m_eri.f90:252-320)  */
  int flags;                 /* RIGW_PROBLEM_DEVICE_POINTERS: outputs in device memory     */
} rigw_ri_problem;
/* (P|Q): v2 [naux_basis][naux_basis]. */
RIGW_API int rigw_eri_2center(rigw_ctx* ctx, const rigw_ri_problem* prob, double* v2);
/* (mu nu|P) without the metric: eri3 [naux_basis][npair]. */
RIGW_API int rigw_eri_3center_raw(rigw_ctx* ctx, const rigw_ri_problem* prob, double* eri3);
/* eri_3center(pair, P) = sum_Q (mu nu|Q) (Q|P)^-1/2 with diagonal pairs halved, as the
 * reference stores it: eri3 [nauxil_kept][npair] (room for naux_basis rows); (P|Q) is
 * diagonalized on the device and eigenvalues <= 1e-6 dropped (*nauxil_kept returns the
 * count).  The kept eigenpairs come in the eigensolver's order: the result equals the
 * reference's up to an orthogonal transformation of the auxiliary index. */
RIGW_API int rigw_eri_3center(rigw_ctx* ctx, const rigw_ri_problem* prob, double* eri3, int* nauxil_kept);

/* ---- GW density matrix from the imaginary axis ----------------------------------
 * Correction to the MO density matrix of one spin channel (gw_density_matrix_imag),
 * with v^1/2 chi v^1/2 of the resident factors of ``wpol`` (its frequencies and
 * weights are wpol_imag's), for p, q in the Sigma range of the window:
 *   P_pq = -spin_fact 2/(2 pi)^2 sum_k w_k sum_s w_s sum_m (p m|W_k - v|q m)
 *          Re{ [1/(i s - e~_m + i w_k) + 1/(i s - e~_m - i w_k)] / ((i s - e~_p)(i s - e~_q)) },
 * e~ = e - mu, the s grid Gauss-Legendre on [0, 1) mapped to [0, inf) with
 * alpha = beta = 1 (nomega_sigma points).  P is symmetric and zero outside the
 * Sigma range; adding diag(occupation) and transforming to the AO basis gives
 * the correlated density matrix (update_density_matrix). */
typedef struct rigw_dm_problem {
  int naux;
  int nstate;                /* window ncore_G+1 .. nvirtual_G-1                           */
  const double* m_full;      /* [nstate][nstate][naux] = eri_3center_mo(naux, q, r) over the window */
  int nsig;                  /* Sigma states nsemin..nsemax                                */
  int sig_first;             /* window index (0-based) of nsemin                           */
  const double* energy;      /* [nstate] host, energies of the window (Ha)                */
  double mu;                 /* centre of the HOMO-LUMO gap (Ha)                          */
  int nomega_sigma;          /* points of the density-matrix frequency grid (<= 256)      */
  double spin_fact;          /* 2 for nspin = 1                                            */
  int flags;                 /* RIGW_PROBLEM_DEVICE_POINTERS (m_full, p_matrix on the device) */
} rigw_dm_problem;
/* p_matrix: [nstate][nstate] over the window, overwritten. */
RIGW_API int rigw_gw_density_matrix_imag(rigw_ctx* ctx, const rigw_wpol* wpol, const rigw_dm_problem* prob,
                                         double* p_matrix);

/* ---- contour deformation ------------------------------------------------------
 * G0W0 by contour deformation (postscf G0W0_CONTOUR), one spin channel
 * (gw_selfenergy_contour): W from the eigenpairs of v^1/2 chi0 v^1/2 at
 * nomega_imag Gauss-Legendre imaginary frequencies and at nomega_real real
 * frequencies spread linearly over 0 .. de_max, keeping the eigenvalues
 * lambda / (1 - lambda) with |.| > 1e-3 (the low-rank W); Sigma_c on the real grid
 * se%omega = step_sigma * (-n .. n), n = nomega_sigma / 2, around energy0 of each
 * state: the imaginary-axis integral plus the residues of the occupied and
 * empty states, W taken at the real frequency closest to the pole (no
 * interpolation); then the linearized and graphical QP energies.  de_max is
 * the largest pole distance over the states and the grid, as the reference
 * computes it. */
typedef struct rigw_contour_problem {
  int naux;
  int nocc_w, nvirt_w;          /* W window: occupied ncore_W+1..nhomo_W, empty nlumo_W..nvirtual_W-1 */
  const double* m_ia;           /* [nocc_w][nvirt_w][naux] = eri_3center_mo(naux, a, i)        */
  const double* e_occ_w;        /* [nocc_w] host, energies of the W window (Ha)                 */
  const double* e_virt_w;       /* [nvirt_w] host                                               */
  const double* occ_occ_w;      /* [nocc_w] host, occupations                                   */
  const double* occ_virt_w;     /* [nvirt_w] host                                               */
  int nomega_imag;              /* nomega_chi_imag (>= 1)                                       */
  int nomega_real;              /* nomega_chi_real (>= 2)                                       */
  int nstate_p;                 /* states p of the sum: ncore_G+1 .. nvirtual_G-1               */
  int p_occ_end;                /* p index (0-based) below which the occupied residues run:
                                   nlumo_G - ncore_G - 1                                        */
  int p_empty_begin;            /* p index from which the empty residues run: nhomo_G - ncore_G */
  const double* energy_p;       /* [nstate_p] host, energies of the states p (energy_g)         */
  int nsig;                     /* Sigma states nsemin..nsemax                                  */
  const double* m_pm;           /* [nsig][nstate_p][naux] = eri_3center_mo(naux, p, m)          */
  const double* energy0;        /* [nsig] host, se%energy0: energy_g of the Sigma states         */
  const double* energy_qp0;     /* [nsig] host, energies of the QP equation (the mean-field
                                   energy of find_qp_energy_*), or NULL: energy0                 */
  const double* exchange_m_vxc; /* [nsig] host, Sigma_x - V_xc, or NULL for zero                */
  int nomega_sigma;             /* se%omega has 2 * (nomega_sigma / 2) + 1 points               */
  double step_sigma;
  double eta;
  int flags;                    /* RIGW_PROBLEM_DEVICE_POINTERS: m_ia and m_pm in device memory  */
} rigw_contour_problem;
typedef struct rigw_contour_result {
  double* sigma;                /* [nsig][2n+1][2] host, or NULL                                */
  double* energy_qp_g;          /* [nsig] graphical QP energies, or NULL                        */
  double* energy_qp_z;          /* [nsig] linearized QP energies, or NULL                       */
  double* zz;                   /* [nsig] Z of the graphical solution, or NULL                  */
  int* rank;                    /* [nomega_imag + nomega_real] eigenpairs kept, or NULL         */
  double* omega_real;           /* [nomega_real] the real frequencies of W, or NULL             */
  double de_max;                /* out: the largest real frequency                              */
} rigw_contour_result;
RIGW_API int rigw_gw_selfenergy_contour(rigw_ctx* ctx, const rigw_contour_problem* prob, rigw_contour_result* result);

/* ---- fused solves ----------------------------------------------------------- */
RIGW_API int rigw_g0w0(rigw_ctx* ctx, const rigw_problem* prob, rigw_result* result);
/* Many problems of different sizes in one launch sequence (one CUDA graph). */
RIGW_API int rigw_g0w0_batch(rigw_ctx* ctx, int nprob, const rigw_problem* probs, rigw_result* results);

/* ---- autotuner ----------------------------------------------------------------
 * No routine of the reference corresponds to this.  Times launch-shape
 * candidates on the given batch (which must fit the device in one plan): the
 * row height of the FP64 chi0 and trailing-update tiles (64 or 128 rows x 128
 * columns), the number of frequency chains, the panels per trailing update and,
 * for split precision, the frequencies per split buffer (automatic, a group
 * whose buffers fit in L2, or 8).  The fastest shapes are kept in the context
 * for every later batch of the same precision class (FP64, BF16x3, Ozaki,
 * mixed); results of a solve do not depend on them beyond floating-point
 * summation order. */
#define RIGW_TUNE_MAX_CANDIDATES 16
typedef struct rigw_tune_report {
  int chi0_rows;             /* FP64 chi0 tile rows chosen (64 or 128)                    */
  int update_rows;           /* trailing-update tile rows chosen (64 or 128)              */
  int split_group;           /* frequencies per split buffer (0: automatic)               */
  int chains;                /* frequency chains (0: automatic)                           */
  int panel_group;           /* panels per trailing update of the factorization (2..32)   */
  int precision_class;       /* 0 FP64, 1 BF16x3, 2 Ozaki INT8, 3 mixed                    */
  int ncandidates;
  int candidate[RIGW_TUNE_MAX_CANDIDATES][5];          /* (chi0_rows, update_rows, split_group, chains,
                                                          panel_group) */
  float candidate_ms[RIGW_TUNE_MAX_CANDIDATES][3];     /* chi0 stage, factorization stage, total      */
  float default_ms, tuned_ms;  /* device time of one solve before and after tuning        */
} rigw_tune_report;
RIGW_API int rigw_autotune(rigw_ctx* ctx, int nprob, const rigw_problem* probs, rigw_tune_report* report);

/* ---- request loop (continuous batching) --------------------------------------
 * No routine of the reference corresponds to this (MOLGW runs one molecule per
 * process); it serves many G0W0 solves on one GPU.  `workers` threads each own a
 * context with hbm_budget_bytes/workers of device memory (0: 85% of the free
 * memory).  Requests are admitted by device footprint into a small and a large
 * lane (footprint above 1/8 of a worker's share); a free worker takes the queued
 * requests of one lane in arrival order while their footprints fit its share (at
 * most max_batch) and solves them as one batch, so requests that arrive while
 * others run are admitted as workers and memory free up, and batches of
 * different workers overlap on the GPU.  Small requests go first; one large
 * request runs at a time, started when no small request waits or when the
 * oldest has waited 5 s.  With two or more workers, worker 0 takes only small
 * requests, on high-priority streams, and the others run on low-priority
 * streams, so that a large request's kernels do not hold up small batches.  The
 * caller keeps the
 * arrays of a submitted problem and its result buffers alive until
 * rigw_server_wait returned for its ticket. */
typedef struct rigw_server rigw_server;
RIGW_API int rigw_server_create(rigw_server** srv, int device, size_t hbm_budget_bytes, int workers,
                                int max_batch);
RIGW_API int rigw_server_submit(rigw_server* srv, const rigw_problem* prob, rigw_result* result,
                                uint64_t* ticket);
RIGW_API int rigw_server_poll(rigw_server* srv, uint64_t ticket, int* done);
/* Waits at most timeout_ns; returns the request's status (RIGW_ERR_TIMEOUT if not
 * done yet, the ticket stays valid), releases the ticket otherwise. */
/* done flag and the steady-clock (CLOCK_MONOTONIC) times of submission and
 * completion of a ticket that has not been waited for. */
RIGW_API int rigw_server_info(rigw_server* srv, uint64_t ticket, int* done, int64_t* submit_ns, int64_t* done_ns);
RIGW_API int rigw_server_wait(rigw_server* srv, uint64_t ticket, int64_t timeout_ns, char* errbuf, size_t errlen);
RIGW_API int rigw_server_counters(rigw_server* srv, long long* completed, long long* batches, long long* queued);
/* Counters of the loop: per lane (0 small, 1 large) batches started, requests
 * completed and queued, batches put back for lack of memory; failed requests;
 * time the small lane was held for a large request; device time per lane; busy
 * (wall) time per worker. */
#define RIGW_SERVER_MAX_WORKERS 16
typedef struct rigw_server_stats {
  long long batches[2], completed[2], queued[2], requeued[2];
  long long failed;
  long long hold_ns;
  double device_ms[2];       /* device time of the lane's batches (CUDA events)          */
  double build_ms[2];        /* host time building plans for the lane                    */
  double capture_ms[2];      /* host time capturing and instantiating CUDA graphs          */
  double alloc_ms[2];        /* host time in device allocations                            */
  long long busy_ns[RIGW_SERVER_MAX_WORKERS];
  int workers;
} rigw_server_stats;
RIGW_API int rigw_server_stats_get(rigw_server* srv, rigw_server_stats* stats);
/* Lets the batches already on the GPU finish, cancels the queued requests
 * (RIGW_ERR_CANCELLED) and stops the workers. */
RIGW_API int rigw_server_destroy(rigw_server* srv);

/* ---- allocation-free variant -------------------------------------------------
 * No counterpart in the reference.  The continuation + QP equation of
 * rigw_qp_solve for callers that may not allocate device memory: a host code
 * with its own device memory pool, an application whose caching allocator owns
 * the GPU, or a request loop whose memory is reserved up front (cudaMalloc
 * would also synchronize the device).  Every array is a CUDA device pointer
 * owned by the caller: sigma_calc [nsig][nomega_sigma_calc][2], e_sig [nsig],
 * exchange_m_vxc [nsig] or NULL, omega_calc [nomega_sigma_calc][2] or NULL
 * (then point k is efermi + i*step_sigma_calc*k, k = 0 .. nomega_sigma_calc-1;
 * RIGW_HOMOLUMO needs the caller's points); outputs energy_qp_g, energy_qp_z
 * (or NULL), zz (or NULL) [nsig] and sigma [nsig][2*(nomega_sigma/2)+1][2] (or
 * NULL).  ``stream`` is a cudaStream_t (NULL: default stream); the call returns
 * after the work on it is done.  Intermediates live in a fixed 1.06 MiB
 * device-resident scratch array that every GPU loading the library keeps until
 * exit; limits: nsig <= 64, nomega_sigma_calc <= 128, 2*(nomega_sigma/2)+1 <=
 * 1025 (larger sizes return RIGW_ERR_ARG).  The first call on a device looks up
 * the scratch address.  Calls share the
 * scratch: calls that overlap on the GPU race.  The message of a failure is
 * written to errbuf (errlen bytes, may be NULL). */
RIGW_API int rigw_qp_solve_noalloc(int device, int nsig, int nomega_sigma_calc, const double* omega_calc,
                                   const double* sigma_calc, const double* e_sig, const double* exchange_m_vxc,
                                   int technique, int nomega_sigma, double step_sigma, double step_sigma_calc,
                                   double eta, double efermi, double* energy_qp_g, double* energy_qp_z, double* zz,
                                   double* sigma, void* stream, char* errbuf, size_t errlen);

#ifdef __cplusplus
}
#endif
#endif /* RIGW_H */
