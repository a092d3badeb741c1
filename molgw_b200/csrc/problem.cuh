// Per-molecule device descriptor of one G0W0 problem and its workspace.
//
// HBM layout of one problem (all float64, row-major, padded):
//   mp      [nia_pad][npad]              W-window M tensor, transition-major (P contiguous)
//   tnorm   [nia_pad]                    |M_t|^2
//   dscale  [nomega][nia_pad]            D_w(t) = 2*docc*de/(w^2+de^2)
//   eps     [nomega][npad][npad]         eps(iw) = 1 - chi0 (upper part), then U with eps = U^T U
//   rhs     [nomega][npad][ldb]          [ I | M_sigma ] -> [ U^-T | U^-T M_sigma ]
//                                        (either part may be absent: moff = 0 / ncm = 0)
//   winv    [nomega][npanel][64][64]     inverse of each diagonal U block
//   colsq   [nomega][npanel][ldb]        per-panel column sums of squares of U^-T [I | M_sigma]
//   logdet  [nomega][npanel]             per-panel sum of log pivots
//   mnorm   [ncm]                        |M_sigma column|^2
//   vchiv   [nomega][ncm]                M_pm^T chi(iw) M_pm
//   ew      [nomega][2]                  per-frequency E_RPA / E_GW integrands
// npad = naux rounded up to the Cholesky panel (64); padded rows/columns hold
// the identity in eps and zeros in M, which leaves every energy term and every
// Sigma contribution unchanged.
#pragma once
#include "common.cuh"

namespace rigw {

struct ProbDev {
  // ---- shapes
  int naux, npad, nocc, nvirt, nia, nia_pad, nomega, npanel;
  int nsig, nstate_p, ncm, ldb;          // ncm = nsig*nstate_p rounded up to 8; ldb = moff + ncm
  int moff;                              // first M_sigma column of rhs (npad when the I-part is present, else 0)
  int nc, nsigma_half;                   // Sigma evaluation points; real grid has 2*nsigma_half+1 points
  int technique;                         // 0: Pade, 1: polynomial (homolumo)
  int want_identity;                     // 1 when the I-part (tr eps^-1 for E_GW) is solved
  double efermi, step_sigma, eta;
  // ---- inputs (device)
  const double* m_in;        // [nia][naux]
  const double* e_occ;       // [nocc]
  const double* e_virt;      // [nvirt]
  const double* occ_occ;     // [nocc]
  const double* occ_virt;    // [nvirt]
  // second spin channel: transitions nia1 .. nia-1 (nocc2 x nvirt2, a fastest)
  int nocc2, nvirt2, nia1;
  const double* m_in2;       // [nocc2*nvirt2][naux]
  const double* e_occ2;      // [nocc2]
  const double* e_virt2;     // [nvirt2]
  const double* occ_occ2;    // [nocc2]
  const double* occ_virt2;   // [nvirt2]
  const double* omega;       // [nomega] imaginary parts
  const double* weight;      // [nomega]
  const double* msig_in;     // [nsig*nstate_p][naux]
  const double* e_p;         // [nstate_p]
  const double* e_sig;       // [nsig]   energy0 of the Sigma states
  const double* xc_sig;      // [nsig]   Sigma_x - V_xc (may be nullptr: zero)
  const double* zcalc;       // [nc] complex (re, im) evaluation points
  // ---- workspace (device)
  double* mp;
  void* xs;                  // split precision: [wgroup][2][npad][kpad] bf16 hi/lo of M sqrt(D_w);
                             // Ozaki: [wgroup][slices][npad][kpad] int8 slices of M sqrt(D_w) 2^-e
  int kpad;                  // transitions padded to the tensor-core K tile (== nia_pad)
  int wgroup;                // frequencies per split group (one buffer, reused group by group)
  int slices;                // Ozaki slices (0: not Ozaki)
  int split_t;               // transitions per item of the split / slice / row-max kernels
  unsigned long long* rmax;  // Ozaki: [nomega][npad] max_t |S_pt| as double bits (atomicMax)
  int* xexp;                 // Ozaki: [nomega][npad] row exponents e_p
  double* tnorm;
  double* dscale;
  double* eps;
  double* rhs;
  double* winv;
  double* colsq;
  double* logdet;
  double* mnorm;
  double* vchiv;
  double* ew;
  double* treps;             // [nomega] tr eps(iw), summed from the matrix that is factorized
  // ---- outputs (device)
  double* out_energies;      // [2]  erpa, egw
  double* sigma_calc;        // [nsig][nc] complex
  double* sigma_real;        // [nsig][2*nsigma_half+1] complex
  double* qp;                // [nsig][4]  energy_qp_g, energy_qp_z, zz (graphical), zz (linearized)
  int* err;                  // device error bitmask
};

}  // namespace rigw
