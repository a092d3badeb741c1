// Non-GEMM kernels of the imaginary-axis G0W0 path.  Every kernel takes the
// problem table and a work list, so one launch covers all frequencies of all
// molecules of a batch.
#include "kernels.cuh"

namespace rigw {

namespace {

struct cplx {
  double re, im;
};
RIGW_DEVICE_INLINE cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
RIGW_DEVICE_INLINE cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
RIGW_DEVICE_INLINE cplx cmul(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
// Smith's algorithm (R. L. Smith, CACM 5 (1962) 435): no overflow for large operands.
RIGW_DEVICE_INLINE cplx cdiv(cplx a, cplx b) {
  if (fabs(b.re) >= fabs(b.im)) {
    const double r = b.im / b.re;
    const double d = b.re + b.im * r;
    return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
  }
  const double r = b.re / b.im;
  const double d = b.re * r + b.im;
  return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}
RIGW_DEVICE_INLINE cplx cconj(cplx a) { return {a.re, -a.im}; }

// Deterministic block-wide sum (fixed tree) for blockDim.x == 256.
__device__ double block_sum_256(double v, double* red /* >= 8 */) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < 8; ++w) s += red[w];
  }
  return s;  // valid in thread 0
}

}  // namespace

// ---------------------------------------------------------------------------
// Pack the W-window tensor into the padded transition-major layout; |M_t|^2 and
// D_w(t) = 2 docc de / (w^2 + de^2), the square of the factor of
// src/m_gw_selfenergy_grid.f90:131-133.
// item: (prob, t0); 8 warps, one transition row each.
__global__ void __launch_bounds__(256) pack_m_kernel(const ProbDev* __restrict__ probs,
                                                     const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int lane = threadIdx.x & 31;
  const int t = wi.a + (threadIdx.x >> 5);
  if (t >= p.nia_pad) return;
  double sq = 0.0;
  if (t < p.nia) {
    const double* src = p.m_in + size_t(t) * p.naux;
    double* dst = p.mp + size_t(t) * p.npad;
    for (int q = lane; q < p.npad; q += 32) {
      const double v = q < p.naux ? src[q] : 0.0;
      dst[q] = v;
      sq += v * v;
    }
  } else {
    double* dst = p.mp + size_t(t) * p.npad;
    for (int q = lane; q < p.npad; q += 32) dst[q] = 0.0;
  }
  sq = warp_sum(sq);
  if (lane == 0) p.tnorm[t] = sq;
  double dcoef = 0.0, de = 0.0;
  if (t < p.nia) {
    const int i = t / p.nvirt, a = t % p.nvirt;
    de = p.e_virt[a] - p.e_occ[i];
    dcoef = 2.0 * (p.occ_occ[i] - p.occ_virt[a]) * de;
  }
  for (int w = lane; w < p.nomega; w += 32) {
    const double om = p.omega[w];
    p.dscale[size_t(w) * p.nia_pad + t] = t < p.nia ? dcoef / (om * om + de * de) : 0.0;
  }
}

// ---------------------------------------------------------------------------
// rhs[w] = [ I | M_sigma^T ] for every frequency (32x32 tiles, transposing copy).
// item: (prob, i0, c0); block (32, 8).
__global__ void __launch_bounds__(256) init_rhs_kernel(const ProbDev* __restrict__ probs,
                                                       const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  __shared__ double tile[32][33];
  const int i0 = wi.a, c0 = wi.b;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int nval = p.nsig * p.nstate_p;
  for (int cc = ty; cc < 32; cc += 8) {
    const int c = c0 + cc, i = i0 + tx;
    double v = 0.0;
    if (c < p.moff) {
      v = (i == c) ? 1.0 : 0.0;
    } else {
      const int cm = c - p.moff;
      if (cm < nval && i < p.naux) v = p.msig_in[size_t(cm) * p.naux + i];
    }
    tile[cc][tx] = v;
  }
  __syncthreads();
  for (int w = 0; w < p.nomega; ++w) {
    double* dst = p.rhs + size_t(w) * p.npad * p.ldb;
    for (int ii = ty; ii < 32; ii += 8) {
      const int i = i0 + ii, c = c0 + tx;
      if (i < p.npad && c < p.ldb) dst[size_t(i) * p.ldb + c] = tile[tx][ii];
    }
  }
}

// |M_sigma column|^2.  item: (prob, cm0); one warp per column.
__global__ void __launch_bounds__(256) mnorm_kernel(const ProbDev* __restrict__ probs,
                                                    const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int lane = threadIdx.x & 31;
  const int cm = wi.a + (threadIdx.x >> 5);
  if (cm >= p.ncm) return;
  double s = 0.0;
  if (cm < p.nsig * p.nstate_p) {
    const double* src = p.msig_in + size_t(cm) * p.naux;
    for (int i = lane; i < p.naux; i += 32) s += src[i] * src[i];
  }
  s = warp_sum(s);
  if (lane == 0) p.mnorm[cm] = s;
}

// ---------------------------------------------------------------------------
// Diagonal block of panel k: A_kk = U^T U (upper Cholesky) and W = U^-1 in one
// sweep.  Gaussian elimination of the symmetric block, with the same row
// operations applied to an identity block stored in the (initially zero)
// strictly lower triangle, leaves D L^T in the upper triangle and L^-1 (unit
// diagonal implicit) in the lower one, where A = L D L^T.  Then U = D^-1/2 (D L^T)
// and W = U^-1 = L^-T D^-1/2, i.e. W[l][m] = (L^-1)[m][l] / sqrt(d_m).
// One CTA of kDiagThreads threads per (prob, frequency); thread t owns column
// l = t % kPanel and rows i = t / kPanel + kDiagGroups * r of the block.
constexpr int kDiagGroups = kDiagThreads / kPanel;        // 4
constexpr int kDiagRows = kPanel / kDiagGroups;           // 32 rows per thread

__global__ void __launch_bounds__(kDiagThreads) chol_diag_kernel(const ProbDev* __restrict__ probs,
                                                                 const WorkItem* __restrict__ items, int k) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int w = wi.a;
  const int ld = p.npad;
  double* A = p.eps + size_t(w) * ld * ld + size_t(k) * kPanel * ld + size_t(k) * kPanel;
  __shared__ double rowbuf[2][kPanel];
  __shared__ double piv[kPanel];
  __shared__ double invd[kPanel];
  const int t = threadIdx.x;
  const int l = t % kPanel;
  const int i0 = t / kPanel;
  double v[kDiagRows];
#pragma unroll
  for (int r = 0; r < kDiagRows; ++r) {
    const int i = i0 + kDiagGroups * r;
    v[r] = (l >= i) ? A[size_t(i) * ld + l] : 0.0;
  }
#pragma unroll
  for (int r = 0; r < kDiagRows; ++r) {
#pragma unroll
    for (int q = 0; q < kDiagGroups; ++q) {
      const int j = kDiagGroups * r + q;
      if (i0 == q) rowbuf[j & 1][l] = v[r];
      __syncthreads();
      const double pj = rowbuf[j & 1][j];
      if (t == 0) piv[j] = pj;
      // multiplier row: A part (l > j) or the L^-1 part (l < j); the implicit unit diagonal at l == j
      const double xj = (l == j ? 1.0 : rowbuf[j & 1][l]) / pj;
#pragma unroll
      for (int rr = r; rr < kDiagRows; ++rr) {
        const int i = i0 + kDiagGroups * rr;
        if (i > j && (l >= i || l <= j)) v[rr] -= rowbuf[j & 1][i] * xj;
      }
    }
  }
  __syncthreads();
  if (t < kPanel) {
    const double pv = piv[t];
    if (!(pv > 0.0)) atomicOr(p.err, kErrNotSPD);
    invd[t] = 1.0 / sqrt(pv);
  }
  __syncthreads();
  double* W = p.winv + (size_t(w) * p.npanel + k) * kPanel * kPanel;
#pragma unroll
  for (int r = 0; r < kDiagRows; ++r) {
    const int i = i0 + kDiagGroups * r;
    if (l >= i) A[size_t(i) * ld + l] = v[r] * invd[i];
    W[l * kPanel + i] = (l < i) ? v[r] * invd[i] : (l == i ? invd[i] : 0.0);
  }
  if (t < 32) {
    double s = 0.0;
    for (int m = t; m < kPanel; m += 32) s += log(piv[m]);
    s = warp_sum(s);
    if (t == 0) p.logdet[size_t(w) * p.npanel + k] = s;
  }
}

// ---------------------------------------------------------------------------
// Per-frequency energy integrands (src/m_gw_selfenergy_grid.f90:171-173) from
// the factorization: sum ln(lambda) = ln det eps = sum of log pivots,
// sum lambda = tr eps = npad + sum_t D_w(t) |M_t|^2, sum 1/lambda = tr eps^-1 = |U^-T|_F^2.
// item: (prob, w).
__global__ void __launch_bounds__(256) energy_kernel(const ProbDev* __restrict__ probs,
                                                     const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int w = wi.a;
  __shared__ double red[8];
  // tr eps from the matrix that was factorized (so that ln det and tr use the
  // same eps in the split-precision mode; in FP64 this equals npad + sum_t D |M_t|^2)
  const double treps = p.treps[w];
  double trinv = 0.0;
  if (p.want_identity) {
    double q = 0.0;
    for (int k = 0; k < p.npanel; ++k) {
      const double* cs = p.colsq + (size_t(w) * p.npanel + k) * p.ldb;
      const int ncol = min((k + 1) * kPanel, p.npad);
      for (int c = threadIdx.x; c < ncol; c += 256) q += cs[c];
    }
    trinv = block_sum_256(q, red);
  }
  if (threadIdx.x == 0) {
    double ld = 0.0;
    for (int k = 0; k < p.npanel; ++k) ld += p.logdet[size_t(w) * p.npanel + k];
    p.ew[2 * w + 0] = ld + p.npad - treps;
    p.ew[2 * w + 1] = p.want_identity ? (2.0 * p.npad - trinv - treps) : __longlong_as_double(0x7ff8000000000000ll);
  }
}

// Identity in the padded rows/columns of eps(iw) (upper part, columns >= naux):
// the FP64 chi0 items cover the naux x naux block only.  item: (prob, w).
__global__ void __launch_bounds__(256) pad_eps_kernel(const ProbDev* __restrict__ probs,
                                                      const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  double* E = p.eps + size_t(wi.a) * p.npad * p.npad;
  const int npadc = p.npad - p.naux;
  for (int idx = threadIdx.x; idx < npadc * p.npad; idx += 256) {
    const int j = p.naux + idx / p.npad, i = idx % p.npad;
    if (i <= j) E[size_t(i) * p.npad + j] = (i == j) ? 1.0 : 0.0;
  }
}

// tr eps(iw) = sum of the diagonal of eps as built by the chi0 stage, before the
// factorization overwrites it.  item: (prob, w).
__global__ void __launch_bounds__(256) trace_kernel(const ProbDev* __restrict__ probs,
                                                    const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int w = wi.a;
  __shared__ double red[8];
  const double* E = p.eps + size_t(w) * p.npad * p.npad;
  double s = 0.0;
  for (int i = threadIdx.x; i < p.npad; i += 256) s += E[size_t(i) * p.npad + i];
  s = block_sum_256(s, red);
  if (threadIdx.x == 0) p.treps[w] = s;
}

// v(p, m, w) = M_pm^T chi(iw) M_pm = |U^-T M_pm|^2 - |M_pm|^2  (chi = eps^-1 - 1).
// item: (prob, w, cm0); one thread per column.
__global__ void __launch_bounds__(256) vchiv_kernel(const ProbDev* __restrict__ probs,
                                                    const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int w = wi.a;
  const int cm = wi.b + threadIdx.x;
  if (cm >= p.ncm) return;
  double s = 0.0;
  for (int k = 0; k < p.npanel; ++k) s += p.colsq[(size_t(w) * p.npanel + k) * p.ldb + p.moff + cm];
  p.vchiv[size_t(w) * p.ncm + cm] = s - p.mnorm[cm];
}

// Sigma_c(z_k) for one Sigma state, src/m_gw_selfenergy_grid.f90:303-319:
//   Sigma(z) -= W(w)/(2 pi) [1/(z - e_p + i w) + 1/(z - e_p - i w)] v(p, m, w).
// item: (prob, s, kz).
__global__ void __launch_bounds__(256) sigma_kernel(const ProbDev* __restrict__ probs,
                                                    const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int s = wi.a, kz = wi.b;
  __shared__ double red[8];
  const double zr = p.zcalc[2 * kz], zi = p.zcalc[2 * kz + 1];
  double sr = 0.0, si = 0.0;
  const int n = p.nomega * p.nstate_p;
  for (int idx = threadIdx.x; idx < n; idx += 256) {
    const int w = idx / p.nstate_p, q = idx % p.nstate_p;
    const double om = p.omega[w];
    const double x = zr - p.e_p[q];
    const cplx f = cadd(cdiv({1.0, 0.0}, {x, zi + om}), cdiv({1.0, 0.0}, {x, zi - om}));
    const double c = p.weight[w] * p.vchiv[size_t(w) * p.ncm + s * p.nstate_p + q] / (2.0 * kPi);
    sr -= c * f.re;
    si -= c * f.im;
  }
  sr = block_sum_256(sr, red);
  si = block_sum_256(si, red);
  if (threadIdx.x == 0) {
    p.sigma_calc[2 * (size_t(s) * p.nc + kz)] = sr;
    p.sigma_calc[2 * (size_t(s) * p.nc + kz) + 1] = si;
  }
}

// ---------------------------------------------------------------------------
// Continuation to the real axis and the QP equation for one Sigma state:
// se_pade_fit (src/m_selfenergy_tools.f90:965-999) with the Thiele coefficients
// of calculate_pade_a (src/m_numerical_tools.f90:120-146; they depend on the
// input points only, so they are formed once per state), or
// self_energy_polynomial (:1005-1033); then find_qp_energy_linearization
// (:202-249) and find_qp_energy_graphical / find_fixed_point (:253-420).
// item: (prob, s); 256 threads; nc <= 128.
__global__ void __launch_bounds__(256) pade_qp_kernel(const ProbDev* __restrict__ probs,
                                                      const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int s = wi.a;
  const int tid = threadIdx.x;
  __shared__ cplx zs[256], row[256], aa[256];
  const int nc = p.nc;
  const int np = 2 * nc - 1;
  const int nreal = 2 * p.nsigma_half + 1;
  const cplx* zc = reinterpret_cast<const cplx*>(p.zcalc);
  const cplx* sc = reinterpret_cast<const cplx*>(p.sigma_calc) + size_t(s) * nc;
  cplx* sr = reinterpret_cast<cplx*>(p.sigma_real) + size_t(s) * nreal;

  if (p.technique == 0) {
    if (tid < np) {
      const int kk = tid - (nc - 1);
      if (kk >= 0) {
        zs[tid] = zc[kk];
        row[tid] = sc[kk];
      } else {
        zs[tid] = cconj(zc[-kk]);
        row[tid] = cconj(sc[-kk]);
      }
    }
    __syncthreads();
    if (tid == 0) aa[0] = row[0];
    for (int ip = 1; ip < np; ++ip) {
      const cplx d = row[ip - 1];
      const cplx zp = zs[ip - 1];
      __syncthreads();
      if (tid >= ip && tid < np) {
        const cplx g = row[tid];
        const cplx den = cmul(csub(zs[tid], zp), g);
        if (den.re == 0.0 && den.im == 0.0) atomicOr(p.err, kErrPade);
        row[tid] = cdiv(csub(d, g), den);
      }
      __syncthreads();
      if (tid == ip) aa[ip] = row[ip];
    }
    __syncthreads();
    for (int j = tid; j < nreal; j += 256) {
      const double wr = p.efermi + p.step_sigma * (j - p.nsigma_half);
      const double sgn = -copysign(1.0, wr - zc[0].re);
      const cplx zo = {wr, p.eta * sgn};
      cplx az_m1 = {0.0, 0.0}, az = aa[0];
      cplx bz_m1 = {1.0, 0.0}, bz = {1.0, 0.0};
      for (int ip = 1; ip < np; ++ip) {
        const cplx tt = cmul(csub(zo, zs[ip - 1]), aa[ip]);
        const cplx an = cadd(az, cmul(tt, az_m1));
        const cplx bn = cadd(bz, cmul(tt, bz_m1));
        az_m1 = az;
        az = an;
        bz_m1 = bz;
        bz = bn;
      }
      sr[j] = cdiv(az, bz);
    }
  } else {
    const int mid = nc / 2;
    const double a0 = sc[mid].re;
    const double span = zc[nc - 1].re - zc[0].re;
    const double a1 = (sc[nc - 1].re - sc[0].re) / span;
    const double a2 = (sc[nc - 1].re + sc[0].re - 2.0 * sc[mid].re) / (span * span) * 2.0;
    for (int j = tid; j < nreal; j += 256) {
      const double wr = p.efermi + p.step_sigma * (j - p.nsigma_half);
      const cplx d = {wr - zc[mid].re, -zc[mid].im};
      const cplx d2 = cmul(d, d);
      sr[j] = {a0 + a1 * d.re + a2 * d2.re, a1 * d.im + a2 * d2.im};
    }
  }
  __syncthreads();
  if (tid != 0) return;
  const double e0 = p.e_sig[s];
  const double xc = p.xc_sig ? p.xc_sig[s] : 0.0;
  const int h = p.nsigma_half;
  double eqp_z, zlin;
  if (h > 0) {
    const double w_p = p.efermi + p.step_sigma * 1.0, w_m = p.efermi - p.step_sigma * 1.0;
    double z = (sr[h + 1].re - sr[h - 1].re) / (w_p - w_m);
    z = 1.0 / (1.0 - z);
    z = fmin(fmax(z, 0.0), 1.0);
    zlin = z;
    eqp_z = z * (e0 + sr[h].re + xc);
  } else {
    zlin = 1.0;
    eqp_z = e0 + sr[h].re + xc;
  }
  double eqp_g, zg;
  if (h > 0) {
    double zw[4] = {-1.0, -1.0, -1.0, -1.0};
    double ef[4] = {0.0, 0.0, 0.0, 0.0};
    double xprev = p.efermi + p.step_sigma * (0 - h);
    double fprev = sr[0].re + xc + e0;
    for (int j = 1; j < nreal; ++j) {
      const double x = p.efermi + p.step_sigma * (j - h);
      const double f = sr[j].re + xc + e0;
      const double g0 = fprev - xprev, g1 = f - x;
      if (g0 * g1 < 0.0) {
        const double zz = 1.0 / (1.0 - (f - fprev) / (x - xprev));
        if (zz >= 0.00001 && zz > zw[3]) {
          int jf = 0;
          while (!(zz > zw[jf])) ++jf;
          for (int m = 3; m > jf; --m) {
            zw[m] = zw[m - 1];
            ef[m] = ef[m - 1];
          }
          zw[jf] = zz;
          const double gp = (g1 - g0) / (x - xprev);
          ef[jf] = xprev - g0 / gp;
        }
      }
      xprev = x;
      fprev = f;
    }
    int iq = 0;
    for (int m = 1; m < 4; ++m)
      if (zw[m] > zw[iq]) iq = m;
    if (zw[iq] > 1.0e-6) {
      eqp_g = ef[iq];
      zg = zw[iq];
    } else {
      eqp_g = e0;
      zg = 1.0;
    }
    int nfixed = 0;
    for (int m = 0; m < 4; ++m) nfixed += zw[m] > 0.0;
    if (nfixed == 0) eqp_g = e0 + sr[h].re + xc;
  } else {
    eqp_g = e0 + sr[h].re + xc;
    zg = 1.0;
  }
  double* q = p.qp + 4 * s;
  q[0] = eqp_g;
  q[1] = eqp_z;
  q[2] = zg;
  q[3] = zlin;
  if (!isfinite(eqp_g) || !isfinite(eqp_z)) atomicOr(p.err, kErrNonFinite);
}

}  // namespace rigw

namespace rigw {
// E_RPA and E_GW: sum of the per-frequency integrands weighted by W(w)/(2 pi),
// accumulated in the frequency order of the reference loop
// (src/m_gw_selfenergy_grid.f90:118-191).  One thread per problem.
__global__ void energy_sum_kernel(const ProbDev* __restrict__ probs, int nprob) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nprob) return;
  const ProbDev& p = probs[i];
  double erpa = 0.0, egw = 0.0;
  for (int w = 0; w < p.nomega; ++w) {
    erpa += p.ew[2 * w] / (2.0 * kPi) * p.weight[w];
    egw += p.ew[2 * w + 1] / (2.0 * kPi) * p.weight[w];
  }
  p.out_energies[0] = erpa;
  p.out_energies[1] = egw;
}
}  // namespace rigw
