// Non-GEMM kernels of the imaginary-axis G0W0 path.  Every kernel takes the
// problem table and a work list, so one launch covers all frequencies of all
// molecules of a batch.
#include "kernels.cuh"
#include "qp_tools.cuh"

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
    const double* src = t < p.nia1 ? p.m_in + size_t(t) * p.naux : p.m_in2 + size_t(t - p.nia1) * p.naux;
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
  if (t < p.nia1) {
    const int i = t / p.nvirt, a = t % p.nvirt;
    de = p.e_virt[a] - p.e_occ[i];
    dcoef = 2.0 * (p.occ_occ[i] - p.occ_virt[a]) * de;
  } else if (t < p.nia) {          // second spin channel
    const int i = (t - p.nia1) / p.nvirt2, a = (t - p.nia1) % p.nvirt2;
    de = p.e_virt2[a] - p.e_occ2[i];
    dcoef = 2.0 * (p.occ_occ2[i] - p.occ_virt2[a]) * de;
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
// Diagonal block of panel k: A_kk = U^T U (upper Cholesky, in place) and
// W = U^-1 (to winv).  One CTA of kDiagThreads threads per (prob, frequency);
// the block lives in shared memory (U in its upper triangle, W^T in its
// strictly lower triangle, W(i,i) = 1/U(i,i) in invd).
//
// Right-looking over 8-wide leaves j with a one-leaf lookahead:
//   a. warp 0 factors and inverts the 8x8 leaf A_jj in registers (lanes 0..7
//      own its columns; Gaussian elimination of [A_jj | I] leaves D L^T above
//      and L^-1 below the diagonal; U_jj = D^-1/2 (D L^T), W_jj = L^-T D^-1/2);
//   b. all warps: U_j,rest = W_jj^T A_j,rest, one 8x8 DMMA tile per warp;
//   c. all warps: A_rest,rest -= U_j,rest^T U_j,rest on the upper 8x8 tiles.
//      Warp 0 takes the next leaf's diagonal tile first and factors that leaf
//      (step a of j + 1) while warps 1..7 finish the update.
// Then W by recursive doubling over blocks of 8, 16, 32, 64 rows: for each
// pair of diagonal blocks (F, G), T = U_FG W_GG and W_FG = -W_FF T (DMMA).
// Two barriers per leaf and two per doubling level; the serial part of the
// block is sixteen 8-step eliminations.
constexpr int kDiagLd = kPanel + 8;      // row stride of the block (doubles): == 8 (mod 32), so the
                                         // DMMA fragment loads (8 rows x 4 columns) hit distinct banks
constexpr int kDiagTl = 72;              // row stride of the product scratch (== 8 mod 32)
constexpr int kLeaf = 8;
constexpr int kNLeaf = kPanel / kLeaf;
constexpr int kDiagWarps = kDiagThreads / 32;

// Steps a of the leaf at rows/columns j0 .. j0+7; all 32 lanes of the calling
// warp take part (lanes 8..31 repeat lanes 0..7 and store nothing).
__device__ __noinline__ void leaf8_factor(double* S, int j0, double* piv, double* invd, int* err) {
  const int lane = threadIdx.x & 31, c = lane & 7;
  const bool owner = lane < kLeaf;
  double col[kLeaf];
#pragma unroll
  for (int i = 0; i < kLeaf; ++i) col[i] = (i <= c) ? S[(j0 + i) * kDiagLd + j0 + c] : 0.0;
  double myd = 0.0;
#pragma unroll
  for (int j = 0; j < kLeaf; ++j) {
    const double d = __shfl_sync(0xffffffffu, col[j], j);
    double aj[kLeaf];
#pragma unroll
    for (int i = j + 1; i < kLeaf; ++i) aj[i] = __shfl_sync(0xffffffffu, col[j], i);   // A(j, i)
    const double xj = ((c == j) ? 1.0 : col[j]) * __drcp_rn(d);
#pragma unroll
    for (int i = j + 1; i < kLeaf; ++i)
      if (c >= i || c <= j) col[i] -= aj[i] * xj;
    if (c == j) myd = d;
  }
  const double r = 1.0 / sqrt(myd);
  if (owner) {
    piv[j0 + c] = myd;
    invd[j0 + c] = r;
    if (!(myd > 0.0)) atomicOr(err, kErrNotSPD);
  }
  // row i <= c: U(i, c); row i > c: W(c, i) = W^T(i, c)
#pragma unroll
  for (int i = 0; i < kLeaf; ++i) {
    const double v = col[i] * __shfl_sync(0xffffffffu, r, i);
    if (owner) S[(j0 + i) * kDiagLd + j0 + c] = v;
  }
}

// W(r, c) of the finished part: r < c stored at S[c][r], the diagonal in invd.
RIGW_DEVICE_INLINE double w_at(const double* S, const double* invd, int r, int c) {
  const double s = S[c * kDiagLd + r], d = invd[r];   // both in bounds for any r, c < kPanel
  return (r < c) ? s : (r == c ? d : 0.0);
}

// Trailing-update tile (rt, ct) of leaf j0: A_rt,ct -= U_j,rt^T U_j,ct (8x8, K = 8).
RIGW_DEVICE_INLINE void leaf8_update_tile(double* S, int j0, int rt, int ct, int g, int q) {
  double c0 = 0.0, c1 = 0.0;
#pragma unroll
  for (int ks = 0; ks < 2; ++ks) {
    const int k = 4 * ks + q;
    dmma_8x8x4(c0, c1, S[(j0 + k) * kDiagLd + 8 * rt + g], S[(j0 + k) * kDiagLd + 8 * ct + g]);
  }
  double2* d = reinterpret_cast<double2*>(S + (8 * rt + g) * kDiagLd + 8 * ct + 2 * q);
  double2 v = *d;
  v.x -= c0;
  v.y -= c1;
  *d = v;
}

// Two independent update tiles: their DMMA chains and shared-memory accesses overlap.
RIGW_DEVICE_INLINE void leaf8_update_tile2(double* S, int j0, int rt0, int ct0, int rt1, int ct1, int g, int q) {
  double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
#pragma unroll
  for (int ks = 0; ks < 2; ++ks) {
    const double* row = S + (j0 + 4 * ks + q) * kDiagLd;
    const double x0 = row[8 * rt0 + g], y0 = row[8 * ct0 + g], x1 = row[8 * rt1 + g], y1 = row[8 * ct1 + g];
    dmma_8x8x4(a0, a1, x0, y0);
    dmma_8x8x4(b0, b1, x1, y1);
  }
  double2* d0 = reinterpret_cast<double2*>(S + (8 * rt0 + g) * kDiagLd + 8 * ct0 + 2 * q);
  double2* d1 = reinterpret_cast<double2*>(S + (8 * rt1 + g) * kDiagLd + 8 * ct1 + 2 * q);
  double2 v0 = *d0, v1 = *d1;
  v0.x -= a0;
  v0.y -= a1;
  v1.x -= b0;
  v1.y -= b1;
  *d0 = v0;
  *d1 = v1;
}

// The upper 8x8 tiles (rt <= ct) of the block listed from the bottom right:
// index t -> m = 15 - rt with m(m+1)/2 <= t < (m+1)(m+2)/2, ct = rt + t - m(m+1)/2.
// The tiles of leaf jb's trailing update (rt > jb) are the first n(n+1)/2 with
// n = 15 - jb, and the next leaf's diagonal tile is index n(n-1)/2.
RIGW_DEVICE_INLINE void tri_tile(int t, int& rt, int& ct) {
  int m = int((sqrtf(8.0f * float(t) + 1.0f) - 1.0f) * 0.5f);
  if ((m + 1) * (m + 2) / 2 <= t) ++m;
  if (m * (m + 1) / 2 > t) --m;
  rt = (kNLeaf - 1) - m;
  ct = rt + t - m * (m + 1) / 2;
}

__global__ void __launch_bounds__(kDiagThreads) chol_diag_kernel(const ProbDev* __restrict__ probs,
                                                                 const WorkItem* __restrict__ items, int k) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int w = wi.a;
  const int ld = p.npad;
  double* A = p.eps + size_t(w) * ld * ld + size_t(k) * kPanel * ld + size_t(k) * kPanel;
  extern __shared__ double dsm[];
  double* S = dsm;                                   // [kPanel][kDiagLd]
  double* Tb = S + kPanel * kDiagLd;                 // [64][kDiagTl] products of the W doubling
  double* piv = Tb + 64 * kDiagTl;                   // [kPanel] pivots D
  double* invd = piv + kPanel;                       // [kPanel] 1/U(i,i) = W(i,i)
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int g = lane >> 2, q = lane & 3;
  // the block: asynchronous 16-byte copies of whole rows, all in flight at once
  // (the lower triangle is loaded too and never read)
  for (int c = t; c < kPanel * kPanel / 2; c += kDiagThreads) {
    const int i = c / (kPanel / 2), l = (c % (kPanel / 2)) * 2;
    cp_async16(S + i * kDiagLd + l, A + size_t(i) * ld + l, 16);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();

  if (warp == 0) leaf8_factor(S, 0, piv, invd, p.err);
  __syncthreads();
  for (int jb = 0; jb < kNLeaf - 1; ++jb) {
    const int j0 = jb * kLeaf;
    const int nb = kNLeaf - 1 - jb;                  // tiles right of the leaf
    // b. U_j,ct = W_jj^T A_j,ct; W_jj^T(m, k) = W(j0 + k, j0 + m)
    for (int tt = warp; tt < nb; tt += kDiagWarps) {
      const int ct = jb + 1 + tt;
      double c0 = 0.0, c1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const int kk = 4 * ks + q;
        dmma_8x8x4(c0, c1, w_at(S, invd, j0 + kk, j0 + g), S[(j0 + kk) * kDiagLd + 8 * ct + g]);
      }
      __syncwarp();
      *reinterpret_cast<double2*>(S + (j0 + g) * kDiagLd + 8 * ct + 2 * q) = make_double2(c0, c1);
    }
    __syncthreads();
    // c. trailing update; warp 0: the next leaf's diagonal tile, then that leaf
    if (warp == 0) {
      leaf8_update_tile(S, j0, jb + 1, jb + 1, g, q);
      __syncwarp();
      leaf8_factor(S, j0 + kLeaf, piv, invd, p.err);
    } else {
      // tiles 0 .. n(n+1)/2 - 1 except the next leaf's diagonal tile n(n-1)/2,
      // two per iteration
      const int ntile = nb * (nb + 1) / 2 - 1, skip = nb * (nb - 1) / 2;
      constexpr int kStride = kDiagWarps - 1;
      for (int u = warp - 1; u < ntile; u += 2 * kStride) {
        int r0, c0, r1, c1;
        tri_tile(u < skip ? u : u + 1, r0, c0);
        const int u1 = u + kStride;
        if (u1 < ntile) {
          tri_tile(u1 < skip ? u1 : u1 + 1, r1, c1);
          leaf8_update_tile2(S, j0, r0, c0, r1, c1, g, q);
        } else {
          leaf8_update_tile(S, j0, r0, c0, g, q);
        }
      }
    }
    __syncthreads();
  }

  // W by recursive doubling: pairs (F, G) of diagonal blocks of b rows
  for (int b = kLeaf; b < kPanel; b *= 2) {
    const int nt = b / kLeaf, ntiles = (kPanel / (2 * b)) * nt * nt;
    for (int tt = warp; tt < ntiles; tt += kDiagWarps) {        // T = U_FG W_GG
      const int pr = tt / (nt * nt), ti = (tt / nt) % nt, tj = tt % nt;
      const int F0 = 2 * pr * b, G0 = F0 + b;
      // two accumulator chains (k-tiles of 8 split in halves) overlap the DMMA latency
      double c0 = 0.0, c1 = 0.0, e0 = 0.0, e1 = 0.0;
      for (int k0 = 0; k0 < 8 * tj + 8; k0 += 8) {
        const int ka = k0 + q, kb = k0 + 4 + q;
        dmma_8x8x4(c0, c1, S[(F0 + 8 * ti + g) * kDiagLd + G0 + ka], w_at(S, invd, G0 + ka, G0 + 8 * tj + g));
        dmma_8x8x4(e0, e1, S[(F0 + 8 * ti + g) * kDiagLd + G0 + kb], w_at(S, invd, G0 + kb, G0 + 8 * tj + g));
      }
      *reinterpret_cast<double2*>(Tb + (pr * b + 8 * ti + g) * kDiagTl + 8 * tj + 2 * q) =
          make_double2(c0 + e0, c1 + e1);
    }
    __syncthreads();
    for (int tt = warp; tt < ntiles; tt += kDiagWarps) {        // W_FG = -W_FF T, stored transposed
      const int pr = tt / (nt * nt), ti = (tt / nt) % nt, tj = tt % nt;
      const int F0 = 2 * pr * b, G0 = F0 + b;
      double c0 = 0.0, c1 = 0.0, e0 = 0.0, e1 = 0.0;
      for (int k0 = 8 * ti; k0 < b; k0 += 8) {
        const int ka = k0 + q, kb = k0 + 4 + q;
        dmma_8x8x4(c0, c1, w_at(S, invd, F0 + 8 * ti + g, F0 + ka), Tb[(pr * b + ka) * kDiagTl + 8 * tj + g]);
        dmma_8x8x4(e0, e1, w_at(S, invd, F0 + 8 * ti + g, F0 + kb), Tb[(pr * b + kb) * kDiagTl + 8 * tj + g]);
      }
      S[(G0 + 8 * tj + 2 * q) * kDiagLd + F0 + 8 * ti + g] = -(c0 + e0);
      S[(G0 + 8 * tj + 2 * q + 1) * kDiagLd + F0 + 8 * ti + g] = -(c1 + e1);
    }
    __syncthreads();
  }

  // U back into eps (upper triangle); W to winv, dense row-major: the strictly
  // lower 32x32 blocks are zeros, the upper ones go through a per-warp
  // transposition tile (warps 0..3, in the product scratch) so that both the
  // shared reads and the global writes are contiguous
  double* W = p.winv + (size_t(w) * p.npanel + k) * kPanel * kPanel;
#pragma unroll 4
  for (int idx = t; idx < kPanel * kPanel; idx += kDiagThreads) {
    const int i = idx / kPanel, l = idx % kPanel;
    if (l >= i) A[size_t(i) * ld + l] = S[i * kDiagLd + l];
    else if ((i >> 5) > (l >> 5)) W[idx] = 0.0;
  }
  if (warp < 4) {
    double* tr = Tb + warp * 32 * 33;
    int n = 0;
    for (int bi = 0; bi < kPanel / 32; ++bi)
      for (int bj = bi; bj < kPanel / 32; ++bj) {
        if (n++ % 4 != warp) continue;
        const int i0 = 32 * bi, l0 = 32 * bj;
        for (int rr = 0; rr < 32; ++rr) tr[lane * 33 + rr] = w_at(S, invd, i0 + lane, l0 + rr);
        __syncwarp();
        for (int rr = 0; rr < 32; ++rr) W[(i0 + rr) * kPanel + l0 + lane] = tr[rr * 33 + lane];
        __syncwarp();
      }
  }
  if (warp == 4) {
    double sl = 0.0;
    for (int m = lane; m < kPanel; m += 32) sl += log(piv[m]);
    sl = warp_sum(sl);
    if (lane == 0) p.logdet[size_t(w) * p.npanel + k] = sl;
  }
}

size_t chol_diag_smem_bytes() {
  return (size_t(kPanel) * kDiagLd + size_t(64) * kDiagTl + 2 * kPanel) * sizeof(double);
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
  double* q = p.qp + 4 * s;
  qp_on_real_grid(reinterpret_cast<const double*>(sr), p.nsigma_half, p.efermi, p.step_sigma, 0.0, p.e_sig[s],
                  p.xc_sig ? p.xc_sig[s] : 0.0, q);
  const double eqp_g = q[0], eqp_z = q[1];
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
