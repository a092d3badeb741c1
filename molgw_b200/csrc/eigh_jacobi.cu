// Batched symmetric eigensolver: block two-sided Jacobi.
//
// The matrix (n a multiple of 64) is cut into nb = n / 32 block rows.  A sweep
// visits every pair of blocks (I, J) once in the round-robin order of Brent and
// Luk (1985): each round takes nb/2 disjoint pairs, nb - 1 rounds make a sweep.
// For a pair, one sweep of the scalar cyclic Jacobi method (Rutishauser's
// rotation formula, round-robin pairs of its 64 indices) runs on the 64 x 64
// subproblem S = [A_II A_IJ; A_JI A_JJ] in shared memory and accumulates the
// orthogonal Q.  (Solving S to convergence instead changes neither the number
// of outer sweeps nor the result: on the test matrices both take 11 outer
// sweeps at n = 512, the single inner sweep with a quarter of the inner work.)
// The whole matrix is then updated with the round's rotation J (the pairs' Q
// embedded at their rows and columns): every row and column belongs to exactly
// one pair, so tile (p, q) of J^T A J is Q_p^T A[P, Q] Q_q and depends only on
// tile (p, q) of A (eigh_apply_kernel, one CTA per upper tile, plus V <- V J by
// 64-row chunks).  A round is two launches over all pairs and all matrices of
// the batch; the update streams A and V once per round, against once per single
// rotation in the scalar method.
//
// A subproblem whose off-diagonal entries are all <= tau = 1e-14 ||A||_F is
// left alone; in one with a larger entry every entry above tau/4 is rotated;
// the sweeps stop when one leaves every pair alone (normwise accuracy, as
// DSYEV's).  The eigenvalues are then the diagonal of A and V[i][k] is
// component i of eigenvector k.  Every loop is bounded: a matrix that does not
// converge in 60 sweeps returns RIGW_ERR_NUMERIC.
#include <vector>

#include "engine.cuh"

namespace rigw {
namespace {

constexpr int kB = 32;            // block size
constexpr int kS = 2 * kB;        // subproblem size
constexpr int kLd = kS + 1;       // shared-memory row stride (conflict-free columns)
constexpr int kThreads = 256;
constexpr int kOuterMaxSweeps = 60;
constexpr double kRelTol = 1.0e-14;
// S, Q, rotations, kS / 2 spare doubles, the 528-entry block-pair table (as ints)
constexpr size_t kPairSmem = size_t(2 * kS * kLd + kS + kS / 2) * sizeof(double) + (kS / 2) * (kS / 2 + 1) / 2 * 4;
constexpr size_t kApplySmem = size_t(3 * kS * (kS + 4)) * sizeof(double);           // tile, two rotations

// Pair k of round r of the round-robin ordering over m (even) indices.
RIGW_DEVICE_INLINE void rr_pair(int r, int k, int m, int& a, int& b) {
  if (k == 0) {
    a = 0;
    b = 1 + r;
  } else {
    a = 1 + (r + k) % (m - 1);
    b = 1 + (r - k + (m - 1)) % (m - 1);
  }
}

// Row or column of the full matrix of index i (0..63) of the subproblem of blocks I, J.
RIGW_DEVICE_INLINE int sub_index(int i, int I, int J) { return i < kB ? I * kB + i : J * kB + (i - kB); }

// V = I and tau = 1e-14 ||A||_F for matrix blockIdx.x.
__global__ void __launch_bounds__(1024) eigh_init_kernel(const double* __restrict__ Aall, double* __restrict__ Vall,
                                                         int n, long long sA, double* __restrict__ tau) {
  const double* A = Aall + size_t(blockIdx.x) * sA;
  double* V = Vall + size_t(blockIdx.x) * sA;
  __shared__ double red[32];
  const long long nn = (long long)n * n;
  double acc = 0.0;
  for (long long idx = threadIdx.x; idx < nn; idx += blockDim.x) {
    const double x = A[idx];
    acc += x * x;
    V[idx] = (idx / n == idx % n) ? 1.0 : 0.0;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) tau[blockIdx.x] = kRelTol * sqrt(v);
  }
}

// One cyclic Jacobi sweep on the 64 x 64 symmetric S (stride kLd) in shared
// memory, accumulating the rotations into Q (starts as the identity).  Per round:
// warp 0 forms the round's 32 rotations (lane k: pair k); then, after one barrier,
// the whole round is applied in one pass: thread t updates the 2 x 2 blocks
// G_k S[{a_k,b_k},{a_l,b_l}] G_l^T for the upper block pairs k <= l of the table
// blk (writing (l, k) as the transpose, so S stays exactly symmetric) and 8 rows
// of columns a_k, b_k of Q.  Rotation: t = p2 / (d + sign(d) sqrt(d^2 + p2^2))
// with d = S_bb - S_aa, p2 = 2 S_ab (Rutishauser's tan of the rotation angle,
// |t| <= 1), c = 1/sqrt(1 + t^2), s = t c.
// G_k X G_l^T for the 2 x 2 block of pairs (k, l) of round r, written at (k, l)
// and, for k != l, transposed at (l, k).
RIGW_DEVICE_INLINE void rotate_block(double* S, int ak, int bk, int al, int bl, bool mirror, double ck, double sk,
                                     double cl, double sl, double x00, double x01, double x10, double x11) {
  // rows: G_k = [[c, -s], [s, c]]; columns: times G_l^T
  const double y00 = ck * x00 - sk * x10, y01 = ck * x01 - sk * x11;
  const double y10 = sk * x00 + ck * x10, y11 = sk * x01 + ck * x11;
  const double z00 = cl * y00 - sl * y01, z01 = sl * y00 + cl * y01;
  const double z10 = cl * y10 - sl * y11, z11 = sl * y10 + cl * y11;
  S[ak * kLd + al] = z00;
  S[ak * kLd + bl] = z01;
  S[bk * kLd + al] = z10;
  S[bk * kLd + bl] = z11;
  if (mirror) {
    S[al * kLd + ak] = z00;
    S[bl * kLd + ak] = z01;
    S[al * kLd + bk] = z10;
    S[bl * kLd + bk] = z11;
  }
}

__device__ void inner_jacobi_sweep(double* S, double* Q, double* cs, double* sn, const int* blk, double tau) {
  const int tid = threadIdx.x;
  constexpr int kNblk = (kS / 2) * (kS / 2 + 1) / 2;   // upper 2 x 2 block pairs (528)
  static_assert(kNblk > 2 * kThreads && kNblk <= 3 * kThreads, "two block pairs per thread plus a tail");
  // this thread's block pairs e = tid and tid + kThreads (both loaded before either is
  // stored), and e = tid + 2 kThreads for the first kNblk - 2 kThreads threads; decoded once
  int bk[3], bl[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const int e = tid + m * kThreads;
    const int kl = e < kNblk ? blk[e] : 0;
    bk[m] = e < kNblk ? (kl & 0xff) : -1;
    bl[m] = kl >> 8;
  }
  const int kq = tid & 31, g = tid >> 5;   // Q: pair kq, rows 8 g .. 8 g + 7
  for (int r = 0; r < kS - 1; ++r) {
    if (tid < 32) {
      int a, b;
      rr_pair(r, tid, kS, a, b);
      const double apq = S[a * kLd + b];
      double c = 1.0, s = 0.0;
      if (fabs(apq) > tau) {
        const double d = S[b * kLd + b] - S[a * kLd + a], p2 = 2.0 * apq;
        const double t = p2 / (d + copysign(sqrt(d * d + p2 * p2), d));
        c = rsqrt(t * t + 1.0);
        s = t * c;
      }
      cs[tid] = c;
      sn[tid] = s;
    }
    __syncthreads();
    {
      double x[2][4];
      int ia[2][4];
      bool act[2];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        act[m] = sn[bk[m]] != 0.0 || sn[bl[m]] != 0.0;
        rr_pair(r, bk[m], kS, ia[m][0], ia[m][1]);
        rr_pair(r, bl[m], kS, ia[m][2], ia[m][3]);
        if (!act[m]) continue;
        x[m][0] = S[ia[m][0] * kLd + ia[m][2]];
        x[m][1] = S[ia[m][0] * kLd + ia[m][3]];
        x[m][2] = S[ia[m][1] * kLd + ia[m][2]];
        x[m][3] = S[ia[m][1] * kLd + ia[m][3]];
      }
#pragma unroll
      for (int m = 0; m < 2; ++m)
        if (act[m])
          rotate_block(S, ia[m][0], ia[m][1], ia[m][2], ia[m][3], bk[m] != bl[m], cs[bk[m]], sn[bk[m]], cs[bl[m]],
                       sn[bl[m]], x[m][0], x[m][1], x[m][2], x[m][3]);
    }
    if (bk[2] >= 0 && (sn[bk[2]] != 0.0 || sn[bl[2]] != 0.0)) {
      int ak, bkk, al, bll;
      rr_pair(r, bk[2], kS, ak, bkk);
      rr_pair(r, bl[2], kS, al, bll);
      const double x00 = S[ak * kLd + al], x01 = S[ak * kLd + bll], x10 = S[bkk * kLd + al], x11 = S[bkk * kLd + bll];
      rotate_block(S, ak, bkk, al, bll, bk[2] != bl[2], cs[bk[2]], sn[bk[2]], cs[bl[2]], sn[bl[2]], x00, x01, x10,
                   x11);
    }
    // Q: columns a, b of pair kq, rows 8 g .. 8 g + 7, loaded before they are stored
    const double sq = sn[kq];
    if (sq != 0.0) {
      const double cq = cs[kq];
      int qa_i, qb_i;
      rr_pair(r, kq, kS, qa_i, qb_i);
      double qa[8], qb[8];
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        qa[jj] = Q[(g * 8 + jj) * kLd + qa_i];
        qb[jj] = Q[(g * 8 + jj) * kLd + qb_i];
      }
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        Q[(g * 8 + jj) * kLd + qa_i] = cq * qa[jj] - sq * qb[jj];
        Q[(g * 8 + jj) * kLd + qb_i] = sq * qa[jj] + cq * qb[jj];
      }
    }
    __syncthreads();
  }
}

// One CTA per (pair k of round r, matrix w = blockIdx.y): one sweep on the
// subproblem, its Q to Qbuf.  flags[w][k] says whether the pair rotated;
// rot[w] whether any pair of matrix w did.
__global__ void __launch_bounds__(kThreads, 3) eigh_pair_kernel(const double* __restrict__ Aall,
                                                             double* __restrict__ Qbuf, int* __restrict__ flags,
                                                             int* __restrict__ rot, const double* __restrict__ tau,
                                                             int n, long long sA, int r) {
  extern __shared__ double smem[];
  double* S = smem;
  double* Q = S + kS * kLd;
  double* cs = Q + kS * kLd;
  double* sn = cs + kS / 2;
  int* blk = reinterpret_cast<int*>(sn + kS / 2) + kS;   // after kS / 2 spare doubles
  const int w = blockIdx.y, k = blockIdx.x, tid = threadIdx.x;
  const int nb = n / kB, npairs = nb / 2;
  const double* A = Aall + size_t(w) * sA;
  int I, J;
  rr_pair(r, k, nb, I, J);
  const double tw = tau[w];
  int big = 0;
  for (int idx = tid; idx < kS * kS; idx += kThreads) {
    const int i = idx / kS, j = idx % kS;
    const double x = A[size_t(sub_index(i, I, J)) * n + sub_index(j, I, J)];
    S[i * kLd + j] = x;
    Q[i * kLd + j] = (i == j) ? 1.0 : 0.0;
    if (i != j && fabs(x) > tw) big = 1;
  }
  if (!__syncthreads_or(big)) {
    if (tid == 0) flags[w * npairs + k] = 0;
    return;
  }
  // hysteresis: inside a flagged subproblem rotate down to tau/4, so that an
  // entry just above tau is not left just below it by the other rotations and
  // recreated above it by the rounding of the 64-wide updates
  for (int e = tid; e < kS / 2; e += kThreads) {   // block pairs (k, l), k <= l, row by row
    const int row0 = e * (kS / 2) - e * (e - 1) / 2;
    for (int l = e; l < kS / 2; ++l) blk[row0 + l - e] = e | (l << 8);
  }
  __syncthreads();
  inner_jacobi_sweep(S, Q, cs, sn, blk, 0.25 * tw);
  if (tid == 0) {
    flags[w * npairs + k] = 1;
    atomicOr(rot + w, 1);
  }
  double* qg = Qbuf + (size_t(w) * npairs + k) * kS * kS;
  for (int idx = tid; idx < kS * kS; idx += kThreads) qg[idx] = Q[(idx / kS) * kLd + idx % kS];
}

// Tiles of the update pass: 64 x 64 with row stride kLdT = 68 (= 4 mod 16 doubles,
// so that the DMMA fragment loads below hit 16 distinct 8-byte banks per half warp).
constexpr int kLdT = kS + 4;

// out = X^T T (transpose_x) or T X, 64 x 64 in shared memory (stride kLdT), on the
// FP64 tensor cores (mma m8n8k4): warp w computes rows 32 (w & 1) .. + 31 and
// columns 16 (w >> 1) .. + 15 as 4 x 2 fragments of 8 x 8; the result goes back into T.
RIGW_DEVICE_INLINE void tile_product(double* T, const double* X, bool transpose_x) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int q = lane >> 2, r = lane & 3;
  const int wm0 = (w & 1) * 32, wn0 = (w >> 1) * 16;
  double acc[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll 4
  for (int k4 = 0; k4 < kS / 4; ++k4) {
    const int k = 4 * k4 + r;
    double a[4], b[2];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = wm0 + 8 * i + q;
      a[i] = transpose_x ? X[k * kLdT + row] : T[row * kLdT + k];
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int col = wn0 + 8 * j + q;
      b[j] = transpose_x ? T[k * kLdT + col] : X[k * kLdT + col];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
  }
  __syncthreads();   // every read of T is done
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int row = wm0 + 8 * i + q, col = wn0 + 8 * j + 2 * r;
      *reinterpret_cast<double2*>(T + row * kLdT + col) = make_double2(acc[i][j][0], acc[i][j][1]);
    }
  __syncthreads();
}

// The rotation of round r applied to the whole matrix in one pass: every row
// and every column belongs to exactly one pair, so output tile (p, q) of
// J^T A J is Q_p^T A[P, Q] Q_q and depends only on input tile (p, q).  CTA t <
// ntri takes the upper tile (p, q), p <= q, of A (writing (q, p) as its
// transpose, which keeps A exactly symmetric); CTA t >= ntri a (64-row chunk,
// pair q) tile of V: V[chunk, Q] <- V[chunk, Q] Q_q.  Tiles whose pairs did not
// rotate are skipped (their Q is the identity).
__global__ void __launch_bounds__(kThreads) eigh_apply_kernel(double* __restrict__ Aall, double* __restrict__ Vall,
                                                              const double* __restrict__ Qbuf,
                                                              const int* __restrict__ flags, int n, long long sA,
                                                              int r) {
  extern __shared__ double smem[];
  double* T = smem;
  double* Qa = T + kS * kLdT;
  double* Qb = Qa + kS * kLdT;
  const int nb = n / kB, npairs = nb / 2, ntri = npairs * (npairs + 1) / 2;
  const int w = blockIdx.y, tid = threadIdx.x;
  const int* fl = flags + w * npairs;
  const double* qw = Qbuf + size_t(w) * npairs * kS * kS;
  int t = blockIdx.x;
  if (t < ntri) {
    int p = 0;
    while (t >= npairs - p) {   // row p of the upper triangle holds npairs - p tiles
      t -= npairs - p;
      ++p;
    }
    const int q = p + t;
    const bool fp = fl[p] != 0, fq = fl[q] != 0;
    if (!fp && !fq) return;
    int Ip, Jp, Iq, Jq;
    rr_pair(r, p, nb, Ip, Jp);
    rr_pair(r, q, nb, Iq, Jq);
    double* A = Aall + size_t(w) * sA;
    // 16-byte asynchronous copies (two doubles; a pair never straddles a 32-wide block)
    for (int c = tid; c < kS * kS / 2; c += kThreads) {
      const int i = c / (kS / 2), j = 2 * (c % (kS / 2));
      cp_async16(T + i * kLdT + j, A + size_t(sub_index(i, Ip, Jp)) * n + sub_index(j, Iq, Jq), 16);
      if (fp) cp_async16(Qa + i * kLdT + j, qw + size_t(p) * kS * kS + i * kS + j, 16);
      if (fq) cp_async16(Qb + i * kLdT + j, qw + size_t(q) * kS * kS + i * kS + j, 16);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    if (fp) tile_product(T, Qa, true);
    if (fq) tile_product(T, Qb, false);
    for (int idx = tid; idx < kS * kS; idx += kThreads) {
      const int i = idx / kS, j = idx % kS;
      // diagonal tile: the upper half mirrored, so the tile stays exactly symmetric
      const double x = (p == q && i > j) ? T[j * kLdT + i] : T[i * kLdT + j];
      A[size_t(sub_index(i, Ip, Jp)) * n + sub_index(j, Iq, Jq)] = x;
      if (p != q) A[size_t(sub_index(j, Iq, Jq)) * n + sub_index(i, Ip, Jp)] = x;
    }
    return;
  }
  t -= ntri;
  const int q = t % npairs, chunk = t / npairs;
  if (!fl[q]) return;
  int Iq, Jq;
  rr_pair(r, q, nb, Iq, Jq);
  double* V = Vall + size_t(w) * sA;
  const int i0 = chunk * kS;
  for (int c = tid; c < kS * kS / 2; c += kThreads) {
    const int i = c / (kS / 2), j = 2 * (c % (kS / 2));
    cp_async16(T + i * kLdT + j, V + size_t(i0 + i) * n + sub_index(j, Iq, Jq), 16);
    cp_async16(Qb + i * kLdT + j, qw + size_t(q) * kS * kS + i * kS + j, 16);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  tile_product(T, Qb, false);
  for (int idx = tid; idx < kS * kS; idx += kThreads) {
    const int i = idx / kS, j = idx % kS;
    V[size_t(i0 + i) * n + sub_index(j, Iq, Jq)] = T[i * kLdT + j];
  }
}

}  // namespace

Status eigh_jacobi_batched(Context& c, double* A, double* V, int n, int nw, cudaStream_t s, int* sweeps,
                           int* launches) {
  if (n <= 0 || n % kS != 0 || nw <= 0)
    return Status::fail(RIGW_ERR_ARG, "eigh_jacobi_batched: n must be a positive multiple of %d", kS);
  // per device (cheap): the current device is the context's
  RIGW_CUDA_TRY(cudaFuncSetAttribute(eigh_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kPairSmem)));
  RIGW_CUDA_TRY(cudaFuncSetAttribute(eigh_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kApplySmem)));
  const int nb = n / kB, npairs = nb / 2, chunks = n / kS, ntri = npairs * (npairs + 1) / 2;
  const long long sA = (long long)n * n;
  DeviceBuffer b_q, b_aux;
  RIGW_TRY(b_q.allocate(&c, size_t(nw) * npairs * kS * kS * 8, "eigensolver block rotations"));
  const size_t aux_bytes = size_t(nw) * 8 + size_t(nw) * npairs * 4 + size_t(nw) * 4;
  RIGW_TRY(b_aux.allocate(&c, aux_bytes, "eigensolver flags"));
  double* qbuf = reinterpret_cast<double*>(b_q.data());
  double* tau = reinterpret_cast<double*>(b_aux.data());
  int* flags = reinterpret_cast<int*>(tau + nw);
  int* rot = flags + size_t(nw) * npairs;
  eigh_init_kernel<<<nw, 1024, 0, s>>>(A, V, n, sA, tau);
  RIGW_CUDA_TRY(cudaGetLastError());
  int nl = 1;
  std::vector<int> host_rot(nw);
  bool converged = false;
  int sweep = 0;
  for (; sweep < kOuterMaxSweeps && !converged; ++sweep) {
    RIGW_CUDA_TRY(cudaMemsetAsync(rot, 0, size_t(nw) * sizeof(int), s));
    for (int r = 0; r < nb - 1; ++r) {
      eigh_pair_kernel<<<dim3(npairs, nw), kThreads, kPairSmem, s>>>(A, qbuf, flags, rot, tau, n, sA, r);
      eigh_apply_kernel<<<dim3(ntri + npairs * chunks, nw), kThreads, kApplySmem, s>>>(A, V, qbuf, flags, n, sA, r);
      nl += 2;
    }
    RIGW_CUDA_TRY(cudaGetLastError());
    RIGW_CUDA_TRY(cudaMemcpyAsync(host_rot.data(), rot, size_t(nw) * sizeof(int), cudaMemcpyDeviceToHost, s));
    RIGW_CUDA_TRY(cudaStreamSynchronize(s));
    converged = true;
    for (int w = 0; w < nw; ++w) converged = converged && host_rot[w] == 0;
  }
  if (!converged)
    return Status::fail(RIGW_ERR_NUMERIC, "eigh_jacobi_batched: no convergence in %d sweeps", kOuterMaxSweeps);
  if (sweeps) *sweeps = sweep;
  if (launches) *launches += nl;
  return Status::ok();
}

}  // namespace rigw
