// FP64 tensor-core (DMMA) tile engine for MN-major operands.
//
//   C[m][n] = alpha * sum_k s_k * A[k][m] * B[k][n]  + beta * Cin[m][n]  (+ I on a diagonal)
//
// Both operands are stored with the output index contiguous (row k holds the
// m (resp. n) elements), which is the natural layout of every product on the
// RI-GW path: the transition-major M tensor for chi0 = M D M^T, and the upper
// Cholesky factor rows U[k][*] for the panel solves and trailing updates.
// One CTA computes one work item (a BM x BN tile of one product); the work
// list lets one launch cover every frequency and every molecule of a batch.
#pragma once
#include "common.cuh"

namespace rigw {

enum GemmFlags : int {
  kAddIdentity = 1,   // C += 1 where (col - row) == diag
  kSubIdentity = 2,   // C -= 1 where (col - row) == diag
  kUpperA = 4,        // A[k][m] = 0 for k > m, with m counted from the item's first row (the
                      // triangular inverse of the panel solves): the warps of rows
                      // m < wm0 + 64 skip the MMAs of k >= wm0 + 64, which add exact zeros
};

struct GemmItem {
  const double* A;      // &A[0][m0], row stride lda
  const double* B;      // &B[0][n0], row stride ldb
  const double* Cin;    // &Cin[m0][n0] or nullptr
  double* C;            // &C[m0][n0], row stride ldc
  const double* kscale; // per-k factor applied to A (nullptr: none)
  double* colsq;        // per-column sum of squares of the stored tile (nullptr: none)
  int lda, ldb, ldc;
  int m, n, k;          // valid extents (m <= BM, n <= BN, all even)
  int diag;
  int flags;
  double alpha, beta;
  // The item covers nw frequencies (nw <= 0: one): CTA (item, j) (blockIdx.y =
  // j < nw) works on the operands advanced by j times these element strides.
  long long sA, sB, sC, sK, sQ;   // A, B, C and Cin, kscale, colsq
  int nw;
};

template <int BM, int BN, int ST = 3>
struct DgemmCfg {
  static constexpr int kWarpsM = BM / 64;
  static constexpr int kWarpsN = BN / 32;
  static constexpr int kThreads = kWarpsM * kWarpsN * 32;
  static constexpr int kBK = 16;
  static constexpr int kStages = ST;
  static constexpr int kLdaS = BM + 2;   // == 2 (mod 16): conflict-free 128-bit A fragment loads
  static constexpr int kLdbS = BN + 4;   // == 4 (mod 16): conflict-free 64-bit B fragment loads
  static constexpr int kStageDoubles = kBK * kLdaS + kBK * kLdbS + kBK;
  static constexpr size_t kSmemBytes = size_t(kStages) * kStageDoubles * sizeof(double);
};

template <int BM, int BN, int STAGES = 3>
__global__ void __launch_bounds__(DgemmCfg<BM, BN, STAGES>::kThreads, 1)
dgemm_mn_kernel(const GemmItem* __restrict__ items) {
  using Cfg = DgemmCfg<BM, BN, STAGES>;
  constexpr int BK = Cfg::kBK;
  constexpr int ST = Cfg::kStages;
  constexpr int NT = Cfg::kThreads;
  extern __shared__ __align__(16) double smem[];

  GemmItem it = items[blockIdx.x];
  const int jw = blockIdx.y;
  if (jw >= (it.nw > 0 ? it.nw : 1)) return;   // nw <= 0: one frequency
  if (jw > 0) {
    it.A += jw * it.sA;
    it.B += jw * it.sB;
    it.C += jw * it.sC;
    if (it.Cin) it.Cin += jw * it.sC;
    if (it.kscale) it.kscale += jw * it.sK;
    if (it.colsq) it.colsq += jw * it.sQ;
  }
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int wm = warp % Cfg::kWarpsM;
  const int wn = warp / Cfg::kWarpsM;
  const int wm0 = wm * 64;
  const int wn0 = wn * 32;
  const int ktiles = (it.k + BK - 1) / BK;
  const bool has_scale = it.kscale != nullptr;
  const int klim = (it.flags & kUpperA) ? min(it.k, wm0 + 64) : it.k;   // warp-uniform

  auto stage_a = [&](int s) { return smem + s * Cfg::kStageDoubles; };
  auto stage_b = [&](int s) { return smem + s * Cfg::kStageDoubles + BK * Cfg::kLdaS; };
  auto stage_k = [&](int s) { return smem + s * Cfg::kStageDoubles + BK * Cfg::kLdaS + BK * Cfg::kLdbS; };

  auto load_stage = [&](int s, int kt) {
    const int k0 = kt * BK;
    double* as = stage_a(s);
    double* bs = stage_b(s);
    constexpr int kChunksA = BK * BM / 2;
#pragma unroll
    for (int c = tid; c < kChunksA; c += NT) {
      const int kk = c / (BM / 2);
      const int mm = (c % (BM / 2)) * 2;
      const bool ok = (k0 + kk < it.k) && (mm < it.m);
      const double* src = ok ? it.A + size_t(k0 + kk) * it.lda + mm : it.A;
      cp_async16(as + kk * Cfg::kLdaS + mm, src, ok ? 16 : 0);
    }
    constexpr int kChunksB = BK * BN / 2;
#pragma unroll
    for (int c = tid; c < kChunksB; c += NT) {
      const int kk = c / (BN / 2);
      const int nn = (c % (BN / 2)) * 2;
      const bool ok = (k0 + kk < it.k) && (nn < it.n);
      const double* src = ok ? it.B + size_t(k0 + kk) * it.ldb + nn : it.B;
      cp_async16(bs + kk * Cfg::kLdbS + nn, src, ok ? 16 : 0);
    }
    if (has_scale && tid < BK) {
      const bool ok = k0 + tid < it.k;
      cp_async8(stage_k(s) + tid, ok ? it.kscale + k0 + tid : it.kscale, ok ? 8 : 0);
    }
  };

  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
  for (int s = 0; s < ST - 1; ++s) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }
  // Pull the tile read by the epilogue into L2 while the mainloop runs.
  if (it.Cin != nullptr) {
    constexpr int kLines = BN / 16;   // 128-byte lines per tile row
    for (int rr = tid; rr < it.m * kLines; rr += NT) {
      const int col = (rr % kLines) * 16;
      const double* line = it.Cin + size_t(rr / kLines) * it.ldc + col;
      if (col < it.n) asm volatile("prefetch.global.L2 [%0];" ::"l"(line));
    }
  }

  const int q = lane >> 2;   // fragment row (A) / column (B) within the 8-wide tile
  const int r = lane & 3;    // fragment k index
  // 8-column fragments of this warp inside the item (warp-uniform); edge tiles
  // skip the MMAs of columns beyond n, whose values are never stored
  const int nfrag = min(4, max(0, (it.n - wn0 + 7) >> 3));
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<ST - 2>();
    __syncthreads();
    {
      const int nk = kt + ST - 1;
      if (nk < ktiles) load_stage(nk % ST, nk);
      cp_async_commit();
    }
    const int s = kt % ST;
    if (kt * BK >= klim) continue;   // this warp's rows see only zeros of A from here on
    const double* as = stage_a(s) + wm0 + 8 * q;
    const double* bs = stage_b(s) + wn0 + q;
    const double* ks = stage_k(s);
#pragma unroll
    for (int k4 = 0; k4 < BK / 4; ++k4) {
      const int kk = k4 * 4 + r;
      double a[8], b[4];
      const double2* ap = reinterpret_cast<const double2*>(as + kk * Cfg::kLdaS);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double2 v = ap[i];
        a[2 * i] = v.x;
        a[2 * i + 1] = v.y;
      }
      if (has_scale) {
        const double sc = ks[kk];
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] *= sc;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = bs[kk * Cfg::kLdbS + 8 * j];
      if (nfrag == 4) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < nfrag)
#pragma unroll
            for (int i = 0; i < 8; ++i) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
    }
  }
  cp_async_wait<0>();

  // Epilogue.  Lane (q, r) of warp (wm, wn) owns rows wm0 + 8q + i (i < 8) and
  // columns wn0 + 8j + 2r + e (j < 4, e < 2).
  const bool ident = (it.flags & (kAddIdentity | kSubIdentity)) != 0;
  const double idv = (it.flags & kSubIdentity) ? -1.0 : 1.0;
  double csq[4][2];
#pragma unroll
  for (int j = 0; j < 4; ++j) csq[j][0] = csq[j][1] = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int row = wm0 + 8 * q + i;
    if (row >= it.m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int col = wn0 + 8 * j + 2 * r;
      if (col >= it.n) continue;
      double v0 = it.alpha * acc[i][j][0];
      double v1 = it.alpha * acc[i][j][1];
      if (it.Cin != nullptr) {
        const double2 c = *reinterpret_cast<const double2*>(it.Cin + size_t(row) * it.ldc + col);
        v0 += it.beta * c.x;
        v1 += it.beta * c.y;
      }
      if (ident) {
        if (col - row == it.diag) v0 += idv;
        if (col + 1 - row == it.diag) v1 += idv;
      }
      *reinterpret_cast<double2*>(it.C + size_t(row) * it.ldc + col) = make_double2(v0, v1);
      csq[j][0] += v0 * v0;
      csq[j][1] += v1 * v1;
    }
  }
  if (it.colsq != nullptr) {
    // reduce over q (lanes with equal r), then over the warps of one column strip
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        double v = csq[j][e];
        v += __shfl_xor_sync(0xffffffffu, v, 4);
        v += __shfl_xor_sync(0xffffffffu, v, 8);
        v += __shfl_xor_sync(0xffffffffu, v, 16);
        csq[j][e] = v;
      }
    __syncthreads();                       // smem is free after the mainloop
    double* red = smem;                    // [kWarpsM][BN]
    if (q == 0) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) red[wm * BN + wn0 + 8 * j + 2 * r + e] = csq[j][e];
    }
    __syncthreads();
    for (int c = tid; c < BN && c < it.n; c += NT) {
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < Cfg::kWarpsM; ++w) v += red[w * BN + c];
      it.colsq[c] = v;
    }
  }
}

}  // namespace rigw
