// Ozaki-sliced INT8 chi0 contraction on the 5th-generation tensor cores.
//
//   eps(iw) = 1 + S S^T,  S = M diag(sqrt(D_w))
//   row p of S is scaled by 2^-e_p, e_p the exponent of max_t |S_pt| (so |x| < 1):
//     x_pt = S_pt 2^-e_p = sum_{k=1..s} q_k(p,t) 2^-7k + r,  q_k integers in [-127, 127],
//   the base-128 digits of trunc(x 2^7s) (an exact 64-bit integer), with the sign of x.
//   (S S^T)_pq ~= 2^(e_p+e_q) sum_{d=2..s+1} 2^-7d L_d(p,q),   L_d = sum_{i+j=d} Q_i Q_j^T
//   (the products of level i+j > s+1 are dropped, as in the Ozaki scheme).
//
// L_d is an exact INT32 sum (tcgen05.mma kind::i8).  K is consumed in chunks of
// kOzChunk k-tiles (4096 transitions): |L_d| <= s * 4096 * 127^2 < 2^31 on one
// chunk, so no sum can overflow; every (chunk, level) accumulator is drained
// into FP64 registers with its weight 2^-7d while the MMA warp fills another of
// the four TMEM accumulators.
//
// ozaki_zero_kernel:   clears the per-row maxima of a problem.
// ozaki_rowmax_kernel: max_t |S_pt| for every frequency and row (atomicMax on the
//                      bit pattern of a non-negative double: order independent).
// ozaki_slice_kernel:  row exponents and the s int8 slices of one frequency group,
//                      K-major (transition-contiguous) for TMA.
// slice_rowmax_kernel, slice_kmajor_kernel: the same slicing for the general
//                      operands of the AO->MO products (row exponents from the
//                      row maxima over K).
// syrk_ozaki_kernel:   one 128x128 upper tile of eps(iw), or one tile of a general
//                      product A B^T, per CTA; warp 0 issues
//                      TMA loads (one A and one B slice tile of 128 rows x 128
//                      transitions per stage, 128-byte swizzle, 6 stages), warp 1
//                      issues the MMAs, warps 2..9 drain.  All waits are bounded.
#include "engine.cuh"
#include "tc_common.cuh"

namespace rigw {

// ---------------------------------------------------------------------------
// item: (prob, first entry); 256 threads clear 4096 entries.
__global__ void __launch_bounds__(256) ozaki_zero_kernel(const ProbDev* __restrict__ probs,
                                                         const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const size_t n = size_t(p.nomega) * p.npad;
  for (int k = threadIdx.x; k < 4096; k += 256) {
    const size_t e = size_t(wi.a) + k;
    if (e < n) p.rmax[e] = 0ull;
  }
}

// item: (prob, t0, p0): split_t transitions from t0 x 64 rows from p0, every
// frequency, in 64-transition sub-tiles.
__global__ void __launch_bounds__(256) ozaki_rowmax_kernel(const ProbDev* __restrict__ probs,
                                                           const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int p0 = wi.b;
  __shared__ double tile[64][65];   // [row p][transition t]
  __shared__ double sc[64];
  __shared__ double part[4][64];
  const int tid = threadIdx.x;
  const int pp = tid & 63, tq = tid >> 6;
  const int tend = min(p.nia_pad, wi.a + p.split_t);
  for (int t0 = wi.a; t0 < tend; t0 += 64) {
    __syncthreads();
    for (int idx = tid; idx < 64 * 64; idx += 256) {
      const int tt = idx >> 6, pq = idx & 63;
      tile[pq][tt] = p.mp[size_t(t0 + tt) * p.npad + p0 + pq];
    }
    for (int w = 0; w < p.nomega; ++w) {
      __syncthreads();
      if (tid < 64) sc[tid] = sqrt(p.dscale[size_t(w) * p.nia_pad + t0 + tid]);
      __syncthreads();
      double m = 0.0;
#pragma unroll
      for (int t = tq * 16; t < tq * 16 + 16; ++t) m = fmax(m, fabs(tile[pp][t] * sc[t]));
      part[tq][pp] = m;
      __syncthreads();
      if (tid < 64) {
        m = fmax(fmax(part[0][tid], part[1][tid]), fmax(part[2][tid], part[3][tid]));
        if (m > 0.0) atomicMax(p.rmax + size_t(w) * p.npad + p0 + tid, (unsigned long long)__double_as_longlong(m));
      }
    }
  }
}

// Base-128 digits of x (|x| < 1) truncated after s digits: X = trunc(x 2^(7s)) is
// exact in 64-bit integers (7s <= 49 bits), and digit k (k = 1..s) of |X|, with
// the sign of x, equals the k-th integer part taken by repeated x <- 128x - trunc(128x).
RIGW_DEVICE_INLINE long long ozaki_fixed(double x, int s) { return (long long)ldexp(x, 7 * s); }
RIGW_DEVICE_INLINE int ozaki_digit(long long X, int s, int k) {
  const long long a = X < 0 ? -X : X;
  const int d = int((a >> (7 * (s - k))) & 127);
  return X < 0 ? -d : d;
}

// item: (prob, t0, p0, w0): the same tiles for the frequencies w0 .. w0+wgroup-1.
__global__ void __launch_bounds__(256) ozaki_slice_kernel(const ProbDev* __restrict__ probs,
                                                          const WorkItem* __restrict__ items) {
  const WorkItem wi = items[blockIdx.x];
  const ProbDev& p = probs[wi.prob];
  const int p0 = wi.b;
  __shared__ double tile[64][65];   // [row p][transition t]
  __shared__ double sc[64];         // sqrt(D_w(t0 + t))
  __shared__ double rs[64];         // 2^-e_p
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int8_t* xq = reinterpret_cast<int8_t*>(p.xs);
  const int ns = p.slices;
  const int w0 = wi.c, w1 = min(p.nomega, w0 + p.wgroup);
  const int tend = min(p.nia_pad, wi.a + p.split_t);
  for (int t0 = wi.a; t0 < tend; t0 += 64) {
    __syncthreads();
    for (int idx = tid; idx < 64 * 64; idx += 256) {
      const int tt = idx >> 6, pp = idx & 63;
      tile[pp][tt] = p.mp[size_t(t0 + tt) * p.npad + p0 + pp];
    }
    for (int w = w0; w < w1; ++w) {
      const int wl = w - w0;
      __syncthreads();
      if (tid < 64) {
        sc[tid] = sqrt(p.dscale[size_t(w) * p.nia_pad + t0 + tid]);
      } else if (tid < 128) {
        const int pp = tid - 64;
        const double m = __longlong_as_double((long long)p.rmax[size_t(w) * p.npad + p0 + pp]);
        int e = 0;
        if (m > 0.0) frexp(m, &e);    // m = f 2^e, f in [0.5, 1): every |S_pt| of the row is < 2^e
        rs[pp] = ldexp(1.0, -e);
        if (t0 == 0) p.xexp[size_t(w) * p.npad + p0 + pp] = e;
      }
      __syncthreads();
      const double s0 = sc[2 * lane], s1 = sc[2 * lane + 1];
#pragma unroll 1
      for (int pr = 0; pr < 8; ++pr) {
        const int pp = warp * 8 + pr;
        const long long X0 = ozaki_fixed(tile[pp][2 * lane] * s0 * rs[pp], ns);
        const long long X1 = ozaki_fixed(tile[pp][2 * lane + 1] * s1 * rs[pp], ns);
        for (int k = 1; k <= ns; ++k) {
          const size_t row = (size_t(wl * ns + k - 1) * p.npad + p0 + pp) * p.kpad + t0;
          reinterpret_cast<char2*>(xq + row)[lane] =
              make_char2(char(ozaki_digit(X0, ns, k)), char(ozaki_digit(X1, ns, k)));
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// General operands (the AO->MO products): 64 x 64 tiles through shared memory,
// read along the source's contiguous index.  Pass 1 takes the row maxima, pass 2
// the row exponents and the digits, written K-contiguous.
__global__ void __launch_bounds__(256) slice_rowmax_kernel(const SliceOp op) {
  __shared__ double tile[64][65];   // [row][k]
  __shared__ double part[4][64];
  const int k0 = blockIdx.x * 64, r0 = blockIdx.y * 64, z = blockIdx.z;
  const double* src = op.src + size_t(z) * op.zs_src;
  const bool rfast = op.rs == 1;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < 64 * 64; idx += 256) {
    const int a = idx >> 6, b = idx & 63;
    const int rr = rfast ? b : a, kk = rfast ? a : b;
    const int r = r0 + rr, k = k0 + kk;
    tile[rr][kk] = (r < op.R && k < op.K) ? fabs(src[r * op.rs + k * op.ks]) : 0.0;
  }
  __syncthreads();
  const int rr = tid & 63, kq = tid >> 6;
  double m = 0.0;
#pragma unroll
  for (int kk = kq * 16; kk < kq * 16 + 16; ++kk) m = fmax(m, tile[rr][kk]);
  part[kq][rr] = m;
  __syncthreads();
  if (tid < 64) {
    m = fmax(fmax(part[0][tid], part[1][tid]), fmax(part[2][tid], part[3][tid]));
    if (m > 0.0) atomicMax(op.rmax + size_t(z) * op.Rpad + r0 + tid, (unsigned long long)__double_as_longlong(m));
  }
}

__global__ void __launch_bounds__(256) slice_kmajor_kernel(const SliceOp op) {
  __shared__ double tile[64][65];   // [row][k]
  __shared__ double rs[64];         // 2^-e_r
  const int k0 = blockIdx.x * 64, r0 = blockIdx.y * 64, z = blockIdx.z;
  const double* src = op.src + size_t(z) * op.zs_src;
  const bool rfast = op.rs == 1;
  const int tid = threadIdx.x, ns = op.slices;
  for (int idx = tid; idx < 64 * 64; idx += 256) {
    const int a = idx >> 6, b = idx & 63;
    const int rr = rfast ? b : a, kk = rfast ? a : b;
    const int r = r0 + rr, k = k0 + kk;
    tile[rr][kk] = (r < op.R && k < op.K) ? src[r * op.rs + k * op.ks] : 0.0;
  }
  if (tid < 64) {
    const size_t e_at = size_t(z) * op.Rpad + r0 + tid;
    const double m = __longlong_as_double((long long)op.rmax[e_at]);
    int e = 0;
    if (m > 0.0) frexp(m, &e);      // every |x| of the row is < 2^e
    rs[tid] = ldexp(1.0, -e);
    if (blockIdx.x == 0) op.exps[e_at] = e;
  }
  __syncthreads();
  int8_t* dst = reinterpret_cast<int8_t*>(op.dst);
  for (int idx = tid; idx < 64 * 32; idx += 256) {
    const int rr = idx >> 5, kp = (idx & 31) * 2;
    const long long X0 = ozaki_fixed(tile[rr][kp] * rs[rr], ns);
    const long long X1 = ozaki_fixed(tile[rr][kp + 1] * rs[rr], ns);
    for (int k = 1; k <= ns; ++k) {
      const size_t row = (size_t(z) * ns + k - 1) * op.Rpad + r0 + rr;
      *reinterpret_cast<char2*>(dst + row * op.Kpad + k0 + kp) =
          make_char2(char(ozaki_digit(X0, ns, k)), char(ozaki_digit(X1, ns, k)));
    }
  }
}

// ---------------------------------------------------------------------------
constexpr int kOzStages = 6;
constexpr int kOzTileBytes = 128 * 128;                 // 128 rows x 128 int8 transitions
constexpr int kOzStageBytes = 2 * kOzTileBytes;
constexpr size_t kOzSmemBytes = size_t(kOzStages) * kOzStageBytes + 1024 + 256;
constexpr int kOzChunk = 32;                            // k-tiles per exact INT32 accumulation
constexpr int kOzAcc = 4;                               // TMEM accumulators of 128 columns
constexpr int kOzThreads = 320;                         // warp 0 TMA, warp 1 MMA, warps 2..9 drain

__global__ void __launch_bounds__(kOzThreads, 1) syrk_ozaki_kernel(const TcItem* __restrict__ items) {
  TcItem it = items[blockIdx.x];
  const int jw = blockIdx.y;
  if (jw >= (it.nw > 0 ? it.nw : 1)) return;   // the whole CTA, before any barrier or TMEM use
  it.C += jw * it.sC;
  it.row_a += jw * it.srow;
  it.row_b += jw * it.srow;
  if (it.ea) {
    it.ea += jw * it.se;
    it.eb += jw * it.se;
  }
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kOzStages * kOzStageBytes);
  uint64_t* empty = full + kOzStages;
  uint64_t* accf = empty + kOzStages;     // [kOzAcc] unit accumulated
  uint64_t* acce = accf + kOzAcc;         // [kOzAcc] unit drained
  uint32_t* tslot = reinterpret_cast<uint32_t*>(acce + kOzAcc);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto tile = [&](int s, int which) { return smem + s * kOzStageBytes + which * kOzTileBytes; };

  if (tid == 0) {
    for (int s = 0; s < kOzStages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < kOzAcc; ++b) {
      tc::mbar_init(&accf[b], 1);
      tc::mbar_init(&acce[b], 8);
    }
    tc::fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(tslot, 128 * kOzAcc);
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  const int nk = it.ktiles;
  const int ns = it.slices;
  const int nchunks = (nk + kOzChunk - 1) / kOzChunk;
  // Work order (identical in the producer and the MMA issuer): chunk c, level
  // d = 2..ns+1, slice pair (i, d-i), k-tile of the chunk.  One unit = (c, d).

  if (tid == 0) {
    // ---- TMA producer
    const void* tmb = it.tmap_b ? it.tmap_b : it.tmap;
    const int lob = it.tmap_b ? it.lo_off_b : it.lo_off;
    tc::tmap_acquire(it.tmap);
    if (it.tmap_b) tc::tmap_acquire(it.tmap_b);
    int issued[kOzStages] = {0, 0, 0, 0, 0, 0};
    bool ok = true;
    int step = 0;
    for (int c = 0; c < nchunks && ok; ++c) {
      const int k0 = c * kOzChunk, k1 = min(nk, k0 + kOzChunk);
      for (int d = 2; d <= ns + 1 && ok; ++d)
        for (int i = max(1, d - ns); i <= min(ns, d - 1) && ok; ++i)
          for (int kt = k0; kt < k1; ++kt, ++step) {
            const int s = step % kOzStages;
            if (step >= kOzStages && !tc::mbar_wait(&empty[s], ((step / kOzStages) - 1) & 1)) {
              ok = false;
              break;
            }
            tc::mbar_arrive_expect_tx(&full[s], kOzStageBytes);
            tc::tma_load_2d(tile(s, 0), it.tmap, &full[s], kt * 128, it.row_a + (i - 1) * it.lo_off);
            tc::tma_load_2d(tile(s, 1), tmb, &full[s], kt * 128, it.row_b + (d - i - 1) * lob);
            ++issued[s];
          }
    }
    if (!ok) atomicOr(it.err, kErrTimeout);
    for (int s = 0; s < kOzStages; ++s)
      if (issued[s] > 0 && !tc::mbar_wait(&full[s], (issued[s] - 1) & 1)) atomicOr(it.err, kErrTimeout);
  } else if (tid == 32) {
    // ---- MMA issuer
    constexpr uint32_t idesc = tc::idesc_s8_s32(128, 128);
    bool ok = true;
    int step = 0, u = 0;
    for (int c = 0; c < nchunks && ok; ++c) {
      const int k0 = c * kOzChunk, k1 = min(nk, k0 + kOzChunk);
      for (int d = 2; d <= ns + 1 && ok; ++d, ++u) {
        const int b = u % kOzAcc;
        if (u >= kOzAcc && !tc::mbar_wait(&acce[b], ((u / kOzAcc) - 1) & 1)) {
          ok = false;
          break;
        }
        tc::tc_fence_after();
        const uint32_t dt = tmem + uint32_t(b * 128);
        bool first = true;
        for (int i = max(1, d - ns); i <= min(ns, d - 1) && ok; ++i)
          for (int kt = k0; kt < k1; ++kt, ++step) {
            const int s = step % kOzStages;
            if (!tc::mbar_wait(&full[s], (step / kOzStages) & 1)) {
              ok = false;
              break;
            }
            tc::tc_fence_after();
            const uint64_t ad = tc::desc_kmajor_sw128(tile(s, 0)), bd = tc::desc_kmajor_sw128(tile(s, 1));
#pragma unroll
            for (int sub = 0; sub < 4; ++sub) {
              const uint64_t o = uint64_t(sub * 2);   // 32 int8 = 32 bytes along K
              tc::mma_s8(dt, ad + o, bd + o, idesc, (first && sub == 0) ? 0u : 1u);
            }
            first = false;
            tc::mma_commit(&empty[s]);
          }
        if (ok) tc::mma_commit(&accf[b]);
      }
    }
    if (!ok) atomicOr(it.err, kErrTimeout);
  } else if (warp >= 2) {
    // ---- drain: every (chunk, level) accumulator into FP64 with weight 2^-7d
    const int quad = warp & 3;                 // TMEM lanes 32*quad .. 32*quad+31 (rows)
    const int half = (warp - 2) >> 2;          // columns 64*half .. 64*half+63
    const int row = quad * 32 + lane;
    double acc[64];
#pragma unroll
    for (int j = 0; j < 64; ++j) acc[j] = 0.0;
    bool ok = true;
    int u = 0;
    for (int c = 0; c < nchunks && ok; ++c)
      for (int d = 2; d <= ns + 1; ++d, ++u) {
        const int b = u % kOzAcc;
        ok = __all_sync(0xffffffffu, tc::mbar_wait(&accf[b], (u / kOzAcc) & 1));
        if (!ok) break;
        tc::tc_fence_after();
        const double wd = ldexp(1.0, -7 * d);
        const uint32_t base = tmem + uint32_t(b * 128 + half * 64) + (uint32_t(quad * 32) << 16);
        uint32_t r[32];
        tc::tmem_ld_32x32(base, r);
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] += double(int(r[j])) * wd;
        tc::tmem_ld_32x32(base + 32, r);
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[32 + j] += double(int(r[j])) * wd;
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&acce[b]);
      }
    if (ok && it.mrows == 0) {
      const int er = it.ea[row];
      double* dst = it.C + size_t(row) * it.ldc + half * 64;
#pragma unroll
      for (int j = 0; j < 64; j += 2) {
        const int col = half * 64 + j;
        double v0 = ldexp(acc[j], er + it.eb[col]), v1 = ldexp(acc[j + 1], er + it.eb[col + 1]);
        if (col - row == it.diag) v0 += 1.0;
        if (col + 1 - row == it.diag) v1 += 1.0;
        *reinterpret_cast<double2*>(dst + j) = make_double2(v0, v1);
      }
    } else if (ok) {
      // edge tile of a general product: rows < mrows, columns < ncols, no identity
      if (row < it.mrows) {
        const int er = it.ea[row];
        double* dst = it.C + size_t(row) * it.ldc;
#pragma unroll
        for (int j = 0; j < 64; ++j) {
          const int col = half * 64 + j;
          if (col < it.ncols) dst[col] = ldexp(acc[j], er + it.eb[col]);
        }
      }
    } else if (lane == 0) {
      atomicOr(it.err, kErrTimeout);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 128 * kOzAcc);
}

// ---------------------------------------------------------------------------
// Ozaki chi0 for s <= 4 slices: every slice pair of a k-tile from one stage.
//
// A stage holds the s A-slice and s B-slice tiles of one k-tile of 64 transitions
// (128 rows x 64 int8 each, 64-byte swizzle, 8 KB), so each tile loaded feeds all
// the pair products it appears in: for s = 4, 20 MMAs (M=128 N=128 K=32) per 64 KB
// staged, against 4 MMAs per 32 KB when one pair is staged at a time.  Level d =
// i+j accumulates in its own TMEM accumulator (d-2: columns 128(d-2)..), exact in
// INT32 over chunks of kOzfChunk k-tiles (4096 transitions: |L_d| <= 4 * 4096 *
// 127^2 < 2^31); after a chunk the eight drain warps add the s levels into FP64
// with weight 2^-7d, and the MMA warp waits for that before the next chunk (the s
// accumulators fill TMEM, so there is no second set).
constexpr int kOzfMaxSlices = 4;
constexpr int kOzfTileBytes = 128 * 64;                            // 128 rows x 64 int8
constexpr int kOzfStageBytes = 2 * kOzfMaxSlices * kOzfTileBytes;  // 64 KB
constexpr int kOzfStages = 3;
constexpr size_t kOzfSmemBytes = size_t(kOzfStages) * kOzfStageBytes + 1024 + 256;
constexpr int kOzfChunk = 64;                                      // k-tiles per exact INT32 accumulation

__global__ void __launch_bounds__(kOzThreads, 1) syrk_ozaki_fused_kernel(const TcItem* __restrict__ items) {
  TcItem it = items[blockIdx.x];
  const int jw = blockIdx.y;
  if (jw >= (it.nw > 0 ? it.nw : 1)) return;   // the whole CTA, before any barrier or TMEM use
  it.C += jw * it.sC;
  it.row_a += jw * it.srow;
  it.row_b += jw * it.srow;
  if (it.ea) {
    it.ea += jw * it.se;
    it.eb += jw * it.se;
  }
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kOzfStages * kOzfStageBytes);
  uint64_t* empty = full + kOzfStages;
  uint64_t* accf = empty + kOzfStages;    // chunk accumulated (all levels)
  uint64_t* acce = accf + 1;              // chunk drained
  uint32_t* tslot = reinterpret_cast<uint32_t*>(acce + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ns = it.slices;               // 3 or 4
  // tile (s, 0, i) = A slice i + 1, tile (s, 1, j) = B slice j + 1
  auto tile = [&](int st, int which, int sl) {
    return smem + st * kOzfStageBytes + (which * kOzfMaxSlices + sl) * kOzfTileBytes;
  };

  if (tid == 0) {
    for (int st = 0; st < kOzfStages; ++st) {
      tc::mbar_init(&full[st], 1);
      tc::mbar_init(&empty[st], 1);
    }
    tc::mbar_init(accf, 1);
    tc::mbar_init(acce, 8);
    tc::fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(tslot, 128 * kOzAcc);
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  const int nk = it.ktiles;
  const int nchunks = (nk + kOzfChunk - 1) / kOzfChunk;

  if (tid == 0) {
    // ---- TMA producer: the 2 ns slice tiles of each k-tile
    tc::tmap_acquire(it.tmap);
    int issued[kOzfStages] = {0, 0, 0};
    bool ok = true;
    const uint32_t bytes = uint32_t(2 * ns * kOzfTileBytes);
    for (int kt = 0; kt < nk && ok; ++kt) {
      const int st = kt % kOzfStages;
      if (kt >= kOzfStages && !tc::mbar_wait(&empty[st], ((kt / kOzfStages) - 1) & 1)) {
        ok = false;
        break;
      }
      tc::mbar_arrive_expect_tx(&full[st], bytes);
      for (int sl = 0; sl < ns; ++sl) {
        tc::tma_load_2d(tile(st, 0, sl), it.tmap, &full[st], kt * 64, it.row_a + sl * it.lo_off);
        tc::tma_load_2d(tile(st, 1, sl), it.tmap, &full[st], kt * 64, it.row_b + sl * it.lo_off);
      }
      ++issued[st];
    }
    if (!ok) atomicOr(it.err, kErrTimeout);
    for (int st = 0; st < kOzfStages; ++st)
      if (issued[st] > 0 && !tc::mbar_wait(&full[st], (issued[st] - 1) & 1)) atomicOr(it.err, kErrTimeout);
  } else if (tid == 32) {
    // ---- MMA issuer: per k-tile every pair (i, j) with i + j <= ns + 1 into level i + j
    constexpr uint32_t idesc = tc::idesc_s8_s32(128, 128);
    bool ok = true;
    for (int kt = 0; kt < nk && ok; ++kt) {
      const int c = kt / kOzfChunk;
      const bool chunk_first = (kt % kOzfChunk) == 0;
      if (chunk_first && c >= 1 && !tc::mbar_wait(acce, (c - 1) & 1)) {
        ok = false;
        break;
      }
      const int st = kt % kOzfStages;
      if (!tc::mbar_wait(&full[st], (kt / kOzfStages) & 1)) {
        ok = false;
        break;
      }
      tc::tc_fence_after();
      for (int d = 2; d <= ns + 1; ++d) {
        const uint32_t dt = tmem + uint32_t((d - 2) * 128);
        bool first = chunk_first;
        for (int i = max(1, d - ns); i <= min(ns, d - 1); ++i) {
          const uint64_t ad = tc::desc_kmajor_sw64(tile(st, 0, i - 1));
          const uint64_t bd = tc::desc_kmajor_sw64(tile(st, 1, d - i - 1));
#pragma unroll
          for (int sub = 0; sub < 2; ++sub) {
            const uint64_t o = uint64_t(sub * 2);   // 32 int8 = 32 bytes along K
            tc::mma_s8(dt, ad + o, bd + o, idesc, (first && sub == 0) ? 0u : 1u);
          }
          first = false;
        }
      }
      tc::mma_commit(&empty[st]);
      if ((kt % kOzfChunk) == kOzfChunk - 1 || kt == nk - 1) tc::mma_commit(accf);
    }
    if (!ok) atomicOr(it.err, kErrTimeout);
  } else if (warp >= 2) {
    // ---- drain: after each chunk, every level into FP64 with weight 2^-7d
    const int quad = warp & 3;                 // TMEM lanes 32*quad .. 32*quad+31 (rows)
    const int half = (warp - 2) >> 2;          // columns 64*half .. 64*half+63
    const int row = quad * 32 + lane;
    double acc[64];
#pragma unroll
    for (int j = 0; j < 64; ++j) acc[j] = 0.0;
    bool ok = true;
    for (int c = 0; c < nchunks && ok; ++c) {
      ok = __all_sync(0xffffffffu, tc::mbar_wait(accf, c & 1));
      if (!ok) break;
      tc::tc_fence_after();
      for (int d = 2; d <= ns + 1; ++d) {
        const double wd = ldexp(1.0, -7 * d);
        const uint32_t base = tmem + uint32_t((d - 2) * 128 + half * 64) + (uint32_t(quad * 32) << 16);
        uint32_t r[32];
        tc::tmem_ld_32x32(base, r);
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] += double(int(r[j])) * wd;
        tc::tmem_ld_32x32(base + 32, r);
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[32 + j] += double(int(r[j])) * wd;
      }
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(acce);
    }
    if (ok) {
      const int er = it.ea[row];
      double* dst = it.C + size_t(row) * it.ldc + half * 64;
#pragma unroll
      for (int j = 0; j < 64; j += 2) {
        const int col = half * 64 + j;
        double v0 = ldexp(acc[j], er + it.eb[col]), v1 = ldexp(acc[j + 1], er + it.eb[col + 1]);
        if (col - row == it.diag) v0 += 1.0;
        if (col + 1 - row == it.diag) v1 += 1.0;
        *reinterpret_cast<double2*>(dst + j) = make_double2(v0, v1);
      }
    } else if (lane == 0) {
      atomicOr(it.err, kErrTimeout);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 128 * kOzAcc);
}

// ---------------------------------------------------------------------------
// Host side
void launch_ozaki_zero(const ProbDev* probs, const WorkItem* items, int n, cudaStream_t s) {
  if (n > 0) ozaki_zero_kernel<<<n, 256, 0, s>>>(probs, items);
}
void launch_ozaki_rowmax(const ProbDev* probs, const WorkItem* items, int n, cudaStream_t s) {
  if (n > 0) ozaki_rowmax_kernel<<<n, 256, 0, s>>>(probs, items);
}
void launch_ozaki_slice(const ProbDev* probs, const WorkItem* items, int n, cudaStream_t s) {
  if (n > 0) ozaki_slice_kernel<<<n, 256, 0, s>>>(probs, items);
}
void launch_slice_kmajor(const SliceOp& op, cudaStream_t s) {
  if (op.Rpad <= 0 || op.Kpad <= 0 || op.nz <= 0) return;
  cudaMemsetAsync(op.rmax, 0, size_t(op.nz) * op.Rpad * sizeof(unsigned long long), s);
  const dim3 grid(op.Kpad / 64, op.Rpad / 64, op.nz);
  slice_rowmax_kernel<<<grid, 256, 0, s>>>(op);
  slice_kmajor_kernel<<<grid, 256, 0, s>>>(op);
}
void launch_syrk_ozaki_fused(const TcItem* items, int n, int ny, cudaStream_t s) {
  if (n > 0 && ny > 0) syrk_ozaki_fused_kernel<<<dim3(n, ny), kOzThreads, kOzfSmemBytes, s>>>(items);
}
void launch_syrk_ozaki(const TcItem* items, int n, int ny, cudaStream_t s) {
  if (n > 0 && ny > 0) syrk_ozaki_kernel<<<dim3(n, ny), kOzThreads, kOzSmemBytes, s>>>(items);
}

cudaError_t prepare_ozaki_kernels() {
  cudaError_t e =
      cudaFuncSetAttribute(syrk_ozaki_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kOzSmemBytes));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(syrk_ozaki_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              int(kOzfSmemBytes));
}

}  // namespace rigw
