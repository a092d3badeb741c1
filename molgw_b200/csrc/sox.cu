// Vertex corrections on the imaginary axis.  GW+SOX: the second-order screened
// exchange on the evaluation points, sox_selfenergy_imag_grid
// (src/m_g3w2_selfenergy.f90:2482-2591); GW+SOSEX further below.
//
//   C_p[q][(j,c)] = (p q|j c) = sum_P M_pq[P] M_jc[P]               FP64 DMMA product
//   Sigma_p(z) = - sum_{i,k occ; b empty} C_p[i][(k,b)] C_p[k][(i,b)] / (z - e_i - e_k + e_b)
//                - sum_{a,c empty; j occ} C_p[a][(j,c)] C_p[c][(j,a)] / (z - e_a - e_c + e_j)
//
// The reference evaluates two RI integrals per (p, i, k, b) and per (p, a, j, c)
// inside its loops (evaluate_eri_mo, :2534-2577).  Here every integral is one
// entry of C_p: one product on the DMMA tile engine per chunk of Sigma states,
// with the auxiliary index as the reduction.  The frequency sums then read C_p
// once per kSoxW evaluation points; the empty-empty sum runs over tile pairs
// a-tile <= c-tile only (the summand is symmetric in a and c).
#include <algorithm>
#include <vector>

#include "engine.cuh"

namespace rigw {
namespace {

constexpr int kSoxThreads = 256;
constexpr int kSoxW = 8;      // evaluation points per pass (register accumulators; 8 leaves room
                              // for two blocks per SM: 8 > 16 by 30%, > 4 by 25% on B200)
constexpr int kSoxTile = 32;  // empty-state tile of the second sum
constexpr int kSoxBlockB = kSoxThreads;   // empty states b per unit of the first sum

inline long long round_up_ll(long long v, long long a) { return (v + a - 1) / a * a; }

// Column of row r = o * group + q in a transposed operand: groups of rows padded
// to group_pad, the rows of a group at or after `split` moved by `shift`, and the
// groups at or after `osplit` moved by `oshift` (even widths for the 16-byte
// operand loads of the DMMA tile engine; zeros stay in the gaps).
struct TransposeMap {
  long long group, group_pad, split, shift, osplit, oshift;
};

// dst[P][column(r)] = src[r][P]: rows of naux values become columns.
__global__ void sox_transpose_kernel(const double* __restrict__ src, long long nrows, int naux, TransposeMap map,
                                     double* __restrict__ dst, long long ld_dst) {
  __shared__ double t[32][33];
  const long long r0 = (long long)blockIdx.x * 32;
  const int p0 = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += 8) {
    const long long r = r0 + y;
    const int p = p0 + threadIdx.x;
    t[y][threadIdx.x] = (r < nrows && p < naux) ? src[r * naux + p] : 0.0;
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += 8) {
    const int p = p0 + y;
    const long long r = r0 + threadIdx.x;
    if (p < naux && r < nrows) {
      const long long o = r / map.group, q = r % map.group;
      const long long col = (o + (o >= map.osplit ? map.oshift : 0)) * map.group_pad + q + (q >= map.split ? map.shift : 0);
      dst[p * ld_dst + col] = t[threadIdx.x][y];
    }
  }
}

struct SoxArgs {
  const double* C;     // [pc][ngp][ldc]: C_p rows q (occupied first), columns (j, c)
  long long sp;        // doubles between the blocks of two Sigma states (ngp * ldc)
  long long ldc;
  int no, nv;
  const double* e;     // [no + nv] energy_g over the window
  const double* z;     // [nw][2]
  int nw;
  int units1;          // first sum: (i, k) x blocks of kSoxBlockB empty states
  int bblocks;
  int vt, tpairs;      // second sum: tiles of the empty states, tile pairs ta <= tc
  int units;           // units1 + no * tpairs
  double* partial;     // [pc][gridDim.x][nw][2]
};

// One block per (unit stripe, Sigma state of the chunk).  Every thread keeps
// sum_e w_e (x / d) and sum_e w_e / d for kSoxW points (x = Re z - delta,
// d = |z - delta|^2), so that sum_e w_e / (z - delta) = ar - i Im(z) as.  The
// per-block sums go to `partial` in a fixed order (deterministic results).
__global__ void __launch_bounds__(kSoxThreads, 2) sox_contract_kernel(SoxArgs a) {
  __shared__ double s1[kSoxTile][kSoxTile + 1];
  __shared__ double s2[kSoxTile][kSoxTile + 1];
  __shared__ double red[kSoxThreads / 32][kSoxW][2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* C = a.C + (long long)blockIdx.y * a.sp;
  const double* ev = a.e + a.no;
  for (int w0 = 0; w0 < a.nw; w0 += kSoxW) {
    const int nwc = min(kSoxW, a.nw - w0);
    double zr[kSoxW], zi2[kSoxW], ar[kSoxW], as[kSoxW];
#pragma unroll
    for (int w = 0; w < kSoxW; ++w) {
      const bool ok = w < nwc;
      zr[w] = ok ? a.z[2 * (w0 + w)] : 0.0;
      const double zi = ok ? a.z[2 * (w0 + w) + 1] : 1.0;   // padded points: finite, discarded
      zi2[w] = zi * zi;
      ar[w] = as[w] = 0.0;
    }
    auto add = [&](double pw, double delta) {
#pragma unroll
      for (int w = 0; w < kSoxW; ++w) {
        const double x = zr[w] - delta;
        const double r = pw * __drcp_rn(fma(x, x, zi2[w]));
        ar[w] = fma(r, x, ar[w]);
        as[w] += r;
      }
    };
    for (int u = blockIdx.x; u < a.units; u += gridDim.x) {   // u is block-uniform
      if (u < a.units1) {
        const int pair = u / a.bblocks, bb = u % a.bblocks;
        const int i = pair / a.no, k = pair % a.no;
        const int b = bb * kSoxBlockB + tid;
        if (b < a.nv) {
          const double v1 = C[i * a.ldc + (long long)k * a.nv + b];   // (p i|b k)
          const double v2 = C[k * a.ldc + (long long)i * a.nv + b];   // (i b|k p)
          add(v1 * v2, a.e[i] + a.e[k] - ev[b]);
        }
      } else {
        const int u2 = u - a.units1;
        const int j = u2 / a.tpairs;
        int rem = u2 % a.tpairs, ta = 0;
        while (rem >= a.vt - ta) {
          rem -= a.vt - ta;
          ++ta;
        }
        const int tc = ta + rem;
        const int a0 = ta * kSoxTile, c0 = tc * kSoxTile;
        const long long col = (long long)j * a.nv;
        __syncthreads();   // the previous tile pair is consumed
        for (int y = warp; y < kSoxTile; y += kSoxThreads / 32) {
          const int ra = a0 + y, rc = c0 + y;
          // s1[y][x] = (p a|j c) with a = a0 + y, c = c0 + x; s2[y][x] = (p c|j a) with c = c0 + y, a = a0 + x
          s1[y][lane] = (ra < a.nv && c0 + lane < a.nv) ? C[(a.no + ra) * a.ldc + col + c0 + lane] : 0.0;
          s2[y][lane] = (rc < a.nv && a0 + lane < a.nv) ? C[(a.no + rc) * a.ldc + col + a0 + lane] : 0.0;
        }
        __syncthreads();
        const double wt = ta == tc ? 1.0 : 2.0;
        const double ej = a.e[j];
        const int c = c0 + lane;
        for (int y = warp; y < kSoxTile; y += kSoxThreads / 32) {
          const int aa = a0 + y;
          if (aa < a.nv && c < a.nv) add(wt * s1[y][lane] * s2[lane][y], ev[aa] + ev[c] - ej);
        }
      }
    }
#pragma unroll
    for (int w = 0; w < kSoxW; ++w)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ar[w] += __shfl_xor_sync(0xffffffffu, ar[w], o);
        as[w] += __shfl_xor_sync(0xffffffffu, as[w], o);
      }
    __syncthreads();   // the previous pass's reads of red are done
    if (lane == 0)
#pragma unroll
      for (int w = 0; w < kSoxW; ++w) {
        red[warp][w][0] = ar[w];
        red[warp][w][1] = as[w];
      }
    __syncthreads();
    if (tid < nwc) {
      double sr = 0.0, ss = 0.0;
      for (int wp = 0; wp < kSoxThreads / 32; ++wp) {
        sr += red[wp][tid][0];
        ss += red[wp][tid][1];
      }
      const double zi = a.z[2 * (w0 + tid) + 1];
      double* out = a.partial + (((long long)blockIdx.y * gridDim.x + blockIdx.x) * a.nw + w0 + tid) * 2;
      out[0] = -sr;       // Sigma^SOX = - sum w / (z - delta)
      out[1] = zi * ss;
    }
  }
}

// out[pl][w] = sum over blocks of partial[pl][blk][w], in block order.
__global__ void sox_reduce_kernel(const double* __restrict__ partial, int nblk, int nw, int pc,
                                  double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= pc * nw) return;
  const int pl = t / nw, w = t % nw;
  double r = 0.0, im = 0.0;
  for (int b = 0; b < nblk; ++b) {
    const double* q = partial + (((long long)pl * nblk + b) * nw + w) * 2;
    r += q[0];
    im += q[1];
  }
  out[2 * (long long)t] = r;
  out[2 * (long long)t + 1] = im;
}

}  // namespace

Status sox_selfenergy_imag(Context& c, const rigw_sox_problem& pr, double* sigma_sox) {
  const int no = pr.nocc, nv = pr.nvirt, naux = pr.naux, nsig = pr.nsig, nw = pr.nomega_calc;
  if (no <= 0 || nv <= 0 || naux <= 0 || nsig <= 0 || nw <= 0 || !pr.m_ov || !pr.m_pq || !pr.energy ||
      !pr.omega_calc || !sigma_sox)
    return Status::fail(RIGW_ERR_ARG, "sox_selfenergy_imag: invalid arguments");
  NvtxRange range("SOX self-energy");
  const bool on_dev = (pr.flags & RIGW_PROBLEM_DEVICE_POINTERS) != 0;
  const int ng = no + nv;
  const long long nov = (long long)no * nv;
  const long long novp = round_up_ll(nov, 2), ngp = round_up_ll(ng, 2);
  const long long lda = (long long)nsig * ngp;
  if (lda >= (1LL << 31) || novp >= (1LL << 31))
    return Status::fail(RIGW_ERR_ARG, "sox_selfenergy_imag: product dimensions beyond 2^31");
  cudaStream_t s = c.stream;
  struct Events {
    cudaEvent_t e[4] = {};
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  for (cudaEvent_t& x : ev.e) RIGW_CUDA_TRY(cudaEventCreate(&x));
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[0], s));

  DeviceBuffer b_mov, b_mpq, b_e, b_z, b_bt, b_at, b_c, b_part, b_out, b_items;
  const double* mov = pr.m_ov;
  const double* mpq = pr.m_pq;
  if (!on_dev) {
    RIGW_TRY(b_mov.allocate(&c, size_t(nov) * naux * 8, "sox m_ov"));
    RIGW_TRY(b_mpq.allocate(&c, size_t(nsig) * ng * naux * 8, "sox m_pq"));
    RIGW_CUDA_TRY(cudaMemcpyAsync(b_mov.data(), pr.m_ov, size_t(nov) * naux * 8, cudaMemcpyHostToDevice, s));
    RIGW_CUDA_TRY(cudaMemcpyAsync(b_mpq.data(), pr.m_pq, size_t(nsig) * ng * naux * 8, cudaMemcpyHostToDevice, s));
    mov = reinterpret_cast<const double*>(b_mov.data());
    mpq = reinterpret_cast<const double*>(b_mpq.data());
  }
  RIGW_TRY(b_e.allocate(&c, size_t(ng) * 8, "sox energies"));
  RIGW_TRY(b_z.allocate(&c, size_t(nw) * 16, "sox omega_calc"));
  RIGW_CUDA_TRY(cudaMemcpyAsync(b_e.data(), pr.energy, size_t(ng) * 8, cudaMemcpyDefault, s));
  RIGW_CUDA_TRY(cudaMemcpyAsync(b_z.data(), pr.omega_calc, size_t(nw) * 16, cudaMemcpyDefault, s));
  // K-major operands of the product: Bt[P][(j,c)], At[P][(p, q)] (rows of ngp per state)
  RIGW_TRY(b_bt.allocate(&c, size_t(naux) * novp * 8, "sox M_ov^T"));
  RIGW_TRY(b_at.allocate(&c, size_t(naux) * lda * 8, "sox M_pq^T"));
  double* bt = reinterpret_cast<double*>(b_bt.data());
  double* at = reinterpret_cast<double*>(b_at.data());
  int launches = 0;
  if (novp != nov) RIGW_CUDA_TRY(cudaMemsetAsync(bt, 0, size_t(naux) * novp * 8, s));
  if (ngp != ng) RIGW_CUDA_TRY(cudaMemsetAsync(at, 0, size_t(naux) * lda * 8, s));
  {
    const dim3 blk(32, 8);
    const long long never = 1LL << 62;
    sox_transpose_kernel<<<dim3(unsigned((nov + 31) / 32), unsigned((naux + 31) / 32)), blk, 0, s>>>(
        mov, nov, naux, TransposeMap{nov, novp, never, 0, never, 0}, bt, novp);
    sox_transpose_kernel<<<dim3(unsigned(((long long)nsig * ng + 31) / 32), unsigned((naux + 31) / 32)), blk, 0,
                           s>>>(mpq, (long long)nsig * ng, naux, TransposeMap{ng, ngp, never, 0, never, 0}, at, lda);
    RIGW_CUDA_TRY(cudaGetLastError());
    launches += 2;
  }
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[1], s));

  // Sigma states per product: C of a chunk stays below ~2 GB and below half of
  // what the context's HBM budget has left
  const size_t per_p = size_t(ngp) * novp * 8;
  size_t cap = size_t(2) << 30;
  if (c.budget > 0) cap = std::min(cap, c.budget > c.in_use ? (c.budget - c.in_use) / 2 : size_t(0));
  const int pc = int(std::max<size_t>(1, std::min<size_t>(size_t(nsig), cap / per_p)));
  RIGW_TRY(b_c.allocate(&c, per_p * pc, "sox (p q|j c)"));
  double* cbuf = reinterpret_cast<double*>(b_c.data());
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
  SoxArgs a{};
  a.sp = ngp * novp;
  a.ldc = novp;
  a.no = no;
  a.nv = nv;
  a.e = reinterpret_cast<const double*>(b_e.data());
  a.z = reinterpret_cast<const double*>(b_z.data());
  a.nw = nw;
  a.bblocks = (nv + kSoxBlockB - 1) / kSoxBlockB;
  a.units1 = no * no * a.bblocks;
  a.vt = (nv + kSoxTile - 1) / kSoxTile;
  a.tpairs = a.vt * (a.vt + 1) / 2;
  a.units = a.units1 + no * a.tpairs;
  const int nblk = std::max(1, std::min(a.units, sms * 4 / pc));
  RIGW_TRY(b_part.allocate(&c, size_t(pc) * nblk * nw * 16, "sox partial sums"));
  a.partial = reinterpret_cast<double*>(b_part.data());
  double* out = sigma_sox;
  if (!on_dev) {
    RIGW_TRY(b_out.allocate(&c, size_t(nsig) * nw * 16, "sox sigma"));
    out = reinterpret_cast<double*>(b_out.data());
  }
  const long long mrows_max = (long long)pc * ngp;
  const size_t max_items = size_t((mrows_max + 127) / 128) * size_t((novp + 127) / 128);
  RIGW_TRY(b_items.allocate(&c, max_items * sizeof(GemmItem), "sox gemm items"));
  std::vector<GemmItem> items;
  items.reserve(max_items);
  double ms_gemm = 0.0, ms_sum = 0.0;
  cudaEvent_t* e = ev.e;
  for (int p0 = 0; p0 < nsig; p0 += pc) {
    const int pcn = std::min(pc, nsig - p0);
    const long long mrows = (long long)pcn * ngp;
    items.clear();
    // column blocks outer: the CTAs in flight share a few 128-column tiles of
    // M_ov^T while all of M_pq^T stays in L2, so M_ov^T comes from HBM about once
    for (long long j0 = 0; j0 < novp; j0 += 128)
      for (long long i0 = 0; i0 < mrows; i0 += 128) {
        GemmItem g{};
        g.A = at + (long long)p0 * ngp + i0;
        g.lda = int(lda);
        g.B = bt + j0;
        g.ldb = int(novp);
        g.C = cbuf + i0 * novp + j0;
        g.ldc = int(novp);
        g.m = int(std::min<long long>(128, mrows - i0));
        g.n = int(std::min<long long>(128, novp - j0));
        g.k = naux;
        g.alpha = 1.0;
        items.push_back(g);
      }
    // the previous chunk's launches read the item list: order the upload after them
    RIGW_CUDA_TRY(cudaMemcpyAsync(b_items.data(), items.data(), items.size() * sizeof(GemmItem),
                                  cudaMemcpyHostToDevice, s));
    RIGW_CUDA_TRY(cudaEventRecord(e[2], s));
    launch_dgemm_128x128(reinterpret_cast<const GemmItem*>(b_items.data()), int(items.size()), 1, s);
    RIGW_CUDA_TRY(cudaGetLastError());
    RIGW_CUDA_TRY(cudaEventRecord(e[3], s));
    a.C = cbuf;
    sox_contract_kernel<<<dim3(nblk, pcn), kSoxThreads, 0, s>>>(a);
    RIGW_CUDA_TRY(cudaGetLastError());
    const int nred = pcn * nw;
    sox_reduce_kernel<<<(nred + 127) / 128, 128, 0, s>>>(a.partial, nblk, nw, pcn, out + size_t(p0) * nw * 2);
    RIGW_CUDA_TRY(cudaGetLastError());
    launches += 3;
    RIGW_CUDA_TRY(cudaEventRecord(e[1], s));
    RIGW_CUDA_TRY(cudaEventSynchronize(e[1]));   // host reuses `items` for the next chunk
    float t1 = 0.0f, t2 = 0.0f;
    cudaEventElapsedTime(&t1, e[2], e[3]);
    cudaEventElapsedTime(&t2, e[3], e[1]);
    ms_gemm += t1;
    ms_sum += t2;
  }
  if (!on_dev)
    RIGW_CUDA_TRY(cudaMemcpyAsync(sigma_sox, out, size_t(nsig) * nw * 16, cudaMemcpyDeviceToHost, s));
  RIGW_CUDA_TRY(cudaEventRecord(e[1], s));
  RIGW_CUDA_TRY(cudaEventSynchronize(e[1]));
  float total = 0.0f;
  cudaEventElapsedTime(&total, e[0], e[1]);
  rigw_stats st{};
  st.stage_ms[0] = double(total) - ms_gemm - ms_sum;   // uploads, transposes, download
  st.stage_ms[1] = ms_gemm;
  st.stage_ms[3] = ms_sum;
  st.total_ms = total;
  st.kernel_launches = launches;
  st.chunks = (nsig + pc - 1) / pc;
  st.waves = 1;
  st.device_bytes_in_use = c.in_use;
  st.device_bytes_peak = c.peak;
  c.last_stats = st;
  return Status::ok();
}


// ---- SOSEX on the imaginary axis (sosex_selfenergy_imag_grid) -----------------
//
// Sigma_m(z) = f/(2 pi) sum_k w_k sum_r [K_k(m, r) / (z + i w_k - e_r) + conj(K_k(m, r)) / (z - i w_k - e_r)]
// K_k(m, r)  = sum_{i,a} T_k(r; i,a) [B1(r; i,a) / (i w_k - D) - B2(r; i,a) / (i w_k + D)],  D = e_a - e_i
// T_k(r; i,a) = (r m|W - v|i a) = sum_Q R_k[Q][r] M[Q](i,a),  R_k = W~_k M(., m),  W~_k = Y_k^T Y_k - 1
// B1 = (r a|i m), B2 = (r i|a m)  (bare, frequency independent)
//
// The reference recomputes its bra-kets for every evaluation point and sign
// (:2262-2466); K_k does not depend on z, and the s = -1 sum is the conjugate of
// the s = +1 one, so the products run once per (Sigma state, frequency).  The
// window tensor is held once, transposed: Mft[P][pos(r) * wq + pos(q)], with the
// occupied and empty blocks each padded to an even width (pos).
namespace {

constexpr int kSosexThreads = 256;

struct SosexKArgs {
  const double* T;     // [pc][wq][niap], rows at window positions, columns i * nvp + a
  const double* B1;
  const double* B2;
  const double* epos;  // [wq] energy_g at window positions (0 in the gaps)
  int no, nv, nop, nvp, wq;
  long long niap;
  double om;           // w_k
  double* K;           // [nsig][nwp][wq][2]
  int k, nwp, p0;
};

// Sum of (a, b) over the block in a fixed order; thread 0 holds the result.
__device__ __forceinline__ void block_sum2(double& a, double& b, double (*red)[2]) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[warp][0] = a;
    red[warp][1] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = b = 0.0;
    for (int wp = 0; wp < kSosexThreads / 32; ++wp) {
      a += red[wp][0];
      b += red[wp][1];
    }
  }
}

// One block per (window row r, Sigma state of the chunk): K_k(m, r).
__global__ void __launch_bounds__(kSosexThreads) sosex_k_kernel(SosexKArgs a) {
  __shared__ double red[kSosexThreads / 32][2];
  const int r = blockIdx.x, ml = blockIdx.y;
  const long long base = ((long long)ml * a.wq + r) * a.niap;
  const double om2 = a.om * a.om;
  double sr = 0.0, si = 0.0;
  for (long long ia = threadIdx.x; ia < a.niap; ia += kSosexThreads) {
    const int i = int(ia / a.nvp), av = int(ia % a.nvp);
    if (i >= a.no || av >= a.nv) continue;
    const double d = a.epos[a.nop + av] - a.epos[i];
    const double t = a.T[base + ia], b1 = a.B1[base + ia], b2 = a.B2[base + ia];
    const double inv = __drcp_rn(fma(d, d, om2));
    // B1 / (i w - D) - B2 / (i w + D) = [-D (B1 + B2) - i w (B1 - B2)] / (D^2 + w^2)
    sr = fma(-t * d * (b1 + b2), inv, sr);
    si = fma(-t * (b1 - b2), inv, si);
  }
  block_sum2(sr, si, red);
  if (threadIdx.x == 0) {
    double* out = a.K + (((long long)(a.p0 + ml) * a.nwp + a.k) * a.wq + r) * 2;
    out[0] = sr;
    out[1] = a.om * si;
  }
}

// One block per (Sigma state, evaluation point): the sum over (k, r).
__global__ void __launch_bounds__(kSosexThreads)
sosex_sigma_kernel(const double* __restrict__ K, const double* __restrict__ omega, const double* __restrict__ weight,
                   const double* __restrict__ epos, const double* __restrict__ z, int nwp, int wq, int nw,
                   double scale, double* __restrict__ out) {
  __shared__ double red[kSosexThreads / 32][2];
  const int m = blockIdx.x, iz = blockIdx.y;
  const double zr = z[2 * iz], zi = z[2 * iz + 1];
  double sr = 0.0, si = 0.0;
  const int n = nwp * wq;
  for (int t = threadIdx.x; t < n; t += kSosexThreads) {
    const int k = t / wq, r = t % wq;
    const double* kk = K + (((long long)m * nwp + k) * wq + r) * 2;
    const double kr = kk[0], ki = kk[1], wk = weight[k], om = omega[k];
    const double x = zr - epos[r];
    // K / (x + i (zi + w)) + conj(K) / (x + i (zi - w))
    const double y1 = zi + om, y2 = zi - om;
    const double i1 = __drcp_rn(fma(x, x, y1 * y1)), i2 = __drcp_rn(fma(x, x, y2 * y2));
    sr += wk * ((kr * x + ki * y1) * i1 + (kr * x - ki * y2) * i2);
    si += wk * ((ki * x - kr * y1) * i1 + (-ki * x - kr * y2) * i2);
  }
  block_sum2(sr, si, red);
  if (threadIdx.x == 0) {
    out[((long long)m * nw + iz) * 2] = scale * sr;
    out[((long long)m * nw + iz) * 2 + 1] = scale * si;
  }
}

// ---------------------------------------------------------------------------
// G3W2 on the imaginary axis (g3w2_selfenergy_imag_grid, src/m_g3w2_selfenergy.f90:2018-2196).
// For one Sigma state p, with X_k[Q][u] = sum_P W~_k[P][Q] M(u, p, P):
//   Gn_k[v][w][u] = (v w|W_k - v|u p) = sum_Q M(v, w, Q) X_k[Q][u]
//   Gp_k[v][w][u] = (u v|W_k - v|w p) = sum_Q X_k[Q][w] M(v, u, Q)     (M symmetric in its states)
//   Sigma_p(z) = (2 pi)^-2 sum_{k', k''} w' w'' sum_v sum_u sum_{s', s''} a_u(z, s') b_v(z, s', s'')
//                sum_w c_w(z, s'') Gn_k'[v][w][u] Gp_k''[v][w][u]
// with a_u = 1/(z + s' i w' - e_u), b_v = 1/(z + s' i w' + s'' i w'' - e_v),
// c_w = 1/(z + s'' i w'' - e_w).  One block per (k', k'', kG3Z points): every
// thread owns states u, keeps the inner sums over w in registers for the
// block's points and both s'', and the products with a_u b_v; one block sum at
// the end.  Both tensors are read along u, so the loads are coalesced.
constexpr int kG3Z = 4;

struct G3w2Args {
  const double* gn;    // [nwp][ng][wq][wq]
  const double* gp;    // [nwp][ng][wq][wq]
  long long sk;        // doubles per frequency: ng * wq * wq
  int ng, wq;
  const double* e;     // [ng] energy_g over the window
  const double* om;    // [nwp] imaginary frequencies
  const double* wt;    // [nwp] quadrature weights
  int nwp;
  const double* z;     // [nz][2]
  int nz;
  double* partial;     // [nwp * nwp][nz][2]
};

RIGW_DEVICE_INLINE void crecip(double x, double y, double& r, double& i) {
  const double inv = 1.0 / fma(x, x, y * y);
  r = x * inv;
  i = -y * inv;
}

__global__ void __launch_bounds__(kSosexThreads) g3w2_contract_kernel(G3w2Args a) {
  extern __shared__ double csm[];   // [ng][kG3Z][2 (s'')][2]: c_w(z, s'')
  __shared__ double red[kSosexThreads / 32][2];
  const int k1 = blockIdx.x / a.nwp, k2 = blockIdx.x % a.nwp;
  const int z0 = blockIdx.y * kG3Z, nzc = min(kG3Z, a.nz - z0);
  const double w1 = a.om[k1], w2 = a.om[k2];
  for (int idx = threadIdx.x; idx < a.ng * kG3Z * 2; idx += kSosexThreads) {
    const int w = idx / (kG3Z * 2), zi = (idx >> 1) % kG3Z, s2 = idx & 1;
    double cr = 0.0, ci = 0.0;
    if (zi < nzc) crecip(a.z[2 * (z0 + zi)] - a.e[w], a.z[2 * (z0 + zi) + 1] + (s2 ? -w2 : w2), cr, ci);
    csm[2 * idx] = cr;
    csm[2 * idx + 1] = ci;
  }
  __syncthreads();
  double accr[kG3Z], acci[kG3Z];
#pragma unroll
  for (int zi = 0; zi < kG3Z; ++zi) accr[zi] = acci[zi] = 0.0;
  const double* g1 = a.gn + k1 * a.sk;
  const double* g2 = a.gp + k2 * a.sk;
  const long long wq2 = (long long)a.wq * a.wq;
  for (int u = threadIdx.x; u < a.ng; u += kSosexThreads) {
    double ar[kG3Z][2], ai[kG3Z][2];
#pragma unroll
    for (int zi = 0; zi < kG3Z; ++zi)
#pragma unroll
      for (int s1 = 0; s1 < 2; ++s1)
        crecip(a.z[2 * (z0 + min(zi, nzc - 1))] - a.e[u], a.z[2 * (z0 + min(zi, nzc - 1)) + 1] + (s1 ? -w1 : w1),
               ar[zi][s1], ai[zi][s1]);
    for (int v = 0; v < a.ng; ++v) {
      double fr[kG3Z][2], fi[kG3Z][2];
#pragma unroll
      for (int zi = 0; zi < kG3Z; ++zi) fr[zi][0] = fr[zi][1] = fi[zi][0] = fi[zi][1] = 0.0;
      const double* p1 = g1 + v * wq2 + u;
      const double* p2 = g2 + v * wq2 + u;
      for (int w = 0; w < a.ng; ++w) {
        const double h = p1[(long long)w * a.wq] * p2[(long long)w * a.wq];
        const double* c = csm + w * kG3Z * 4;
#pragma unroll
        for (int zi = 0; zi < kG3Z; ++zi)
#pragma unroll
          for (int s2 = 0; s2 < 2; ++s2) {
            fr[zi][s2] = fma(h, c[(zi * 2 + s2) * 2], fr[zi][s2]);
            fi[zi][s2] = fma(h, c[(zi * 2 + s2) * 2 + 1], fi[zi][s2]);
          }
      }
      const double ev = a.e[v];
#pragma unroll
      for (int zi = 0; zi < kG3Z; ++zi) {
        const double zr = a.z[2 * (z0 + min(zi, nzc - 1))] - ev, zm = a.z[2 * (z0 + min(zi, nzc - 1)) + 1];
#pragma unroll
        for (int s1 = 0; s1 < 2; ++s1)
#pragma unroll
          for (int s2 = 0; s2 < 2; ++s2) {
            double br, bi;
            crecip(zr, zm + (s1 ? -w1 : w1) + (s2 ? -w2 : w2), br, bi);
            const double tr = ar[zi][s1] * br - ai[zi][s1] * bi, ti = ar[zi][s1] * bi + ai[zi][s1] * br;
            accr[zi] += tr * fr[zi][s2] - ti * fi[zi][s2];
            acci[zi] += tr * fi[zi][s2] + ti * fr[zi][s2];
          }
      }
    }
  }
  const double scale = a.wt[k1] * a.wt[k2] / (4.0 * kPi * kPi);
  for (int zi = 0; zi < nzc; ++zi) {
    double sr = accr[zi], si = acci[zi];
    block_sum2(sr, si, red);
    if (threadIdx.x == 0) {
      double* o = a.partial + ((long long)blockIdx.x * a.nz + z0 + zi) * 2;
      o[0] = scale * sr;
      o[1] = scale * si;
    }
    __syncthreads();   // red is reused by the next point
  }
}

// out[iz] = sum over the frequency pairs of the partial sums, in a fixed order.
__global__ void __launch_bounds__(kSosexThreads) g3w2_reduce_kernel(const double* __restrict__ partial, int npair,
                                                                     int nz, double* __restrict__ out) {
  __shared__ double red[kSosexThreads / 32][2];
  const int iz = blockIdx.x;
  double sr = 0.0, si = 0.0;
  for (int j = threadIdx.x; j < npair; j += kSosexThreads) {
    sr += partial[((long long)j * nz + iz) * 2];
    si += partial[((long long)j * nz + iz) * 2 + 1];
  }
  block_sum2(sr, si, red);
  if (threadIdx.x == 0) {
    out[2 * iz] = sr;
    out[2 * iz + 1] = si;
  }
}

Status upload_items(Context& c, DeviceBuffer* buf, const std::vector<GemmItem>& items, const char* what) {
  if (items.empty()) return Status::ok();
  RIGW_TRY(buf->allocate(&c, items.size() * sizeof(GemmItem), what));
  RIGW_CUDA_TRY(cudaMemcpyAsync(buf->data(), items.data(), items.size() * sizeof(GemmItem), cudaMemcpyHostToDevice,
                                c.stream));
  return Status::ok();
}

}  // namespace

Status sosex_selfenergy_imag(Context& c, const Wpol& w, const rigw_sosex_problem& pr, double* sigma) {
  const int no = pr.nocc, nv = pr.nvirt, naux = pr.naux, nsig = pr.nsig, nw = pr.nomega_calc;
  const int ng = no + nv;
  if (no <= 0 || nv <= 0 || naux <= 0 || nsig <= 0 || nw <= 0 || nw > 65535 || !pr.m_full || !pr.energy ||
      !pr.omega_calc || !sigma || pr.sig_first < 0 || pr.sig_first + nsig > ng)
    return Status::fail(RIGW_ERR_ARG, "sosex_selfenergy_imag: invalid arguments");
  const ProbDev& pd = w.plan->problems()[0].dev;
  if (naux != pd.naux) return Status::fail(RIGW_ERR_ARG, "sosex_selfenergy_imag: naux differs from the polarizability");
  if (!pd.want_identity)
    return Status::fail(RIGW_ERR_UNSUPPORTED, "sosex_selfenergy_imag: the polarizability was solved without W (QP-only)");
  NvtxRange range("SOSEX self-energy");
  const bool on_dev = (pr.flags & RIGW_PROBLEM_DEVICE_POINTERS) != 0;
  const int nop = no + (no & 1), nvp = nv + (nv & 1), wq = nop + nvp;
  const long long niap = (long long)nop * nvp, ldm = (long long)wq * wq;
  const int naux_e = naux + (naux & 1), npad = pd.npad, nwp = pd.nomega;
  if (ldm >= (1LL << 31) || niap >= (1LL << 31))
    return Status::fail(RIGW_ERR_ARG, "sosex_selfenergy_imag: window beyond 2^31 operand columns");
  auto pos = [&](int q) { return q < no ? q : q + (nop - no); };
  cudaStream_t s = c.stream;
  struct Events {
    cudaEvent_t e[4] = {};
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  for (cudaEvent_t& x : ev.e) RIGW_CUDA_TRY(cudaEventCreate(&x));
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[0], s));

  // window tensor, transposed once: Mft[P][pos(r) * wq + pos(q)]
  DeviceBuffer b_in, b_mft, b_e, b_z;
  const double* min = pr.m_full;
  if (!on_dev) {
    RIGW_TRY(b_in.allocate(&c, size_t(ng) * ng * naux * 8, "sosex window tensor"));
    RIGW_CUDA_TRY(cudaMemcpyAsync(b_in.data(), pr.m_full, size_t(ng) * ng * naux * 8, cudaMemcpyHostToDevice, s));
    min = reinterpret_cast<const double*>(b_in.data());
  }
  RIGW_TRY(b_mft.allocate(&c, size_t(naux) * ldm * 8, "sosex window tensor^T"));
  double* mft = reinterpret_cast<double*>(b_mft.data());
  RIGW_CUDA_TRY(cudaMemsetAsync(mft, 0, size_t(naux) * ldm * 8, s));
  sox_transpose_kernel<<<dim3(unsigned(((long long)ng * ng + 31) / 32), unsigned((naux + 31) / 32)), dim3(32, 8), 0,
                         s>>>(min, (long long)ng * ng, naux, TransposeMap{ng, wq, no, nop - no, no, nop - no}, mft, ldm);
  RIGW_CUDA_TRY(cudaGetLastError());
  int launches = 1;
  std::vector<double> epos(wq, 0.0);
  {
    std::vector<double> e(ng);
    RIGW_CUDA_TRY(cudaMemcpy(e.data(), pr.energy, size_t(ng) * 8, cudaMemcpyDefault));
    for (int q = 0; q < ng; ++q) epos[pos(q)] = e[q];
  }
  std::vector<double> om(nwp);
  RIGW_CUDA_TRY(cudaMemcpy(om.data(), pd.omega, size_t(nwp) * 8, cudaMemcpyDeviceToHost));
  RIGW_TRY(b_e.allocate(&c, size_t(wq) * 8, "sosex energies"));
  RIGW_TRY(b_z.allocate(&c, size_t(nw) * 16, "sosex omega_calc"));
  RIGW_CUDA_TRY(cudaMemcpyAsync(b_e.data(), epos.data(), size_t(wq) * 8, cudaMemcpyHostToDevice, s));
  RIGW_CUDA_TRY(cudaMemcpyAsync(b_z.data(), pr.omega_calc, size_t(nw) * 16, cudaMemcpyDefault, s));
  const double* de = reinterpret_cast<const double*>(b_e.data());
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[1], s));

  // Sigma states per pass: T, B1, B2 and R of a chunk below ~2 GB and below half
  // of what the HBM budget has left
  const size_t per_m = (size_t(3) * wq * niap + size_t(naux_e) * wq) * 8;
  size_t cap = size_t(2) << 30;
  if (c.budget > 0) cap = std::min(cap, c.budget > c.in_use ? (c.budget - c.in_use) / 2 : size_t(0));
  const int pc = int(std::max<size_t>(1, std::min<size_t>(size_t(nsig), cap / per_m)));
  DeviceBuffer b_t, b_b1, b_b2, b_r, b_wt, b_k, b_out, b_iw;
  RIGW_TRY(b_t.allocate(&c, size_t(pc) * wq * niap * 8, "sosex T"));
  RIGW_TRY(b_b1.allocate(&c, size_t(pc) * wq * niap * 8, "sosex B1"));
  RIGW_TRY(b_b2.allocate(&c, size_t(pc) * wq * niap * 8, "sosex B2"));
  RIGW_TRY(b_r.allocate(&c, size_t(pc) * naux_e * wq * 8, "sosex R"));
  RIGW_TRY(b_wt.allocate(&c, size_t(npad) * npad * 8, "sosex W~"));
  RIGW_TRY(b_k.allocate(&c, size_t(nsig) * nwp * wq * 16, "sosex K"));
  double* dt = reinterpret_cast<double*>(b_t.data());
  double* db1 = reinterpret_cast<double*>(b_b1.data());
  double* db2 = reinterpret_cast<double*>(b_b2.data());
  double* dr = reinterpret_cast<double*>(b_r.data());
  double* wt = reinterpret_cast<double*>(b_wt.data());
  double* dk = reinterpret_cast<double*>(b_k.data());
  // rows at the gaps of the window positions stay zero in B1 and B2 (no item writes them)
  RIGW_CUDA_TRY(cudaMemsetAsync(db1, 0, size_t(pc) * wq * niap * 8, s));
  RIGW_CUDA_TRY(cudaMemsetAsync(db2, 0, size_t(pc) * wq * niap * 8, s));
  double* out = sigma;
  if (!on_dev) {
    RIGW_TRY(b_out.allocate(&c, size_t(nsig) * nw * 16, "sosex sigma"));
    out = reinterpret_cast<double*>(b_out.data());
  }
  // W~_k = Y_k^T Y_k - 1 for every frequency (Y_k = U_k^-T, the identity part of the resident solve)
  std::vector<GemmItem> iw;
  for (int k = 0; k < nwp; ++k) {
    const double* y = pd.rhs + size_t(k) * npad * pd.ldb;
    for (int i0 = 0; i0 < npad; i0 += 128)
      for (int j0 = 0; j0 < npad; j0 += 128) {
        GemmItem g{};
        g.A = y + i0;
        g.lda = pd.ldb;
        g.B = y + j0;
        g.ldb = pd.ldb;
        g.C = wt + size_t(i0) * npad + j0;
        g.ldc = npad;
        g.m = std::min(128, npad - i0);
        g.n = std::min(128, npad - j0);
        g.k = npad;
        g.flags = kSubIdentity;
        g.diag = i0 - j0;
        g.alpha = 1.0;
        iw.push_back(g);
      }
  }
  const int nwt = int(iw.size()) / nwp;
  RIGW_TRY(upload_items(c, &b_iw, iw, "sosex W~ items"));
  const GemmItem* d_iw = reinterpret_cast<const GemmItem*>(b_iw.data());
  for (int p0 = 0; p0 < nsig; p0 += pc) {
    const int pcn = std::min(pc, nsig - p0);
    std::vector<GemmItem> ib, ir, it;
    for (int ml = 0; ml < pcn; ++ml) {
      const long long colm = (long long)pos(pr.sig_first + p0 + ml) * wq;   // columns of M(., m) in Mft
      for (int q = 0; q < ng; ++q) {
        const int r = pos(q);
        for (int i0 = 0; i0 < nop; i0 += 64)   // 64-row items of the 64 x 128 tile engine
          for (int a0 = 0; a0 < nvp; a0 += 128) {
            GemmItem g{};
            g.ldc = nvp;
            g.m = std::min(64, nop - i0);
            g.n = std::min(128, nvp - a0);
            g.k = naux;
            g.alpha = 1.0;
            g.lda = g.ldb = int(ldm);
            // B1[r][i][a] = sum_P M[P](i, m) M[P](r, a)
            g.A = mft + colm + i0;
            g.B = mft + (long long)r * wq + nop + a0;
            g.C = db1 + ((long long)ml * wq + r) * niap + (long long)i0 * nvp + a0;
            ib.push_back(g);
            // B2[r][i][a] = sum_P M[P](r, i) M[P](a, m)
            g.A = mft + (long long)r * wq + i0;
            g.B = mft + colm + nop + a0;
            g.C = db2 + ((long long)ml * wq + r) * niap + (long long)i0 * nvp + a0;
            ib.push_back(g);
          }
      }
      // R[Q][r] = sum_P W~[P][Q] M[P](r, m)
      for (int q0 = 0; q0 < naux_e; q0 += 128)
        for (int r0 = 0; r0 < wq; r0 += 128) {
          GemmItem g{};
          g.A = wt + q0;
          g.lda = npad;
          g.B = mft + colm + r0;
          g.ldb = int(ldm);
          g.C = dr + (size_t(ml) * naux_e + q0) * wq + r0;
          g.ldc = wq;
          g.m = std::min(128, naux_e - q0);
          g.n = std::min(128, wq - r0);
          g.k = naux;
          g.alpha = 1.0;
          ir.push_back(g);
        }
      // T[r][i][a] = sum_Q R[Q][r] M[Q](i, a)
      for (int r0 = 0; r0 < wq; r0 += 128)
        for (int i = 0; i < no; ++i)
          for (int a0 = 0; a0 < nvp; a0 += 128) {
            GemmItem g{};
            g.A = dr + size_t(ml) * naux_e * wq + r0;
            g.lda = wq;
            g.B = mft + (long long)i * wq + nop + a0;
            g.ldb = int(ldm);
            g.C = dt + ((long long)ml * wq + r0) * niap + (long long)i * nvp + a0;
            g.ldc = int(niap);
            g.m = std::min(128, wq - r0);
            g.n = std::min(128, nvp - a0);
            g.k = naux;
            g.alpha = 1.0;
            it.push_back(g);
          }
    }
    DeviceBuffer b_ib, b_ir, b_it;
    RIGW_TRY(upload_items(c, &b_ib, ib, "sosex B items"));
    RIGW_TRY(upload_items(c, &b_ir, ir, "sosex R items"));
    RIGW_TRY(upload_items(c, &b_it, it, "sosex T items"));
    launch_dgemm_64x128(reinterpret_cast<const GemmItem*>(b_ib.data()), int(ib.size()), 1, s);
    RIGW_CUDA_TRY(cudaGetLastError());
    ++launches;
    for (int k = 0; k < nwp; ++k) {
      launch_dgemm_128x128(d_iw + size_t(k) * nwt, nwt, 1, s);
      launch_dgemm_128x128(reinterpret_cast<const GemmItem*>(b_ir.data()), int(ir.size()), 1, s);
      launch_dgemm_128x128(reinterpret_cast<const GemmItem*>(b_it.data()), int(it.size()), 1, s);
      RIGW_CUDA_TRY(cudaGetLastError());
      SosexKArgs a{dt, db1, db2, de, no, nv, nop, nvp, wq, niap, om[k], dk, k, nwp, p0};
      sosex_k_kernel<<<dim3(wq, pcn), kSosexThreads, 0, s>>>(a);
      RIGW_CUDA_TRY(cudaGetLastError());
      launches += 4;
    }
    // the item buffers of this chunk are released at the end of the iteration
    RIGW_CUDA_TRY(cudaStreamSynchronize(s));
  }
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[2], s));
  sosex_sigma_kernel<<<dim3(nsig, nw), kSosexThreads, 0, s>>>(dk, pd.omega, pd.weight, de,
                                                              reinterpret_cast<const double*>(b_z.data()), nwp, wq,
                                                              nw, pr.factor_sosex / (2.0 * M_PI), out);
  RIGW_CUDA_TRY(cudaGetLastError());
  ++launches;
  if (!on_dev) RIGW_CUDA_TRY(cudaMemcpyAsync(sigma, out, size_t(nsig) * nw * 16, cudaMemcpyDeviceToHost, s));
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[3], s));
  RIGW_CUDA_TRY(cudaEventSynchronize(ev.e[3]));
  float t01 = 0.0f, t12 = 0.0f, t23 = 0.0f;
  cudaEventElapsedTime(&t01, ev.e[0], ev.e[1]);
  cudaEventElapsedTime(&t12, ev.e[1], ev.e[2]);
  cudaEventElapsedTime(&t23, ev.e[2], ev.e[3]);
  rigw_stats st{};
  st.stage_ms[0] = t01;   // upload and transpose of the window tensor
  st.stage_ms[1] = t12;   // products (B1, B2, W~, R, T) and the K reductions
  st.stage_ms[3] = t23;   // sums over (frequency, r) and the download
  st.total_ms = double(t01) + t12 + t23;
  st.kernel_launches = launches;
  st.chunks = (nsig + pc - 1) / pc;
  st.waves = 1;
  st.device_bytes_in_use = c.in_use;
  st.device_bytes_peak = c.peak;
  c.last_stats = st;
  return Status::ok();
}

Status g3w2_selfenergy_imag(Context& c, const Wpol& w, const rigw_g3w2_problem& pr, double* sigma) {
  const int ng = pr.nstate, naux = pr.naux, nsig = pr.nsig, nz = pr.nomega_calc;
  if (ng <= 0 || naux <= 0 || nsig <= 0 || nz <= 0 || nz > 65535 || !pr.m_full || !pr.energy || !pr.omega_calc ||
      !sigma || pr.sig_first < 0 || pr.sig_first + nsig > ng)
    return Status::fail(RIGW_ERR_ARG, "g3w2_selfenergy_imag: invalid arguments");
  const ProbDev& pd = w.plan->problems()[0].dev;
  if (naux != pd.naux) return Status::fail(RIGW_ERR_ARG, "g3w2_selfenergy_imag: naux differs from the polarizability");
  if (!pd.want_identity)
    return Status::fail(RIGW_ERR_UNSUPPORTED, "g3w2_selfenergy_imag: the polarizability was solved without W (QP-only)");
  const int wq = ng + (ng & 1), naux_e = naux + (naux & 1), npad = pd.npad, nwp = pd.nomega;
  const long long ldm = (long long)wq * wq, sk = (long long)ng * ldm;
  const size_t smem = size_t(ng) * kG3Z * 4 * sizeof(double);
  if (ldm >= (1LL << 31) || smem > 200 * 1024)
    return Status::fail(RIGW_ERR_ARG, "g3w2_selfenergy_imag: window of %d states beyond the contraction's limit", ng);
  // Gn and Gp of every frequency stay resident for the frequency pairs
  const size_t need = (size_t(2) * nwp * sk + size_t(nwp) * npad * npad + size_t(nwp) * naux_e * wq +
                       size_t(naux) * ldm + size_t(nwp) * nwp * nz * 2) * 8;
  if (c.budget > 0 && need > (c.budget > c.in_use ? c.budget - c.in_use : 0))
    return Status::fail(RIGW_ERR_NOMEM, "g3w2_selfenergy_imag: %zu bytes needed beyond the HBM budget", need);
  NvtxRange range("G3W2 self-energy");
  const bool on_dev = (pr.flags & RIGW_PROBLEM_DEVICE_POINTERS) != 0;
  cudaStream_t s = c.stream;
  struct Events {
    cudaEvent_t e[4] = {};
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  for (cudaEvent_t& x : ev.e) RIGW_CUDA_TRY(cudaEventCreate(&x));
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[0], s));

  // window tensor, transposed once: Mft[P][a * wq + b]
  DeviceBuffer b_in, b_mft, b_e, b_z;
  const double* min = pr.m_full;
  if (!on_dev) {
    RIGW_TRY(b_in.allocate(&c, size_t(ng) * ng * naux * 8, "g3w2 window tensor"));
    RIGW_CUDA_TRY(cudaMemcpyAsync(b_in.data(), pr.m_full, size_t(ng) * ng * naux * 8, cudaMemcpyHostToDevice, s));
    min = reinterpret_cast<const double*>(b_in.data());
  }
  RIGW_TRY(b_mft.allocate(&c, size_t(naux) * ldm * 8, "g3w2 window tensor^T"));
  double* mft = reinterpret_cast<double*>(b_mft.data());
  RIGW_CUDA_TRY(cudaMemsetAsync(mft, 0, size_t(naux) * ldm * 8, s));
  sox_transpose_kernel<<<dim3(unsigned(((long long)ng * ng + 31) / 32), unsigned((naux + 31) / 32)), dim3(32, 8), 0,
                         s>>>(min, (long long)ng * ng, naux, TransposeMap{ng, wq, ng, 0, ng, 0}, mft, ldm);
  RIGW_CUDA_TRY(cudaGetLastError());
  int launches = 1;
  RIGW_TRY(b_e.allocate(&c, size_t(ng) * 8, "g3w2 energies"));
  RIGW_TRY(b_z.allocate(&c, size_t(nz) * 16, "g3w2 omega_calc"));
  RIGW_CUDA_TRY(cudaMemcpyAsync(b_e.data(), pr.energy, size_t(ng) * 8, cudaMemcpyDefault, s));
  RIGW_CUDA_TRY(cudaMemcpyAsync(b_z.data(), pr.omega_calc, size_t(nz) * 16, cudaMemcpyDefault, s));
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[1], s));

  DeviceBuffer b_wt, b_x, b_gn, b_gp, b_part, b_out, b_iw;
  RIGW_TRY(b_wt.allocate(&c, size_t(nwp) * npad * npad * 8, "g3w2 W~"));
  RIGW_TRY(b_x.allocate(&c, size_t(nwp) * naux_e * wq * 8, "g3w2 X"));
  RIGW_TRY(b_gn.allocate(&c, size_t(nwp) * sk * 8, "g3w2 Gn"));
  RIGW_TRY(b_gp.allocate(&c, size_t(nwp) * sk * 8, "g3w2 Gp"));
  RIGW_TRY(b_part.allocate(&c, size_t(nwp) * nwp * nz * 16, "g3w2 partial sums"));
  double* wt = reinterpret_cast<double*>(b_wt.data());
  double* dx = reinterpret_cast<double*>(b_x.data());
  double* gn = reinterpret_cast<double*>(b_gn.data());
  double* gp = reinterpret_cast<double*>(b_gp.data());
  double* out = sigma;
  if (!on_dev) {
    RIGW_TRY(b_out.allocate(&c, size_t(nsig) * nz * 16, "g3w2 sigma"));
    out = reinterpret_cast<double*>(b_out.data());
  }
  // W~_k = Y_k^T Y_k - 1 for every frequency (Y_k = U_k^-T, the identity part of the resident solve)
  std::vector<GemmItem> iw;
  for (int k = 0; k < nwp; ++k) {
    const double* y = pd.rhs + size_t(k) * npad * pd.ldb;
    for (int i0 = 0; i0 < npad; i0 += 128)
      for (int j0 = 0; j0 < npad; j0 += 128) {
        GemmItem g{};
        g.A = y + i0;
        g.lda = pd.ldb;
        g.B = y + j0;
        g.ldb = pd.ldb;
        g.C = wt + size_t(k) * npad * npad + size_t(i0) * npad + j0;
        g.ldc = npad;
        g.m = std::min(128, npad - i0);
        g.n = std::min(128, npad - j0);
        g.k = npad;
        g.flags = kSubIdentity;
        g.diag = i0 - j0;
        g.alpha = 1.0;
        iw.push_back(g);
      }
  }
  RIGW_TRY(upload_items(c, &b_iw, iw, "g3w2 W~ items"));
  launch_dgemm_128x128(reinterpret_cast<const GemmItem*>(b_iw.data()), int(iw.size()), 1, s);
  RIGW_CUDA_TRY(cudaGetLastError());
  ++launches;
  if (smem > 48 * 1024)
    RIGW_CUDA_TRY(cudaFuncSetAttribute(g3w2_contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  for (int ml = 0; ml < nsig; ++ml) {
    const long long colp = (long long)(pr.sig_first + ml) * wq;   // columns of M(p, .) in Mft
    std::vector<GemmItem> ix, ig;
    for (int k = 0; k < nwp; ++k) {
      double* xk = dx + size_t(k) * naux_e * wq;
      // X_k[Q][u] = sum_P W~_k[P][Q] M(p, u, P)
      for (int q0 = 0; q0 < naux_e; q0 += 128)
        for (int u0 = 0; u0 < wq; u0 += 128) {
          GemmItem g{};
          g.A = wt + size_t(k) * npad * npad + q0;
          g.lda = npad;
          g.B = mft + colp + u0;
          g.ldb = int(ldm);
          g.C = xk + size_t(q0) * wq + u0;
          g.ldc = wq;
          g.m = std::min(128, naux_e - q0);
          g.n = std::min(128, wq - u0);
          g.k = naux;
          g.alpha = 1.0;
          ix.push_back(g);
        }
      for (int v = 0; v < ng; ++v)
        for (int w0 = 0; w0 < wq; w0 += 64)
          for (int u0 = 0; u0 < wq; u0 += 128) {
            GemmItem g{};
            g.m = std::min(64, wq - w0);
            g.n = std::min(128, wq - u0);
            g.k = naux;
            g.alpha = 1.0;
            g.ldc = wq;
            // Gn_k[v][w][u] = sum_Q M(v, w, Q) X_k[Q][u]
            g.A = mft + (long long)v * wq + w0;
            g.lda = int(ldm);
            g.B = xk + u0;
            g.ldb = wq;
            g.C = gn + size_t(k) * sk + (size_t(v) * wq + w0) * wq + u0;
            ig.push_back(g);
            // Gp_k[v][w][u] = sum_Q X_k[Q][w] M(v, u, Q)
            g.A = xk + w0;
            g.lda = wq;
            g.B = mft + (long long)v * wq + u0;
            g.ldb = int(ldm);
            g.C = gp + size_t(k) * sk + (size_t(v) * wq + w0) * wq + u0;
            ig.push_back(g);
          }
    }
    DeviceBuffer b_ix, b_ig;
    RIGW_TRY(upload_items(c, &b_ix, ix, "g3w2 X items"));
    RIGW_TRY(upload_items(c, &b_ig, ig, "g3w2 G items"));
    launch_dgemm_128x128(reinterpret_cast<const GemmItem*>(b_ix.data()), int(ix.size()), 1, s);
    launch_dgemm_64x128(reinterpret_cast<const GemmItem*>(b_ig.data()), int(ig.size()), 1, s);
    RIGW_CUDA_TRY(cudaGetLastError());
    G3w2Args a{gn, gp, sk, ng, wq, reinterpret_cast<const double*>(b_e.data()), pd.omega, pd.weight, nwp,
               reinterpret_cast<const double*>(b_z.data()), nz, reinterpret_cast<double*>(b_part.data())};
    g3w2_contract_kernel<<<dim3(unsigned(nwp * nwp), unsigned((nz + kG3Z - 1) / kG3Z)), kSosexThreads, smem, s>>>(a);
    g3w2_reduce_kernel<<<nz, kSosexThreads, 0, s>>>(reinterpret_cast<const double*>(b_part.data()), nwp * nwp, nz,
                                                     out + size_t(ml) * nz * 2);
    RIGW_CUDA_TRY(cudaGetLastError());
    launches += 4;
    RIGW_CUDA_TRY(cudaStreamSynchronize(s));   // the item buffers of this state are released below
  }
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[2], s));
  if (!on_dev) RIGW_CUDA_TRY(cudaMemcpyAsync(sigma, out, size_t(nsig) * nz * 16, cudaMemcpyDeviceToHost, s));
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[3], s));
  RIGW_CUDA_TRY(cudaEventSynchronize(ev.e[3]));
  float t01 = 0.0f, t12 = 0.0f, t23 = 0.0f;
  cudaEventElapsedTime(&t01, ev.e[0], ev.e[1]);
  cudaEventElapsedTime(&t12, ev.e[1], ev.e[2]);
  cudaEventElapsedTime(&t23, ev.e[2], ev.e[3]);
  rigw_stats st{};
  st.stage_ms[0] = t01;   // upload and transpose of the window tensor
  st.stage_ms[1] = t12;   // W~, X, Gn, Gp products and the frequency-pair contractions
  st.stage_ms[3] = t23;   // download
  st.total_ms = double(t01) + t12 + t23;
  st.kernel_launches = launches;
  st.chunks = nsig;
  st.waves = 1;
  st.device_bytes_in_use = c.in_use;
  st.device_bytes_peak = c.peak;
  c.last_stats = st;
  return Status::ok();
}

}  // namespace rigw
