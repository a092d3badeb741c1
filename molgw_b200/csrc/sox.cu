// GW+SOX on the imaginary axis: the second-order screened exchange on the
// evaluation points, sox_selfenergy_imag_grid (src/m_g3w2_selfenergy.f90:2482-2591).
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

// dst[P][(r / group) * group_pad + r % group] = src[r][P]: rows of naux values
// become columns, each group of rows padded to an even width (zeros stay in the pad).
__global__ void sox_transpose_kernel(const double* __restrict__ src, long long nrows, int naux, long long group,
                                     long long group_pad, double* __restrict__ dst, long long ld_dst) {
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
    if (p < naux && r < nrows) dst[p * ld_dst + (r / group) * group_pad + r % group] = t[threadIdx.x][y];
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
    sox_transpose_kernel<<<dim3(unsigned((nov + 31) / 32), unsigned((naux + 31) / 32)), blk, 0, s>>>(
        mov, nov, naux, nov, novp, bt, novp);
    sox_transpose_kernel<<<dim3(unsigned(((long long)nsig * ng + 31) / 32), unsigned((naux + 31) / 32)), blk, 0,
                           s>>>(mpq, (long long)nsig * ng, naux, ng, ngp, at, lda);
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

}  // namespace rigw
