// GW density matrix from the imaginary axis (pt_density_matrix GW_IMAGINARY:
// gw_density_matrix_imag, src/m_mbpt_density_matrix.f90:491-640), one spin
// channel, from the resident W of rigw_polarizability_imag.
//
//   W~_k = Y_k^T Y_k - 1 = v^1/2 chi(i w_k) v^1/2      (DMMA, every frequency; Y_k = U_k^-T)
//   per Sigma state q:
//     X_k[Q][m] = sum_P W~_k[P][Q] M(q, m, P)        (DMMA, every frequency in one launch)
//     dm_contract_kernel, one warp per (p >= q, k), lanes over m:
//       v(m) = sum_Q M(p, m, Q) X_k[Q][m]
//       F(m) = sum_s w_s Re{ [1/(i s - e~_m + i w_k) + 1/(i s - e~_m - i w_k)]
//                            / ((i s - e~_p)(i s - e~_q)) }
//       partial[p][k] = w_k sum_m v(m) F(m)
//   P_pq = -spin_fact 2/(2 pi)^2 sum_k partial[p][k]    (fixed order over k; P_qp = P_pq)
// e~ = e - mu; the s grid is Gauss-Legendre on [0, 1) mapped with alpha = beta = 1.
#include <cmath>
#include <vector>

#include "engine.cuh"

namespace rigw {
namespace {

constexpr int kDmThreads = 128;
constexpr int kDmMaxS = 256;   // points of the density-matrix frequency grid

// Mft[P][a * wq + b] = M[a][b][P] (zero padded columns stay as set by the caller).
__global__ void dm_transpose_kernel(const double* __restrict__ m, int ng, int naux, int wq, long long ldm,
                                    double* __restrict__ mft) {
  __shared__ double t[32][33];
  const long long r0 = (long long)blockIdx.x * 32;   // rows (a, b) of M
  const int c0 = blockIdx.y * 32;                    // auxiliary index
  const long long nrows = (long long)ng * ng;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const long long r = r0 + y;
    const int c = c0 + threadIdx.x;
    if (r < nrows && c < naux) t[y][threadIdx.x] = m[r * naux + c];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y;
    const long long r = r0 + threadIdx.x;
    if (r < nrows && c < naux) {
      const long long a = r / ng, b = r % ng;
      mft[(long long)c * ldm + a * wq + b] = t[threadIdx.x][y];
    }
  }
}

struct DmArgs {
  const double* mft;    // [naux][ldm]
  const double* x;      // [nw][naux_e][wq]
  const double* e;      // [ng] window energies
  const double* om;     // [nw] imaginary frequencies of W
  const double* wt;     // [nw] their weights
  const double* oms;    // [ns] density-matrix grid
  const double* ws;     // [ns]
  double* partial;      // [ng][nw]
  long long ldm;
  int ng, wq, naux, naux_e, nw, ns, q, pend;
  double mu;
};

__global__ void __launch_bounds__(kDmThreads) dm_contract_kernel(DmArgs a) {
  const int warp = int((blockIdx.x * (unsigned)kDmThreads + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  const int np = a.pend - a.q;
  if (warp >= np * a.nw) return;
  const int p = a.q + warp % np, k = warp / np;
  const double y = __ldg(a.om + k);
  const double ep = __ldg(a.e + p) - a.mu, eq = __ldg(a.e + a.q) - a.mu;
  const double* xk = a.x + (size_t)k * a.naux_e * a.wq;
  double acc = 0.0;
  for (int m = lane; m < a.ng; m += 32) {
    double v = 0.0;
    const double* mp = a.mft + (long long)p * a.wq + m;
    for (int Q = 0; Q < a.naux; ++Q) v += mp[(long long)Q * a.ldm] * xk[(size_t)Q * a.wq + m];
    const double em = __ldg(a.e + m) - a.mu;
    double f = 0.0;
    for (int s = 0; s < a.ns; ++s) {
      const double z = __ldg(a.oms + s);
      // 1/(-em + i(z + y)) + 1/(-em + i(z - y))
      const double d1 = em * em + (z + y) * (z + y), d2 = em * em + (z - y) * (z - y);
      const double ar = -em / d1 - em / d2;
      const double ai = -(z + y) / d1 - (z - y) / d2;
      // b = (-ep + i z)(-eq + i z)
      const double br = ep * eq - z * z, bi = -z * (ep + eq);
      f += __ldg(a.ws + s) * (ar * br + ai * bi) / (br * br + bi * bi);
    }
    acc += v * f;
  }
  acc = warp_sum(acc);
  if (lane == 0) a.partial[(size_t)p * a.nw + k] = __ldg(a.wt + k) * acc;
}

// P[p][q] = P[q][p] = factor * sum_k partial[p][k] for the p >= q of state q.
__global__ void dm_reduce_kernel(const double* __restrict__ partial, int nw, int q, int pend, double factor,
                                 double* __restrict__ pm, int ng) {
  const int p = q + blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pend) return;
  double s = 0.0;
  for (int k = 0; k < nw; ++k) s += partial[(size_t)p * nw + k];
  pm[(size_t)p * ng + q] = factor * s;
  pm[(size_t)q * ng + p] = factor * s;
}

}  // namespace

Status gw_density_matrix_imag(Context& c, const Wpol& w, const rigw_dm_problem& pr, double* p_matrix) {
  const int ng = pr.nstate, naux = pr.naux, nsig = pr.nsig, ns = pr.nomega_sigma;
  if (ng <= 0 || naux <= 0 || nsig <= 0 || ns <= 0 || ns > kDmMaxS || !pr.m_full || !pr.energy || !p_matrix ||
      pr.sig_first < 0 || pr.sig_first + nsig > ng)
    return Status::fail(RIGW_ERR_ARG, "gw_density_matrix_imag: invalid arguments");
  const ProbDev& pd = w.plan->problems()[0].dev;
  if (naux != pd.naux)
    return Status::fail(RIGW_ERR_ARG, "gw_density_matrix_imag: naux differs from the polarizability");
  if (!pd.want_identity)
    return Status::fail(RIGW_ERR_UNSUPPORTED,
                        "gw_density_matrix_imag: the polarizability was solved without W (QP-only)");
  const int wq = ng + (ng & 1), naux_e = naux + (naux & 1), npad = pd.npad, nwp = pd.nomega;
  const long long ldm = (long long)wq * wq;
  if (ldm >= (1LL << 31)) return Status::fail(RIGW_ERR_ARG, "gw_density_matrix_imag: window too large");
  const size_t need = (size_t(nwp) * npad * npad + size_t(nwp) * naux_e * wq + size_t(naux) * ldm +
                       size_t(ng) * nwp + size_t(ng) * ng) * 8;
  if (c.budget > 0 && need > (c.budget > c.in_use ? c.budget - c.in_use : 0))
    return Status::fail(RIGW_ERR_NOMEM, "gw_density_matrix_imag: %zu bytes needed beyond the HBM budget", need);
  NvtxRange range("GW density matrix");
  const bool on_dev = (pr.flags & RIGW_PROBLEM_DEVICE_POINTERS) != 0;
  cudaStream_t s = c.stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  RIGW_CUDA_TRY(cudaEventCreate(&e0));
  RIGW_CUDA_TRY(cudaEventCreate(&e1));
  struct EvGuard {
    cudaEvent_t* a;
    cudaEvent_t* b;
    ~EvGuard() {
      cudaEventDestroy(*a);
      cudaEventDestroy(*b);
    }
  } guard{&e0, &e1};
  RIGW_CUDA_TRY(cudaEventRecord(e0, s));

  // density-matrix frequency grid: the map of imag_grid with beta = 1 instead of 2 (exact halving)
  std::vector<double> oms(ns), ws(ns);
  imag_grid(ns, oms.data(), ws.data());
  for (int i = 0; i < ns; ++i) {
    oms[i] *= 0.5;
    ws[i] *= 0.5;
  }
  DeviceBuffer b_in, b_mft, b_small, b_wt, b_x, b_part, b_pm, b_items;
  const double* min = pr.m_full;
  if (!on_dev) {
    RIGW_TRY(b_in.allocate(&c, size_t(ng) * ng * naux * 8, "dm window tensor"));
    RIGW_CUDA_TRY(cudaMemcpyAsync(b_in.data(), pr.m_full, size_t(ng) * ng * naux * 8, cudaMemcpyHostToDevice, s));
    min = reinterpret_cast<const double*>(b_in.data());
  }
  RIGW_TRY(b_mft.allocate(&c, size_t(naux) * ldm * 8, "dm window tensor^T"));
  double* mft = reinterpret_cast<double*>(b_mft.data());
  RIGW_CUDA_TRY(cudaMemsetAsync(mft, 0, size_t(naux) * ldm * 8, s));
  dm_transpose_kernel<<<dim3(unsigned(((long long)ng * ng + 31) / 32), unsigned((naux + 31) / 32)), dim3(32, 8), 0,
                        s>>>(min, ng, naux, wq, ldm, mft);
  RIGW_CUDA_TRY(cudaGetLastError());
  int launches = 1;
  std::vector<double> small(size_t(ng) + 2 * ns);
  std::copy(pr.energy, pr.energy + ng, small.begin());
  std::copy(oms.begin(), oms.end(), small.begin() + ng);
  std::copy(ws.begin(), ws.end(), small.begin() + ng + ns);
  RIGW_TRY(b_small.allocate(&c, small.size() * 8, "dm energies and grid"));
  double* d_small = reinterpret_cast<double*>(b_small.data());
  RIGW_CUDA_TRY(cudaMemcpyAsync(d_small, small.data(), small.size() * 8, cudaMemcpyHostToDevice, s));

  RIGW_TRY(b_wt.allocate(&c, size_t(nwp) * npad * npad * 8, "dm W~"));
  RIGW_TRY(b_x.allocate(&c, size_t(nwp) * naux_e * wq * 8, "dm X"));
  RIGW_TRY(b_part.allocate(&c, size_t(ng) * nwp * 8, "dm partial sums"));
  double* wt = reinterpret_cast<double*>(b_wt.data());
  double* dx = reinterpret_cast<double*>(b_x.data());
  double* part = reinterpret_cast<double*>(b_part.data());
  double* pm = p_matrix;
  if (!on_dev) {
    RIGW_TRY(b_pm.allocate(&c, size_t(ng) * ng * 8, "dm P"));
    pm = reinterpret_cast<double*>(b_pm.data());
  }
  RIGW_CUDA_TRY(cudaMemsetAsync(pm, 0, size_t(ng) * ng * 8, s));
  RIGW_CUDA_TRY(cudaMemsetAsync(dx, 0, size_t(nwp) * naux_e * wq * 8, s));

  // item lists: W~ for every frequency, then X_k for one Sigma state (rebuilt per state)
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
  size_t nx = 0;
  for (int q0 = 0; q0 < naux_e; q0 += 128)
    for (int u0 = 0; u0 < wq; u0 += 128) ++nx;
  RIGW_TRY(b_items.allocate(&c, iw.size() * sizeof(GemmItem), "dm W~ items"));
  GemmItem* d_items = reinterpret_cast<GemmItem*>(b_items.data());
  RIGW_CUDA_TRY(cudaMemcpyAsync(d_items, iw.data(), iw.size() * sizeof(GemmItem), cudaMemcpyHostToDevice, s));
  launch_dgemm_128x128(d_items, int(iw.size()), 1, s);
  RIGW_CUDA_TRY(cudaGetLastError());
  ++launches;

  DmArgs a{};
  a.mft = mft;
  a.x = dx;
  a.e = d_small;
  a.om = pd.omega;
  a.wt = pd.weight;
  a.oms = d_small + ng;
  a.ws = d_small + ng + ns;
  a.partial = part;
  a.ldm = ldm;
  a.ng = ng;
  a.wq = wq;
  a.naux = naux;
  a.naux_e = naux_e;
  a.nw = nwp;
  a.ns = ns;
  a.mu = pr.mu;
  const double factor = -pr.spin_fact * 2.0 / ((2.0 * 3.14159265358979323) * (2.0 * 3.14159265358979323));
  // X_k[Q][u] = sum_P W~_k[P][Q] M(q, u, P), every frequency (grid y): one item list per state, uploaded once
  const int pend = pr.sig_first + nsig;
  std::vector<GemmItem> ix;
  ix.reserve(size_t(nsig) * nx);
  for (int q = pr.sig_first; q < pend; ++q)
    for (int q0 = 0; q0 < naux_e; q0 += 128)
      for (int u0 = 0; u0 < wq; u0 += 128) {
        GemmItem g{};
        g.A = wt + q0;
        g.lda = npad;
        g.B = mft + (long long)q * wq + u0;
        g.ldb = int(ldm);
        g.C = dx + size_t(q0) * wq + u0;
        g.ldc = wq;
        g.m = std::min(128, naux_e - q0);
        g.n = std::min(128, wq - u0);
        g.k = naux;
        g.alpha = 1.0;
        g.nw = nwp;
        g.sA = (long long)npad * npad;
        g.sC = (long long)naux_e * wq;
        ix.push_back(g);
      }
  DeviceBuffer b_xitems;
  RIGW_TRY(b_xitems.allocate(&c, ix.size() * sizeof(GemmItem), "dm X items"));
  GemmItem* d_xitems = reinterpret_cast<GemmItem*>(b_xitems.data());
  RIGW_CUDA_TRY(cudaMemcpyAsync(d_xitems, ix.data(), ix.size() * sizeof(GemmItem), cudaMemcpyHostToDevice, s));
  a.pend = pend;
  for (int q = pr.sig_first; q < pend; ++q) {
    launch_dgemm_128x128(d_xitems + size_t(q - pr.sig_first) * nx, int(nx), nwp, s);
    a.q = q;
    const long long nwarps = (long long)(pend - q) * nwp;
    dm_contract_kernel<<<unsigned((nwarps * 32 + kDmThreads - 1) / kDmThreads), kDmThreads, 0, s>>>(a);
    dm_reduce_kernel<<<(pend - q + 127) / 128, 128, 0, s>>>(part, nwp, q, pend, factor, pm, ng);
    RIGW_CUDA_TRY(cudaGetLastError());
    launches += 3;
  }
  if (!on_dev) RIGW_CUDA_TRY(cudaMemcpyAsync(p_matrix, pm, size_t(ng) * ng * 8, cudaMemcpyDeviceToHost, s));
  RIGW_CUDA_TRY(cudaEventRecord(e1, s));
  RIGW_CUDA_TRY(cudaEventSynchronize(e1));
  float total = 0.0f;
  cudaEventElapsedTime(&total, e0, e1);
  rigw_stats st{};
  st.stage_ms[3] = total;
  st.total_ms = total;
  st.kernel_launches = launches;
  st.chunks = nsig;
  st.waves = 1;
  st.device_bytes_in_use = c.in_use;
  st.device_bytes_peak = c.peak;
  c.last_stats = st;
  return Status::ok();
}

}  // namespace rigw
