// Contour-deformation G0W0 self-energy on the device (gw_selfenergy_contour,
// src/m_gw_selfenergy_grid.f90:342-551) for one spin channel.
//
//   chi0(w) = M^T F(w) M, F_t = REAL(2 docc de / (w^2 - de^2))   (DMMA, lower tiles, mirrored)
//           at nomega_imag Gauss-Legendre imaginary frequencies and nomega_real
//           real frequencies 0 .. de_max                          (src/m_spectral_function.f90:779-921)
//   chi0(w) = V diag(lambda) V^T                                  (block Jacobi, eigh_jacobi.cu)
//   g_k = lambda_k / (1 - lambda_k), dropped where |g_k| <= 1e-3   (the low-rank W)
//   v(w, m, p) = sum_k g_k (V_k . M_mp)^2                         (DMMA Z = V^T M^T, then a weighted
//                                                                   column sum of squares)
//   Sigma_m(x_j) = imaginary-axis integral over the v(i w) + residues of the
//                  occupied and empty states with v at the real frequency
//                  closest to |de| (no interpolation, :440-538)
//   QP: linearized and graphical on that real grid (qp_tools.cuh).
//
// The auxiliary dimension is padded with zeros to a multiple of 64 (the block
// size of the eigensolver); the padded rows and columns stay decoupled and give
// zero eigenvalues, which the low-rank filter drops.
#include <algorithm>
#include <cmath>
#include <vector>

#include "engine.cuh"
#include "qp_tools.cuh"

namespace rigw {
namespace {

constexpr double kTolLowEigval = 1.0e-3;   // TOL_LOW_EIGVAL, src/m_spectral_function.f90:783
constexpr double kPi = 3.14159265358979323;

enum ContourErr : int {
  kCErrRange = 2,       // a residue asked for a real frequency outside 0 .. de_max
  kCErrNonFinite = 4,   // non-finite QP energy
};

inline long long round_up(long long v, long long a) { return (v + a - 1) / a * a; }

// F[w][t] = REAL(2 docc de / (omega_w^2 - de^2)) (src/m_spectral_function.f90:861-872);
// om2[w] is the real part of omega_w^2 (-y^2 on the imaginary axis, x^2 on the real one).
__global__ void contour_factor_kernel(const double* __restrict__ eo, const double* __restrict__ ev,
                                      const double* __restrict__ oo, const double* __restrict__ ov, int no, int nv,
                                      int ntp, const double* __restrict__ om2, double* __restrict__ f) {
  const int w = blockIdx.y;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntp; t += gridDim.x * blockDim.x) {
    double v = 0.0;
    if (t < no * nv) {
      const int i = t / nv, a = t % nv;
      const double docc = oo[i] - ov[a];
      const double de = ev[a] - eo[i];
      v = 2.0 * docc * de / (om2[w] - de * de);
    }
    f[size_t(w) * ntp + t] = v;
  }
}

// dst[c][r] = src[r][c] for r < rows, c < cols (dst rows are ldd apart).
__global__ void contour_transpose_kernel(const double* __restrict__ src, int rows, int cols,
                                         double* __restrict__ dst, int ldd) {
  __shared__ double t[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[y][threadIdx.x] = src[size_t(r) * cols + c];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    if (r < rows && c < cols) dst[size_t(c) * ldd + r] = t[threadIdx.x][y];
  }
}

// Copy the strict lower triangle of each n x n matrix (blockIdx.z) to the upper one.
__global__ void contour_mirror_kernel(double* __restrict__ A, int n, long long sA) {
  const int rt = blockIdx.y, ct = blockIdx.x;   // destination tile (rows rt, columns ct), upper: rt <= ct
  if (rt > ct) return;
  double* a = A + size_t(blockIdx.z) * sA;
  __shared__ double t[32][33];
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = ct * 32 + y, c = rt * 32 + threadIdx.x;   // source: rows ct, columns rt
    t[y][threadIdx.x] = (r < n && c < n) ? a[size_t(r) * n + c] : 0.0;
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = rt * 32 + y, c = ct * 32 + threadIdx.x;
    if (r < n && c < n && r < c) a[size_t(r) * n + c] = t[threadIdx.x][y];
  }
}

// g[w][k] = lambda_k / (1 - lambda_k) where |.| > 1e-3, else 0 (src/m_spectral_function.f90:898-913);
// rank[w] counts the kept eigenpairs.
__global__ void contour_lowrank_kernel(const double* __restrict__ A, int n, long long sA, double* __restrict__ g,
                                       int* __restrict__ rank) {
  const int w = blockIdx.x;
  const double* a = A + size_t(w) * sA;
  int kept = 0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double lam = a[size_t(k) * n + k];
    double x = lam / (1.0 - lam);
    if (!(fabs(x) > kTolLowEigval)) x = 0.0;
    else ++kept;
    g[size_t(w) * n + k] = x;
  }
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  if (kept) atomicAdd(&cnt, kept);
  __syncthreads();
  if (threadIdx.x == 0) rank[w] = cnt;
}

// v[w][col] = sum_k g[w][k] Z[w][k][col]^2 for col < ncols (Z rows are ncp apart).
__global__ void contour_vchiv_kernel(const double* __restrict__ Z, const double* __restrict__ g, int n, int ncp,
                                     int ncols, double* __restrict__ v) {
  const int w = blockIdx.y;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncols) return;
  const double* z = Z + size_t(w) * n * ncp + col;
  const double* gw = g + size_t(w) * n;
  double s = 0.0;
  for (int k = 0; k < n; ++k) {
    const double gk = gw[k];
    if (gk == 0.0) continue;
    const double x = z[size_t(k) * ncp];
    s += x * x * gk;
  }
  v[size_t(w) * ncp + col] = s;
}

struct ContourArgs {
  const double* v;      // [nimag + nreal][ncp], column m * np + p
  const double* ep;     // [np]
  const double* e0;     // [nsig] se%energy0
  const double* eq;     // [nsig] energies of the QP equation
  const double* xc;     // [nsig] or nullptr
  const double* y;      // [nimag] imaginary frequencies
  const double* wq;     // [nimag] quadrature weights
  const double* omr;    // [nreal] real frequencies
  double* sigma;        // [nsig][2h+1][2]
  double* qp;           // [nsig][4]
  int* status;
  int np, nsig, nimag, nreal, ncp, h, p_occ_end, p_empty_begin;
  double step, eta;
};

// First closest real frequency (MINLOC), src/m_spectral_function.f90:925-950.
RIGW_DEVICE_INLINE int nearest_real(const double* omr, int nreal, double w, int* status) {
  if (w > omr[nreal - 1] || w < omr[0]) atomicOr(status, kCErrRange);
  int best = 0;
  double d = fabs(omr[0] - w);
  for (int k = 1; k < nreal; ++k) {
    const double dk = fabs(omr[k] - w);
    if (dk < d) {
      d = dk;
      best = k;
    }
  }
  return best;
}

// Sigma_m on its real grid (src/m_gw_selfenergy_grid.f90:440-538): one block per state m.
__global__ void contour_sigma_kernel(ContourArgs a) {
  const int m = blockIdx.x;
  const int nreal_sig = 2 * a.h + 1;
  const double e0 = a.e0[m];
  for (int j = threadIdx.x; j < nreal_sig; j += blockDim.x) {
    const double x0 = e0 + a.step * (j - a.h);   // se%energy0 + se%omega
    double sum = 0.0;
    for (int iw = 0; iw < a.nimag; ++iw) {
      const double y = a.y[iw], wq = a.wq[iw];
      const double* vw = a.v + size_t(iw) * a.ncp + size_t(m) * a.np;
      for (int p = 0; p < a.np; ++p) {
        const double x = x0 - a.ep[p];
        if (!(fabs(x) > a.eta)) continue;
        // 1/(x + i y) + 1/(x - i y)
        sum -= wq * (2.0 * x / (x * x + y * y)) * vw[p] / (2.0 * kPi);
      }
    }
    for (int p = 0; p < a.p_occ_end; ++p) {   // occupied states: poles in the first quadrant
      const double de = a.ep[p] - x0;
      if (de < -a.eta) continue;
      const int k = nearest_real(a.omr, a.nreal, fabs(de), a.status);
      const double fac = fabs(de) < a.eta ? 0.5 : 1.0;
      sum -= a.v[size_t(a.nimag + k) * a.ncp + size_t(m) * a.np + p] * fac;
    }
    for (int p = a.p_empty_begin; p < a.np; ++p) {   // empty states: poles in the third quadrant
      const double de = x0 - a.ep[p];
      if (de < -a.eta) continue;
      const int k = nearest_real(a.omr, a.nreal, fabs(de), a.status);
      const double fac = fabs(de) < a.eta ? 0.5 : 1.0;
      sum += a.v[size_t(a.nimag + k) * a.ncp + size_t(m) * a.np + p] * fac;
    }
    double* out = a.sigma + (size_t(m) * nreal_sig + j) * 2;
    out[0] = sum;
    out[1] = 0.0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double* q = a.qp + 4 * m;
    qp_on_real_grid(a.sigma + size_t(m) * nreal_sig * 2, a.h, 0.0, a.step, e0, a.eq[m], a.xc ? a.xc[m] : 0.0, q);
    if (!isfinite(q[0]) || !isfinite(q[1])) atomicOr(a.status, kCErrNonFinite);
  }
}

}  // namespace

Status gw_selfenergy_contour(Context& c, const rigw_contour_problem& pr, rigw_contour_result& res) {
  const int naux = pr.naux, no = pr.nocc_w, nv = pr.nvirt_w, nimag = pr.nomega_imag, nreal = pr.nomega_real;
  const int np = pr.nstate_p, nsig = pr.nsig;
  if (naux <= 0 || no <= 0 || nv <= 0 || nimag < 1 || nreal < 2 || np <= 0 || nsig <= 0 || pr.nomega_sigma < 1 ||
      !(pr.step_sigma > 0.0) || !(pr.eta >= 0.0) || !pr.m_ia || !pr.m_pm || !pr.e_occ_w || !pr.e_virt_w ||
      !pr.occ_occ_w || !pr.occ_virt_w || !pr.energy_p || !pr.energy0 || pr.p_occ_end < 0 || pr.p_occ_end > np ||
      pr.p_empty_begin < 0 || pr.p_empty_begin > np)
    return Status::fail(RIGW_ERR_ARG, "gw_selfenergy_contour: invalid arguments");
  NvtxRange range("GW self-energy (contour deformation)");
  const bool on_dev = (pr.flags & RIGW_PROBLEM_DEVICE_POINTERS) != 0;
  const int h = pr.nomega_sigma / 2, nrs = 2 * h + 1;
  const int nw = nimag + nreal;
  const long long npad = round_up(naux, 64), ntrans = (long long)no * nv, ntp = round_up(ntrans, 2);
  const long long ncols = (long long)nsig * np, ncp = round_up(ncols, 2);
  if (npad * npad >= (1LL << 31) || ntp >= (1LL << 31) || npad * ncp >= (1LL << 31) || npad > 16384)
    return Status::fail(RIGW_ERR_ARG, "gw_selfenergy_contour: dimensions beyond the supported range");

  // largest real frequency of the residues (:390-414)
  double de_max = 0.0;
  for (int m = 0; m < nsig; ++m) {
    for (int p = 0; p < pr.p_empty_begin; ++p)
      for (int j = -h; j <= h; ++j) {
        const double de = pr.energy_p[p] - (pr.energy0[m] + pr.step_sigma * j);
        if (de < -pr.eta) continue;
        de_max = std::max(de_max, de);
      }
    for (int p = pr.p_occ_end; p < np; ++p)
      for (int j = -h; j <= h; ++j) {
        const double de = pr.energy0[m] + pr.step_sigma * j - pr.energy_p[p];
        if (de < -pr.eta) continue;
        de_max = std::max(de_max, de);
      }
  }
  std::vector<double> y(nimag), wq(nimag), omr(nreal), om2(nw);
  imag_grid(nimag, y.data(), wq.data());
  for (int k = 0; k < nreal; ++k) omr[k] = double(k) / double(nreal - 1) * de_max;   // REAL_LINEAR (:308-316)
  for (int k = 0; k < nimag; ++k) om2[k] = -(y[k] * y[k]);
  for (int k = 0; k < nreal; ++k) om2[nimag + k] = omr[k] * omr[k];

  cudaStream_t s = c.stream;
  struct Events {
    cudaEvent_t e[5] = {};
    ~Events() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } ev;
  for (cudaEvent_t& x : ev.e) RIGW_CUDA_TRY(cudaEventCreate(&x));
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[0], s));

  DeviceBuffer b_mt, b_mT, b_mpm, b_f, b_chi, b_v, b_g, b_z, b_vc, b_small, b_sig, b_items, b_status;
  RIGW_TRY(b_mt.allocate(&c, size_t(ntp) * npad * 8, "contour M (transition-major)"));
  RIGW_TRY(b_mT.allocate(&c, size_t(npad) * ncp * 8, "contour M_sigma^T"));
  RIGW_TRY(b_f.allocate(&c, size_t(nw) * ntp * 8, "contour chi0 factors"));
  RIGW_TRY(b_chi.allocate(&c, size_t(nw) * npad * npad * 8, "contour chi0 / eigenvalues"));
  RIGW_TRY(b_v.allocate(&c, size_t(nw) * npad * npad * 8, "contour eigenvectors"));
  RIGW_TRY(b_g.allocate(&c, size_t(nw) * npad * 8, "contour low-rank weights"));
  RIGW_TRY(b_z.allocate(&c, size_t(nw) * npad * ncp * 8, "contour V^T M"));
  RIGW_TRY(b_vc.allocate(&c, size_t(nw) * ncp * 8, "contour v chi v"));
  const size_t nsmall = size_t(2 * no + 2 * nv + np + 3 * nsig + 2 * nimag + nreal + nw);
  RIGW_TRY(b_small.allocate(&c, nsmall * 8, "contour energies and grids"));
  RIGW_TRY(b_sig.allocate(&c, size_t(nsig) * (nrs * 2 + 4) * 8, "contour sigma and QP"));
  RIGW_TRY(b_status.allocate(&c, size_t(nw + 1) * sizeof(int), "contour status and ranks"));
  double* mt = reinterpret_cast<double*>(b_mt.data());
  double* mT = reinterpret_cast<double*>(b_mT.data());
  double* f = reinterpret_cast<double*>(b_f.data());
  double* chi = reinterpret_cast<double*>(b_chi.data());
  double* vv = reinterpret_cast<double*>(b_v.data());
  double* g = reinterpret_cast<double*>(b_g.data());
  double* z = reinterpret_cast<double*>(b_z.data());
  double* vc = reinterpret_cast<double*>(b_vc.data());
  double* sm = reinterpret_cast<double*>(b_small.data());
  double* sig = reinterpret_cast<double*>(b_sig.data());
  double* qp = sig + size_t(nsig) * nrs * 2;
  int* status = reinterpret_cast<int*>(b_status.data());
  int* rank = status + 1;
  double *d_eo = sm, *d_ev = d_eo + no, *d_oo = d_ev + nv, *d_ov = d_oo + no, *d_ep = d_ov + nv;
  double *d_e0 = d_ep + np, *d_eq = d_e0 + nsig, *d_xc = d_eq + nsig, *d_y = d_xc + nsig;
  double *d_wq = d_y + nimag, *d_omr = d_wq + nimag;
  double* d_om2 = d_omr + nreal;

  // inputs
  std::vector<double> small(nsmall, 0.0);
  std::copy(pr.e_occ_w, pr.e_occ_w + no, small.begin());
  std::copy(pr.e_virt_w, pr.e_virt_w + nv, small.begin() + no);
  std::copy(pr.occ_occ_w, pr.occ_occ_w + no, small.begin() + no + nv);
  std::copy(pr.occ_virt_w, pr.occ_virt_w + nv, small.begin() + 2 * no + nv);
  std::copy(pr.energy_p, pr.energy_p + np, small.begin() + 2 * no + 2 * nv);
  std::copy(pr.energy0, pr.energy0 + nsig, small.begin() + (d_e0 - sm));
  const double* eq0 = pr.energy_qp0 ? pr.energy_qp0 : pr.energy0;
  std::copy(eq0, eq0 + nsig, small.begin() + (d_eq - sm));
  if (pr.exchange_m_vxc) std::copy(pr.exchange_m_vxc, pr.exchange_m_vxc + nsig, small.begin() + (d_xc - sm));
  std::copy(y.begin(), y.end(), small.begin() + (d_y - sm));
  std::copy(wq.begin(), wq.end(), small.begin() + (d_wq - sm));
  std::copy(omr.begin(), omr.end(), small.begin() + (d_omr - sm));
  std::copy(om2.begin(), om2.end(), small.begin() + (d_om2 - sm));
  RIGW_CUDA_TRY(cudaMemcpyAsync(sm, small.data(), nsmall * 8, cudaMemcpyHostToDevice, s));
  RIGW_CUDA_TRY(cudaMemsetAsync(status, 0, size_t(nw + 1) * sizeof(int), s));
  // the host tensors go up contiguous (one copy each); the pitched copy into the
  // padded layout runs device to device
  const double* mia = pr.m_ia;
  const double* mpm = pr.m_pm;
  if (!on_dev) {
    RIGW_TRY(b_mpm.allocate(&c, size_t(ncols + ntrans) * naux * 8, "contour M uploads"));
    double* up = reinterpret_cast<double*>(b_mpm.data());
    RIGW_CUDA_TRY(cudaMemcpyAsync(up, pr.m_pm, size_t(ncols) * naux * 8, cudaMemcpyHostToDevice, s));
    RIGW_CUDA_TRY(cudaMemcpyAsync(up + size_t(ncols) * naux, pr.m_ia, size_t(ntrans) * naux * 8,
                                  cudaMemcpyHostToDevice, s));
    mpm = up;
    mia = up + size_t(ncols) * naux;
  }
  RIGW_CUDA_TRY(cudaMemsetAsync(mt, 0, size_t(ntp) * npad * 8, s));
  RIGW_CUDA_TRY(cudaMemcpy2DAsync(mt, size_t(npad) * 8, mia, size_t(naux) * 8, size_t(naux) * 8, size_t(ntrans),
                                  cudaMemcpyDeviceToDevice, s));
  RIGW_CUDA_TRY(cudaMemsetAsync(mT, 0, size_t(npad) * ncp * 8, s));
  int launches = 0;
  contour_transpose_kernel<<<dim3(unsigned((naux + 31) / 32), unsigned((ncols + 31) / 32)), dim3(32, 8), 0, s>>>(
      mpm, int(ncols), naux, mT, int(ncp));
  contour_factor_kernel<<<dim3(unsigned(std::min<long long>((ntp + 255) / 256, 1024)), unsigned(nw)), 256, 0, s>>>(
      d_eo, d_ev, d_oo, d_ov, no, nv, int(ntp), d_om2, f);
  RIGW_CUDA_TRY(cudaGetLastError());
  launches += 2;
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[1], s));

  // chi0: lower 128 x 128 tiles of every frequency, then mirrored
  std::vector<GemmItem> items;
  for (long long i0 = 0; i0 < npad; i0 += 128)
    for (long long j0 = 0; j0 <= i0; j0 += 128) {
      GemmItem it{};
      it.A = mt + i0;
      it.lda = int(npad);
      it.B = mt + j0;
      it.ldb = int(npad);
      it.C = chi + i0 * npad + j0;
      it.ldc = int(npad);
      it.kscale = f;
      it.m = int(std::min<long long>(128, npad - i0));
      it.n = int(std::min<long long>(128, npad - j0));
      it.k = int(ntp);
      it.alpha = 1.0;
      it.nw = nw;
      it.sC = npad * npad;
      it.sK = ntp;
      items.push_back(it);
    }
  const size_t nchi_items = items.size();
  for (long long i0 = 0; i0 < npad; i0 += 128)
    for (long long j0 = 0; j0 < ncp; j0 += 128) {
      GemmItem it{};
      it.A = vv + i0;   // A[k = aux][m = eigenpair] = V[aux][i0 + m]
      it.lda = int(npad);
      it.B = mT + j0;
      it.ldb = int(ncp);
      it.C = z + i0 * ncp + j0;
      it.ldc = int(ncp);
      it.m = int(std::min<long long>(128, npad - i0));
      it.n = int(std::min<long long>(128, ncp - j0));
      it.k = int(npad);
      it.alpha = 1.0;
      it.nw = nw;
      it.sA = npad * npad;
      it.sC = npad * ncp;
      items.push_back(it);
    }
  RIGW_TRY(b_items.allocate(&c, items.size() * sizeof(GemmItem), "contour gemm items"));
  const GemmItem* d_items = reinterpret_cast<const GemmItem*>(b_items.data());
  RIGW_CUDA_TRY(cudaMemcpyAsync(b_items.data(), items.data(), items.size() * sizeof(GemmItem),
                                cudaMemcpyHostToDevice, s));
  launch_dgemm_128x128(d_items, int(nchi_items), nw, s);
  const unsigned tiles = unsigned((npad + 31) / 32);
  contour_mirror_kernel<<<dim3(tiles, tiles, unsigned(nw)), dim3(32, 8), 0, s>>>(chi, int(npad), npad * npad);
  RIGW_CUDA_TRY(cudaGetLastError());
  launches += 2;
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[2], s));

  // eigenpairs, low-rank weights
  int sweeps = 0;
  RIGW_TRY(eigh_jacobi_batched(c, chi, vv, int(npad), nw, s, &sweeps, &launches));
  contour_lowrank_kernel<<<nw, 256, 0, s>>>(chi, int(npad), npad * npad, g, rank);
  RIGW_CUDA_TRY(cudaGetLastError());
  launches += 1;
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[3], s));

  // v(w, m, p), Sigma on the real grids, QP
  launch_dgemm_128x128(d_items + nchi_items, int(items.size() - nchi_items), nw, s);
  contour_vchiv_kernel<<<dim3(unsigned((ncols + 127) / 128), unsigned(nw)), 128, 0, s>>>(z, g, int(npad), int(ncp),
                                                                                       int(ncols), vc);
  ContourArgs a{};
  a.v = vc;
  a.ep = d_ep;
  a.e0 = d_e0;
  a.eq = d_eq;
  a.xc = pr.exchange_m_vxc ? d_xc : nullptr;
  a.y = d_y;
  a.wq = d_wq;
  a.omr = d_omr;
  a.sigma = sig;
  a.qp = qp;
  a.status = status;
  a.np = np;
  a.nsig = nsig;
  a.nimag = nimag;
  a.nreal = nreal;
  a.ncp = int(ncp);
  a.h = h;
  a.p_occ_end = pr.p_occ_end;
  a.p_empty_begin = pr.p_empty_begin;
  a.step = pr.step_sigma;
  a.eta = pr.eta;
  contour_sigma_kernel<<<nsig, 128, 0, s>>>(a);
  RIGW_CUDA_TRY(cudaGetLastError());
  launches += 3;
  std::vector<double> host_sig(size_t(nsig) * (nrs * 2 + 4));
  std::vector<int> host_status(nw + 1);
  RIGW_CUDA_TRY(cudaMemcpyAsync(host_sig.data(), sig, host_sig.size() * 8, cudaMemcpyDeviceToHost, s));
  RIGW_CUDA_TRY(cudaMemcpyAsync(host_status.data(), status, host_status.size() * sizeof(int), cudaMemcpyDeviceToHost,
                                s));
  RIGW_CUDA_TRY(cudaEventRecord(ev.e[4], s));
  RIGW_CUDA_TRY(cudaEventSynchronize(ev.e[4]));
  if (host_status[0] & kCErrRange)
    return Status::fail(RIGW_ERR_NUMERIC, "gw_selfenergy_contour: requested real frequency out of range");
  if (host_status[0] & kCErrNonFinite)
    return Status::fail(RIGW_ERR_NUMERIC, "gw_selfenergy_contour: non-finite QP energy");

  const double* hq = host_sig.data() + size_t(nsig) * nrs * 2;
  if (res.sigma) std::copy(host_sig.begin(), host_sig.begin() + size_t(nsig) * nrs * 2, res.sigma);
  for (int m = 0; m < nsig; ++m) {
    if (res.energy_qp_g) res.energy_qp_g[m] = hq[4 * m + 0];
    if (res.energy_qp_z) res.energy_qp_z[m] = hq[4 * m + 1];
    if (res.zz) res.zz[m] = hq[4 * m + 2];
  }
  if (res.rank) std::copy(host_status.begin() + 1, host_status.end(), res.rank);
  if (res.omega_real) std::copy(omr.begin(), omr.end(), res.omega_real);
  res.de_max = de_max;

  float t[4] = {0, 0, 0, 0}, total = 0.0f;
  for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&t[k], ev.e[k], ev.e[k + 1]);
  cudaEventElapsedTime(&total, ev.e[0], ev.e[4]);
  rigw_stats st{};
  for (int k = 0; k < 4; ++k) st.stage_ms[k] = t[k];   // inputs, chi0, eigensolver, v + Sigma + QP
  st.total_ms = total;
  st.kernel_launches = launches;
  st.chunks = 1;
  st.waves = 1;
  st.device_bytes_in_use = c.in_use;
  st.device_bytes_peak = c.peak;
  c.last_stats = st;
  return Status::ok();
}

}  // namespace rigw
