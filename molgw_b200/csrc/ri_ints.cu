// RI Coulomb integrals on the device: (P|Q) over the auxiliary basis and (mu nu|P)
// over the orbital-basis pairs, then B(mu nu, P) = sum_Q (mu nu|Q) (Q|P)^-1/2 in the
// pair-packed layout the AO->MO transform reads (calculate_eri_2center /
// calculate_eri_3center_scalapack, src/m_eri_calculate.f90:1049-1262, 1584-1950).
//
// The integrals follow the McMurchie-Davidson scheme (Helgaker, Jorgensen, Olsen,
// "Molecular Electronic-Structure Theory", ch. 9): Hermite expansion coefficients
// E^{ij}_t of the Gaussian products and Hermite Coulomb integrals R_tuv from the
// Boys function.  A block is one (orbital shell pair, auxiliary shell) or one
// auxiliary shell pair.  The 3-center blocks come in three classes, launched
// together on three streams: up to 32 Cartesian components and 4 primitive
// triples on one warp per CTA, contracted blocks (>= 20 triples, <= 128
// components) on four warp teams per CTA that share the triples, the rest on
// 128 threads per CTA.  For every primitive pair/triple the E tables, the Boys
// values (one thread per order, from a table and its Taylor expansion) and the
// R table (level-by-level recursion in shared memory over the live (t, u, v)
// only, two tetrahedral arrays) are built once; the ket step and the bra step
// contract them into the Cartesian block, which is then transformed to pure
// functions (real solid harmonics) or normalized per component (CART) in shared
// memory and stored.  Shared memory is laid out per class for the angular
// momenta it holds.
//
// The metric: (P|Q) is diagonalized by the device eigensolver (eigh_jacobi.cu),
// eigenvalues <= 1e-6 are dropped (TOO_LOW_EIGENVAL, src/m_eri.f90:27) and
// (P|Q)^-1/2 = V[:, kept] / sqrt(lambda[kept]).  The kept eigenpairs are taken in
// the eigensolver's order; B is defined up to that orthogonal transformation of
// the auxiliary index, like the reference's (every product M M^T downstream is
// invariant to it).
#include <algorithm>
#include <cmath>
#include <vector>

#include "engine.cuh"

namespace rigw {
namespace {

constexpr int kRiLmax = 4;                                   // highest angular momentum of a shell
constexpr int kRiThreads = 128;
constexpr double kRiTooLowEigval = 1.0e-6;
// Boys table: F_m(T) at T_i = i * 0.1, i = 0..400, m = 0..19 (orders up to 3 kRiLmax
// plus the 7 derivatives of the Taylor expansion).  Beyond T = 40, F_0 = sqrt(pi/T)/2
// (erfc(sqrt(40)) < 1e-18) and the upward recursion.
constexpr int kBoysOrders = 3 * kRiLmax + 8;
constexpr int kBoysRows = 401;
constexpr double kBoysStep = 0.1;
constexpr double kBoysTmax = 40.0;
constexpr double kTwoPi52 = 34.98683665524972569;            // 2 pi^(5/2)

struct DevShell {
  double x, y, z;
  int l, nprim, p0, f0;   // angular momentum, primitives, first primitive, first function
};

struct RiArgs {
  const DevShell* sh;     // orbital shells
  const DevShell* ax;     // auxiliary shells
  const double* alpha;    // primitives of both bases
  const double* coeff;
  const double* trans;    // per l and basis: [nfun][ncart] transforms, at toff[l] (orbital), toff[5 + l] (aux)
  const int* toff;
  const int* shellpair;   // [nsp][2] orbital shell pairs (A >= B)
  const int* pairmap;     // [nbf][nbf] pair index or -1
  const double* boys;     // [kBoysRows][kBoysOrders]
  const int* tet;         // (t, u, v) of each tetrahedral index, packed t | u << 8 | v << 16
  double* out;            // 3-center: [naux][npair]; 2-center: [naux][naux]
  int nbf, naux, npair;
  int pure_orb, pure_aux;
  // shared-memory layout of the launch (doubles): two R arrays of ntet, the bra E
  // tables (entry (i, j, t) of an axis at i * ld_ei + j * ld_ej + t, axis stride
  // e_axis), the ket tables (i * ld_fk + t, axis stride f_axis), the Cartesian
  // block (nacc) and its transform scratch, which also holds the ket-contracted
  // Hermite integrals during the primitive loops, the scaled Boys values, 8 scalars,
  // the packed Cartesian exponents of each component (nacc ints)
  int ntet, ld_ei, ld_ej, e_axis, ld_fk, f_axis;
  int off_e, off_f, off_acc, off_tmp, off_boys, off_scal, off_code, smem_doubles;
};

RIGW_DEVICE_INLINE int ncart(int l) { return (l + 1) * (l + 2) / 2; }
RIGW_DEVICE_INLINE int nfun(int l, int pure) { return pure ? 2 * l + 1 : ncart(l); }

// Cartesian component c of shell l: nx from l down, nz from 0 up (the reference's order).
RIGW_DEVICE_INLINE void cart_comp(int l, int c, int& nx, int& ny, int& nz) {
  int k = 0;
  for (int x = l; x >= 0; --x)
    for (int z = 0; z <= l - x; ++z) {
      if (k == c) {
        nx = x;
        ny = l - x - z;
        nz = z;
        return;
      }
      ++k;
    }
  nx = ny = nz = 0;
}

// (-2 al)^m F_m(T) for one order m <= mmax, into F[m].  T < 40: the Taylor
// expansion about the nearest table point T_i (|T_i - T| <= 0.05), eight terms,
// F_m(T) = sum_k F_{m+k}(T_i) (T_i - T)^k / k! (dF_m/dT = -F_{m+1}; the first
// omitted term is below 1e-15 F_m).  T >= 40: thread m == 0 alone fills every
// order with F_0 = sqrt(pi/T)/2 and F_{m+1} = ((2m+1) F_m - e^-T) / (2T), stable
// there since (2m+1)/(2T) < 1.
__device__ __forceinline__ void boys_scaled(int m, int mmax, double al, double T, const double* __restrict__ tab,
                                            double* F) {
  if (T < kBoysTmax) {
    const int i = __double2int_rn(T * 10.0);
    const double d = i * kBoysStep - T;
    const double* r = tab + i * kBoysOrders + m;
    double v = __ldg(r + 7);
    v = __ldg(r + 6) + v * d * (1.0 / 7.0);
    v = __ldg(r + 5) + v * d * (1.0 / 6.0);
    v = __ldg(r + 4) + v * d * (1.0 / 5.0);
    v = __ldg(r + 3) + v * d * (1.0 / 4.0);
    v = __ldg(r + 2) + v * d * (1.0 / 3.0);
    v = __ldg(r + 1) + v * d * 0.5;
    v = __ldg(r) + v * d;
    double sc = 1.0;
    for (int k = 0; k < m; ++k) sc *= -2.0 * al;
    F[m] = sc * v;
    return;
  }
  if (m != 0) return;
  const double e = exp(-T), h = 0.5 / T;
  double f = 0.5 * sqrt(3.14159265358979323846 / T), sc = 1.0;
  for (int k = 0; k <= mmax; ++k) {
    F[k] = sc * f;
    f = ((2 * k + 1) * f - e) * h;
    sc *= -2.0 * al;
  }
}

// E^{ij}_t along one axis for i <= imax, j <= jmax (Q = A - B), into E[i * ld_i + j * ld_j + t].
__device__ __forceinline__ void hermite_e(int imax, int jmax, double a, double b, double qx, double* E, int ld_i,
                                          int ld_j) {
  const double p = a + b, mu = a * b / p;
  const double xpa = -b / p * qx, xpb = a / p * qx, h = 0.5 / p;
  E[0] = exp(-mu * qx * qx);
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j) {
      if (i == 0 && j == 0) continue;
      const int tp = i + j - 1;
      const double* Ep = i > 0 ? E + (i - 1) * ld_i + j * ld_j : E + i * ld_i + (j - 1) * ld_j;
      const double x = i > 0 ? xpa : xpb;
      for (int t = 0; t <= i + j; ++t) {
        double v = (t <= tp ? x * Ep[t] : 0.0) + (t + 1 <= tp ? (t + 1) * Ep[t + 1] : 0.0);
        if (t > 0) v += h * Ep[t - 1];
        E[i * ld_i + j * ld_j + t] = v;
      }
    }
}

// Tetrahedral index of (t, u, v): ordered by s = t + u + v, then t, then u.
RIGW_DEVICE_INLINE int tet(int t, int u, int v) {
  const int s = t + u + v;
  return s * (s + 1) * (s + 2) / 6 + t * (2 * s + 3 - t) / 2 + u;
}

// Barrier of a team of NT threads: one warp (a team inside a larger CTA) or the CTA.
template <int NT>
RIGW_DEVICE_INLINE void team_sync() {
  if constexpr (NT == 32)
    __syncwarp();
  else
    __syncthreads();
}

// R_tuv of order 0 for t + u + v <= L (tetrahedral), the whole team working level
// by level between two arrays; F[n] = (-2 al)^n F_n(T) = R^{(n)}_000, so F + L is
// level L.  Returns the array holding level 0 (F itself when L = 0).
template <int NT>
__device__ __forceinline__ const double* hermite_r(int L, double X, double Y, double Z, const double* F,
                                                   const int* __restrict__ code, double* R0, double* R1) {
  const int lane = threadIdx.x & (NT - 1);
  const double* cur = F + L;
  for (int n = L - 1; n >= 0; --n) {
    double* nxt = (n & 1) ? R1 : R0;
    const int lim = L - n;
    const int ntet = (lim + 1) * (lim + 2) * (lim + 3) / 6;   // (t, u, v) with t + u + v <= lim
    for (int idx = lane; idx < ntet; idx += NT) {
      const int c = __ldg(code + idx);
      const int t = c & 255, u = (c >> 8) & 255, v = c >> 16;
      double val;
      if (idx == 0) {
        val = F[n];
      } else if (t > 0) {
        val = X * cur[tet(t - 1, u, v)] + (t > 1 ? (t - 1) * cur[tet(t - 2, u, v)] : 0.0);
      } else if (u > 0) {
        val = Y * cur[tet(t, u - 1, v)] + (u > 1 ? (u - 1) * cur[tet(t, u - 2, v)] : 0.0);
      } else {
        val = Z * cur[tet(t, u, v - 1)] + (v > 1 ? (v - 1) * cur[tet(t, u, v - 2)] : 0.0);
      }
      nxt[idx] = val;
    }
    team_sync<NT>();
    cur = nxt;
  }
  return cur;
}

// Cartesian block of one shell triple (bra A, B; ket Q, a single function) or,
// with B == nullptr, one auxiliary pair (bra P as a single function, ket Q), into
// smem + off_acc, by a CTA of NT threads.  Per primitive triple, in one phase: the
// bra E tables (threads 0-2, for a new primitive pair), the ket tables (three
// threads from kKet, for a new ket primitive), the Boys values (one thread per
// order from kBoys, the first also publishing the prefactor and P - Q); then the
// R recursion, the ket step and the bra step.  The Cartesian exponents of every component are decoded once per block.
template <int NT>
__device__ __forceinline__ void shell_block(const RiArgs& g, const DevShell& A, const DevShell* B, const DevShell& Q,
                                            double* smem, int na, int nb, int nq, int tr0, int trstep) {
  constexpr int kKet = NT >= 64 ? 32 : 3;    // first of the three threads building the ket tables
  constexpr int kBoys = NT >= 128 ? 64 : 8;  // thread of Boys order 0 (orders up to 3 kRiLmax follow)
  static_assert(kBoys + 3 * kRiLmax < NT, "a thread per Boys order");
  double* R0 = smem;
  double* R1 = smem + g.ntet;
  double* E = smem + g.off_e;
  double* Fk = smem + g.off_f;
  double* acc = smem + g.off_acc;
  double* F = smem + g.off_boys;
  double* G = smem + g.off_tmp;     // ket-contracted Hermite integrals (the transform scratch until the end)
  double* sc = smem + g.off_scal;   // pref, X, Y, Z of the triple
  int* code = reinterpret_cast<int*>(smem + g.off_code);
  const double* alpha = g.alpha;
  const double* coeff = g.coeff;
  const int tid = threadIdx.x & (NT - 1);
  const int lb = B ? B->l : 0;
  const int nblk = na * nb * nq;
  for (int o = tid; o < nblk; o += NT) {
    acc[o] = 0.0;
    const int i = o / (nb * nq), j = (o / nq) % nb, k = o % nq;
    int ix, iy, iz, jx = 0, jy = 0, jz = 0, kx, ky, kz;
    cart_comp(A.l, i, ix, iy, iz);
    if (B) cart_comp(lb, j, jx, jy, jz);
    cart_comp(Q.l, k, kx, ky, kz);
    code[o] = ix | iy << 3 | iz << 6 | jx << 9 | jy << 12 | jz << 15 | kx << 18 | ky << 21 | kz << 24;
  }
  const int L = A.l + lb + Q.l;
  const int lab = A.l + lb, ntab = (lab + 1) * (lab + 2) * (lab + 3) / 6;
  const int pbn = B ? B->nprim : 1;
  const double bx = B ? B->x : A.x, by = B ? B->y : A.y, bz = B ? B->z : A.z;
  const int ntri = A.nprim * pbn * Q.nprim;
  int cur_pair = -1, cur_q = -1;   // primitive pair and ket primitive whose tables are in place
  for (int tr = tr0; tr < ntri; tr += trstep) {
    const int pq = tr % Q.nprim, pab = tr / Q.nprim, pb = pab % pbn, pa = pab / pbn;
    team_sync<NT>();   // the previous triple's tables, R and Hermite integrals are no longer read
    if (tid < 3) {
      if (pab != cur_pair) {
        const double a = alpha[A.p0 + pa], b = B ? alpha[B->p0 + pb] : 0.0;
        const double qx = tid == 0 ? A.x - bx : (tid == 1 ? A.y - by : A.z - bz);
        hermite_e(A.l, lb, a, b, qx, E + tid * g.e_axis, g.ld_ei, g.ld_ej);
      }
    } else if (tid >= kKet && tid < kKet + 3) {
      if (pq != cur_q) hermite_e(Q.l, 0, alpha[Q.p0 + pq], 0.0, 0.0, Fk + (tid - kKet) * g.f_axis, g.ld_fk, 0);
    } else if (tid >= kBoys && tid <= kBoys + L) {
      const double a = alpha[A.p0 + pa], b = B ? alpha[B->p0 + pb] : 0.0, q = alpha[Q.p0 + pq];
      const double p = a + b, ip = 1.0 / p;
      const double X = (a * A.x + b * bx) * ip - Q.x, Y = (a * A.y + b * by) * ip - Q.y,
                   Z = (a * A.z + b * bz) * ip - Q.z;
      const double ipq = 1.0 / (p + q), al = p * q * ipq;
      boys_scaled(tid - kBoys, L, al, al * (X * X + Y * Y + Z * Z), g.boys, F);
      if (tid == kBoys) {
        const double cab = coeff[A.p0 + pa] * (B ? coeff[B->p0 + pb] : 1.0);
        sc[0] = cab * coeff[Q.p0 + pq] * kTwoPi52 * sqrt(ipq) / (p * q);
        sc[1] = X;
        sc[2] = Y;
        sc[3] = Z;
      }
    }
    cur_pair = pab;
    cur_q = pq;
    team_sync<NT>();
    const double* R = hermite_r<NT>(L, sc[1], sc[2], sc[3], F, g.tet, R0, R1);   // ends with a barrier when L > 0
    // ket step: G[k][tuv] = sum_{t2 u2 v2} E^k_t2 E^k_u2 E^k_v2 R_{t+t2, u+u2, v+v2} for t + u + v <= lab;
    // the ket is a single centre, so E^{i0}_t vanishes unless t = i (mod 2) and the sign
    // (-1)^(t2+u2+v2) of the ket's Hermite functions is (-1)^lq throughout (folded into pref)
    for (int w = tid; w < nq * ntab; w += NT) {
      const int k = w / ntab, idx = w - k * ntab;
      const int tc = __ldg(g.tet + idx);
      const int t = tc & 255, u = (tc >> 8) & 255, v = tc >> 16;
      const int c = code[k];
      const int kx = (c >> 18) & 7, ky = (c >> 21) & 7, kz = (c >> 24) & 7;
      const double* Fx = Fk + kx * g.ld_fk;
      const double* Fy = Fk + g.f_axis + ky * g.ld_fk;
      const double* Fz = Fk + 2 * g.f_axis + kz * g.ld_fk;
      double sum = 0.0;
      for (int t2 = kx & 1; t2 <= kx; t2 += 2)
        for (int u2 = ky & 1; u2 <= ky; u2 += 2) {
          const double fxy = Fx[t2] * Fy[u2];
          for (int v2 = kz & 1; v2 <= kz; v2 += 2) sum += fxy * Fz[v2] * R[tet(t + t2, u + u2, v + v2)];
        }
      G[w] = sum;
    }
    team_sync<NT>();
    // bra step: acc[i][j][k] += pref sum_{tuv} E^{ij}_t E^{ij}_u E^{ij}_v G[k][tuv]
    const double pref = (Q.l & 1) ? -sc[0] : sc[0];
    for (int o = tid; o < nblk; o += NT) {
      const int c = code[o];
      const int ix = c & 7, iy = (c >> 3) & 7, iz = (c >> 6) & 7, jx = (c >> 9) & 7, jy = (c >> 12) & 7,
                jz = (c >> 15) & 7;
      const double* Ex = E + ix * g.ld_ei + jx * g.ld_ej;
      const double* Ey = E + g.e_axis + iy * g.ld_ei + jy * g.ld_ej;
      const double* Ez = E + 2 * g.e_axis + iz * g.ld_ei + jz * g.ld_ej;
      const double* Gk = G + (o % nq) * ntab;
      double tot = 0.0;
      for (int t = 0; t <= ix + jx; ++t) {
        const double ex = Ex[t];
        if (ex == 0.0) continue;
        for (int u = 0; u <= iy + jy; ++u) {
          const double exy = ex * Ey[u];
          if (exy == 0.0) continue;
          for (int v = 0; v <= iz + jz; ++v) tot += exy * Ez[v] * Gk[tet(t, u, v)];
        }
      }
      acc[o] += pref * tot;
    }
  }
  team_sync<NT>();
}

// Transform of the Cartesian block acc[na][nb][nq] to functions: out[fa][fb][fq]
// = sum Ta[fa][i] Tb[fb][j] Tq[fq][k] acc[i][j][k] (three passes through tmp).
__device__ __forceinline__ void transform_block(const double* Ta, int fa, int na, const double* Tb, int fb, int nb,
                                                const double* Tq, int fq, int nq, double* acc, double* tmp) {
  const int tid = threadIdx.x;
  // k: tmp[i][j][q] = sum_k Tq[q][k] acc[i][j][k]
  for (int o = tid; o < na * nb * fq; o += blockDim.x) {
    const int i = o / (nb * fq), j = (o / fq) % nb, q = o % fq;
    double s = 0.0;
    for (int k = 0; k < nq; ++k) s += Tq[q * nq + k] * acc[(i * nb + j) * nq + k];
    tmp[o] = s;
  }
  __syncthreads();
  // j: acc[i][b][q] = sum_j Tb[b][j] tmp[i][j][q]
  for (int o = tid; o < na * fb * fq; o += blockDim.x) {
    const int i = o / (fb * fq), bb = (o / fq) % fb, q = o % fq;
    double s = 0.0;
    for (int j = 0; j < nb; ++j) s += Tb[bb * nb + j] * tmp[(i * nb + j) * fq + q];
    acc[o] = s;
  }
  __syncthreads();
  // i: tmp[a][b][q] = sum_i Ta[a][i] acc[i][b][q]
  for (int o = tid; o < fa * fb * fq; o += blockDim.x) {
    const int aa = o / (fb * fq), bb = (o / fq) % fb, q = o % fq;
    double s = 0.0;
    for (int i = 0; i < na; ++i) s += Ta[aa * na + i] * acc[(i * fb + bb) * fq + q];
    tmp[o] = s;
  }
  __syncthreads();
}

// One CTA per (orbital shell pair, auxiliary shell) of a block list: blocks[b] =
// shell pair | auxiliary shell << 32.  W teams of NT threads share the primitive
// triples (triple tr to team tr mod W), each in its own smem_doubles of shared
// memory; their Cartesian blocks are summed in team order, then the CTA
// transforms and stores the block.
template <int NT, int W>
__global__ void __launch_bounds__(NT * W) ri_3center_kernel(RiArgs a, const long long* __restrict__ blocks) {
  extern __shared__ double smem[];
  const long long code = __ldg(blocks + blockIdx.x);
  const int sp = int(code & 0xFFFFFFFFLL), qs = int(code >> 32);
  const DevShell A = a.sh[a.shellpair[2 * sp]], B = a.sh[a.shellpair[2 * sp + 1]], Q = a.ax[qs];
  const int na = ncart(A.l), nb = ncart(B.l), nq = ncart(Q.l);
  const int team = W > 1 ? int(threadIdx.x) / NT : 0;
  shell_block<NT>(a, A, &B, Q, smem + (size_t)team * a.smem_doubles, na, nb, nq, team, W);
  double* acc = smem + a.off_acc;
  double* tmp = smem + a.off_tmp;
  if constexpr (W > 1) {
    __syncthreads();
    for (int o = threadIdx.x; o < na * nb * nq; o += NT * W) {
      double v = acc[o];
      for (int w = 1; w < W; ++w) v += acc[(size_t)w * a.smem_doubles + o];
      acc[o] = v;
    }
    __syncthreads();
  }
  const int fa = nfun(A.l, a.pure_orb), fb = nfun(B.l, a.pure_orb), fq = nfun(Q.l, a.pure_aux);
  transform_block(a.trans + a.toff[A.l], fa, na, a.trans + a.toff[B.l], fb, nb, a.trans + a.toff[5 + Q.l], fq, nq,
                  acc, tmp);
  for (int o = threadIdx.x; o < fa * fb * fq; o += blockDim.x) {
    const int i = o / (fb * fq), j = (o / fq) % fb, k = o % fq;
    const int mu = A.f0 + i, nu = B.f0 + j;
    if (mu < nu) continue;   // A == B: (mu nu|P) = (nu mu|P), stored once
    const int pr = a.pairmap[mu * a.nbf + nu];
    if (pr >= 0) a.out[(size_t)(Q.f0 + k) * a.npair + pr] = tmp[o];
  }
}

__global__ void __launch_bounds__(kRiThreads) ri_2center_kernel(RiArgs a) {
  extern __shared__ double smem[];
  const int ps = blockIdx.x, qs = blockIdx.y;
  if (qs > ps) return;
  const DevShell P = a.ax[ps], Q = a.ax[qs];
  const int np = ncart(P.l), nq = ncart(Q.l);
  shell_block<kRiThreads>(a, P, nullptr, Q, smem, np, 1, nq, 0, 1);
  double* acc = smem + a.off_acc;
  double* tmp = smem + a.off_tmp;
  const double one = 1.0;
  const int fp = nfun(P.l, a.pure_aux), fq = nfun(Q.l, a.pure_aux);
  transform_block(a.trans + a.toff[5 + P.l], fp, np, &one, 1, 1, a.trans + a.toff[5 + Q.l], fq, nq, acc, tmp);
  for (int o = threadIdx.x; o < fp * fq; o += blockDim.x) {
    const int i = o / fq, k = o % fq;
    a.out[(size_t)(P.f0 + i) * a.naux + Q.f0 + k] = tmp[o];
    a.out[(size_t)(Q.f0 + k) * a.naux + P.f0 + i] = tmp[o];
  }
}

// sqrtinv[P][c] = V[P][k_c] / sqrt(lambda_{k_c}) for the kept eigenpairs, in order;
// A holds the eigenvalues on its diagonal (n x n, padded).
__global__ void ri_sqrtinv_kernel(const double* __restrict__ A, const double* __restrict__ V, int n, int naux,
                                  const int* __restrict__ kept, int nkept, double* __restrict__ out, int ldo) {
  const int c = blockIdx.x;
  const int k = kept[c];
  const double s = 1.0 / sqrt(A[(size_t)k * n + k]);
  for (int p = threadIdx.x; p < naux; p += blockDim.x) out[(size_t)p * ldo + c] = V[(size_t)p * n + k] * s;
}

// Halve the diagonal pairs (the reference's convention, src/m_eri_calculate.f90:1841,1854).
__global__ void ri_halve_diag_kernel(double* __restrict__ raw, int naux, int npair, const int* __restrict__ diag,
                                     int ndiag) {
  const int p = blockIdx.y;
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < ndiag; d += gridDim.x * blockDim.x)
    raw[(size_t)p * npair + diag[d]] *= 0.5;
}

// ---- host: solid harmonics and the basis upload
double dfact(int n) {
  double r = 1.0;
  for (int k = n; k > 1; k -= 2) r *= k;
  return r;
}
double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}
double fact(int n) {
  double r = 1.0;
  for (int k = 2; k <= n; ++k) r *= k;
  return r;
}

// Transform of shell l acting on monomials of the common normalization
// (2/pi)^{3/4} 2^l alpha^{(2l+3)/4} (the reference's shell coefficients): pure:
// real solid harmonics m = -l..l (Helgaker et al. eq. 6.4.73) over sqrt((2l-1)!!);
// Cartesian: 1 / sqrt((2nx-1)!! (2ny-1)!! (2nz-1)!!) (src/m_cart_to_pure.f90:262-279).
std::vector<double> shell_transform(int l, bool pure) {
  const int nc = (l + 1) * (l + 2) / 2;
  std::vector<int> cx, cy, cz;
  for (int x = l; x >= 0; --x)
    for (int z = 0; z <= l - x; ++z) {
      cx.push_back(x);
      cy.push_back(l - x - z);
      cz.push_back(z);
    }
  auto index = [&](int x, int y, int z) {
    for (int k = 0; k < nc; ++k)
      if (cx[k] == x && cy[k] == y && cz[k] == z) return k;
    return -1;
  };
  if (!pure) {
    std::vector<double> t(size_t(nc) * nc, 0.0);
    for (int k = 0; k < nc; ++k) t[size_t(k) * nc + k] = 1.0 / std::sqrt(dfact(2 * cx[k] - 1) * dfact(2 * cy[k] - 1) *
                                                                        dfact(2 * cz[k] - 1));
    return t;
  }
  const int nf = 2 * l + 1;
  std::vector<double> t(size_t(nf) * nc, 0.0);
  for (int row = 0; row < nf; ++row) {
    const int m = row - l, am = std::abs(m);
    const double vm = m >= 0 ? 0.0 : 0.5;
    const double nlm = 1.0 / (std::pow(2.0, am) * fact(l)) *
                       std::sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0));
    for (int tt = 0; tt <= (l - am) / 2; ++tt)
      for (int u = 0; u <= tt; ++u) {
        const double vtop = std::floor(am / 2.0 - vm) + vm;
        for (double v = vm; v <= vtop + 1e-9; v += 1.0) {
          const int iv2 = int(std::lround(2 * v));
          const double sgn = (int(std::lround(tt + v - vm)) % 2 == 0) ? 1.0 : -1.0;
          const double c = sgn * std::pow(0.25, tt) * binom(l, tt) * binom(l - tt, am + tt) * binom(tt, u) * binom(am, iv2);
          const int ex = int(std::lround(2 * tt + am - 2 * (u + v))), ey = int(std::lround(2 * (u + v))),
                    ez = l - 2 * tt - am;
          const int k = index(ex, ey, ez);
          if (k >= 0) t[size_t(row) * nc + k] += nlm * c / std::sqrt(dfact(2 * l - 1));
        }
      }
  }
  return t;
}

struct RiBasis {
  std::vector<DevShell> sh, ax;
  std::vector<double> alpha, coeff, trans;
  std::vector<int> toff, shellpair, pairmap, diag;
  int nbf = 0, naux = 0;
};

Status build_basis(const rigw_ri_problem& pr, RiBasis& b) {
  auto add = [&](const rigw_shell* src, int n, std::vector<DevShell>& dst, bool pure, int& nf) -> Status {
    for (int i = 0; i < n; ++i) {
      const rigw_shell& s = src[i];
      if (s.am < 0 || s.am > kRiLmax || s.nprim <= 0 || !s.alpha || !s.coeff)
        return Status::fail(RIGW_ERR_ARG, "ri integrals: shell %d: angular momentum beyond %d or no primitives", i,
                            kRiLmax);
      DevShell d{};
      d.x = s.center[0];
      d.y = s.center[1];
      d.z = s.center[2];
      d.l = s.am;
      d.nprim = s.nprim;
      d.p0 = int(b.alpha.size());
      d.f0 = nf;
      for (int k = 0; k < s.nprim; ++k) {
        b.alpha.push_back(s.alpha[k]);
        b.coeff.push_back(s.coeff[k]);
      }
      nf += pure ? 2 * s.am + 1 : (s.am + 1) * (s.am + 2) / 2;
      dst.push_back(d);
    }
    return Status::ok();
  };
  RIGW_TRY(add(pr.shells, pr.nshell, b.sh, pr.pure != 0, b.nbf));
  RIGW_TRY(add(pr.aux_shells, pr.nshell_aux, b.ax, pr.pure_aux != 0, b.naux));
  b.toff.assign(10, 0);
  for (int basis = 0; basis < 2; ++basis)
    for (int l = 0; l <= kRiLmax; ++l) {
      b.toff[basis * 5 + l] = int(b.trans.size());
      const std::vector<double> t = shell_transform(l, basis == 0 ? pr.pure != 0 : pr.pure_aux != 0);
      b.trans.insert(b.trans.end(), t.begin(), t.end());
    }
  for (int A = 0; A < int(b.sh.size()); ++A)
    for (int B = 0; B <= A; ++B) {
      b.shellpair.push_back(A);
      b.shellpair.push_back(B);
    }
  if (pr.npair > 0) {
    b.pairmap.assign(size_t(b.nbf) * b.nbf, -1);
    for (int k = 0; k < pr.npair; ++k) {
      const int i = pr.index_basis[2 * k] - 1, j = pr.index_basis[2 * k + 1] - 1;
      if (i < 0 || j < 0 || i >= b.nbf || j >= b.nbf)
        return Status::fail(RIGW_ERR_ARG, "ri integrals: pair %d outside the basis", k);
      b.pairmap[size_t(i) * b.nbf + j] = k;
      b.pairmap[size_t(j) * b.nbf + i] = k;
      if (i == j) b.diag.push_back(k);
    }
  }
  return Status::ok();
}

// F_m(T_i) for the table points T_i = i * 0.1 (the double the device forms), from
// the series e^-T sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)) in extended precision.
const std::vector<double>& boys_table() {
  static const std::vector<double> tab = [] {
    std::vector<double> t(size_t(kBoysRows) * kBoysOrders);
    for (int i = 0; i < kBoysRows; ++i) {
      const long double T = (long double)(i * kBoysStep);
      const long double e = std::exp(-T);
      for (int m = 0; m < kBoysOrders; ++m) {
        long double term = 1.0L / (2 * m + 1), sum = term;
        for (int k = 1; k < 2000; ++k) {
          term *= 2.0L * T / (2 * m + 2 * k + 1);
          sum += term;
          if (term < 1.0e-21L * sum) break;
        }
        t[size_t(i) * kBoysOrders + m] = double(e * sum);
      }
    }
    return t;
  }();
  return tab;
}

// (t, u, v) of every tetrahedral index up to t + u + v = 3 kRiLmax.
std::vector<int> tet_codes() {
  std::vector<int> c;
  for (int s = 0; s <= 3 * kRiLmax; ++s)
    for (int t = 0; t <= s; ++t)
      for (int u = 0; u <= s - t; ++u) c.push_back(t | (u << 8) | ((s - t - u) << 16));
  return c;
}

// Shared-memory layout for bra shells up to la and lb, ket shells up to lk, blocks
// of total angular momentum up to L, Cartesian blocks of up to nacc components and
// ket-contracted Hermite tables of up to ngk entries.
void set_layout(RiArgs& g, int la, int lb, int lk, int L, int nacc, int ngk) {
  g.ntet = (L + 1) * (L + 2) * (L + 3) / 6;
  g.ld_ej = la + lb + 1;
  g.ld_ei = (lb + 1) * g.ld_ej;
  g.e_axis = (la + 1) * g.ld_ei;
  g.ld_fk = lk + 1;
  g.f_axis = (lk + 1) * g.ld_fk;
  g.off_e = 2 * g.ntet;
  g.off_f = g.off_e + 3 * g.e_axis;
  g.off_acc = g.off_f + 3 * g.f_axis;
  g.off_tmp = g.off_acc + nacc;
  g.off_boys = g.off_tmp + std::max(nacc, ngk);
  g.off_scal = g.off_boys + L + 1;
  g.off_code = g.off_scal + 8;
  g.smem_doubles = g.off_code + (nacc + 1) / 2;
}

int ncart_host(int l) { return (l + 1) * (l + 2) / 2; }
int ntet_host(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }

// A class of 3-center blocks launched together: the block list and the layout maxima.
struct BlockClass {
  std::vector<long long> blocks;
  int la = 0, lb = 0, lk = 0, L = 0, nacc = 1, ngk = 1;
  void add(long long code, const DevShell& A, const DevShell& B, const DevShell& Q) {
    blocks.push_back(code);
    const int nblk = ncart_host(A.l) * ncart_host(B.l) * ncart_host(Q.l);
    la = std::max(la, A.l);
    lb = std::max(lb, B.l);
    lk = std::max(lk, Q.l);
    L = std::max(L, A.l + B.l + Q.l);
    nacc = std::max(nacc, nblk);
    ngk = std::max(ngk, ncart_host(Q.l) * ntet_host(A.l + B.l));
  }
};

template <class T>
Status upload(Context& c, DeviceBuffer& buf, const std::vector<T>& v, const char* name, cudaStream_t s) {
  RIGW_TRY(buf.allocate(&c, std::max<size_t>(v.size(), 1) * sizeof(T), name));
  if (!v.empty()) RIGW_CUDA_TRY(cudaMemcpyAsync(buf.data(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return Status::ok();
}

}  // namespace

Status ri_integrals(Context& c, const rigw_ri_problem& pr, int what, double* out, int* nkept_out) {
  if (pr.nshell_aux <= 0 || !pr.aux_shells || (what != 2 && (pr.nshell <= 0 || !pr.shells || pr.npair <= 0 ||
                                                             !pr.index_basis)) || !out)
    return Status::fail(RIGW_ERR_ARG, "ri integrals: invalid arguments");
  NvtxRange range(what == 2 ? "2-center integrals" : "3-center integrals");
  RiBasis b;
  RIGW_TRY(build_basis(pr, b));
  cudaStream_t s = c.stream;
  const bool on_dev = (pr.flags & RIGW_PROBLEM_DEVICE_POINTERS) != 0;
  DeviceBuffer b_sh, b_ax, b_al, b_co, b_tr, b_to, b_sp, b_pm, b_out, b_v2, b_vec, b_kept, b_diag, b_items, b_boys,
      b_tet;
  RIGW_TRY(upload(c, b_sh, b.sh, "ri shells", s));
  RIGW_TRY(upload(c, b_ax, b.ax, "ri auxiliary shells", s));
  RIGW_TRY(upload(c, b_al, b.alpha, "ri exponents", s));
  RIGW_TRY(upload(c, b_co, b.coeff, "ri coefficients", s));
  RIGW_TRY(upload(c, b_tr, b.trans, "ri transforms", s));
  RIGW_TRY(upload(c, b_to, b.toff, "ri transform offsets", s));
  RIGW_TRY(upload(c, b_boys, boys_table(), "ri Boys table", s));
  RIGW_TRY(upload(c, b_tet, tet_codes(), "ri Hermite index table", s));
  RiArgs a{};
  a.sh = reinterpret_cast<const DevShell*>(b_sh.data());
  a.ax = reinterpret_cast<const DevShell*>(b_ax.data());
  a.alpha = reinterpret_cast<const double*>(b_al.data());
  a.coeff = reinterpret_cast<const double*>(b_co.data());
  a.trans = reinterpret_cast<const double*>(b_tr.data());
  a.toff = reinterpret_cast<const int*>(b_to.data());
  a.nbf = b.nbf;
  a.naux = b.naux;
  a.npair = pr.npair;
  a.pure_orb = pr.pure != 0;
  a.pure_aux = pr.pure_aux != 0;
  a.boys = reinterpret_cast<const double*>(b_boys.data());
  a.tet = reinterpret_cast<const int*>(b_tet.data());
  int lorb = 0, laux = 0;
  for (const DevShell& d : b.sh) lorb = std::max(lorb, d.l);
  for (const DevShell& d : b.ax) laux = std::max(laux, d.l);
  const int nax = int(b.ax.size());
  if (what == 2 || what == 0) {
    // (P|Q); for the metric, into a matrix padded to a multiple of 64 for the eigensolver
    const int n = what == 2 ? b.naux : int((b.naux + 63) / 64 * 64);
    double* v2 = nullptr;
    if (what == 2 && on_dev) {
      v2 = out;
    } else {
      RIGW_TRY(b_v2.allocate(&c, size_t(n) * n * 8, "ri (P|Q)"));
      v2 = reinterpret_cast<double*>(b_v2.data());
    }
    RIGW_CUDA_TRY(cudaMemsetAsync(v2, 0, size_t(n) * n * 8, s));
    RiArgs a2 = a;
    a2.out = v2;
    a2.naux = n;   // row stride
    set_layout(a2, laux, 0, laux, 2 * laux, ncart_host(laux) * ncart_host(laux), ncart_host(laux) * ntet_host(laux));
    const size_t smem2 = size_t(a2.smem_doubles) * sizeof(double);
    RIGW_CUDA_TRY(cudaFuncSetAttribute(ri_2center_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem2)));
    ri_2center_kernel<<<dim3(nax, nax), kRiThreads, smem2, s>>>(a2);
    RIGW_CUDA_TRY(cudaGetLastError());
    if (what == 2) {
      if (!on_dev) RIGW_CUDA_TRY(cudaMemcpyAsync(out, v2, size_t(n) * n * 8, cudaMemcpyDeviceToHost, s));
      RIGW_CUDA_TRY(cudaStreamSynchronize(s));
      return Status::ok();
    }
  }
  // (mu nu|P) over the pairs: [naux][npair]
  const int nsp = int(b.shellpair.size() / 2);
  RIGW_TRY(upload(c, b_sp, b.shellpair, "ri shell pairs", s));
  RIGW_TRY(upload(c, b_pm, b.pairmap, "ri pair map", s));
  a.shellpair = reinterpret_cast<const int*>(b_sp.data());
  a.pairmap = reinterpret_cast<const int*>(b_pm.data());
  double* raw = nullptr;
  if (what == 3 && on_dev) {
    raw = out;
  } else {
    RIGW_TRY(b_out.allocate(&c, size_t(b.naux) * pr.npair * 8, "ri (mu nu|P)"));
    raw = reinterpret_cast<double*>(b_out.data());
  }
  a.out = raw;
  // Three classes of blocks: at least 20 primitive triples and up to 128 Cartesian
  // components (contracted shells on both sides) run four one-warp teams per CTA
  // that share the triples; the others up to 32 components (most blocks) one warp
  // per CTA; the rest 128 threads per CTA.
  // Shell pairs with the most primitive pairs come first, so that the last wave
  // holds short blocks.
  std::vector<int> order(nsp);
  for (int i = 0; i < nsp; ++i) order[i] = i;
  auto prims = [&](int sp) { return b.sh[b.shellpair[2 * sp]].nprim * b.sh[b.shellpair[2 * sp + 1]].nprim; };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return prims(x) > prims(y); });
  constexpr int kTeams = 4;
  BlockClass cls[3];   // warp CTAs, teams of warps, 128-thread CTAs
  cls[0].blocks.reserve(size_t(nsp) * nax);
  for (const int sp : order)
    for (int qs = 0; qs < nax; ++qs) {
      const DevShell& A = b.sh[b.shellpair[2 * sp]];
      const DevShell& B = b.sh[b.shellpair[2 * sp + 1]];
      const DevShell& Q = b.ax[qs];
      const int nblk = ncart_host(A.l) * ncart_host(B.l) * ncart_host(Q.l);
      const int ntri = A.nprim * B.nprim * Q.nprim;
      const int k = ntri >= 20 && nblk <= 128 ? 1 : (nblk <= 32 ? 0 : 2);
      cls[k].add((long long)sp | ((long long)qs << 32), A, B, Q);
    }
  DeviceBuffer b_list[3];
  for (int k = 0; k < 3; ++k) RIGW_TRY(upload(c, b_list[k], cls[k].blocks, "ri block list", s));
  // the three launches run concurrently (each fills the others' tails): classes 0 and 1
  // on two side streams that fork from and join back into the call's stream
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> ev;
  RIGW_TRY(c.borrow(2, 3, &side, &ev));
  RIGW_CUDA_TRY(cudaEventRecord(ev[0], s));
  for (int k = 0; k < 2; ++k) RIGW_CUDA_TRY(cudaStreamWaitEvent(side[k], ev[0], 0));
  for (const int k : {2, 1, 0}) {
    const BlockClass& bc = cls[k];
    if (bc.blocks.empty()) continue;
    RiArgs ak = a;
    set_layout(ak, bc.la, bc.lb, bc.lk, bc.L, bc.nacc, bc.ngk);
    const long long* list = reinterpret_cast<const long long*>(b_list[k].data());
    const unsigned nb = unsigned(bc.blocks.size());
    const cudaStream_t sk = k == 2 ? s : side[k];
    if (k == 0) {
      const size_t smem3 = size_t(ak.smem_doubles) * sizeof(double);
      RIGW_CUDA_TRY(cudaFuncSetAttribute(ri_3center_kernel<32, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(smem3)));
      ri_3center_kernel<32, 1><<<nb, 32, smem3, sk>>>(ak, list);
    } else if (k == 1) {
      const size_t smem3 = size_t(kTeams) * ak.smem_doubles * sizeof(double);
      RIGW_CUDA_TRY(cudaFuncSetAttribute(ri_3center_kernel<32, kTeams>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem3)));
      ri_3center_kernel<32, kTeams><<<nb, 32 * kTeams, smem3, sk>>>(ak, list);
    } else {
      const size_t smem3 = size_t(ak.smem_doubles) * sizeof(double);
      RIGW_CUDA_TRY(cudaFuncSetAttribute(ri_3center_kernel<kRiThreads, 1>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem3)));
      ri_3center_kernel<kRiThreads, 1><<<nb, kRiThreads, smem3, sk>>>(ak, list);
    }
    RIGW_CUDA_TRY(cudaGetLastError());
  }
  for (int k = 0; k < 2; ++k) {
    RIGW_CUDA_TRY(cudaEventRecord(ev[1 + k], side[k]));
    RIGW_CUDA_TRY(cudaStreamWaitEvent(s, ev[1 + k], 0));
  }
  RIGW_CUDA_TRY(cudaGetLastError());
  if (what == 3) {
    if (!on_dev)
      RIGW_CUDA_TRY(cudaMemcpyAsync(out, raw, size_t(b.naux) * pr.npair * 8, cudaMemcpyDeviceToHost, s));
    RIGW_CUDA_TRY(cudaStreamSynchronize(s));
    return Status::ok();
  }
  // the metric: eigenpairs of (P|Q), kept where lambda > 1e-6
  const int n = int((b.naux + 63) / 64 * 64);
  double* v2 = reinterpret_cast<double*>(b_v2.data());
  RIGW_TRY(b_vec.allocate(&c, size_t(n) * n * 8, "ri metric eigenvectors"));
  double* vec = reinterpret_cast<double*>(b_vec.data());
  int sweeps = 0, launches = 0;
  RIGW_TRY(eigh_jacobi_batched(c, v2, vec, n, 1, s, &sweeps, &launches));
  std::vector<double> diag(size_t(n) * n);
  RIGW_CUDA_TRY(cudaMemcpyAsync(diag.data(), v2, size_t(n) * n * 8, cudaMemcpyDeviceToHost, s));
  RIGW_CUDA_TRY(cudaStreamSynchronize(s));
  // the padding rows and columns are zero: their eigenvalues are 0 and never kept
  std::vector<int> kept;
  for (int k = 0; k < n; ++k)
    if (diag[size_t(k) * n + k] > kRiTooLowEigval) kept.push_back(k);
  const int nkept = int(kept.size());
  RIGW_TRY(upload(c, b_kept, kept, "ri kept eigenpairs", s));
  // sqrtinv [naux][nkept padded to even]
  const int ldk = nkept + (nkept & 1);
  DeviceBuffer b_si;
  RIGW_TRY(b_si.allocate(&c, size_t(b.naux) * ldk * 8, "ri (P|Q)^-1/2"));
  double* si = reinterpret_cast<double*>(b_si.data());
  RIGW_CUDA_TRY(cudaMemsetAsync(si, 0, size_t(b.naux) * ldk * 8, s));
  if (nkept > 0)
    ri_sqrtinv_kernel<<<nkept, 128, 0, s>>>(v2, vec, n, b.naux, reinterpret_cast<const int*>(b_kept.data()), nkept,
                                            si, ldk);
  // halve the diagonal pairs, then B[c][pair] = sum_P sqrtinv[P][c] raw[P][pair] (DMMA)
  RIGW_TRY(upload(c, b_diag, b.diag, "ri diagonal pairs", s));
  if (!b.diag.empty())
    ri_halve_diag_kernel<<<dim3(unsigned((b.diag.size() + 255) / 256), unsigned(b.naux)), 256, 0, s>>>(
        raw, b.naux, pr.npair, reinterpret_cast<const int*>(b_diag.data()), int(b.diag.size()));
  RIGW_CUDA_TRY(cudaGetLastError());
  // pairs padded to even for the product: copy raw into an even-strided buffer when npair is odd
  const int npp = pr.npair + (pr.npair & 1);
  DeviceBuffer b_rawp, b_res;
  const double* rawp = raw;
  if (npp != pr.npair) {
    RIGW_TRY(b_rawp.allocate(&c, size_t(b.naux) * npp * 8, "ri (mu nu|P) padded"));
    double* rp = reinterpret_cast<double*>(b_rawp.data());
    RIGW_CUDA_TRY(cudaMemsetAsync(rp, 0, size_t(b.naux) * npp * 8, s));
    RIGW_CUDA_TRY(cudaMemcpy2DAsync(rp, size_t(npp) * 8, raw, size_t(pr.npair) * 8, size_t(pr.npair) * 8, b.naux,
                                    cudaMemcpyDeviceToDevice, s));
    rawp = rp;
  }
  RIGW_TRY(b_res.allocate(&c, size_t(ldk) * npp * 8, "ri B"));
  double* res = reinterpret_cast<double*>(b_res.data());
  std::vector<GemmItem> items;
  for (int i0 = 0; i0 < ldk; i0 += 128)
    for (int j0 = 0; j0 < npp; j0 += 128) {
      GemmItem g{};
      g.A = si + i0;   // A[k = P][m = c]
      g.lda = ldk;
      g.B = rawp + j0;   // B[k = P][n = pair]
      g.ldb = npp;
      g.C = res + size_t(i0) * npp + j0;
      g.ldc = npp;
      g.m = std::min(128, ldk - i0);
      g.n = std::min(128, npp - j0);
      g.k = b.naux;
      g.alpha = 1.0;
      items.push_back(g);
    }
  RIGW_TRY(upload(c, b_items, items, "ri product items", s));
  launch_dgemm_128x128(reinterpret_cast<const GemmItem*>(b_items.data()), int(items.size()), 1, s);
  RIGW_CUDA_TRY(cudaGetLastError());
  const cudaMemcpyKind kind = on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  RIGW_CUDA_TRY(cudaMemcpy2DAsync(out, size_t(pr.npair) * 8, res, size_t(npp) * 8, size_t(pr.npair) * 8, nkept, kind,
                                  s));
  RIGW_CUDA_TRY(cudaStreamSynchronize(s));
  if (nkept_out) *nkept_out = nkept;
  return Status::ok();
}

}  // namespace rigw
