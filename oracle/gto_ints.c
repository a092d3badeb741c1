/* Gaussian integrals for the oracle's front end (TEST INFRASTRUCTURE ONLY).
 *
 * MOLGW takes its integrals from LIBCINT, a third-party library absent here.
 * This file restates them with the published McMurchie-Davidson scheme
 * (Helgaker, Jorgensen, Olsen, "Molecular Electronic-Structure Theory", ch. 9):
 * Hermite expansion coefficients E^{ij}_t of Gaussian products, Hermite Coulomb
 * integrals R_{tuv} from the Boys function, contracted over primitives.  It
 * produces the overlap, kinetic and nuclear-attraction matrices and the 2- and
 * 3-center Coulomb integrals over contracted Cartesian shells; the caller
 * normalizes the primitives (coefficients include their norms) and transforms
 * to pure functions.  Cartesian components of a shell of angular momentum l are
 * ordered with nx from l down and, for each nx, nz from 0 up (x^l first), the
 * order of the reference (src/m_basis_set.f90:281-315).
 *
 * Loops run over shells and primitive pairs/triples: one Boys evaluation and
 * one R table per primitive combination serve every Cartesian component.
 *
 * Built by oracle/gaussian_ri.py:build_library (gcc -O2 -shared -fPIC, next to this file).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LMAX 6                      /* highest angular momentum of a shell */
#define NE (LMAX + 3)               /* E arrays carry j up to lb + 2 (kinetic) */
#define NT (2 * LMAX + 4)
#define LTOT (3 * LMAX)             /* highest Hermite order of a 3-center integral */
#define NR (LTOT + 1)
#define NCMAX ((LMAX + 1) * (LMAX + 2) / 2)

typedef struct {
  double x, y, z;
  int l, nprim;
  const double* a;                  /* exponents */
  const double* c;                  /* contraction coefficients including primitive norms */
} shell_t;

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

static void cart_list(int l, int (*out)[3]) {
  int k = 0;
  for (int nx = l; nx >= 0; --nx)
    for (int nz = 0; nz <= l - nx; ++nz) {
      out[k][0] = nx;
      out[k][1] = l - nx - nz;
      out[k][2] = nz;
      ++k;
    }
}

typedef double etab_t[NE][NE][NT];

/* E^{ij}_t for i <= imax, j <= jmax along one axis, Q = A - B (Helgaker eq. 9.5.6-9.5.7). */
static void hermite_e(int imax, int jmax, double a, double b, double qx, etab_t E) {
  const double p = a + b, mu = a * b / p;
  const double xpa = -b / p * qx, xpb = a / p * qx, h = 0.5 / p;
  E[0][0][0] = exp(-mu * qx * qx);
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; ++t) {
        double v;
        /* E[i'][j'][t] vanishes for t > i' + j' */
        const int tp = i + j - 1;
        if (i > 0) {
          v = (t <= tp ? xpa * E[i - 1][j][t] : 0.0) + (t + 1 <= tp ? (t + 1) * E[i - 1][j][t + 1] : 0.0);
          if (t > 0) v += h * E[i - 1][j][t - 1];
        } else {
          v = (t <= tp ? xpb * E[i][j - 1][t] : 0.0) + (t + 1 <= tp ? (t + 1) * E[i][j - 1][t + 1] : 0.0);
          if (t > 0) v += h * E[i][j - 1][t - 1];
        }
        E[i][j][t] = v;
      }
    }
}

/* Boys function F_m(T), m = 0..mmax: series for the highest order and
 * downward recursion; for large T the asymptotic F_0 and upward recursion. */
static void boys(int mmax, double T, double* F) {
  if (T < 1e-14) {
    for (int m = 0; m <= mmax; ++m) F[m] = 1.0 / (2 * m + 1) - T / (2 * m + 3);
    return;
  }
  const double e = exp(-T);
  if (T > 50.0 && T > 2.0 * mmax) {
    F[0] = 0.5 * sqrt(M_PI / T);    /* erf(sqrt(T)) = 1 to below 1e-22 */
    for (int m = 0; m < mmax; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
    return;
  }
  double term = 1.0 / (2 * mmax + 1), sum = term;
  for (int k = 1; k < 4000; ++k) {
    term *= 2.0 * T / (2 * mmax + 2 * k + 1);
    sum += term;
    if (term < 1e-17 * sum) break;
  }
  F[mmax] = e * sum;
  for (int m = mmax; m > 0; --m) F[m - 1] = (2.0 * T * F[m] + e) / (2 * m - 1);
}

typedef double rtab_t[NR][NR][NR];

/* R_{tuv} of order 0 for t + u + v <= L (Helgaker eq. 9.9.18-9.9.20). */
static void hermite_r(int L, double p, double X, double Y, double Z, rtab_t Rout) {
  static __thread double R[NR][NR][NR][NR];
  double F[NR];
  boys(L, p * (X * X + Y * Y + Z * Z), F);
  double fac = 1.0;
  for (int n = 0; n <= L; ++n) {
    R[n][0][0][0] = fac * F[n];
    fac *= -2.0 * p;
  }
  for (int n = L - 1; n >= 0; --n)
    for (int t = 0; t <= L - n; ++t)
      for (int u = 0; u <= L - n - t; ++u)
        for (int v = 0; v <= L - n - t - u; ++v) {
          if (t + u + v == 0) continue;
          double val;
          if (t > 0)
            val = X * R[n + 1][t - 1][u][v] + (t > 1 ? (t - 1) * R[n + 1][t - 2][u][v] : 0.0);
          else if (u > 0)
            val = Y * R[n + 1][t][u - 1][v] + (u > 1 ? (u - 1) * R[n + 1][t][u - 2][v] : 0.0);
          else
            val = Z * R[n + 1][t][u][v - 1] + (v > 1 ? (v - 1) * R[n + 1][t][u][v - 2] : 0.0);
          R[n][t][u][v] = val;
        }
  for (int t = 0; t <= L; ++t)
    for (int u = 0; u <= L - t; ++u)
      for (int v = 0; v <= L - t - u; ++v) Rout[t][u][v] = R[0][t][u][v];
}

static int shell_offsets(int nsh, const shell_t* sh, int* off) {
  int n = 0;
  for (int s = 0; s < nsh; ++s) {
    off[s] = n;
    n += ncart(sh[s].l);
  }
  return n;
}

/* Overlap, kinetic and nuclear attraction (-sum_C Z_C <a|1/r_C|b>) over
 * Cartesian functions, each [n][n].  Returns n. */
int gto_one_body(int nsh, const shell_t* sh, int nnuc, const double* zc, const double* xyz, double* S, double* T,
                 double* V) {
  int* off = (int*)malloc(sizeof(int) * nsh);
  const int n = shell_offsets(nsh, sh, off);
  etab_t* E = (etab_t*)malloc(sizeof(etab_t) * 3);
  rtab_t* R = (rtab_t*)malloc(sizeof(rtab_t));
  memset(S, 0, sizeof(double) * n * n);
  memset(T, 0, sizeof(double) * n * n);
  memset(V, 0, sizeof(double) * n * n);
  for (int A = 0; A < nsh; ++A)
    for (int B = 0; B < nsh; ++B) {
      const shell_t *sa = &sh[A], *sb = &sh[B];
      int ca[NCMAX][3], cb[NCMAX][3];
      cart_list(sa->l, ca);
      cart_list(sb->l, cb);
      const int na = ncart(sa->l), nb = ncart(sb->l), L = sa->l + sb->l;
      const double XA[3] = {sa->x, sa->y, sa->z}, XB[3] = {sb->x, sb->y, sb->z};
      for (int pa = 0; pa < sa->nprim; ++pa)
        for (int pb = 0; pb < sb->nprim; ++pb) {
          const double a = sa->a[pa], b = sb->a[pb], p = a + b, cc = sa->c[pa] * sb->c[pb];
          for (int d = 0; d < 3; ++d) hermite_e(sa->l, sb->l + 2, a, b, XA[d] - XB[d], E[d]);
          const double P[3] = {(a * XA[0] + b * XB[0]) / p, (a * XA[1] + b * XB[1]) / p, (a * XA[2] + b * XB[2]) / p};
          const double sfac = pow(M_PI / p, 1.5);
          for (int i = 0; i < na; ++i)
            for (int j = 0; j < nb; ++j) {
              double s1[3], t1[3];
              for (int d = 0; d < 3; ++d) {
                const int ii = ca[i][d], jj = cb[j][d];
                s1[d] = E[d][ii][jj][0];
                /* d^2/dx^2 of x_B^j exp(-b x_B^2), projected on the bra */
                t1[d] = 4.0 * b * b * E[d][ii][jj + 2][0] - 2.0 * b * (2 * jj + 1) * s1[d] +
                        (jj >= 2 ? jj * (jj - 1) * E[d][ii][jj - 2][0] : 0.0);
              }
              S[(off[A] + i) * n + off[B] + j] += cc * sfac * s1[0] * s1[1] * s1[2];
              T[(off[A] + i) * n + off[B] + j] +=
                  -0.5 * cc * sfac * (t1[0] * s1[1] * s1[2] + s1[0] * t1[1] * s1[2] + s1[0] * s1[1] * t1[2]);
            }
          for (int C = 0; C < nnuc; ++C) {
            hermite_r(L, p, P[0] - xyz[3 * C], P[1] - xyz[3 * C + 1], P[2] - xyz[3 * C + 2], *R);
            const double pref = -cc * zc[C] * 2.0 * M_PI / p;
            for (int i = 0; i < na; ++i)
              for (int j = 0; j < nb; ++j) {
                const int ix = ca[i][0], iy = ca[i][1], iz = ca[i][2];
                const int jx = cb[j][0], jy = cb[j][1], jz = cb[j][2];
                double v = 0.0;
                for (int t = 0; t <= ix + jx; ++t)
                  for (int u = 0; u <= iy + jy; ++u) {
                    const double etu = E[0][ix][jx][t] * E[1][iy][jy][u];
                    for (int w = 0; w <= iz + jz; ++w) v += etu * E[2][iz][jz][w] * (*R)[t][u][w];
                  }
                V[(off[A] + i) * n + off[B] + j] += pref * v;
              }
          }
        }
    }
  free(R);
  free(E);
  free(off);
  return n;
}

/* Hermite expansions of all Cartesian components of one primitive pair:
 * H[c][t][u][v] for component c = (i, j) of the pair (j = 0 and b = 0 for a
 * single function). */
#define NH (2 * LMAX + 1)
typedef double htab_t[NH][NH][NH];

static void pair_hermite(const shell_t* sa, int pa, const shell_t* sb, int pb, etab_t* E, htab_t* H, double* P,
                         double* p_out) {
  const double a = sa->a[pa], b = sb ? sb->a[pb] : 0.0;
  const double XA[3] = {sa->x, sa->y, sa->z};
  const double XB[3] = {sb ? sb->x : sa->x, sb ? sb->y : sa->y, sb ? sb->z : sa->z};
  const int lb = sb ? sb->l : 0;
  const double p = a + b;
  for (int d = 0; d < 3; ++d) {
    hermite_e(sa->l, lb, a, b, XA[d] - XB[d], E[d]);
    P[d] = (a * XA[d] + b * XB[d]) / p;
  }
  *p_out = p;
  int ca[NCMAX][3], cb[NCMAX][3];
  cart_list(sa->l, ca);
  cart_list(lb, cb);
  const int nb = ncart(lb);
  for (int i = 0; i < ncart(sa->l); ++i)
    for (int j = 0; j < nb; ++j) {
      double(*h)[NH][NH] = H[i * nb + j];
      const int ix = ca[i][0], iy = ca[i][1], iz = ca[i][2];
      const int jx = cb[j][0], jy = cb[j][1], jz = cb[j][2];
      for (int t = 0; t <= ix + jx; ++t)
        for (int u = 0; u <= iy + jy; ++u)
          for (int v = 0; v <= iz + jz; ++v) h[t][u][v] = E[0][ix][jx][t] * E[1][iy][jy][u] * E[2][iz][jz][v];
    }
}

/* Sum over two Hermite expansions (per-axis orders e1, e2) of
 * E1_{tuv} (-1)^{t'+u'+v'} E2_{t'u'v'} R_{t+t',u+u',v+v'}. */
static double hermite_contract(const double (*h1)[NH][NH], const int* e1, const double (*h2)[NH][NH], const int* e2,
                               const double (*R)[NR][NR]) {
  double tot = 0.0;
  for (int t = 0; t <= e1[0]; ++t)
    for (int u = 0; u <= e1[1]; ++u)
      for (int v = 0; v <= e1[2]; ++v) {
        const double c1 = h1[t][u][v];
        if (c1 == 0.0) continue;
        double s = 0.0;
        for (int t2 = 0; t2 <= e2[0]; ++t2)
          for (int u2 = 0; u2 <= e2[1]; ++u2)
            for (int v2 = 0; v2 <= e2[2]; ++v2) {
              const double c2 = h2[t2][u2][v2];
              s += (((t2 + u2 + v2) & 1) ? -c2 : c2) * R[t + t2][u + u2][v + v2];
            }
        tot += c1 * s;
      }
  return tot;
}

/* (P|Q) over the Cartesian functions of the auxiliary shells, [n][n].  Returns n. */
int gto_coulomb2(int nsh, const shell_t* sh, double* out) {
  int* off = (int*)malloc(sizeof(int) * nsh);
  const int n = shell_offsets(nsh, sh, off);
  etab_t* E = (etab_t*)malloc(sizeof(etab_t) * 3);
  htab_t* H1 = (htab_t*)malloc(sizeof(htab_t) * NCMAX);
  htab_t* H2 = (htab_t*)malloc(sizeof(htab_t) * NCMAX);
  rtab_t* R = (rtab_t*)malloc(sizeof(rtab_t));
  double* blk = (double*)malloc(sizeof(double) * NCMAX * NCMAX);
  for (int A = 0; A < nsh; ++A)
    for (int B = 0; B <= A; ++B) {
      const shell_t *sa = &sh[A], *sb = &sh[B];
      int ca[NCMAX][3], cb[NCMAX][3];
      cart_list(sa->l, ca);
      cart_list(sb->l, cb);
      const int na = ncart(sa->l), nb = ncart(sb->l);
      memset(blk, 0, sizeof(double) * na * nb);
      for (int pa = 0; pa < sa->nprim; ++pa) {
        double P1[3], p;
        pair_hermite(sa, pa, NULL, 0, E, H1, P1, &p);
        for (int pb = 0; pb < sb->nprim; ++pb) {
          double P2[3], q;
          pair_hermite(sb, pb, NULL, 0, E, H2, P2, &q);
          hermite_r(sa->l + sb->l, p * q / (p + q), P1[0] - P2[0], P1[1] - P2[1], P1[2] - P2[2], *R);
          const double pref = sa->c[pa] * sb->c[pb] * 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q));
          for (int i = 0; i < na; ++i)
            for (int j = 0; j < nb; ++j)
              blk[i * nb + j] += pref * hermite_contract((const double(*)[NH][NH])H1[i], ca[i],
                                                         (const double(*)[NH][NH])H2[j], cb[j],
                                                         (const double(*)[NR][NR])*R);
        }
      }
      for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j) {
          out[(size_t)(off[A] + i) * n + off[B] + j] = blk[i * nb + j];
          out[(size_t)(off[B] + j) * n + off[A] + i] = blk[i * nb + j];
        }
    }
  free(blk);
  free(R);
  free(H2);
  free(H1);
  free(E);
  free(off);
  return n;
}

/* (mu nu|P) over Cartesian functions, [n][n][naux].  Returns n. */
int gto_coulomb3(int nsh, const shell_t* sh, int nsha, const shell_t* ax, double* out) {
  int* off = (int*)malloc(sizeof(int) * nsh);
  int* offa = (int*)malloc(sizeof(int) * nsha);
  const int n = shell_offsets(nsh, sh, off);
  const int naux = shell_offsets(nsha, ax, offa);
  etab_t* E = (etab_t*)malloc(sizeof(etab_t) * 3);
  htab_t* H1 = (htab_t*)malloc(sizeof(htab_t) * NCMAX * NCMAX);
  htab_t* H2 = (htab_t*)malloc(sizeof(htab_t) * NCMAX);
  rtab_t* R = (rtab_t*)malloc(sizeof(rtab_t));
  double* blk = (double*)malloc(sizeof(double) * NCMAX * NCMAX * NCMAX);
  for (int A = 0; A < nsh; ++A)
    for (int B = 0; B <= A; ++B) {
      const shell_t *sa = &sh[A], *sb = &sh[B];
      int ca[NCMAX][3], cb[NCMAX][3];
      cart_list(sa->l, ca);
      cart_list(sb->l, cb);
      const int na = ncart(sa->l), nb = ncart(sb->l);
      for (int Q = 0; Q < nsha; ++Q) {
        const shell_t* sq = &ax[Q];
        int cq[NCMAX][3];
        cart_list(sq->l, cq);
        const int nq = ncart(sq->l), L = sa->l + sb->l + sq->l;
        memset(blk, 0, sizeof(double) * na * nb * nq);
        for (int pa = 0; pa < sa->nprim; ++pa)
          for (int pb = 0; pb < sb->nprim; ++pb) {
            double P1[3], p;
            pair_hermite(sa, pa, sb, pb, E, H1, P1, &p);
            const double cab = sa->c[pa] * sb->c[pb];
            for (int pq = 0; pq < sq->nprim; ++pq) {
              double P2[3], q;
              pair_hermite(sq, pq, NULL, 0, E, H2, P2, &q);
              hermite_r(L, p * q / (p + q), P1[0] - P2[0], P1[1] - P2[1], P1[2] - P2[2], *R);
              const double pref = cab * sq->c[pq] * 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q));
              for (int i = 0; i < na; ++i)
                for (int j = 0; j < nb; ++j) {
                  const int e1[3] = {ca[i][0] + cb[j][0], ca[i][1] + cb[j][1], ca[i][2] + cb[j][2]};
                  for (int k = 0; k < nq; ++k)
                    blk[(i * nb + j) * nq + k] +=
                        pref * hermite_contract((const double(*)[NH][NH])H1[i * nb + j], e1,
                                                (const double(*)[NH][NH])H2[k], cq[k], (const double(*)[NR][NR])*R);
                }
            }
          }
        for (int i = 0; i < na; ++i)
          for (int j = 0; j < nb; ++j)
            for (int k = 0; k < nq; ++k) {
              const double v = blk[(i * nb + j) * nq + k];
              out[((size_t)(off[A] + i) * n + off[B] + j) * naux + offa[Q] + k] = v;
              out[((size_t)(off[B] + j) * n + off[A] + i) * naux + offa[Q] + k] = v;
            }
      }
    }
  free(blk);
  free(R);
  free(H2);
  free(H1);
  free(E);
  free(offa);
  free(off);
  return n;
}
