// QP equation on a real frequency grid, shared by the imaginary-axis path (after
// the continuation) and the contour-deformation path (Sigma evaluated there):
// find_qp_energy_linearization (src/m_selfenergy_tools.f90:202-249) and
// find_qp_energy_graphical with find_fixed_point (:253-420) for one state.
#pragma once
#include "common.cuh"

namespace rigw {

// ``sr`` holds Sigma at the 2h+1 points se%omega_j = omega0 + step (j - h)
// shifted by se%energy0 = se_e0, i.e. at x_j = se%omega_j + se_e0, as
// interleaved (re, im) pairs.  Imaginary-axis path: omega0 = efermi, se_e0 = 0;
// contour path: omega0 = 0, se_e0 = the mean-field energy.  e0 is the
// mean-field energy, xc = Sigma_x - V_xc.  Writes q[0..3] = graphical QP energy,
// linearized QP energy, graphical Z, linearized Z.
RIGW_DEVICE_INLINE void qp_on_real_grid(const double* sr, int h, double omega0, double step, double se_e0,
                                        double e0, double xc, double* q) {
  const int nreal = 2 * h + 1;
  double eqp_z, zlin;
  if (h > 0) {
    const double w_p = omega0 + step * 1.0, w_m = omega0 - step * 1.0;
    double z = (sr[2 * (h + 1)] - sr[2 * (h - 1)]) / (w_p - w_m);
    z = 1.0 / (1.0 - z);
    z = fmin(fmax(z, 0.0), 1.0);
    zlin = z;
    eqp_z = se_e0 + z * (e0 - se_e0 + sr[2 * h] + xc);
  } else {
    zlin = 1.0;
    eqp_z = e0 + sr[2 * h] + xc;
  }
  double eqp_g, zg;
  if (h > 0) {
    // up to four crossings of x and Sigma(x) + xc + e0, ranked by spectral weight
    double zw[4] = {-1.0, -1.0, -1.0, -1.0};
    double ef[4] = {0.0, 0.0, 0.0, 0.0};
    double xprev = omega0 + step * (0 - h) + se_e0;
    double fprev = sr[0] + xc + e0;
    for (int j = 1; j < nreal; ++j) {
      const double x = omega0 + step * (j - h) + se_e0;
      const double f = sr[2 * j] + xc + e0;
      const double g0 = fprev - xprev, g1 = f - x;
      if (g0 * g1 < 0.0) {
        const double zz = 1.0 / (1.0 - (f - fprev) / (x - xprev));
        if (zz >= 0.00001 && zz > zw[3]) {
          int jf = 0;
          while (!(zz > zw[jf])) ++jf;
          for (int m = 3; m > jf; --m) {
            zw[m] = zw[m - 1];
            ef[m] = ef[m - 1];
          }
          zw[jf] = zz;
          const double gp = (g1 - g0) / (x - xprev);
          ef[jf] = xprev - g0 / gp;
        }
      }
      xprev = x;
      fprev = f;
    }
    int iq = 0;
    for (int m = 1; m < 4; ++m)
      if (zw[m] > zw[iq]) iq = m;
    if (zw[iq] > 1.0e-6) {
      eqp_g = ef[iq];
      zg = zw[iq];
    } else {
      eqp_g = e0;
      zg = 1.0;
    }
    int nfixed = 0;
    for (int m = 0; m < 4; ++m) nfixed += zw[m] > 0.0;
    if (nfixed == 0) eqp_g = e0 + sr[2 * h] + xc;
  } else {
    eqp_g = e0 + sr[2 * h] + xc;
    zg = 1.0;
  }
  q[0] = eqp_g;
  q[1] = eqp_z;
  q[2] = zg;
  q[3] = zlin;
}

}  // namespace rigw
