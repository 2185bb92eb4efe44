// analytic_api.cpp - include/bh_analytic.h: the closed-form helpers on the
// host, from the same header as the image tracer's analytic integrator
// (device/kerr_analytic.cuh compiled as C++).
#include <cmath>
#include <limits>
#include <utility>

#include "../../../include/bh_analytic.h"
#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wunknown-pragmas"  // the header's loop pragmas are for nvcc
#include "../device/kerr_analytic.cuh"
#pragma GCC diagnostic pop

namespace {
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();
}  // namespace

extern "C" {

double bh_analytic_radial_potential(double r, double a, double xi, double eta) {
  const double A = (r * r + a * a) - a * xi;
  const double D = (r * r - 2.0 * r) + a * a;
  return A * A - D * (eta + (xi - a) * (xi - a));
}

void bh_analytic_quartic_coeffs(double a, double xi, double eta, double out[3]) {
  if (!out) return;
  const double a2l = a * a - a * xi, K = eta + (xi - a) * (xi - a);
  out[0] = 2.0 * a2l - K;
  out[1] = 2.0 * K;
  out[2] = a2l * a2l - a * a * K;
}

int bh_analytic_radial_roots(double c2, double c1, double c0, double re[4], double im[4], int *motion) {
  if (!re || !im) return -1;
  double al, be, ga;
  if (!bhan::ferrari_factor(c2, c1, c0, al, be, ga)) {
    for (int k = 0; k < 4; ++k) re[k] = im[k] = kNaN;
    if (motion) *motion = BH_MOTION_INVALID;
    return -1;
  }
  // x^2 + al x + be and x^2 - al x + ga
  double rr[4], ci[4];
  int nr = 0, nc = 0;
  const double q[2][2] = {{al, be}, {-al, ga}};
  for (const auto &f : q) {
    const double disc = f[0] * f[0] - 4.0 * f[1];
    if (disc >= 0.0) {
      const double s = std::sqrt(disc);
      rr[nr++] = bhan::newton_root(c2, c1, c0, 0.5 * (-f[0] + s));
      rr[nr++] = bhan::newton_root(c2, c1, c0, 0.5 * (-f[0] - s));
    } else {
      ci[nc++] = -0.5 * f[0];
      ci[nc++] = 0.5 * std::sqrt(-disc);
    }
  }
  for (int i = 1; i < nr; ++i)  // descending
    for (int j = i; j > 0 && rr[j] > rr[j - 1]; --j) std::swap(rr[j], rr[j - 1]);
  int k = 0;
  for (int i = 0; i < nr; ++i, ++k) {
    re[k] = rr[i];
    im[k] = 0.0;
  }
  for (int i = 0; i < nc; i += 2) {
    re[k] = ci[i];
    im[k++] = ci[i + 1];
    re[k] = ci[i];
    im[k++] = -ci[i + 1];
  }
  if (motion) *motion = nr == 4 ? BH_MOTION_TRANSIT : (nr == 2 ? BH_MOTION_SCATTER : BH_MOTION_PLUNGE);
  return nr;
}

double bh_analytic_r_bound(double lambda, const double roots[4], double lambda0) {
  if (!roots) return kNaN;
  const double r1 = roots[0], r2 = roots[1], r3 = roots[2], r4 = roots[3];
  if (!(r1 >= r2 && r2 >= r3 && r3 >= r4)) return kNaN;
  const double den = (r1 - r3) * (r2 - r4);
  if (!(den > 0.0)) return kNaN;
  const double m1 = (r1 - r2) * (r3 - r4) / den;  // 1 - m without cancellation
  const double u = 0.5 * std::sqrt(den) * (lambda - lambda0);
  double sn, cn, dn;
  bhan::sncndn(u, m1, sn, cn, dn);
  const double s2 = sn * sn;
  return (r3 * (r2 - r4) - r4 * (r2 - r3) * s2) / ((r2 - r4) - (r2 - r3) * s2);
}

double bh_analytic_radial_half_period(const double roots[4]) {
  if (!roots) return kNaN;
  const double r1 = roots[0], r2 = roots[1], r3 = roots[2], r4 = roots[3];
  const double den = (r1 - r3) * (r2 - r4);
  if (!(den > 0.0) || !(r1 >= r2 && r2 >= r3 && r3 >= r4)) return kNaN;
  const double m1 = (r1 - r2) * (r3 - r4) / den;
  return bhan::carlson_rf(0.0, m1, 1.0) / (0.5 * std::sqrt(den));
}

void bh_analytic_critical_impact_params(double r_ph, double a, double out[2]) {
  if (!out) return;
  if (std::fabs(a) < 1e-15) {
    out[0] = 0.0;
    out[1] = 27.0;
    return;
  }
  const double D = r_ph * r_ph - 2.0 * r_ph + a * a, Dp = 2.0 * r_ph - 2.0;
  if (std::fabs(Dp) < 1e-15) {
    out[0] = out[1] = 0.0;
    return;
  }
  const double xi = (r_ph * r_ph + a * a) / a - 4.0 * r_ph * D / (a * Dp);
  out[0] = xi;
  out[1] = 16.0 * r_ph * r_ph * D / (Dp * Dp) - (xi - a) * (xi - a);
}

double bh_analytic_prograde_photon_orbit(double a) {
  return 2.0 * (1.0 + std::cos((2.0 / 3.0) * std::acos(-std::fabs(a))));
}

double bh_analytic_retrograde_photon_orbit(double a) {
  return 2.0 * (1.0 + std::cos((2.0 / 3.0) * std::acos(std::fabs(a))));
}

void bh_analytic_ellpj(double u, double m, double out[3]) {
  if (!out) return;
  if (!(m <= 1.0)) {
    out[0] = out[1] = out[2] = kNaN;
  } else if (m == 1.0) {
    out[0] = std::tanh(u);
    out[1] = out[2] = 1.0 / std::cosh(u);
  } else if (m >= 0.0) {
    bhan::sncndn(u, 1.0 - m, out[0], out[1], out[2]);
  } else {
    bhan::sncndn_neg(u, 1.0 - m, out[0], out[1], out[2]);
  }
}

double bh_analytic_ellint_k(double k) {
  const double m1 = 1.0 - k * k;
  if (!(m1 > 0.0)) return m1 == 0.0 ? std::numeric_limits<double>::infinity() : kNaN;
  return bhan::carlson_rf(0.0, m1, 1.0);
}

}  // extern "C"
