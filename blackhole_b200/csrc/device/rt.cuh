// rt.cuh - the medium and the emission of the along-ray radiative transfer
// (FP64, device): grid sampling, the emitter's redshift, thermal synchrotron
// emission and absorption, and one front-to-back segment of the formal
// solution.
//
// Physics restated from the reference: synchrotronThermalEmissivity /
// synchrotronThermalAbsorption (src/physics/rte_integrator.h:291-356:
// Mahadevan 1996 with K_2(1/Theta) ~ 2 Theta^2, the branch the reference
// builds without Boost), planckFunction (:221-230), grTransformEmission /
// Absorption (:480-512: j g^2, alpha / g), rteStep (:138-187: exact for
// constant coefficients, (1 - e^-tau) ~ tau (1 - tau/2) below tau = 1e-4),
// here in front-to-back form (I += T S (1 - e^-tau), T *= e^-tau), the
// reference GPU kernel's order (src/cuda/device_physics.cuh:1988-2173).
#pragma once

#include "launch.h"

namespace bhrt {

constexpr double kE = 4.80320425e-10;     // esu
constexpr double kMe = 9.1093837015e-28;  // g
constexpr double kC = 2.99792458e10;      // cm / s
constexpr double kKb = 1.380649e-16;      // erg / K
constexpr double kH = 6.62607015e-27;     // erg s (2 pi hbar)
constexpr double kTwoPi = 6.283185307179586;

// Trilinear (n_e, Theta_e, |B|) at (r, theta, phi); false outside [r_min, r_max].
__device__ __forceinline__ bool sample(const BhkRtParams &q, double r, double u, double phi, double &n, double &th,
                                       double &b) {
  if (!(r >= q.r_min && r <= q.r_max)) return false;
  const double fr = (log(r / q.r_min) * q.inv_log_range) * (double)(q.n_r - 1);
  int i0 = (int)floor(fr);
  i0 = i0 < 0 ? 0 : (i0 > q.n_r - 2 ? q.n_r - 2 : i0);
  double tr = fr - (double)i0;
  tr = tr < 0.0 ? 0.0 : (tr > 1.0 ? 1.0 : tr);
  const double theta = acos(u < -1.0 ? -1.0 : (u > 1.0 ? 1.0 : u));
  const double ft = (theta * (1.0 / 3.141592653589793)) * (double)q.n_th - 0.5;
  int j0 = (int)floor(ft);
  j0 = j0 < 0 ? 0 : (j0 > q.n_th - 2 ? q.n_th - 2 : j0);
  double tt = ft - (double)j0;
  tt = tt < 0.0 ? 0.0 : (tt > 1.0 ? 1.0 : tt);
  const double fp = (phi * (1.0 / kTwoPi)) * (double)q.n_ph;
  const double fl = floor(fp);
  const double tp = fp - fl;
  long long k0 = (long long)fl % q.n_ph;
  if (k0 < 0) k0 += q.n_ph;
  const long long k1 = (k0 + 1) % q.n_ph;
  const float4 *c = reinterpret_cast<const float4 *>(q.cells);
  double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        const double w = (di ? tr : 1.0 - tr) * (dj ? tt : 1.0 - tt) * (dk ? tp : 1.0 - tp);
        const long long idx = ((long long)(i0 + di) * q.n_th + (j0 + dj)) * q.n_ph + (dk ? k1 : k0);
        const float4 v = __ldg(c + idx);
        acc[0] = acc[0] + w * (double)v.x;
        acc[1] = acc[1] + w * (double)v.y;
        acc[2] = acc[2] + w * (double)v.z;
      }
  n = acc[0];
  th = acc[1];
  b = acc[2];
  return true;
}

// Redshift nu_obs / nu_emit of an emitter on a circular orbit of angular
// velocity Omega = 1 / (r^(3/2) + a) at (r, theta) for a photon of lambda;
// 0 where that orbit is not timelike.
__device__ __forceinline__ double redshift(double a, double r, double u, double lam) {
  const double u2 = u * u;
  const double s2 = (1.0 - u) * (1.0 + u);
  const double sig = r * r + a * a * u2;
  const double delta = r * r - 2.0 * r + a * a;
  const double A = (r * r + a * a) * (r * r + a * a) - a * a * delta * s2;
  const double om = 1.0 / (r * sqrt(r) + a);
  const double gtt = -(1.0 - 2.0 * r / sig);
  const double gtp = -2.0 * a * r * s2 / sig;
  const double gpp = A * s2 / sig;
  const double norm = -(gtt + 2.0 * gtp * om + gpp * om * om);
  if (!(norm > 0.0)) return 0.0;
  const double ut = 1.0 / sqrt(norm);
  const double den = ut * (1.0 - om * lam);
  return den > 0.0 ? 1.0 / den : 0.0;
}

// Planck B_nu(T) (reference planckFunction).
__device__ __forceinline__ double planck(double nu, double temp) {
  const double x = (kH * nu) / (kKb * temp);
  const double den = (x > 500.0) ? exp(x) : expm1(x);
  if (!(den > 0.0)) return 0.0;
  return (2.0 * kH * nu * nu * nu / (kC * kC)) / den;
}

// Emission and absorption in the emitter's frame at frequency nu_e (the
// table holds ln(j / (n_e nu_B)), interpolated bilinearly).
__device__ __forceinline__ void synchrotron(const BhkRtParams &q, double n, double theta_e, double b, double nu_e,
                                            double &j, double &alpha) {
  j = 0.0;
  alpha = 0.0;
  if (!(n > 0.0 && theta_e > 0.0 && b > 0.0 && nu_e > 0.0)) return;
  const double nu_b = kE * b / (kTwoPi * kMe * kC);
  const double nu_s = 1.5 * nu_b * theta_e * theta_e;
  const double lx = log(nu_e / nu_s);
  if (lx > q.lx1) return;  // beyond the table: exp(-1.89 x^(1/3)) below any use
  const double lt = log(theta_e);
  double ft = (lt - q.lt0) / (q.lt1 - q.lt0) * (double)(q.n_lt - 1);
  double fx = (lx - q.lx0) / (q.lx1 - q.lx0) * (double)(q.n_lx - 1);
  ft = ft < 0.0 ? 0.0 : (ft > (double)(q.n_lt - 1) ? (double)(q.n_lt - 1) : ft);
  fx = fx < 0.0 ? 0.0 : (fx > (double)(q.n_lx - 1) ? (double)(q.n_lx - 1) : fx);
  int i0 = (int)floor(ft), k0 = (int)floor(fx);
  i0 = i0 > q.n_lt - 2 ? q.n_lt - 2 : i0;
  k0 = k0 > q.n_lx - 2 ? q.n_lx - 2 : k0;
  const double ti = ft - (double)i0, tk = fx - (double)k0;
  const float *L = q.lut;
  const double v00 = (double)__ldg(L + i0 * q.n_lx + k0), v01 = (double)__ldg(L + i0 * q.n_lx + k0 + 1);
  const double v10 = (double)__ldg(L + (i0 + 1) * q.n_lx + k0), v11 = (double)__ldg(L + (i0 + 1) * q.n_lx + k0 + 1);
  const double J = ((1.0 - ti) * ((1.0 - tk) * v00 + tk * v01)) + (ti * ((1.0 - tk) * v10 + tk * v11));
  j = n * nu_b * exp(J);
  const double bnu = planck(nu_e, theta_e * kMe * kC * kC / kKb);
  alpha = bnu > 0.0 ? j / bnu : 0.0;
}

}  // namespace bhrt
