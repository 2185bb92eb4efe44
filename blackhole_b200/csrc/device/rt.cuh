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

// ---- FP32 variants (the mixed-precision transfer) ------------------------------
//
// The same physics in FP32 with the emission and the source function carried
// as logarithms: ln j = ln n_e + ln nu_B + J (J the table value), Kirchhoff
// alpha = j / B_nu, so the observed source function g^3 B_nu and the
// observed opacity alpha / g never leave the FP32 exponent range (j itself
// reaches 1e-40 and below, under FP32's normal range).

namespace bhrt {

struct MediumF {
  const float4 *cells;
  const float *lut;
  int n_r, n_th, n_ph, n_lt, n_lx;
  float r_min, r_max, fr_scale;  // (n_r - 1) / log(r_max / r_min)
  float lt0, lt_scale, lx0, lx1, lx_scale;
  float ln_nu, ln_len, ds_max, min_transmit;
  float x_coef;        // h nu / (m_e c^2): x = x_coef / (g Theta_e)
  float ln_nub_gauss;  // ln(e / (2 pi m_e c)): ln nu_B per ln gauss
  float ln_2h_c2;      // ln(2 h / c^2)
};

__host__ __device__ inline MediumF medium_f(const BhkRtParams &q) {
  MediumF m;
  m.cells = reinterpret_cast<const float4 *>(q.cells);
  m.lut = q.lut;
  m.n_r = q.n_r;
  m.n_th = q.n_th;
  m.n_ph = q.n_ph;
  m.n_lt = q.n_lt;
  m.n_lx = q.n_lx;
  m.r_min = (float)q.r_min;
  m.r_max = (float)q.r_max;
  m.fr_scale = (float)(q.inv_log_range * (double)(q.n_r - 1));
  m.lt0 = (float)q.lt0;
  m.lt_scale = (float)((double)(q.n_lt - 1) / (q.lt1 - q.lt0));
  m.lx0 = (float)q.lx0;
  m.lx1 = (float)q.lx1;
  m.lx_scale = (float)((double)(q.n_lx - 1) / (q.lx1 - q.lx0));
  m.ln_nu = (float)log(q.nu);
  m.ln_len = (float)log(q.length_cm);
  m.ds_max = (float)q.ds_max;
  m.min_transmit = (float)q.min_transmit;
  m.x_coef = (float)(kH * q.nu / (kMe * kC * kC));
  m.ln_nub_gauss = (float)log(kE / (kTwoPi * kMe * kC));
  m.ln_2h_c2 = (float)log(2.0 * kH / (kC * kC));
  return m;
}

#ifdef __CUDACC__
__device__ __forceinline__ bool sample_f(const MediumF &q, float r, float u, float phi, float &n, float &th,
                                         float &b) {
  if (!(r >= q.r_min && r <= q.r_max)) return false;
  const float fr = __logf(r / q.r_min) * q.fr_scale;
  const int i0 = min(max((int)floorf(fr), 0), q.n_r - 2);
  const float tr = fminf(fmaxf(fr - (float)i0, 0.0f), 1.0f);
  const float theta = acosf(fminf(fmaxf(u, -1.0f), 1.0f));
  const float ft = theta * (0.31830988618f * (float)q.n_th) - 0.5f;
  const int j0 = min(max((int)floorf(ft), 0), q.n_th - 2);
  const float tt = fminf(fmaxf(ft - (float)j0, 0.0f), 1.0f);
  const float fp = phi * (0.15915494309f * (float)q.n_ph);
  const float fl = floorf(fp);
  const float tp = fp - fl;
  int k0 = (int)fmodf(fl, (float)q.n_ph);
  if (k0 < 0) k0 += q.n_ph;
  const int k1 = (k0 + 1 == q.n_ph) ? 0 : k0 + 1;
  float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        const float w = (di ? tr : 1.0f - tr) * (dj ? tt : 1.0f - tt) * (dk ? tp : 1.0f - tp);
        const float4 v = __ldg(q.cells + ((long long)(i0 + di) * q.n_th + (j0 + dj)) * q.n_ph + (dk ? k1 : k0));
        a0 = fmaf(w, v.x, a0);
        a1 = fmaf(w, v.y, a1);
        a2 = fmaf(w, v.z, a2);
      }
  n = a0;
  th = a1;
  b = a2;
  return true;
}

// FP32 redshift of the circular-orbit emitter (see redshift above).
__device__ __forceinline__ float redshift_f(float a, float r, float u, float lam) {
  const float u2 = u * u;
  const float s2 = (1.0f - u) * (1.0f + u);
  const float sig = fmaf(r, r, a * a * u2);
  const float delta = fmaf(r, r - 2.0f, a * a);
  const float rr = fmaf(r, r, a * a);
  const float A = fmaf(rr, rr, -a * a * delta * s2);
  const float om = 1.0f / fmaf(r, sqrtf(r), a);
  const float inv_sig = 1.0f / sig;
  const float gtt = -(1.0f - 2.0f * r * inv_sig);
  const float gtp = -2.0f * a * r * s2 * inv_sig;
  const float gpp = A * s2 * inv_sig;
  const float norm = -(gtt + om * fmaf(gpp, om, 2.0f * gtp));
  if (!(norm > 0.0f)) return 0.0f;
  const float den = (1.0f - om * lam) * rsqrtf(norm);
  return den > 0.0f ? 1.0f / den : 0.0f;
}

// ln(j_obs) - ln(S_obs) and ln(S_obs) of one sample: S_obs = g^3 B_nu(nu/g),
// alpha_obs = (j / B_nu) / g. Returns false where there is no emission.
__device__ __forceinline__ bool ln_emission_f(const MediumF &q, float n, float theta_e, float b, float g,
                                              float &ln_alpha_obs, float &ln_s_obs) {
  if (!(n > 0.0f && theta_e > 0.0f && b > 0.0f && g > 0.0f)) return false;
  const float ln_g = __logf(g);
  const float ln_nu_e = q.ln_nu - ln_g;
  const float ln_nub = __logf(b) + q.ln_nub_gauss;
  const float lt = __logf(theta_e);
  const float lx = ln_nu_e - 0.40546511f - ln_nub - 2.0f * lt;  // ln(nu_e / nu_s), nu_s = 3/2 nu_B Theta^2
  if (lx > q.lx1) return false;
  const float ft = fminf(fmaxf((lt - q.lt0) * q.lt_scale, 0.0f), (float)(q.n_lt - 1));
  const float fx = fminf(fmaxf((lx - q.lx0) * q.lx_scale, 0.0f), (float)(q.n_lx - 1));
  const int i0 = min((int)ft, q.n_lt - 2), k0 = min((int)fx, q.n_lx - 2);
  const float ti = ft - (float)i0, tk = fx - (float)k0;
  const float *L = q.lut + i0 * q.n_lx + k0;
  const float J = (1.0f - ti) * fmaf(tk, __ldg(L + 1) - __ldg(L), __ldg(L)) +
                  ti * fmaf(tk, __ldg(L + q.n_lx + 1) - __ldg(L + q.n_lx), __ldg(L + q.n_lx));
  const float ln_j = __logf(n) + ln_nub + J;
  // ln B_nu(nu_e, T) = ln(2 h / c^2) + 3 ln nu_e - ln(e^x - 1), x = h nu_e / (k T) = x_coef / (g Theta_e)
  const float x = __fdividef(q.x_coef, g * theta_e);
  const float ln_em1 = x > 20.0f ? x : __logf(expm1f(x));
  const float ln_bnu = q.ln_2h_c2 + 3.0f * ln_nu_e - ln_em1;
  ln_alpha_obs = ln_j - ln_bnu - ln_g;
  ln_s_obs = 3.0f * ln_g + ln_bnu;
  return true;
}
#endif

}  // namespace bhrt
