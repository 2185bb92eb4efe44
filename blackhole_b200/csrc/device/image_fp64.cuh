// image_fp64.cuh - FP64 device math of the image-plane tracer.
//
// The Mino-time Kerr system of the reference's potentials
// (src/physics/kerr.cpp:69-97: R(r) = A^2 - Delta (q + (Lz - a E)^2),
// Theta = q + a^2 E^2 cos^2 - Lz^2 / sin^2) in second-order form with
// u = cos(theta) and E = 1:
//   r'  = p_r          p_r' = R'(r)/2 = 2 r A - (r - 1) K,  K = q_R + (lambda - a)^2
//   u'  = p_u          p_u' = U'(u)/2 = u (a^2 - q_Th - 2 a^2 u^2),
//                      U(u) = sin^2 Theta = (q_Th + a^2 u^2)(1 - u^2) - lambda^2
//   psi' = a - lambda / sin^2 - a (A + p_r) / Delta  (psi = phi - a G(r), G' = 1/Delta:
//          kerr.cpp:61 time-reversed, made regular at the horizon)
// Every expression is written in a fixed evaluation order and the translation
// units that include this header are compiled with -fmad=false, so each FP64
// operation rounds exactly once, as on the CPU: results are bit-identical to
// a host build of the same arithmetic.
#pragma once

#include "launch.h"

namespace bhk {

struct RayC {
  double a, a2, lam, qTh, K;
};

struct Yd {
  double r, u, phi, pr, pu;
};

__device__ __forceinline__ double dmax_(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin_(double a, double b) { return (b < a) ? b : a; }

__device__ __forceinline__ Yd rhs(const Yd &y, const RayC &c) {
  const double r = y.r, u = y.u;
  const double A = ((r * r) + c.a2) - (c.a * c.lam);
  const double D = ((r * r) - (2.0 * r)) + c.a2;
  const double u2 = u * u;
  const double s2 = dmax_(1.0 - u2, 1e-12);
  Yd d;
  d.r = y.pr;
  d.u = y.pu;
  d.pr = ((2.0 * r) * A) - ((r - 1.0) * c.K);
  d.pu = u * ((c.a2 - c.qTh) - ((2.0 * c.a2) * u2));
  // horizon-regular azimuth psi = phi - a G(r), G' = 1/Delta: psi' = a -
  // lambda/sin^2 - a (A + p_r)/Delta, with (A + p_r)/Delta = K/(A - p_r) on
  // the first integral for ingoing rays (the rationalization of the
  // reference's GPU step, src/cuda/device_physics.cuh:453-525)
  const bool in = y.pr < 0.0;
  const double num = in ? c.K : (A + y.pr);
  const double den = in ? (A - y.pr) : D;
  d.phi = (c.a - (c.lam / s2)) - (c.a * (num / den));
  return d;
}

// phi = psi + a (G(r) - G(r_obs)), G(r) = ln((r - r+)/(r - r-)) / (r+ - r-).
__device__ __forceinline__ double phi_of_psi(double psi, double r, const BhkImageParams &p) {
  if (p.a == 0.0) return psi;
  const double q = ((r - p.r_plus) * (p.r_obs - p.r_minus)) / ((r - p.r_minus) * (p.r_obs - p.r_plus));
  return psi + p.a * (log(q) / (p.r_plus - p.r_minus));
}

__device__ __forceinline__ Yd axpy(const Yd &y, double h, const Yd &k) {
  Yd o;
  o.r = y.r + h * k.r;
  o.u = y.u + h * k.u;
  o.phi = y.phi + h * k.phi;
  o.pr = y.pr + h * k.pr;
  o.pu = y.pu + h * k.pu;
  return o;
}

// R(r) with E = 1, M = 1.
__device__ __forceinline__ double pot_R(double r, const RayC &c) {
  const double A = ((r * r) + (c.a * c.a)) - (c.a * c.lam);
  const double D = ((r * r) - (2.0 * r)) + (c.a * c.a);
  return (A * A) - (D * c.K);
}

// U(u) = sin^2 Theta = (q_Th + a^2 u^2)(1 - u^2) - lambda^2.
__device__ __forceinline__ double pot_U(double u, const RayC &c) {
  const double u2 = u * u;
  return ((c.qTh + ((c.a * c.a) * u2)) * (1.0 - u2)) - (c.lam * c.lam);
}

// Threshold of the first-integral projection (R > tau r^4, U > tau (|q|+a^2)).
constexpr double kProjTau = 1e-6;

// Resets the Mino-time momenta to the first integrals p_r^2 = R(r) and
// p_u^2 = U(u), keeping their signs, where those are well conditioned (away
// from turning points). Without it the second-order form lets b^2 drift by
// ~rtol r^2 per step at r ~ 1000, where b enters R only at order b^2/r^2.
// With want_drift, returns the Carter-constant residual the projection
// removed, |eta(state) - eta| / (|q_Th| + a^2) with eta(state) - eta =
// (p_u^2 - U(u)) / (1 - u^2), where the polar momentum was projected (0 near
// a polar turning point); otherwise 0, and the division is skipped.
__device__ __forceinline__ double project(Yd &y, const RayC &c, bool want_drift = false) {
  const double Rv = pot_R(y.r, c);
  const double r2 = y.r * y.r;
  if (Rv > kProjTau * (r2 * r2)) {
    const double m = sqrt(Rv);
    y.pr = (y.pr < 0.0) ? -m : m;
  }
  const double Uv = pot_U(y.u, c);
  const double scale = fabs(c.qTh) + (c.a * c.a);
  double drift = 0.0;
  if (Uv > kProjTau * scale) {
    if (want_drift) drift = fabs((y.pu * y.pu) - Uv) / ((1.0 - (y.u * y.u)) * scale);
    const double m = sqrt(Uv);
    y.pu = (y.pu < 0.0) ? -m : m;
  }
  return drift;
}

// Classical RK4 step of size h (k1 = rhs(y) given).
__device__ __forceinline__ Yd rk4(const Yd &y, double h, const RayC &c, const Yd &k1) {
  const double hh = 0.5 * h;
  const Yd k2 = rhs(axpy(y, hh, k1), c);
  Yd s;
  s.r = k1.r + 2.0 * k2.r;
  s.u = k1.u + 2.0 * k2.u;
  s.phi = k1.phi + 2.0 * k2.phi;
  s.pr = k1.pr + 2.0 * k2.pr;
  s.pu = k1.pu + 2.0 * k2.pu;
  const Yd k3 = rhs(axpy(y, hh, k2), c);
  s.r = s.r + 2.0 * k3.r;
  s.u = s.u + 2.0 * k3.u;
  s.phi = s.phi + 2.0 * k3.phi;
  s.pr = s.pr + 2.0 * k3.pr;
  s.pu = s.pu + 2.0 * k3.pu;
  const Yd k4 = rhs(axpy(y, h, k3), c);
  const double w = h / 6.0;
  Yd n;
  n.r = y.r + w * (s.r + k4.r);
  n.u = y.u + w * (s.u + k4.u);
  n.phi = y.phi + w * (s.phi + k4.phi);
  n.pr = y.pr + w * (s.pr + k4.pr);
  n.pu = y.pu + w * (s.pu + k4.pu);
  return n;
}

// Dormand & Prince (1980) 5(4) coefficients.
namespace dp {
constexpr double a21 = 1.0 / 5.0;
constexpr double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
constexpr double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
constexpr double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0, a53 = 64448.0 / 6561.0, a54 = -212.0 / 729.0;
constexpr double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0, a64 = 49.0 / 176.0,
                 a65 = -5103.0 / 18656.0;
constexpr double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0, b5 = -2187.0 / 6784.0,
                 b6 = 11.0 / 84.0;
constexpr double e1 = 35.0 / 384.0 - 5179.0 / 57600.0;
constexpr double e3 = 500.0 / 1113.0 - 7571.0 / 16695.0;
constexpr double e4 = 125.0 / 192.0 - 393.0 / 640.0;
constexpr double e5 = -2187.0 / 6784.0 + 92097.0 / 339200.0;
constexpr double e6 = 11.0 / 84.0 - 187.0 / 2100.0;
constexpr double e7 = -1.0 / 40.0;
}  // namespace dp

struct DPRes {
  Yd y5;
  Yd k7;
  double err;
};

// One Dormand-Prince attempt of size h from y with k1 = rhs(y). With
// want_err the FSAL stage k7 = rhs(y5) and the scaled RMS error over the five
// components, sc_i = atol + rtol max(|y_i|, |y5_i|), are returned.
__device__ __forceinline__ DPRes dp45(const Yd &y, double h, const RayC &c, const Yd &k1, double rtol,
                                      double atol, bool want_err) {
  Yd s;
  s = axpy(y, h * dp::a21, k1);
  const Yd k2 = rhs(s, c);
  s = axpy(axpy(y, h * dp::a31, k1), h * dp::a32, k2);
  const Yd k3 = rhs(s, c);
  s = axpy(axpy(axpy(y, h * dp::a41, k1), h * dp::a42, k2), h * dp::a43, k3);
  const Yd k4 = rhs(s, c);
  s = axpy(axpy(axpy(axpy(y, h * dp::a51, k1), h * dp::a52, k2), h * dp::a53, k3), h * dp::a54, k4);
  const Yd k5 = rhs(s, c);
  s = axpy(axpy(axpy(axpy(axpy(y, h * dp::a61, k1), h * dp::a62, k2), h * dp::a63, k3), h * dp::a64, k4),
           h * dp::a65, k5);
  const Yd k6 = rhs(s, c);
  DPRes o;
  o.y5 = axpy(axpy(axpy(axpy(axpy(y, h * dp::b1, k1), h * dp::b3, k3), h * dp::b4, k4), h * dp::b5, k5),
              h * dp::b6, k6);
  o.err = 0.0;
  if (!want_err) {
    o.k7 = k1;
    return o;
  }
  o.k7 = rhs(o.y5, c);
#define BHK_ECOMP(f)                                                                                    \
  (h * ((((((dp::e1 * k1.f) + (dp::e3 * k3.f)) + (dp::e4 * k4.f)) + (dp::e5 * k5.f)) + (dp::e6 * k6.f)) + \
        (dp::e7 * o.k7.f)))
#define BHK_SC(f) (atol + rtol * dmax_(fabs(y.f), fabs(o.y5.f)))
  const double q0 = BHK_ECOMP(r) / BHK_SC(r);
  const double q1 = BHK_ECOMP(u) / BHK_SC(u);
  const double q2 = BHK_ECOMP(phi) / BHK_SC(phi);
  const double q3 = BHK_ECOMP(pr) / BHK_SC(pr);
  const double q4 = BHK_ECOMP(pu) / BHK_SC(pu);
#undef BHK_ECOMP
#undef BHK_SC
  o.err = sqrt(((((q0 * q0) + (q1 * q1)) + (q2 * q2)) + (q3 * q3) + (q4 * q4)) / 5.0);
  return o;
}

// x^(-1/5) for finite x > 0 with frexp/ldexp (exact) and correctly rounded
// arithmetic: x = m 2^e, e = 5k + j, z = m 2^j in [0.5, 16); Newton's
// iteration y <- y (6 - z y^5) / 5 from 2^(-j/5) rises monotonically to
// z^(-1/5). Free of libm, so host and device give the same bits.
__device__ __forceinline__ double inv_fifth_root(double x) {
  int e = 0;
  const double m = frexp(x, &e);
  int k = e / 5;
  int j = e - 5 * k;
  if (j < 0) {
    j += 5;
    k -= 1;
  }
  const double z = ldexp(m, j);
  double y = (j == 0)   ? 1.0
             : (j == 1) ? 0.87055056329612412
             : (j == 2) ? 0.75785828325519899
             : (j == 3) ? 0.65975395538644710
                        : 0.57434917749851755;
#pragma unroll
  for (int it = 0; it < 6; ++it) {
    const double y2 = y * y;
    const double y5 = (y2 * y2) * y;
    y = (y * (6.0 - (z * y5))) / 5.0;
  }
  return ldexp(y, -k);
}

// Step factor of the Hairer-Norsett-Wanner controller (safety 0.9, bounds
// [0.1, 2] after acceptance, [0.1, 1] after rejection).
__device__ __forceinline__ double step_factor(double err, bool accepted) {
  const double hi = accepted ? 2.0 : 1.0;
  if (!(err < 1e300)) return 0.1;
  if (!(err > 0.0)) return hi;
  const double f = 0.9 * inv_fifth_root(err);
  return (f < 0.1) ? 0.1 : ((hi < f) ? hi : f);
}

// Keplerian prograde emitter (Bardeen, Press & Teukolsky 1972):
// g = sqrt(x^3 (x^3 - 3x + 2a)) / (x^3 + a - lambda), x = sqrt(r).
__device__ __forceinline__ double disk_g(double r, double a, double lam) {
  const double x = sqrt(r);
  const double x3 = (x * x) * x;
  const double v = x3 * ((x3 - (3.0 * x)) + (2.0 * a));
  if (v <= 0.0) return 0.0;
  return sqrt(v) / ((x3 + a) - lam);
}

// NovikovThorneDisk::normalizedFlux (src/physics/novikov_thorne.h:170-190)
// with its scene constants r_isco and flux(1.5 r_isco) precomputed.
__device__ __forceinline__ double nt_flux(double r, double r_isco, double flux_peak) {
  if (r < r_isco) return 0.0;
  const double t = 1.0 - sqrt(r_isco / r);
  const double fR = (0.0 < t) ? t : 0.0;
  const double flux = fR / ((r * r) * r);
  const double v = flux / flux_peak;
  return (v < 1.0) ? v : 1.0;
}

}  // namespace bhk
