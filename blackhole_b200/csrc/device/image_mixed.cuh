// image_mixed.cuh - mixed-precision device math of the image-plane tracer.
//
// Same Mino-time second-order system as image_fp64.cuh, evaluated in FP32:
//   p_r' = 2 r A - (r - 1) K, p_u' = u (a^2 - q_Th - 2 a^2 u^2),
//   psi' = a - lambda / sin^2 - a (A + p_r) / Delta (horizon-regular azimuth,
// rationalized for ingoing rays; both quotients share one division). Positions r, u, phi carry an
// FP32 compensation term (TwoSum), so the accumulated position keeps ~48
// bits while each step's increment is computed in FP32; the momenta are
// reset to the first integrals every accepted step (projection), so they
// never accumulate. FP64 is used for the per-ray set-up (constants of
// motion, initial momenta) and for the outputs (crossing radius, g).
#pragma once

#include "launch.h"

namespace bhm {

struct RayCf {
  float a, a2, lam, qTh, K;
  float a2_minus_alam;   // a^2 - a lambda
  float c_pu;            // a^2 - q_Th
};

struct Yf {
  float r, u, phi, pr, pu;
};

struct Lof {
  float r, u, phi;  // compensation terms of the positions
};

__device__ __forceinline__ Yf rhs(const Yf &y, const RayCf &c) {
  const float r = y.r, u = y.u;
  const float A = fmaf(r, r, c.a2_minus_alam);
  const float D = fmaf(r, r - 2.0f, c.a2);
  const float u2 = u * u;
  const float s2 = fmaxf((1.0f - u) * (1.0f + u), 1e-12f);  // no cancellation near the poles
  Yf d;
  d.r = y.pr;
  d.u = y.pu;
  d.pr = fmaf(2.0f * r, A, -(r - 1.0f) * c.K);
  d.pu = u * fmaf(-2.0f * c.a2, u2, c.c_pu);
  // psi' = a - lambda/s2 - a num/den (image_fp64.cuh), as one quotient:
  // (s2 a (den - num) - lambda den) / (s2 den)
  const bool in = y.pr < 0.0f;
  const float num = in ? c.K : (A + y.pr);
  const float den = in ? (A - y.pr) : D;
  d.phi = __fdividef(fmaf(s2, c.a * (den - num), -c.lam * den), s2 * den);
  return d;
}

__device__ __forceinline__ Yf axpy(const Yf &y, float h, const Yf &k) {
  Yf o;
  o.r = fmaf(h, k.r, y.r);
  o.u = fmaf(h, k.u, y.u);
  o.phi = fmaf(h, k.phi, y.phi);
  o.pr = fmaf(h, k.pr, y.pr);
  o.pu = fmaf(h, k.pu, y.pu);
  return o;
}

__device__ __forceinline__ float pot_R(float r, const RayCf &c) {
  const float A = fmaf(r, r, c.a2_minus_alam);
  const float D = fmaf(r, r - 2.0f, c.a2);
  return fmaf(A, A, -D * c.K);
}

__device__ __forceinline__ float pot_U(float u, const RayCf &c) {
  const float u2 = u * u;
  return fmaf(fmaf(c.a2, u2, c.qTh), 1.0f - u2, -c.lam * c.lam);
}

// Constants of motion in FP64 for the first-integral projection.
struct RayCd {
  double a, lam, qTh, K;
};

constexpr double kProjTau = 1e-6;

// First-integral projection (see image_fp64.cuh) with R and U evaluated in
// FP64 from the compensated positions. In FP32 both potentials carry an
// absolute error ~1e-7 of their largest term (A^2, resp. q + a^2), which near
// a turning point, where R ~ 1e-4 r^4, would already move p_r by 4e-4; in
// FP64 the reset is exact at the 1e-6 threshold of the FP64 path. Only the
// square root's argument is FP64: the result is rounded to FP32 once.
// With want_drift, returns the Carter-constant residual the projection
// removed, |eta(state) - eta| / (|q_Th| + a^2) with eta(state) - eta =
// (p_u^2 - U(u)) / (1 - u^2), where the polar momentum was projected (0 near
// a polar turning point): the difference in FP64 (p_u^2 and U nearly
// cancel), the quotient in FP32; otherwise 0.
__device__ __forceinline__ float project(Yf &y, const Lof &lo, const RayCd &c, bool want_drift = false) {
  const double r = (double)y.r + (double)lo.r;
  const double u = (double)y.u + (double)lo.u;
  const double A = r * r + c.a * c.a - c.a * c.lam;
  const double D = r * r - 2.0 * r + c.a * c.a;
  const double Rv = A * A - D * c.K;
  const double r2 = r * r;
  if (Rv > kProjTau * (r2 * r2)) y.pr = copysignf(sqrtf((float)Rv), y.pr);
  const double u2 = u * u;
  const double Uv = (c.qTh + c.a * c.a * u2) * (1.0 - u2) - c.lam * c.lam;
  const double scale = fabs(c.qTh) + c.a * c.a;
  float drift = 0.0f;
  if (Uv > kProjTau * scale) {
    if (want_drift) {
      const double pu = (double)y.pu;
      drift = __fdividef((float)fabs(pu * pu - Uv), (float)((1.0 - u2) * scale));
    }
    y.pu = copysignf(sqrtf((float)Uv), y.pu);
  }
  return drift;
}

// hi + lo += d (TwoSum then renormalise): exact error-free accumulation of
// an FP32 increment into a compensated FP32 pair.
__device__ __forceinline__ void comp_add(float &hi, float &lo, float d) {
  const float s = hi + d;
  const float bp = s - hi;
  const float e = (hi - (s - bp)) + (d - bp);
  const float t = lo + e;
  const float nh = s + t;
  lo = t - (nh - s);
  hi = nh;
}

__device__ __forceinline__ double to_f64(float hi, float lo) { return (double)hi + (double)lo; }

// Dormand & Prince (1980) coefficients in FP32.
namespace dpf {
constexpr float a21 = 1.0f / 5.0f;
constexpr float a31 = 3.0f / 40.0f, a32 = 9.0f / 40.0f;
constexpr float a41 = 44.0f / 45.0f, a42 = -56.0f / 15.0f, a43 = 32.0f / 9.0f;
constexpr float a51 = 19372.0f / 6561.0f, a52 = -25360.0f / 2187.0f, a53 = 64448.0f / 6561.0f,
                a54 = -212.0f / 729.0f;
constexpr float a61 = 9017.0f / 3168.0f, a62 = -355.0f / 33.0f, a63 = 46732.0f / 5247.0f, a64 = 49.0f / 176.0f,
                a65 = -5103.0f / 18656.0f;
constexpr float b1 = 35.0f / 384.0f, b3 = 500.0f / 1113.0f, b4 = 125.0f / 192.0f, b5 = -2187.0f / 6784.0f,
                b6 = 11.0f / 84.0f;
constexpr float e1 = (float)(35.0 / 384.0 - 5179.0 / 57600.0);
constexpr float e3 = (float)(500.0 / 1113.0 - 7571.0 / 16695.0);
constexpr float e4 = (float)(125.0 / 192.0 - 393.0 / 640.0);
constexpr float e5 = (float)(-2187.0 / 6784.0 + 92097.0 / 339200.0);
constexpr float e6 = (float)(11.0 / 84.0 - 187.0 / 2100.0);
constexpr float e7 = (float)(-1.0 / 40.0);
}  // namespace dpf

// Increment of one Dormand-Prince step (d = y5 - y, computed from the
// stages so that no large position is subtracted), its FSAL stage and the
// scaled RMS error.
struct DPf {
  Yf d;    // y5 - y
  Yf k7;   // rhs(y5)
  float err;
};

__device__ __forceinline__ DPf dp45(const Yf &y, float h, const RayCf &c, const Yf &k1, float rtol, float atol,
                                    bool want_err) {
  const Yf k2 = rhs(axpy(y, h * dpf::a21, k1), c);
  Yf s = axpy(axpy(y, h * dpf::a31, k1), h * dpf::a32, k2);
  const Yf k3 = rhs(s, c);
  s = axpy(axpy(axpy(y, h * dpf::a41, k1), h * dpf::a42, k2), h * dpf::a43, k3);
  const Yf k4 = rhs(s, c);
  s = axpy(axpy(axpy(axpy(y, h * dpf::a51, k1), h * dpf::a52, k2), h * dpf::a53, k3), h * dpf::a54, k4);
  const Yf k5 = rhs(s, c);
  s = axpy(axpy(axpy(axpy(axpy(y, h * dpf::a61, k1), h * dpf::a62, k2), h * dpf::a63, k3), h * dpf::a64, k4),
           h * dpf::a65, k5);
  const Yf k6 = rhs(s, c);
  DPf o;
#define BHM_INC(f) (h * fmaf(dpf::b1, k1.f, fmaf(dpf::b3, k3.f, fmaf(dpf::b4, k4.f, fmaf(dpf::b5, k5.f, dpf::b6 * k6.f)))))
  o.d.r = BHM_INC(r);
  o.d.u = BHM_INC(u);
  o.d.phi = BHM_INC(phi);
  o.d.pr = BHM_INC(pr);
  o.d.pu = BHM_INC(pu);
#undef BHM_INC
  o.err = 0.0f;
  if (!want_err) {
    o.k7 = k1;
    return o;
  }
  Yf y5;
  y5.r = y.r + o.d.r;
  y5.u = y.u + o.d.u;
  y5.phi = y.phi + o.d.phi;
  y5.pr = y.pr + o.d.pr;
  y5.pu = y.pu + o.d.pu;
  o.k7 = rhs(y5, c);
#define BHM_E(f)                                                                                          \
  (h * fmaf(dpf::e1, k1.f,                                                                               \
            fmaf(dpf::e3, k3.f, fmaf(dpf::e4, k4.f, fmaf(dpf::e5, k5.f, fmaf(dpf::e6, k6.f, dpf::e7 * o.k7.f))))))
  // Error scale: atol + rtol max(|y|, |y5|), plus a floor of 1e-7 |y5 - y|.
  // The FP32 estimate h sum e_j k_j carries rounding noise ~1e-8 |y5 - y|;
  // where rtol |y| falls below that (momenta near a turning point, phi near
  // its start value of 0) the floor keeps the controller from chasing it.
  // Near a pole, lambda / sin^2 inherits the FP32 rounding of u as a
  // relative error ~6e-8 / (1 - |u|), hence the wider floor for psi there.
#define BHM_Q(f) __fdividef(BHM_E(f), fmaf(1e-7f, fabsf(o.d.f), fmaf(rtol, fmaxf(fabsf(y.f), fabsf(y5.f)), atol)))
  const float q0 = BHM_Q(r), q1 = BHM_Q(u), q3 = BHM_Q(pr), q4 = BHM_Q(pu);
  const float pole = 1e-7f + __fdividef(1e-8f, fmaxf(1.0f - fabsf(y.u), 1e-7f));
  const float q2 = __fdividef(BHM_E(phi), fmaf(pole, fabsf(o.d.phi), fmaf(rtol, fmaxf(fabsf(y.phi), fabsf(y5.phi)), atol)));
#undef BHM_Q
#undef BHM_E
  o.err = sqrtf(0.2f * fmaf(q0, q0, fmaf(q1, q1, fmaf(q2, q2, fmaf(q3, q3, q4 * q4)))));
  return o;
}

// Classical RK4 increment (y_{n+1} - y_n) of step h.
__device__ __forceinline__ Yf rk4_inc(const Yf &y, float h, const RayCf &c, const Yf &k1) {
  const float hh = 0.5f * h;
  const Yf k2 = rhs(axpy(y, hh, k1), c);
  const Yf k3 = rhs(axpy(y, hh, k2), c);
  const Yf k4 = rhs(axpy(y, h, k3), c);
  const float w = h * (1.0f / 6.0f);
  Yf d;
  d.r = w * (k1.r + 2.0f * (k2.r + k3.r) + k4.r);
  d.u = w * (k1.u + 2.0f * (k2.u + k3.u) + k4.u);
  d.phi = w * (k1.phi + 2.0f * (k2.phi + k3.phi) + k4.phi);
  d.pr = w * (k1.pr + 2.0f * (k2.pr + k3.pr) + k4.pr);
  d.pu = w * (k1.pu + 2.0f * (k2.pu + k3.pu) + k4.pu);
  return d;
}

// Step factor 0.9 err^(-1/5) in [0.1, 2] (accepted) or [0.1, 1] (rejected).
__device__ __forceinline__ float step_factor(float err, bool accepted) {
  const float hi = accepted ? 2.0f : 1.0f;
  if (!(err < 1e30f)) return 0.1f;
  if (!(err > 0.0f)) return hi;
  const float f = 0.9f * __powf(err, -0.2f);
  return fminf(hi, fmaxf(0.1f, f));
}

}  // namespace bhm
