// kerr_oracle.hpp - CPU oracle for the Kerr geodesic tracer.
//
// TEST INFRASTRUCTURE ONLY. This is the checker the CUDA path is compared
// against; nothing in the product library links, loads or calls it.
//
// Part A restates the reference's FP64 Mino-time Kerr stepper operation for
// operation:
//   kerr_potentials   <- physics::kerrPotentials        (src/physics/kerr.cpp:69-97)
//   kerr_mino_derivs  <- kerrMinoDerivatives            (src/physics/kerr.cpp:40-66)
//   kerr_step_mino    <- physics::kerrStepMino          (src/physics/kerr.cpp:99-134)
//   kerr_trace        <- physics::KerrRaytracer::trace  (src/physics/raytracer.h:324-378)
//   horizon / ISCO / photon orbit <- src/physics/kerr.h:132-274
//   nt_normalized_flux <- NovikovThorneDisk::normalizedFlux (src/physics/novikov_thorne.h:170-190)
// Part A is pinned bit for bit against the reference's own kerr.cpp compiled
// into oracle/_ref (tests/test_oracle_ref.py).
//
// Part B is the image-plane tracer, new work built on Part A's potentials:
//   - Bardeen (1973) image-plane initial data (alpha, beta) -> (lambda, eta);
//   - the Mino-time system in second-order form, r'' = R'(r)/2 (R' is the
//     reference's dRdr, kerr.cpp:86-88) and, with u = cos(theta),
//     u'' = U'(u)/2 where U(u) = sin^2(theta) Theta(theta) is the reference's
//     Theta (kerr.cpp:89) times sin^2;
//   - classical RK4 on the affine step h = c min(r, rcap), dsigma = h / Sigma,
//     or Dormand & Prince (1980) 5(4) with the step controller of Hairer,
//     Norsett & Wanner (1993) II.4 (safety 0.9, factor in [0.1, 2]) as the
//     reference states it in src/physics/verified/rk4.h:254-265;
//   - equatorial crossings located inside the accepted step by quintic
//     Hermite interpolation, root bracketed as in event_detection.h:127-180;
//   - Keplerian redshift g = 1 / (u^t (1 - Omega lambda)) with the
//     Bardeen-Press-Teukolsky (1972) u^t and Omega (as in src/physics/iron_kline.h:25-40).
// Templated on the scalar so that a counting scalar can count its FLOPs and
// long double / __float128 can check rounding.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numbers>

#include "scalars.hpp"

namespace bho {

// ---------------------------------------------------------------------------
// Scalar helpers (overloadable for counting / extended-precision scalars)
// ---------------------------------------------------------------------------
inline double s_sqrt(double x) { return std::sqrt(x); }
inline double s_sin(double x) { return std::sin(x); }
inline double s_cos(double x) { return std::cos(x); }
inline double s_abs(double x) { return std::fabs(x); }
inline double s_acos(double x) { return std::acos(x); }
inline double s_cbrt(double x) { return std::cbrt(x); }
inline double s_pow(double x, double y) { return std::pow(x, y); }
inline double s_log(double x) { return std::log(x); }
inline double s_exp(double x) { return std::exp(x); }
inline double s_expm1(double x) { return std::expm1(x); }
inline double s_floor(double x) { return std::floor(x); }
inline double s_ceil(double x) { return std::ceil(x); }
inline long double s_sqrt(long double x) { return std::sqrt(x); }
inline long double s_sin(long double x) { return std::sin(x); }
inline long double s_cos(long double x) { return std::cos(x); }
inline long double s_abs(long double x) { return std::fabs(x); }
inline long double s_acos(long double x) { return std::acos(x); }
inline long double s_cbrt(long double x) { return std::cbrt(x); }
inline long double s_pow(long double x, long double y) { return std::pow(x, y); }

template <class T> inline T s_max(T a, T b) { return (a < b) ? b : a; }  // std::max semantics
template <class T> inline T s_min(T a, T b) { return (b < a) ? b : a; }  // std::min semantics
template <class T> inline T s_clamp(T v, T lo, T hi) {                   // std::clamp semantics
  return (v < lo) ? lo : ((hi < v) ? hi : v);
}

// CGS constants of src/physics/constants.h:23-29 (CODATA 2018 G, exact c).
inline constexpr double kC = 2.99792458e10;
inline constexpr double kC2 = kC * kC;
inline constexpr double kG = 6.67430e-8;
inline constexpr double kPI = std::numbers::pi;
// Mass [g] for which G * mass / C2 == 1.0 exactly in double: geometric units.
inline constexpr double kUnitMass = kC2 / kG;

// ===========================================================================
// Part A - the reference stepper
// ===========================================================================

template <class T> struct Consts { T e, lz, q; };
template <class T> struct State { T r, theta, phi, t, signR, signTheta; };
template <class T> struct Pot { T rPot, dRdr, thetaPot, dThetadtheta; };
template <class T> struct Derivs { T dr, dtheta, dphi, dt; };

// kerr.cpp:69-97
template <class T>
inline Pot<T> kerr_potentials(T r, T theta, T mass, T a, const Consts<T> &c) {
  const T mGeom = T(kG) * mass / T(kC2);
  const T rr = r * r;
  const T aa = a * a;
  const T sinTheta = s_sin(theta);
  const T cosTheta = s_cos(theta);
  const T sin2 = s_max(sinTheta * sinTheta, T(1e-12));
  const T cos2 = cosTheta * cosTheta;
  const T delta = rr - (T(2.0) * mGeom * r) + aa;
  const T aFactor = ((rr + aa) * c.e) - (a * c.lz);
  const T lzMinusAe = c.lz - (a * c.e);
  Pot<T> p{};
  p.rPot = (aFactor * aFactor) - (delta * (c.q + (lzMinusAe * lzMinusAe)));
  const T dAdR = T(2.0) * r * c.e;
  const T dDeltaDr = (T(2.0) * r) - (T(2.0) * mGeom);
  p.dRdr = (T(2.0) * aFactor * dAdR) - (dDeltaDr * (c.q + (lzMinusAe * lzMinusAe)));
  p.thetaPot = c.q + (aa * c.e * c.e * cos2) - (c.lz * c.lz / sin2);
  p.dThetadtheta = -(T(2.0) * aa * c.e * c.e * cosTheta * sinTheta) +
                   (T(2.0) * c.lz * c.lz * cosTheta / (sin2 * sinTheta));
  return p;
}

// kerr.cpp:40-66
template <class T>
inline Derivs<T> kerr_mino_derivs(const State<T> &s, T mass, T a, const Consts<T> &c) {
  const T mGeom = T(kG) * mass / T(kC2);
  const T r = s.r;
  const T theta = s.theta;
  const Pot<T> p = kerr_potentials(r, theta, mass, a, c);
  const T rPot = s_max(p.rPot, T(0.0));
  const T thetaPot = s_max(p.thetaPot, T(0.0));
  const T drDlam = s.signR * s_sqrt(rPot);
  const T dthetaDlam = s.signTheta * s_sqrt(thetaPot);
  const T sinTheta = s_sin(theta);
  const T sin2 = s_max(sinTheta * sinTheta, T(1e-12));
  const T delta = (r * r) - (T(2.0) * mGeom * r) + (a * a);
  const T aFactor = (((r * r) + (a * a)) * c.e) - (a * c.lz);
  const T deltaSafe = s_max(delta, T(1e-12));
  Derivs<T> d{};
  d.dr = drDlam;
  d.dtheta = dthetaDlam;
  d.dphi = (c.lz / sin2) - (a * c.e) + (a * aFactor / deltaSafe);
  d.dt = ((((r * r) + (a * a)) * aFactor) / deltaSafe) + (a * (c.lz - (a * c.e * sin2)));
  return d;
}

// kerr.cpp:99-134
template <class T>
inline State<T> kerr_step_mino(const State<T> &state, T mass, T a, const Consts<T> &c, T dlam) {
  State<T> next = state;
  const Derivs<T> k1 = kerr_mino_derivs(state, mass, a, c);
  State<T> s2 = state;
  s2.r += T(0.5) * dlam * k1.dr;
  s2.theta += T(0.5) * dlam * k1.dtheta;
  s2.phi += T(0.5) * dlam * k1.dphi;
  s2.t += T(0.5) * dlam * k1.dt;
  const Derivs<T> k2 = kerr_mino_derivs(s2, mass, a, c);
  State<T> s3 = state;
  s3.r += T(0.5) * dlam * k2.dr;
  s3.theta += T(0.5) * dlam * k2.dtheta;
  s3.phi += T(0.5) * dlam * k2.dphi;
  s3.t += T(0.5) * dlam * k2.dt;
  const Derivs<T> k3 = kerr_mino_derivs(s3, mass, a, c);
  State<T> s4 = state;
  s4.r += dlam * k3.dr;
  s4.theta += dlam * k3.dtheta;
  s4.phi += dlam * k3.dphi;
  s4.t += dlam * k3.dt;
  const Derivs<T> k4 = kerr_mino_derivs(s4, mass, a, c);
  next.r += dlam * (k1.dr + (T(2.0) * k2.dr) + (T(2.0) * k3.dr) + k4.dr) / T(6.0);
  next.theta += dlam * (k1.dtheta + (T(2.0) * k2.dtheta) + (T(2.0) * k3.dtheta) + k4.dtheta) / T(6.0);
  next.phi += dlam * (k1.dphi + (T(2.0) * k2.dphi) + (T(2.0) * k3.dphi) + k4.dphi) / T(6.0);
  next.t += dlam * (k1.dt + (T(2.0) * k2.dt) + (T(2.0) * k3.dt) + k4.dt) / T(6.0);
  next.theta = s_clamp(next.theta, T(1e-6), T(kPI - 1e-6));
  return next;
}

// kerr.h:132-141 (outer horizon, geometric mass m)
template <class T> inline T outer_horizon_geom(T m, T a) {
  const T disc = (m * m) - (a * a);
  if (disc < T(0)) return T(NAN);
  return m + s_sqrt(disc);
}

// kerr.h:203-225 (BPT 1972 ISCO, cbrt form), returns r_isco in units of m
template <class T> inline T isco_geom(T m, T a, bool prograde = true) {
  const T aStar = a / m;
  if (s_abs(aStar) > T(1.0)) return T(NAN);
  const T oneMinusA2 = T(1.0) - (aStar * aStar);
  const T cbrtFactor = s_cbrt(oneMinusA2);
  const T cbrtPlus = s_cbrt(T(1.0) + aStar);
  const T cbrtMinus = s_cbrt(T(1.0) - aStar);
  const T z1 = T(1.0) + (cbrtFactor * (cbrtPlus + cbrtMinus));
  const T z2 = s_sqrt((T(3.0) * aStar * aStar) + (z1 * z1));
  const T sq = s_sqrt((T(3.0) - z1) * (T(3.0) + z1 + (T(2.0) * z2)));
  const T rOverM = prograde ? (T(3.0) + z2 - sq) : (T(3.0) + z2 + sq);
  return rOverM * m;
}

// kerr.h:246-256 (prograde photon orbit)
template <class T> inline T photon_orbit_prograde_geom(T m, T a) {
  const T aStar = a / m;
  if (s_abs(aStar) > T(1.0)) return T(NAN);
  const T angle = (T(2.0) / T(3.0)) * s_acos(-aStar);
  return T(2.0) * m * (T(1.0) + s_cos(angle));
}
template <class T> inline T photon_orbit_retrograde_geom(T m, T a) {
  const T aStar = a / m;
  if (s_abs(aStar) > T(1.0)) return T(NAN);
  const T angle = (T(2.0) / T(3.0)) * s_acos(aStar);
  return T(2.0) * m * (T(1.0) + s_cos(angle));
}

// kerr.h:361-378 (static-observer redshift z = 1/sqrt(1 - r_s r / Sigma) - 1)
template <class T> inline T kerr_redshift_geom(T r, T theta, T m, T a) {
  const T rS = T(2.0) * m;
  const T cosTheta = s_cos(theta);
  const T sigma = (r * r) + (a * a * cosTheta * cosTheta);
  const T factor = T(1.0) - ((rS * r) / sigma);
  if (factor <= T(0)) return T(INFINITY);
  return (T(1.0) / s_sqrt(factor)) - T(1.0);
}

// novikov_thorne.h:81-90 (ISCO in M, pow/copysign form, spin clamped to +-0.9999)
inline double nt_isco(double aStar) {
  aStar = std::clamp(aStar, -0.9999, 0.9999);
  const double z1 = 1.0 + (std::pow(1.0 - (aStar * aStar), 1.0 / 3.0) *
                           (std::pow(1.0 + aStar, 1.0 / 3.0) + std::pow(1.0 - aStar, 1.0 / 3.0)));
  const double z2 = std::sqrt((3.0 * aStar * aStar) + (z1 * z1));
  return 3.0 + z2 - std::copysign(std::sqrt((3.0 - z1) * (3.0 + z1 + (2.0 * z2))), aStar);
}

// novikov_thorne.h:50-72 (radiative efficiency 1 - E_isco, E_isco = sqrt(1 - 2/(3 r_isco)))
inline double nt_radiative_efficiency(double aStar) {
  aStar = std::clamp(aStar, -0.9999, 0.9999);
  const double z1 = 1.0 + (std::pow(1.0 - (aStar * aStar), 1.0 / 3.0) *
                           (std::pow(1.0 + aStar, 1.0 / 3.0) + std::pow(1.0 - aStar, 1.0 / 3.0)));
  const double z2 = std::sqrt((3.0 * aStar * aStar) + (z1 * z1));
  const double rIsco = 3.0 + z2 - std::copysign(std::sqrt((3.0 - z1) * (3.0 + z1 + (2.0 * z2))), aStar);
  const double eIsco = std::sqrt(1.0 - (2.0 / (3.0 * rIsco)));
  return 1.0 - eIsco;
}

// novikov_thorne.h:170-190
inline double nt_normalized_flux(double r, double aStar) {
  const double rIsco = nt_isco(aStar);
  if (r < rIsco) return 0.0;
  const double fR = std::max(0.0, 1.0 - std::sqrt(rIsco / r));
  const double flux = fR / (r * r * r);
  const double rPeak = 1.5 * rIsco;
  const double fPeak = std::max(0.0, 1.0 - std::sqrt(rIsco / rPeak));
  const double fluxPeak = fPeak / (rPeak * rPeak * rPeak);
  return std::min(1.0, flux / fluxPeak);
}

// Status values of physics::RayStatus (raytracer.h:46-52)
enum RayStatus : int32_t { PROPAGATING = 0, ESCAPED = 1, CAPTURED = 2, HIT_DISK = 3, MAX_STEPS = 4 };

template <class T> struct TraceResult {
  T r, theta, phi;
  T totalDistance;
  T redshift;
  int32_t steps;
  int32_t status;
};

// raytracer.h:324-378, with the parameters of the KerrRaytracer constructor
// (raytracer.h:311-318) passed in explicitly.
template <class T>
inline TraceResult<T> kerr_trace(const State<T> &initial, const Consts<T> &c, T mass, T a,
                                 T rHorizon, T rEscape, T stepSize, int32_t maxSteps) {
  TraceResult<T> res{};
  res.steps = 0;
  res.totalDistance = T(0.0);
  res.redshift = T(1.0);
  res.status = PROPAGATING;
  State<T> state = initial;
  for (int32_t step = 0; step < maxSteps; ++step) {
    if (state.r <= (rHorizon * T(1.001))) { res.status = CAPTURED; break; }
    if (state.r >= rEscape) { res.status = ESCAPED; break; }
    const Pot<T> p = kerr_potentials(state.r, state.theta, mass, a, c);
    State<T> next = state;
    if (p.rPot < T(0.0)) next.signR = -next.signR;
    if (p.thetaPot < T(0.0)) next.signTheta = -next.signTheta;
    next = kerr_step_mino(next, mass, a, c, stepSize);
    state = next;
    res.totalDistance += stepSize;
    ++res.steps;
  }
  if (res.status == PROPAGATING) res.status = (res.steps >= maxSteps) ? MAX_STEPS : ESCAPED;
  res.r = state.r;
  res.theta = state.theta;
  res.phi = state.phi;
  if (state.r > (rHorizon * T(1.001))) {
    const T mGeom = T(kG) * mass / T(kC2);
    res.redshift = T(1.0) + kerr_redshift_geom(state.r, state.theta, mGeom, a);
  }
  return res;
}

// ===========================================================================
// Part B - image-plane tracer (geometric units, M = 1)
// ===========================================================================

enum PixelClass : int32_t { CLS_CAPTURED = 0, CLS_DISK = 1, CLS_ESCAPED = 2, CLS_MAX_STEPS = 3 };

// Per-ray constants. E = 1. qR enters R(r), qTh enters Theta(theta).
template <class T> struct RayConsts {
  T a;      // spin a/M
  T lam;    // lambda = L_z / E
  T qR;     // Carter constant as used in R(r)
  T qTh;    // Carter constant as used in Theta(theta)
  T K;      // qR + (lam - a)^2
};

// Second-order state: position, Mino-time velocities, azimuth.
template <class T> struct Y { T r, u, phi, pr, pu; };

// R(r) = A^2 - Delta K  (kerr.cpp:81 with E = 1, M = 1)
template <class T> inline T pot_R(T r, const RayConsts<T> &c) {
  const T A = r * r + c.a * c.a - c.a * c.lam;
  const T D = r * r - T(2) * r + c.a * c.a;
  return A * A - D * c.K;
}
// U(u) = sin^2 Theta = (qTh + a^2 u^2)(1 - u^2) - lam^2  (kerr.cpp:89 times sin^2)
template <class T> inline T pot_U(T u, const RayConsts<T> &c) {
  const T u2 = u * u;
  return (c.qTh + c.a * c.a * u2) * (T(1) - u2) - c.lam * c.lam;
}

// Right-hand side in Mino time sigma for a ray traced BACKWARD from the
// observer: r' = p_r, u' = p_u, p_r' = R'(r)/2, p_u' = U'(u)/2.
//
// Azimuth. With Phi = lam / sin^2 - a + a A / Delta the forward-time rate of
// kerr.cpp:61 (E = 1), the emitter's azimuth obeys phi' = -Phi (time reversed
// along the ray), which diverges as 1/Delta at the horizon. The state carries
// instead psi = phi - a G(r), G' = 1/Delta (the horizon-regular azimuth the
// reference's GPU step uses, src/cuda/device_physics.cuh:453-525):
//   psi' = -lam / sin^2 + a - a (A + p_r) / Delta,
// and on the first integral p_r^2 = R, A^2 - R = Delta K gives
//   (A + p_r) / Delta = K / (A - p_r),
// finite at the horizon for an ingoing ray (p_r < 0); that form is used there
// and (A + p_r) / Delta for outgoing rays (which stay off the horizon).
// phi = psi + a (G(r) - G(r_obs)) is restored at the outputs (phi_of_psi).
template <class T> inline Y<T> img_rhs(const Y<T> &y, const RayConsts<T> &c) {
  const T r = y.r, u = y.u;
  const T a2 = c.a * c.a;
  const T A = r * r + a2 - c.a * c.lam;
  const T D = r * r - T(2) * r + a2;
  const T u2 = u * u;
  const T s2 = s_max(T(1) - u2, T(1e-12));
  Y<T> d;
  d.r = y.pr;
  d.u = y.pu;
  d.pr = T(2) * r * A - (r - T(1)) * c.K;                  // R'(r) / 2
  d.pu = u * (a2 - c.qTh - T(2) * a2 * u2);                // U'(u) / 2
  const bool in = y.pr < T(0);
  const T num = in ? c.K : (A + y.pr);
  const T den = in ? (A - y.pr) : D;
  d.phi = (c.a - c.lam / s2) - c.a * (num / den);
  return d;
}

// phi = psi + a (G(r) - G(r_obs)), G(r) = ln((r - r+) / (r - r-)) / (r+ - r-).
template <class T> inline T phi_of_psi(T psi, T r, T r_obs, T a, T r_plus, T r_minus) {
  if (a == T(0)) return psi;
  const T q = ((r - r_plus) * (r_obs - r_minus)) / ((r - r_minus) * (r_obs - r_plus));
  return psi + a * (T(std::log(double(q))) / (r_plus - r_minus));
}

template <class T> inline Y<T> y_axpy(const Y<T> &y, T h, const Y<T> &k) {
  return Y<T>{y.r + h * k.r, y.u + h * k.u, y.phi + h * k.phi, y.pr + h * k.pr, y.pu + h * k.pu};
}

// First-integral projection threshold: the momenta are reset to the first
// integrals p_r^2 = R(r), p_u^2 = U(u) only where those are well conditioned,
// R > tau r^4 and U > tau (|q_Th| + a^2), i.e. away from turning points.
inline constexpr double kProjTau = 1e-6;

// Projection of the Mino-time momenta onto p_r^2 = R(r), p_u^2 = U(u),
// keeping their signs. In the second-order form these first integrals are
// not enforced by the integrator; at r ~ 1000 the impact parameter enters R
// only at relative order b^2/r^2 ~ 1e-4, so a step error of rtol in p_r
// moves b^2 by ~rtol r^2. Resetting the momenta after each accepted step
// keeps b and q exact while the second-order form still carries the ray
// through its turning points.
template <class T> inline T with_sign_of(T mag, T s) { return (s < T(0)) ? -mag : mag; }

template <class T> struct PolyRhs {
  const RayConsts<T> &c;
  Y<T> operator()(const Y<T> &y) const { return img_rhs(y, c); }
  void project(Y<T> &y) const {
    const T Rv = pot_R(y.r, c);
    const T r2 = y.r * y.r;
    if (Rv > T(kProjTau) * (r2 * r2)) y.pr = with_sign_of(s_sqrt(Rv), y.pr);
    const T Uv = pot_U(y.u, c);
    if (Uv > T(kProjTau) * (s_abs(c.qTh) + c.a * c.a)) y.pu = with_sign_of(s_sqrt(Uv), y.pu);
  }
};

// Classical RK4 step of size h in Mino time.
template <class T, class F> inline Y<T> img_rk4(const Y<T> &y, T h, const F &f, const Y<T> &k1) {
  const Y<T> k2 = f(y_axpy(y, T(0.5) * h, k1));
  const Y<T> k3 = f(y_axpy(y, T(0.5) * h, k2));
  const Y<T> k4 = f(y_axpy(y, h, k3));
  const T w = h / T(6);
  Y<T> n;
  n.r = y.r + w * (k1.r + T(2) * k2.r + T(2) * k3.r + k4.r);
  n.u = y.u + w * (k1.u + T(2) * k2.u + T(2) * k3.u + k4.u);
  n.phi = y.phi + w * (k1.phi + T(2) * k2.phi + T(2) * k3.phi + k4.phi);
  n.pr = y.pr + w * (k1.pr + T(2) * k2.pr + T(2) * k3.pr + k4.pr);
  n.pu = y.pu + w * (k1.pu + T(2) * k2.pu + T(2) * k3.pu + k4.pu);
  return n;
}

// Dormand & Prince (1980) 5(4) tableau (also listed in src/physics/verified/rk4.h:182-223).
struct DP {
  static constexpr double a21 = 1.0 / 5.0;
  static constexpr double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
  static constexpr double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
  static constexpr double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0, a53 = 64448.0 / 6561.0,
                          a54 = -212.0 / 729.0;
  static constexpr double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0,
                          a64 = 49.0 / 176.0, a65 = -5103.0 / 18656.0;
  static constexpr double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0,
                          b5 = -2187.0 / 6784.0, b6 = 11.0 / 84.0;
  // e = b(5th) - b(4th)
  static constexpr double e1 = 35.0 / 384.0 - 5179.0 / 57600.0;
  static constexpr double e3 = 500.0 / 1113.0 - 7571.0 / 16695.0;
  static constexpr double e4 = 125.0 / 192.0 - 393.0 / 640.0;
  static constexpr double e5 = -2187.0 / 6784.0 + 92097.0 / 339200.0;
  static constexpr double e6 = 11.0 / 84.0 - 187.0 / 2100.0;
  static constexpr double e7 = -1.0 / 40.0;
};

template <class T> struct DPOut { Y<T> y5; Y<T> k7; T err; };

// x^(-1/5) for finite x > 0 with only frexp/ldexp (exact) and correctly
// rounded +, -, *: x = m 2^e, e = 5k + j, z = m 2^j in [0.5, 16); Newton's
// iteration y <- y (6 - z y^5) / 5 for y^-5 = z, started at 2^(-j/5) <= z^(-1/5),
// rises monotonically to the root (6 iterations reach double precision).
// Being free of libm calls it gives the same bits on the CPU and the GPU, so
// the DP45 step sequence is reproducible across the two.
inline double inv_fifth_root(double x) {
  int e = 0;
  const double m = std::frexp(x, &e);
  int k = e / 5;
  int j = e - 5 * k;
  if (j < 0) { j += 5; k -= 1; }
  const double z = std::ldexp(m, j);
  static constexpr double y0[5] = {1.0, 0.87055056329612412, 0.75785828325519899, 0.65975395538644710,
                                   0.57434917749851755};
  double y = y0[j];
  for (int it = 0; it < 6; ++it) {
    const double y2 = y * y;
    const double y5 = (y2 * y2) * y;
    y = (y * (6.0 - (z * y5))) / 5.0;
  }
  return std::ldexp(y, -k);
}

// Step-size factor of the controller (Hairer, Norsett & Wanner 1993, II.4):
// 0.9 err^(-1/5), within [0.1, 2] after an accepted step and [0.1, 1] after a
// rejected one; err == 0 gives 2, a non-finite err gives 0.1.
inline double step_factor(double err, bool accepted) {
  const double hi = accepted ? 2.0 : 1.0;
  if (!(err < 1e300)) return 0.1;
  if (!(err > 0.0)) return hi;
  const double f = 0.9 * inv_fifth_root(err);
  return (f < 0.1) ? 0.1 : ((hi < f) ? hi : f);
}

// One Dormand-Prince attempt; err is the scaled RMS norm over the 5 components.
template <class T, class F>
inline DPOut<T> img_dp45(const Y<T> &y, T h, const F &f, const Y<T> &k1, T rtol, T atol, bool want_err) {
  auto comb = [&](std::initializer_list<std::pair<T, const Y<T> *>> terms) {
    Y<T> s = y;
    for (auto &t : terms) s = y_axpy(s, h * t.first, *t.second);
    return s;
  };
  const Y<T> k2 = f(comb({{T(DP::a21), &k1}}));
  const Y<T> k3 = f(comb({{T(DP::a31), &k1}, {T(DP::a32), &k2}}));
  const Y<T> k4 = f(comb({{T(DP::a41), &k1}, {T(DP::a42), &k2}, {T(DP::a43), &k3}}));
  const Y<T> k5 = f(comb({{T(DP::a51), &k1}, {T(DP::a52), &k2}, {T(DP::a53), &k3}, {T(DP::a54), &k4}}));
  const Y<T> k6 = f(comb({{T(DP::a61), &k1}, {T(DP::a62), &k2}, {T(DP::a63), &k3}, {T(DP::a64), &k4},
                          {T(DP::a65), &k5}}));
  DPOut<T> o;
  o.y5 = comb({{T(DP::b1), &k1}, {T(DP::b3), &k3}, {T(DP::b4), &k4}, {T(DP::b5), &k5}, {T(DP::b6), &k6}});
  o.err = T(0);
  if (!want_err) { o.k7 = k1; return o; }
  o.k7 = f(o.y5);
  auto ecomp = [&](T k1v, T k3v, T k4v, T k5v, T k6v, T k7v) {
    return h * (T(DP::e1) * k1v + T(DP::e3) * k3v + T(DP::e4) * k4v + T(DP::e5) * k5v +
                T(DP::e6) * k6v + T(DP::e7) * k7v);
  };
  const T er = ecomp(k1.r, k3.r, k4.r, k5.r, k6.r, o.k7.r);
  const T eu = ecomp(k1.u, k3.u, k4.u, k5.u, k6.u, o.k7.u);
  const T ep = ecomp(k1.phi, k3.phi, k4.phi, k5.phi, k6.phi, o.k7.phi);
  const T epr = ecomp(k1.pr, k3.pr, k4.pr, k5.pr, k6.pr, o.k7.pr);
  const T epu = ecomp(k1.pu, k3.pu, k4.pu, k5.pu, k6.pu, o.k7.pu);
  auto sc = [&](T a0, T a1) { return atol + rtol * s_max(s_abs(a0), s_abs(a1)); };
  const T q0 = er / sc(y.r, o.y5.r), q1 = eu / sc(y.u, o.y5.u), q2 = ep / sc(y.phi, o.y5.phi),
          q3 = epr / sc(y.pr, o.y5.pr), q4 = epu / sc(y.pu, o.y5.pu);
  o.err = s_sqrt((q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3 + q4 * q4) / T(5));
  return o;
}

// Keplerian prograde emitter in the equatorial plane (BPT 1972):
// g = 1 / (u^t (1 - Omega lambda)) = sqrt(x^3 (x^3 - 3x + 2a)) / (x^3 + a - lambda), x = sqrt(r).
template <class T> inline T disk_g(T r, T a, T lam) {
  const T x = s_sqrt(r);
  const T x3 = x * x * x;
  const T v = x3 * (x3 - T(3) * x + T(2) * a);
  if (v <= T(0)) return T(0);
  return s_sqrt(v) / (x3 + a - lam);
}

// Scene description used by the oracle (mirrors BH_KerrScene).
struct Scene {
  double spin, r_obs, theta_obs;
  double alpha_min, alpha_max, beta_min, beta_max;
  int32_t width, height;
  int32_t integrator;      // 0 RK4, 1 DP45
  int32_t potential_form;  // 0 reference, 1 Carter
  int32_t max_crossings;
  int32_t max_steps;
  double step_coeff, step_rcap, rtol, atol;
  double horizon_factor, escape_factor;
  double disk_r_in, disk_r_out;
};

template <class T> struct PixelResult {
  int32_t cls, steps, n_cross;
  T r_hit[3], phi_hit[3], g[3];
  T flux, intensity, theta_inf, phi_inf;
  T u_inf;  // cos(theta_inf) before the arc cosine (sky lookups)
  T r_end, pr_end, pu_end, dphi_end;  // escape point: radius, momenta, d(phi)/d(Mino time)
};

// Derived per-scene constants.
template <class T> struct SceneDerived {
  T a, r_plus, r_minus, r_hor, r_esc, r_in, r_out, sin_o, cos_o, u_o;
};

template <class T> inline SceneDerived<T> derive(const Scene &s) {
  SceneDerived<T> d{};
  d.a = T(s.spin);
  d.r_plus = outer_horizon_geom(T(1), d.a);
  d.r_minus = T(1) - s_sqrt(T(1) - d.a * d.a);
  d.r_hor = T(s.horizon_factor) * d.r_plus;
  d.r_esc = T(s.escape_factor) * T(s.r_obs);
  d.r_in = (s.disk_r_in > 0) ? T(s.disk_r_in) : isco_geom(T(1), d.a, true);
  d.r_out = T(s.disk_r_out);
  d.sin_o = s_sin(T(s.theta_obs));
  d.cos_o = s_cos(T(s.theta_obs));
  d.u_o = d.cos_o;
  return d;
}

// Pixel centre -> image-plane coordinates.
inline void pixel_alpha_beta(const Scene &s, int64_t pix, double &alpha, double &beta) {
  const int64_t i = pix % s.width, j = pix / s.width;
  alpha = s.alpha_min + (double(i) + 0.5) * ((s.alpha_max - s.alpha_min) / double(s.width));
  beta = s.beta_min + (double(j) + 0.5) * ((s.beta_max - s.beta_min) / double(s.height));
}

// Bardeen (1973) image-plane initial data for the photon that reaches the
// observer at (r_obs, theta_obs) with image coordinates (alpha, beta):
//   lambda = -alpha sin(theta_o),  eta = beta^2 + (alpha^2 - a^2) cos^2(theta_o).
// Backward ray: p_r = -sqrt(R(r_obs)) (inward), p_theta = -beta (beta > 0 heads
// toward the spin axis), p_u = -sin(theta_o) p_theta = beta sin(theta_o).
template <class T>
inline void init_ray(const SceneDerived<T> &d, const Scene &s, T alpha, T beta, RayConsts<T> &c, Y<T> &y) {
  c.a = d.a;
  c.lam = -alpha * d.sin_o;
  const T eta = beta * beta + (alpha * alpha - d.a * d.a) * d.cos_o * d.cos_o;
  c.qTh = eta + c.lam * c.lam;
  c.qR = (s.potential_form == 1) ? eta : c.qTh;
  c.K = c.qR + (c.lam - c.a) * (c.lam - c.a);
  y.r = T(s.r_obs);
  y.u = d.u_o;
  y.phi = T(0);
  y.pr = -s_sqrt(s_max(pot_R(y.r, c), T(0)));
  y.pu = beta * d.sin_o;
}

// Affine step -> Mino step: dsigma = h / Sigma, h = coeff * min(r, rcap).
template <class T> inline T mino_step(const Scene &s, const Y<T> &y, T a) {
  const T h = T(s.step_coeff) * s_min(y.r, T(s.step_rcap));
  const T sigma = y.r * y.r + a * a * y.u * y.u;
  return h / sigma;
}

// ---------------------------------------------------------------------------
// Equatorial crossing by Hermite interpolation of the accepted step.
//
// In the second-order form every position x in {r, u} has x' = p_x and
// x'' = F_x(position) known at both ends of a step (F from the right-hand
// side at y0 and at y1), so the quintic Hermite interpolant through (x, h x',
// h^2 x'') at t = 0 and t = 1 approximates x(t0 + t h) with an error of
// O(h^6) -- below the step's own truncation error -- without any further
// integration. phi' is known at both ends: cubic Hermite. The root of u on
// [0, 1] is bracketed by u0, u1 of opposite signs and found with the
// Illinois variant of regula falsi (Dowell & Jarratt 1971) on the polynomial
// (the bracketing pattern of bisectRadialCrossing, event_detection.h:127-180),
// stopping at |u| <= 1e-15 (|u0| + |u1|) or a bracket narrower than 1e-14.
// ---------------------------------------------------------------------------
template <class T> struct Quintic { T c0, c1, c2, c3, c4, c5; };

template <class T> inline Quintic<T> quintic_hermite(T p0, T v0, T a0, T p1, T v1, T a1) {
  const T A = ((p1 - p0) - v0) - T(0.5) * a0;
  const T B = (v1 - v0) - a0;
  const T Cc = a1 - a0;
  Quintic<T> q;
  q.c0 = p0;
  q.c1 = v0;
  q.c2 = T(0.5) * a0;
  q.c3 = (T(10) * A - T(4) * B) + T(0.5) * Cc;
  q.c4 = (T(7) * B - T(15) * A) - Cc;
  q.c5 = (T(6) * A - T(3) * B) + T(0.5) * Cc;
  return q;
}

template <class T> inline T eval_quintic(const Quintic<T> &q, T t) {
  return q.c0 + t * (q.c1 + t * (q.c2 + t * (q.c3 + t * (q.c4 + t * q.c5))));
}

template <class T> inline T eval_cubic_hermite(T p0, T v0, T p1, T v1, T t) {
  const T A = (p1 - p0) - v0;
  const T B = v1 - v0;
  const T c2 = T(3) * A - B;
  const T c3 = B - T(2) * A;
  return p0 + t * (v0 + t * (c2 + t * c3));
}

inline constexpr int kRootMaxIter = 60;

// Crossing state (r, phi) of the step y0 -> y1 of Mino size h, k0 = rhs(y0),
// k1 = rhs(y1) (y1 before projection).
template <class T>
inline Y<T> hermite_crossing(const Y<T> &y0, const Y<T> &k0, const Y<T> &y1, const Y<T> &k1, T h) {
  const T h2 = h * h;
  const Quintic<T> qu = quintic_hermite(y0.u, h * y0.pu, h2 * k0.pu, y1.u, h * y1.pu, h2 * k1.pu);
  T a = T(0), fa = y0.u, b = T(1), fb = y1.u;
  const T tol = T(1e-15) * (s_abs(fa) + s_abs(fb));
  int side = 0;
  T t = T(0.5);
  for (int i = 0; i < kRootMaxIter; ++i) {
    t = (a * fb - b * fa) / (fb - fa);
    if (!(t > a && t < b)) t = T(0.5) * (a + b);
    const T fc = eval_quintic(qu, t);
    if (s_abs(fc) <= tol || (b - a) <= T(1e-14)) break;
    if ((fc * fb) > T(0)) {
      b = t;
      fb = fc;
      if (side == -1) fa = T(0.5) * fa;
      side = -1;
    } else {
      a = t;
      fa = fc;
      if (side == 1) fb = T(0.5) * fb;
      side = 1;
    }
  }
  const Quintic<T> qr = quintic_hermite(y0.r, h * y0.pr, h2 * k0.pr, y1.r, h * y1.pr, h2 * k1.pr);
  Y<T> yc;
  yc.r = eval_quintic(qr, t);
  yc.u = eval_quintic(qu, t);
  yc.phi = eval_cubic_hermite(y0.phi, h * k0.phi, y1.phi, h * k1.phi, t);
  yc.pr = T(0);
  yc.pu = T(0);
  return yc;
}

template <class T>
inline void record_crossing(const Scene &s, const SceneDerived<T> &d, const RayConsts<T> &c, const Y<T> &yc,
                            PixelResult<T> &out) {
  const int k = out.n_cross;
  out.r_hit[k] = yc.r;
  out.phi_hit[k] = phi_of_psi(yc.phi, yc.r, T(s.r_obs), d.a, d.r_plus, d.r_minus);
  out.g[k] = disk_g(yc.r, d.a, c.lam);
  const T q = d.r_in / yc.r;
  const T g2 = out.g[k] * out.g[k];
  out.intensity += g2 * g2 * q * q * q;
  if (k == 0) out.flux = T(nt_normalized_flux(double(yc.r), s.spin));
  out.n_cross = k + 1;
}

// Trace one pixel. Loop order follows raytracer.h:338-365: step budget,
// horizon test, escape test, step; then the equatorial-crossing test.
// MakeRhs(c) returns the right-hand-side callable for the ray constants c.
// A camera at finite distance (the library's legacy renderer): pixel (i, j)
// looks along d = normalize(-u right - v up + fwd), u = (2 (i + 1/2) / W - 1)
// fov aspect + shift_x, v = (2 (j + 1/2) / H - 1) fov + shift_y; d is the
// direction in the locally non-rotating frame (Bardeen, Press & Teukolsky
// 1972) at the camera (r0, u0 = cos theta0, azimuth 0 after rotating the
// world by -phi_cam). The photon seen arrives along -d: with lapse
// alpha_L = sqrt(Sigma Delta / A), omega = 2 a r / A, varpi = sqrt(A / Sigma)
// sin theta, lambda = varpi v_phi / (alpha_L + omega varpi v_phi) and
// Theta = (sqrt(Sigma) v_theta / (alpha_L + omega varpi v_phi))^2 for
// v = -d; eta = Theta - a^2 cos^2 + lambda^2 cot^2 (textbook Carter form).
struct Camera {
  double right[3], up[3], fwd[3];
  double fov, aspect, shift_x, shift_y;
  double r0, u0, cphi, sphi;
  int32_t width, height;
};

inline void init_ray_camera(const SceneDerived<double> &dd, const Camera &cam, int64_t pix, RayConsts<double> &c,
                            Y<double> &y) {
  const int64_t i = pix % cam.width, j = pix / cam.width;
  const double uu = (2.0 * (double(i) + 0.5) / double(cam.width) - 1.0) * cam.fov * cam.aspect + cam.shift_x;
  const double vv = (2.0 * (double(j) + 0.5) / double(cam.height) - 1.0) * cam.fov + cam.shift_y;
  double d[3];
  for (int k = 0; k < 3; ++k) d[k] = -uu * cam.right[k] - vv * cam.up[k] + cam.fwd[k];
  const double dn = 1.0 / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  for (double &v : d) v *= dn;
  const double u0 = cam.u0, s0 = std::sqrt(std::max(0.0, (1.0 - u0) * (1.0 + u0)));
  const double dx = cam.cphi * d[0] + cam.sphi * d[1], dy = -cam.sphi * d[0] + cam.cphi * d[1], dz = d[2];
  const double n_r = s0 * dx + u0 * dz, n_th = u0 * dx - s0 * dz, n_ph = dy;
  const double a = dd.a, a2 = a * a, r = cam.r0;
  const double sig = r * r + a2 * u0 * u0;
  const double del = r * r - 2.0 * r + a2;
  const double AA = (r * r + a2) * (r * r + a2) - a2 * del * s0 * s0;
  const double lapse = std::sqrt(sig * del / AA);
  const double omega = 2.0 * a * r / AA;
  const double varpi = std::sqrt(AA / sig) * s0;
  const double e = lapse + omega * varpi * (-n_ph);
  c.a = a;
  c.lam = varpi * (-n_ph) / e;
  const double pth = std::sqrt(sig) * (-n_th) / e;
  const double cot2 = s0 > 1e-12 ? (u0 * u0) / (s0 * s0) : 0.0;
  const double eta = pth * pth - a2 * u0 * u0 + c.lam * c.lam * cot2;
  c.qTh = eta + c.lam * c.lam;
  c.qR = eta;
  c.K = eta + (c.lam - a) * (c.lam - a);
  y.r = r;
  y.u = u0;
  y.phi = 0.0;
  const double mr = std::sqrt(std::max(pot_R(r, c), 0.0)), mu = std::sqrt(std::max(pot_U(u0, c), 0.0));
  y.pr = n_r < 0.0 ? -mr : mr;
  y.pu = n_th > 0.0 ? -mu : mu;
}

template <class T, class MakeRhs>
inline PixelResult<T> trace_pixel_from(const Scene &s, const SceneDerived<T> &d, const RayConsts<T> &c, Y<T> y,
                                       const MakeRhs &make_rhs) {
  PixelResult<T> out{};
  out.cls = CLS_MAX_STEPS;
  const auto f = make_rhs(c);
  // Start on the first integrals too: the projection is then idempotent on
  // any state it has produced, so re-applying it to an unchanged state (a
  // rejected DP45 attempt on the GPU) changes nothing.
  f.project(y);
  const int maxc = std::max(1, std::min(3, int(s.max_crossings)));
  auto in_disk = [&](T r) { return r >= d.r_in && r <= d.r_out; };
  auto finish_escape = [&](const Y<T> &yy) {
    out.u_inf = s_clamp(yy.u, T(-1), T(1));
    {  // direction of motion for the sky: dphi = dpsi + a p_r / Delta
      const Y<T> k = img_rhs(yy, c);
      const T delta = ((yy.r * yy.r) - (T(2) * yy.r)) + d.a * d.a;
      out.r_end = yy.r;
      out.pr_end = yy.pr;
      out.pu_end = yy.pu;
      out.dphi_end = k.phi + (d.a * yy.pr) / delta;
    }
    out.theta_inf = s_acos(out.u_inf);
    out.phi_inf = phi_of_psi(yy.phi, yy.r, T(s.r_obs), d.a, d.r_plus, d.r_minus);
  };

  if (s.integrator == 0) {
    for (;;) {
      if (out.steps >= s.max_steps) { out.cls = CLS_MAX_STEPS; break; }
      if (y.r <= d.r_hor) { out.cls = CLS_CAPTURED; break; }
      if (y.r >= d.r_esc) { out.cls = CLS_ESCAPED; finish_escape(y); break; }
      const T h = mino_step(s, y, d.a);
      const Y<T> k0 = f(y);
      Y<T> yn = img_rk4(y, h, f, k0);
      ++out.steps;
      if ((y.u * yn.u) < T(0)) {
        const Y<T> yc = hermite_crossing(y, k0, yn, f(yn), h);
        if (in_disk(yc.r)) {
          record_crossing(s, d, c, yc, out);
          if (out.n_cross >= maxc) { out.cls = CLS_DISK; break; }
        }
      }
      f.project(yn);
      y = yn;
    }
  } else {
    const T rtol = T(s.rtol), atol = T(s.atol);
    T h = mino_step(s, y, d.a);
    Y<T> k1 = f(y);
    int64_t attempts = 0;
    const int64_t max_attempts = int64_t(4) * s.max_steps + 64;
    for (;;) {
      if (out.steps >= s.max_steps || attempts >= max_attempts) { out.cls = CLS_MAX_STEPS; break; }
      if (y.r <= d.r_hor) { out.cls = CLS_CAPTURED; break; }
      if (y.r >= d.r_esc) { out.cls = CLS_ESCAPED; finish_escape(y); break; }
      ++attempts;
      const DPOut<T> o = img_dp45(y, h, f, k1, rtol, atol, true);
      const T err = o.err;
      bool stop = false;
      if (err <= T(1)) {
        ++out.steps;
        if ((y.u * o.y5.u) < T(0)) {
          const Y<T> yc = hermite_crossing(y, k1, o.y5, o.k7, h);
          if (in_disk(yc.r)) {
            record_crossing(s, d, c, yc, out);
            if (out.n_cross >= maxc) { out.cls = CLS_DISK; stop = true; }
          }
        }
        y = o.y5;
        k1 = o.k7;
        f.project(y);
        k1.r = y.pr;  // projection moves only the momenta: k1's other components stand
        k1.u = y.pu;
        h = h * T(step_factor(double(err), true));
      } else {
        h = h * T(step_factor(double(err), false));
      }
      if (stop) break;
    }
  }
  return out;
}

template <class T, class MakeRhs>
inline PixelResult<T> trace_pixel(const Scene &s, const SceneDerived<T> &d, T alpha, T beta,
                                  const MakeRhs &make_rhs) {
  RayConsts<T> c;
  Y<T> y;
  init_ray(d, s, alpha, beta, c, y);
  return trace_pixel_from(s, d, c, y, make_rhs);
}

template <class T> inline PixelResult<T> trace_pixel(const Scene &s, const SceneDerived<T> &d, T alpha, T beta) {
  return trace_pixel(s, d, alpha, beta, [](const RayConsts<T> &c) { return PolyRhs<T>{c}; });
}

}  // namespace bho
