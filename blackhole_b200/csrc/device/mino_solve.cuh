// mino_solve.cuh - exact equatorial crossings of a Kerr image-plane ray
// without stepping (FP64; device code under nvcc, plain C++ elsewhere).
//
// The image tracer integrates r'' = R'(r)/2, u'' = U'(u)/2 in Mino time tau
// with p_r^2 = R, p_u^2 = U (u = cos theta). Both motions separate, so the
// Mino times of the equatorial crossings and the radius reached at a given
// Mino time follow from one-dimensional integrals:
//
// * theta: U = (z+ - u^2)(a^2 u^2 + w) with z+ w = q_Th - lambda^2. With
//   u = sqrt(z+) sin(chi), d tau = d chi / sqrt(w + a^2 z+ sin^2 chi): the
//   crossings (chi = n pi) are at tau_1 + 2(n-1)K, from Legendre's integral
//   of the first kind, evaluated with Carlson's R_F (B. C. Carlson, "Numerical
//   computation of real or complex elliptic integrals", Numer. Algorithms 10
//   (1995) 13-26, duplication algorithm).
// * r: x = 1/r, P(x) = x^4 R(1/x) = 1 + p2 x^2 + p1 x^3 + p0 x^4. A ray with a
//   turning point x_tp (smallest positive root of P below 1/r+) is described
//   by sigma with x = x_tp - sigma^2 (sigma < 0 inbound, > 0 outbound), so
//   d tau / d sigma = 2 / sqrt(P(x) / (x_tp - x)) is smooth and positive
//   through the turning point; a ray without one uses x itself, d tau / dx =
//   1 / sqrt(P(x)). tau(sigma) is then a smooth increasing function evaluated
//   by composite 16-point Gauss-Legendre quadrature and inverted by
//   bracketed Newton iteration.
// * phi: the tracer's azimuth is -(Phi_r + Phi_th). Phi_r = int a (2r - a
//   lambda) / Delta dtau rides on the same quadrature nodes as tau (a second
//   integrand, rational in x); Phi_th = lambda int dtau / (1 - u^2) is closed
//   form in the polar amplitude: Carlson's R_J at the observer and at the end
//   point, Bulirsch's cel for the complete integral.
//
// Accuracy degrades where P has a near-double root (rays next to the
// critical curve): critical_distance() gives a first-order image-plane
// distance to the critical curve so callers can send those rays to the
// integrator.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define BHM_HD __device__ __forceinline__
#else
#define BHM_HD inline
#endif

namespace bhmino {

#ifdef __CUDACC__
BHM_HD double inv_sqrt(double x) { return rsqrt(x); }
BHM_HD float inv_sqrt(float x) { return rsqrtf(x); }
#else
BHM_HD double inv_sqrt(double x) { return 1.0 / std::sqrt(x); }
BHM_HD float inv_sqrt(float x) { return 1.0f / std::sqrt(x); }
#endif

// Gauss-Legendre, 16 points on [-1, 1]: the 8 positive nodes and weights.
struct GlNode {
  double x, w;
};
#ifdef __CUDACC__
__constant__
#endif
    static const GlNode kGl16[8] = {
        {9.50125098376374405e-02, 1.89450610455068641e-01}, {2.81603550779258915e-01, 1.82603415044923639e-01},
        {4.58016777657227370e-01, 1.69156519395002647e-01}, {6.17876244402643771e-01, 1.49595988816576708e-01},
        {7.55404408355002999e-01, 1.24628971255534071e-01}, {8.65631202387831755e-01, 9.51585116824926053e-02},
        {9.44575023073232600e-01, 6.22535239386474565e-02}, {9.89400934991649939e-01, 2.71524594117541762e-02}};

// Gauss-Legendre, 8 points on [-1, 1]: the 4 positive nodes and weights.
#ifdef __CUDACC__
__constant__
#endif
    static const GlNode kGl8[4] = {{1.83434642495649805e-01, 3.62683783378361983e-01},
                                   {5.25532409916328986e-01, 3.13706645877887287e-01},
                                   {7.96666477413626740e-01, 2.22381034453374471e-01},
                                   {9.60289856497536232e-01, 1.01228536290376259e-01}};

// The same nodes and weights in FP32 (the FP32 quadrature of the fast path).
struct GlNodeF {
  float x, w;
};
#ifdef __CUDACC__
__constant__
#endif
    static const GlNodeF kGl16f[8] = {{9.50125098376374405e-02f, 1.89450610455068641e-01f},
                                      {2.81603550779258915e-01f, 1.82603415044923639e-01f},
                                      {4.58016777657227370e-01f, 1.69156519395002647e-01f},
                                      {6.17876244402643771e-01f, 1.49595988816576708e-01f},
                                      {7.55404408355002999e-01f, 1.24628971255534071e-01f},
                                      {8.65631202387831755e-01f, 9.51585116824926053e-02f},
                                      {9.44575023073232600e-01f, 6.22535239386474565e-02f},
                                      {9.89400934991649939e-01f, 2.71524594117541762e-02f}};
#ifdef __CUDACC__
__constant__
#endif
    static const GlNodeF kGl8f[4] = {{1.83434642495649805e-01f, 3.62683783378361983e-01f},
                                     {5.25532409916328986e-01f, 3.13706645877887287e-01f},
                                     {7.96666477413626740e-01f, 2.22381034453374471e-01f},
                                     {9.60289856497536232e-01f, 1.01228536290376259e-01f}};

// Unrolling of the FP32 quadrature's node loops (4 node pairs of a short
// interval, 8 of a panel). By 2: the refinement kernel then fits in 80
// registers (see BH_REFINE_MIN_CTAS) without spilling its hot loop; a 2048^2
// render with azimuths measured 3.41 ms against 3.61 ms fully unrolled at
// 80 registers and 3.72 ms fully unrolled at 148.
#ifndef BHM_GL_UNROLL
#define BHM_GL_UNROLL 2
#endif
constexpr int kGlUnroll = BHM_GL_UNROLL;

// a / b: IEEE division in FP64 (the closed-form tracer's results stay those
// of plain division); in FP32 on the device the 2-ulp __fdividef, ample for
// elliptic integrals carried to FP32's ~1e-7.
template <class T>
BHM_HD T qdiv(T a, T b) {
#ifdef __CUDA_ARCH__
  if constexpr (sizeof(T) == 4) return __fdividef(a, b);
#endif
  return a / b;
}

// Carlson's symmetric integral R_F(x, y, z) = 1/2 int_0^inf dt / sqrt((t+x)(t+y)(t+z)),
// x, y, z >= 0 with at most one zero.
template <class T>
BHM_HD T carlson_rf(T x, T y, T z) {
  const T tol = sizeof(T) == 4 ? T(3e-2) : T(1e-3);  // series error ~ tol^6
  for (int it = 0; it < 60; ++it) {
    const T sx = sqrt(x), sy = sqrt(y), sz = sqrt(z);
    const T lam = sx * sy + sy * sz + sz * sx;
    x = T(0.25) * (x + lam);
    y = T(0.25) * (y + lam);
    z = T(0.25) * (z + lam);
    const T A = (x + y + z) * T(1.0 / 3.0);
    const T dx = T(1) - qdiv(x, A), dy = T(1) - qdiv(y, A);
    const T dz = -(dx + dy);
    if (fmax(fabs(dx), fmax(fabs(dy), fabs(dz))) < tol) {
      const T e2 = dx * dy - dz * dz, e3 = dx * dy * dz;
      return (T(1) - T(0.1) * e2 + e3 * T(1.0 / 14.0) + e2 * e2 * T(1.0 / 24.0) - e2 * e3 * T(3.0 / 44.0)) *
             inv_sqrt(A);
    }
  }
  return T(NAN);
}

// int_0^{pi/2} dchi / sqrt(w + m sin^2 chi) = pi / (2 AGM(sqrt(w), sqrt(w + m)))
// (Gauss's arithmetic-geometric mean; quadratic convergence).
template <class T>
BHM_HD T quarter_period(T w, T m) {
  const T eps = sizeof(T) == 4 ? T(1e-7) : T(1e-15);
  T a = sqrt(w + m), g = sqrt(w);
  for (int it = 0; it < 12 && fabs(a - g) > eps * a; ++it) {
    const T an = T(0.5) * (a + g);
    g = sqrt(a * g);
    a = an;
  }
  return T(1.5707963267948966) / (T(0.5) * (a + g));
}

// ---- elliptic integrals of the third kind --------------------------------------
// (B. C. Carlson, Numer. Algorithms 10 (1995) 13-26; R. Bulirsch, Numer. Math.
// 13 (1969) 305-315.) T = double is the closed-form tracer's precision; T =
// float serves the surrogate's refinement, where each integral enters an
// azimuth of order one and FP32's ~1e-7 relative is the stated budget.

// R_C(1, 1 + e) (e > -1): atan(sqrt e) / sqrt e, atanh(sqrt -e) / sqrt -e, or
// its series for |e| < 1e-3.
template <class T>
BHM_HD T rc1(T e) {
  if (fabs(e) < T(1e-3))
    return T(1) - e * (T(1.0 / 3.0) - e * (T(0.2) - e * (T(1.0 / 7.0) - e * (T(1.0 / 9.0) - e * T(1.0 / 11.0)))));
  if (e > T(0)) {
    const T se = sqrt(e);
    return qdiv(atan(se), se);
  }
  const T se = sqrt(-e);
  return qdiv(atanh(se), se);
}

// The fifth-order expansion of R_J about the mean of its arguments.
template <class T>
BHM_HD T rj_series(T X, T Y, T Z, T P) {
  const T E2 = X * Y + X * Z + Y * Z - T(3) * P * P;
  const T E3 = X * Y * Z + T(2) * E2 * P + T(4) * P * P * P;
  const T E4 = (T(2) * X * Y * Z + E2 * P + T(3) * P * P * P) * P;
  const T E5 = X * Y * Z * P * P;
  return T(1) - T(3.0 / 14.0) * E2 + E3 * T(1.0 / 6.0) + T(9.0 / 88.0) * E2 * E2 - T(3.0 / 22.0) * E4 -
         T(9.0 / 52.0) * E2 * E3 + T(3.0 / 26.0) * E5;
}

// R_J(x, y, z, p) for p > 0 in Carlson's 1995 form: R_J = 4^-n A_n^-3/2 S +
// 6 sum_m 4^-m R_C(1, 1 + e_m) / d_m, d_m = (sqrt p_m + sqrt x_m)(sqrt p_m + sqrt y_m)
// (sqrt p_m + sqrt z_m), e_m = 4^-3m delta / d_m^2, delta = (p - x)(p - y)(p - z):
// e_m falls by 64 per step, so all but the first terms take the series.
// The series error is ~tol^6: 1e-3 in FP64, 3e-2 in FP32.
template <class T>
BHM_HD T rj_pos(T x, T y, T z, T p) {
  const T tol = sizeof(T) == 4 ? T(3e-2) : T(1e-3);
  const T delta = (p - x) * (p - y) * (p - z);
  T sum = T(0), fac = T(1), f3 = T(1);
  for (int it = 0; it < 60; ++it) {
    const T sx = sqrt(x), sy = sqrt(y), sz = sqrt(z), sp = sqrt(p);
    const T lam = sx * sy + sy * sz + sz * sx;
    const T d = (sp + sx) * (sp + sy) * (sp + sz);
    sum += qdiv(fac * rc1<T>(qdiv(f3 * delta, d * d)), d);
    fac *= T(0.25);
    f3 *= T(1.0 / 64.0);
    x = T(0.25) * (x + lam);
    y = T(0.25) * (y + lam);
    z = T(0.25) * (z + lam);
    p = T(0.25) * (p + lam);
    const T A = (x + y + z + T(2) * p) * T(0.2);
    const T X = qdiv(A - x, A), Y = qdiv(A - y, A), Z = qdiv(A - z, A), P = qdiv(A - p, A);
    if (fmax(fmax(fabs(X), fabs(Y)), fmax(fabs(Z), fabs(P))) < tol)
      return T(6) * sum + qdiv(fac * rj_series<T>(X, Y, Z, P) * inv_sqrt(A), A);
  }
  return T(NAN);
}

// Bulirsch's complete integral cel(kc, p, a, b) = int_0^(pi/2) (a cos^2 + b sin^2) /
// ((cos^2 + p sin^2) sqrt(cos^2 + kc^2 sin^2)) dphi, a Gauss-type iteration with
// quadratic convergence (stops once the relative step is below sqrt(eps));
// p < 0 gives the Cauchy principal value.
template <class T>
BHM_HD T cel(T kc, T p, T a, T b) {
  const T ca = sizeof(T) == 4 ? T(3e-4) : T(1e-15);
  kc = fabs(kc);
  T e = kc, em = T(1);
  if (p > T(0)) {
    p = sqrt(p);
    b = qdiv(b, p);
  } else {
    T f = kc * kc, q = T(1) - f;
    const T g = T(1) - p;
    f -= p;
    q *= (b - a * p);
    p = sqrt(qdiv(f, g));
    a = qdiv(a - b, g);
    b = -qdiv(q, g * g * p) + a * p;
  }
  for (int it = 0; it < 40; ++it) {
    const T f = a;
    a += qdiv(b, p);
    T g = qdiv(e, p);
    b += f * g;
    b += b;
    p = g + p;
    g = em;
    em += kc;
    if (fabs(g - kc) <= g * ca) break;
    kc = sqrt(e);
    kc += kc;
    e = kc * em;
  }
  return qdiv(T(1.5707963267948966) * (b + a * em), em * (em + p));
}

// ---- polar motion ---------------------------------------------------------------
//
// U = (z+ - u^2)(a^2 u^2 + w), u = sqrt(z+) sin chi, d tau = d chi / sqrt(w +
// mm sin^2 chi) (mm = a^2 z+): Phi(chi) = int_0^chi d tau is F(chi | -mm / w) /
// sqrt(w). chi increases along the ray; the equator is at chi = j pi, the
// turning points at chi = pi/2 + j pi. The polar part of the azimuth is
// lambda int dtau / (1 - u^2) = lambda (tau + (z+ / sqrt w) (Q(chi) - Q(chi0)))
// with Q(chi) = int_0^chi sin^2 / ((1 - z+ sin^2) dn) dchi, Q(chi + pi) = Q(chi) + 2 Q_c.
// 1 - z+ ~ lambda^2 is formed without cancellation (it falls below FP64
// resolution as lambda -> 0, where the azimuth turns by pi at each pass over
// the pole within a Mino time ~|lambda|).

struct Polar {
  bool crosses;          // U(0) > 0: the ray oscillates about the equator
  double zp, zc;         // z+ and 1 - z+
  double w, mm, m1;      // m1 = 1 + mm / w (complementary parameter of -mm / w)
  double sw, sz;         // sqrt(w), sqrt(z+)
  double K, period;      // quarter and half period (Mino time)
  double phi_start;      // Phi(chi0): chi0 the observer's amplitude
  double tau1;           // Mino time of the first crossing
  double s0, c0;         // sin, cos chi0 (c0 has the sign of du/dtau)
  double qc, q0;         // Q_c and Q(chi0) (azimuths requested; else NaN)
};

// Q(chi) for chi in [0, pi/2] from s = sin chi, c = cos chi (nc = 1 - z+).
template <class T>
BHM_HD T q_part(T nc, T s, T c, T m1) {
  return s * s * s * rj_pos<T>(c * c, c * c + m1 * s * s, T(1), c * c + nc * s * s) * T(1.0 / 3.0);
}

// u0 = cos theta_obs, pu0 = du/dtau at the observer. T: precision of the
// elliptic integrals (z+, w and the period bookkeeping stay FP64). az: also
// the observer's Q (for azimuths).
template <class T = double>
BHM_HD Polar polar_motion(double a2, double qTh, double lam, double u0, double pu0, bool az) {
  Polar t{};
  t.crosses = false;
  t.tau1 = t.period = INFINITY;
  t.qc = t.q0 = NAN;
  const double c0 = qTh - lam * lam;  // U(0)
  if (!(c0 > 0.0)) return t;
  const double b2 = a2 - qTh;
  const double sq = sqrt(b2 * b2 + 4.0 * a2 * c0);
  t.zp = (b2 > 0.0) ? (b2 + sq) / (2.0 * a2) : 2.0 * c0 / (sq - b2);
  t.zc = 2.0 * lam * lam / (a2 + qTh + sq);  // (a^2 + qTh)^2 - sq^2 = 4 a^2 lambda^2
  t.w = c0 / t.zp;
  t.mm = a2 * t.zp;
  t.m1 = 1.0 + t.mm / t.w;
  t.sw = sqrt(t.w);
  t.sz = sqrt(t.zp);
  t.s0 = fmax(-1.0, fmin(1.0, u0 / t.sz));
  // cos^2 chi0 = pu0^2 / ((a^2 u0^2 + w) z+) (U(u0) = pu0^2): no cancellation near |s0| = 1
  const double c2 = fmin(1.0, pu0 * pu0 / ((a2 * u0 * u0 + t.w) * t.zp));
  t.c0 = (pu0 >= 0.0 ? 1.0 : -1.0) * sqrt(c2);
  const double phi_x = (double)(T(t.s0) * carlson_rf<T>(T(t.w * c2), T(t.w + t.mm * t.s0 * t.s0), T(t.w)));
  t.K = (double)quarter_period<T>(T(t.w), T(t.mm));
  t.period = 2.0 * t.K;
  // moving away from the equator (du/dtau has the sign of u): chi0 in (pi/2, 3 pi/2)
  t.phi_start = (pu0 >= 0.0) ? phi_x : t.period - phi_x;
  t.tau1 = ((pu0 * u0) < 0.0) ? fabs(phi_x) : t.period - fabs(phi_x);
  t.crosses = true;
  if (az) {
    t.qc = (double)cel<T>(T(sqrt(t.m1)), T(t.zc), T(0), T(1));
    const double qp = (double)q_part<T>(T(t.zc), T(fabs(t.s0)), T(fabs(t.c0)), T(t.m1));
    // chi0 in [-pi/2, pi/2] (c0 >= 0): Q odd in chi; else chi0 = pi - chi' (Q = 2 Q_c - Q(chi'))
    const double qs = t.s0 < 0.0 ? -qp : qp;
    t.q0 = t.c0 >= 0.0 ? qs : 2.0 * t.qc - qs;
  }
  return t;
}

// Passes over the pole (chi = pi/2 + j pi) between the observer and Mino time tau.
BHM_HD double pole_passes(const Polar& t, double tau) {
  return floor((t.phi_start + tau - t.K) / t.period) - floor((t.phi_start - t.K) / t.period);
}

// lambda int_0^tau dtau / (1 - u^2) at an equatorial crossing (chi = j pi,
// Q(j pi) = 2 j Q_c). With 1 - z+ == 0 (lambda == 0, or lambda^2 below the
// smallest double) the integral is the limit lambda -> 0 of either sign: a
// turn by copysign(pi, lambda) at each pass over the pole, so lambda = +0 and
// -0 continue the two sides, which agree modulo 2 pi.
BHM_HD double phi_theta_crossing(const Polar& t, double lam, double tau) {
  if (!(t.zc > 0.0)) return copysign(3.141592653589793, lam) * pole_passes(t, tau);
  const double j = rint((t.phi_start + tau) / t.period);
  return lam * (tau + t.zp / t.sw * (2.0 * j * t.qc - t.q0));
}

// u = cos theta reached at Mino time tau (the ray must cross the equator:
// t.crosses) and, with az, the polar part of the azimuth there (as
// phi_theta_crossing). T: precision of the elliptic integrals and of the
// Newton iteration on chi; T = float gives u to a few 1e-7.
template <class T = double>
BHM_HD double polar_at(const Polar& t, double lam, double tau, bool az, double& phi_th) {
  const double total = t.phi_start + tau;
  const double n = floor(total / t.period);
  double rem = total - n * t.period;  // in [0, 2K)
  const bool second = rem > t.K;
  if (second) rem = t.period - rem;   // chi' -> pi - chi' has the same sine
  // Phi(chi') = rem on [0, pi/2]: bracketed Newton.
  const T wT = T(t.w), mT = T(t.mm), remT = T(rem);
  T lo = T(0), hi = T(1.5707963267948966), chi = T(rem * sqrt(t.w + 0.5 * t.mm));
  chi = fmin(fmax(chi, lo), hi);
  const T tol = sizeof(T) == 4 ? T(2e-7) : T(1e-15);
  for (int it = 0; it < 60; ++it) {
    const T s = sin(chi), c = cos(chi);
    const T f = s * carlson_rf<T>(wT * c * c, wT + mT * s * s, wT) - remT;
    if (f < T(0)) lo = chi; else hi = chi;
    T nc = chi - f * sqrt(wT + mT * s * s);
    if (!(nc > lo && nc < hi)) nc = T(0.5) * (lo + hi);
    const T step = nc - chi;
    chi = nc;
    if (fabs(step) < tol) break;
  }
  const T s = sin(chi), c = cos(chi);
  if (az) {
    if (!(t.zc > 0.0)) {
      phi_th = copysign(3.141592653589793, lam) * pole_passes(t, tau);
    } else {
      const double qp = (double)q_part<T>(T(t.zc), s, c, T(t.m1));
      const double q = 2.0 * n * t.qc + (second ? 2.0 * t.qc - qp : qp);
      phi_th = lam * (tau + t.zp / t.sw * (q - t.q0));
    }
  }
  const double sgn = (fmod(n, 2.0) != 0.0) ? -1.0 : 1.0;
  return sgn * t.sz * (double)s;
}

struct Radial {
  int kind;            // 1: turning point (escapes), 0: none (falls in), -1: not handled
  double p2, p1, p0;   // R = r^4 + p2 r^2 + p1 r + p0
  double x_tp;         // kind 1: 1 / r_tp
  double q3, q2, q1, q0;  // kind 1: P(x) / (x_tp - x)
  double v_obs;        // variable at the observer (kind 1: -sqrt(x_tp - x_obs); kind 0: x_obs)
  double v_end;        // variable where the tracer stops (escape or horizon)
  double r_min;        // largest local minimum of R (0 if none above r+)
  double R_min;        // R there
  double a, alam, a2;  // spin, a lambda, a^2: the radial part of the azimuth
};

BHM_HD double poly_R(const Radial& q, double r) {
  const double r2 = r * r;
  return (r2 + q.p2) * r2 + q.p1 * r + q.p0;
}

// Largest real root of R'(r) / 4 = r^3 + (p2/2) r + p1/4.
BHM_HD double largest_dR_root(double p2, double p1) {
  // FP32 closed form (trigonometric or Cardano), then two FP64 Newton steps.
  const double p = 0.5 * p2, qq = 0.25 * p1;
  const double disc = qq * qq * 0.25 + p * p * p * (1.0 / 27.0);
  float t;
  if (disc < 0.0) {  // three real roots (p < 0)
    const float rr = sqrtf((float)(-p * (1.0 / 3.0)));
    float c = (float)(-0.5 * qq) / (rr * rr * rr);
    c = fmaxf(-1.0f, fminf(1.0f, c));
    t = 2.0f * rr * cosf(acosf(c) * (1.0f / 3.0f));
  } else {
    const float sd = sqrtf((float)disc);
    t = cbrtf((float)(-0.5 * qq) + sd) + cbrtf((float)(-0.5 * qq) - sd);
  }
  double r = (double)t;
  for (int it = 0; it < 2; ++it) {
    const double g = (r * r + p) * r + qq;
    const double dg = 3.0 * r * r + p;
    if (dg != 0.0) r -= g / dg;
  }
  return r;
}

// The radial part of the azimuth: Phi_r = int a (2 r - a lambda) / Delta dtau,
// in x = 1/r a rational function, a x (2 - a lambda x) / (1 - 2 x + a^2 x^2),
// regular on every path the solve integrates (its poles are the horizons).
BHM_HD double phi_weight(const Radial& q, double x) {
  return q.a * x * (2.0 - q.alam * x) / ((q.a2 * x - 2.0) * x + 1.0);
}

// d tau / dv (and x(v)) in the ray's variable.
BHM_HD double integrand_x(const Radial& q, double v, double& x) {
  if (q.kind == 1) {
    x = q.x_tp - v * v;
    const double pt = ((q.q3 * x + q.q2) * x + q.q1) * x + q.q0;
    return 2.0 * inv_sqrt(pt);
  }
  x = v;
  const double x2 = x * x;
  const double P = 1.0 + x2 * (q.p2 + x * (q.p1 + x * q.p0));
  return inv_sqrt(P);
}

BHM_HD double integrand(const Radial& q, double v) {
  double x;
  return integrand_x(q, v, x);
}

// The same integrands entirely in FP32 (coefficients rounded once per ray).
struct RadialF {
  float x_tp, q3, q2, q1, q0;  // turning-point form
  float p2, p1, p0;            // direct form
  float a, alam, a2;           // azimuth weight
};

BHM_HD RadialF to_f32(const Radial& q) {
  return RadialF{(float)q.x_tp, (float)q.q3, (float)q.q2, (float)q.q1, (float)q.q0, (float)q.p2,
                 (float)q.p1,   (float)q.p0, (float)q.a,  (float)q.alam, (float)q.a2};
}

template <int KIND>
BHM_HD float integrand_fx(const RadialF& q, float v, float& x) {
  if (KIND == 1) {
    x = q.x_tp - v * v;
    const float pt = ((q.q3 * x + q.q2) * x + q.q1) * x + q.q0;
    return 2.0f * inv_sqrt(pt);
  }
  x = v;
  const float P = 1.0f + v * v * (q.p2 + v * (q.p1 + v * q.p0));
  return inv_sqrt(P);
}

template <int KIND>
BHM_HD float integrand_f(const RadialF& q, float v) {
  float x;
  return integrand_fx<KIND>(q, v, x);
}

BHM_HD float phi_weight_f(const RadialF& q, float x) {
#ifdef __CUDACC__
  return __fdividef(q.a * x * (2.0f - q.alam * x), (q.a2 * x - 2.0f) * x + 1.0f);
#else
  return q.a * x * (2.0f - q.alam * x) / ((q.a2 * x - 2.0f) * x + 1.0f);
#endif
}

BHM_HD double radius_of(const Radial& q, double v) { return q.kind == 1 ? 1.0 / (q.x_tp - v * v) : 1.0 / v; }

// Mino time and, with PHI, the radial azimuth integral over an interval of v.
struct TauPhi {
  double t, ph;
};

// int_{v0}^{v1} d tau (and Phi_r): composite Gauss-Legendre with panels no
// wider than hmax, 16 points per panel (ORDER 16), or 8 points on intervals
// shorter than hmax / 4 (the Newton increments near convergence).
template <int ORDER = 16, bool PHI = false>
BHM_HD TauPhi integrate2(const Radial& q, double v0, double v1, double hmax) {
  const double len = v1 - v0;
  if (len == 0.0) return TauPhi{0.0, 0.0};
  if ((ORDER == 8 || fabs(len) <= 0.25 * hmax) && fabs(len) <= hmax) {
    const double c = v0 + 0.5 * len, hh = 0.5 * len;
    double s = 0.0, sp = 0.0;
    for (int k = 0; k < 4; ++k) {
      double xa, xb;
      const double fa = integrand_x(q, c - hh * kGl8[k].x, xa), fb = integrand_x(q, c + hh * kGl8[k].x, xb);
      s += kGl8[k].w * (fa + fb);
      if (PHI) sp += kGl8[k].w * (fa * phi_weight(q, xa) + fb * phi_weight(q, xb));
    }
    return TauPhi{s * hh, sp * hh};
  }
  int n = (int)ceil(fabs(len) / hmax);
  n = n < 1 ? 1 : (n > 64 ? 64 : n);
  const double h = len / n;
  double sum = 0.0, sump = 0.0;
  for (int p = 0; p < n; ++p) {
    const double c = v0 + (p + 0.5) * h, hh = 0.5 * h;
    double s = 0.0, sp = 0.0;
    for (int k = 0; k < 8; ++k) {
      double xa, xb;
      const double fa = integrand_x(q, c - hh * kGl16[k].x, xa), fb = integrand_x(q, c + hh * kGl16[k].x, xb);
      s += kGl16[k].w * (fa + fb);
      if (PHI) sp += kGl16[k].w * (fa * phi_weight(q, xa) + fb * phi_weight(q, xb));
    }
    sum += s * hh;
    sump += sp * hh;
  }
  return TauPhi{sum, sump};
}

template <int ORDER = 16>
BHM_HD double integrate(const Radial& q, double v0, double v1, double hmax) {
  return integrate2<ORDER, false>(q, v0, v1, hmax).t;
}

// The FP32 version for radial kind KIND: nodes, integrands and panel sums in
// FP32; the sums over panels and the interval ends stay FP64.
template <int KIND, bool PHI = false>
BHM_HD TauPhi integrate_f2(const RadialF& q, double v0, double v1, double hmax) {
  const double len = v1 - v0;
  if (len == 0.0) return TauPhi{0.0, 0.0};
  if (fabs(len) <= 0.25 * hmax) {
    const float c = (float)(v0 + 0.5 * len), hh = (float)(0.5 * len);
    float s = 0.0f, sp = 0.0f;
#pragma unroll kGlUnroll
    for (int k = 0; k < 4; ++k) {
      float xa, xb;
      const float fa = integrand_fx<KIND>(q, c - hh * kGl8f[k].x, xa);
      const float fb = integrand_fx<KIND>(q, c + hh * kGl8f[k].x, xb);
      s += kGl8f[k].w * (fa + fb);
      if (PHI) sp += kGl8f[k].w * (fa * phi_weight_f(q, xa) + fb * phi_weight_f(q, xb));
    }
    return TauPhi{(double)s * (0.5 * len), (double)sp * (0.5 * len)};
  }
  int n = (int)ceil(fabs(len) / hmax);
  n = n < 1 ? 1 : (n > 64 ? 64 : n);
  const double h = len / n;
  double sum = 0.0, sump = 0.0;
  for (int p = 0; p < n; ++p) {
    const float c = (float)(v0 + (p + 0.5) * h), hh = (float)(0.5 * h);
    float s = 0.0f, sp = 0.0f;
#pragma unroll kGlUnroll
    for (int k = 0; k < 8; ++k) {
      float xa, xb;
      const float fa = integrand_fx<KIND>(q, c - hh * kGl16f[k].x, xa);
      const float fb = integrand_fx<KIND>(q, c + hh * kGl16f[k].x, xb);
      s += kGl16f[k].w * (fa + fb);
      if (PHI) sp += kGl16f[k].w * (fa * phi_weight_f(q, xa) + fb * phi_weight_f(q, xb));
    }
    sum += (double)s * (0.5 * h);
    sump += (double)sp * (0.5 * h);
  }
  return TauPhi{sum, sump};
}

template <int KIND>
BHM_HD double integrate_f(const RadialF& q, double v0, double v1, double hmax) {
  return integrate_f2<KIND, false>(q, v0, v1, hmax).t;
}

// Radial set-up. C = K of the tracer (q_R + (lambda - a)^2); a2_alam = a^2 - a lambda.
BHM_HD Radial radial_motion(double a2, double a2_alam, double C, double r_obs, double r_plus, double r_hor,
                            double r_esc) {
  Radial q{};
  q.p2 = 2.0 * a2_alam - C;
  q.p1 = 2.0 * C;
  q.p0 = a2_alam * a2_alam - a2 * C;
  q.a2 = a2;
  q.kind = -1;
  if (q.p0 > 0.0) return q;  // q_R < 0: more than two roots possible above r+
  const double rm = largest_dR_root(q.p2, q.p1);
  q.r_min = 0.0;
  q.R_min = 0.0;
  if (rm > r_plus) {
    q.r_min = rm;
    q.R_min = poly_R(q, rm);
  }
  if (q.r_min > 0.0 && q.R_min < 0.0) {
    // Largest root of R: Newton from the right on the convex branch.
    const double d2 = 12.0 * rm * rm + 2.0 * q.p2;
    double r = rm + sqrt(-2.0 * q.R_min / fmax(d2, 1e-300));
    for (int it = 0; it < 100; ++it) {
      const double r2 = r * r;
      const double R = (r2 + q.p2) * r2 + q.p1 * r + q.p0;
      const double dR = 4.0 * r2 * r + 2.0 * q.p2 * r + q.p1;
      const double dr = R / dR;
      r -= dr;
      if (fabs(dr) <= 1e-15 * r) break;
    }
    if (!(r > r_hor) || !(r < r_obs)) return q;  // turning point inside the horizon cut or beyond the observer
    q.kind = 1;
    q.x_tp = 1.0 / r;
    // P(x) = (x - x_tp) Q(x) (synthetic division, remainder dropped); P / (x_tp - x) = -Q.
    const double b3 = q.p0;
    const double b2 = q.p1 + q.x_tp * b3;
    const double b1 = q.p2 + q.x_tp * b2;
    const double b0 = q.x_tp * b1;
    q.q3 = -b3;
    q.q2 = -b2;
    q.q1 = -b1;
    q.q0 = -b0;
    q.v_obs = -sqrt(q.x_tp - 1.0 / r_obs);
    q.v_end = sqrt(q.x_tp - 1.0 / r_esc);
  } else {
    q.kind = 0;
    q.v_obs = 1.0 / r_obs;
    q.v_end = 1.0 / r_hor;
  }
  return q;
}

// The azimuth weight's constants (spin a, lambda).
BHM_HD void set_azimuth(Radial& q, double a, double lam) {
  q.a = a;
  q.alam = a * lam;
}

// Solve tau(v) = T on [lo, hi] given tau(lo) = tlo <= T, where tau is
// increasing: Newton steps safeguarded by bisection of the bracket, each new
// tau(v) from the last by an increment of quadrature. Returns 1 with (v, tau)
// when found, 0 when tau(hi) < T (the ray stops before reaching T), -1 if
// the iteration did not settle. seed: a first guess inside (lo, hi), or NaN.
// FAST: FP32 quadrature (radial kind KIND), whose ~1e-8 noise in tau sets
// the acceptance tolerance. PHI: Phi_r is carried along the same increments
// (it telescopes exactly like tau, so it ends as Phi_r(v_out)).
template <bool FAST, int KIND, bool PHI>
struct Quad {
  const Radial& q;
  RadialF f;
  BHM_HD double integ(double a, double b, double hmax) const {
    return FAST ? integrate_f<KIND>(f, a, b, hmax) : integrate<16>(q, a, b, hmax);
  }
  BHM_HD TauPhi integ2(double a, double b, double hmax) const {
    return FAST ? integrate_f2<KIND, PHI>(f, a, b, hmax) : integrate2<16, PHI>(q, a, b, hmax);
  }
  BHM_HD double at(double v) const { return FAST ? (double)integrand_f<KIND>(f, (float)v) : integrand(q, v); }
};

template <bool FAST, int KIND, bool PHI>
BHM_HD int solve_tau(const Quad<FAST, KIND, PHI>& Q, double T, double lo, double tlo, double plo, double hi,
                     double seed, double hmax, double& v_out, double& t_out, double& p_out) {
  double v = lo, tv = tlo, pv = plo;
  if (seed > lo && seed < hi) {
    v = seed;
    const TauPhi d = Q.integ2(lo, seed, hmax);
    tv = tlo + d.t;
    pv = plo + d.ph;
  }
  bool end_known = false;  // tau(hi) evaluated once, when Newton first aims past the end of the ray
  for (int it = 0; it < 80; ++it) {
    if (tv <= T) {
      lo = v;
      tlo = tv;
    } else {
      hi = v;
      end_known = true;
    }
    double vn = v + (T - tv) / Q.at(v);
    if (!(vn < hi) && !end_known) {
      const double t_hi = tv + Q.integ(v, hi, hmax);
      if (t_hi < T) {
        v_out = hi;
        t_out = t_hi;
        p_out = NAN;  // not carried: the ray ends before T
        return 0;
      }
      end_known = true;
    }
    if (!(vn > lo && vn < hi)) vn = 0.5 * (lo + hi);
    const double step = vn - v;
    const TauPhi d = Q.integ2(v, vn, hmax);
    tv += d.t;
    pv += d.ph;
    v = vn;
    // Newton converges quadratically here: once a step is below tol_v the
    // error left is of order tol_v^2 relative, far below FP32 quadrature
    // noise (~1e-8) in the fast path.
    const double tol_v = FAST ? 1e-6 : 1e-14;
    if (fabs(step) <= tol_v * fmax(1e-3, fabs(v))) {
      v_out = v;
      t_out = tv;
      p_out = pv;
      if (fabs(tv - T) <= (FAST ? 1e-6 : 1e-9) * fmax(1.0, T)) return 1;
      return (tv < T) ? 0 : -1;  // pinned at the end of the ray: no crossing before it stops
    }
  }
  return -1;
}

struct Crossings {
  int status;      // 0 ok, -1 radial form not handled, -2 no convergence
  int kind;        // radial kind (1 escapes, 0 falls in)
  int n_hits;      // disk hits found (<= max_hits)
  double r[3];     // their radii
  double tau[3];   // their Mino times (the polar crossing times)
  double phr[3];   // Phi_r at each (with azimuths)
  double v_last;   // variable, Mino time and Phi_r of the last solved crossing (or the observer)
  double t_last;
  double p_last;
  double r_min;    // largest local minimum of R above r+ (0 if none) ...
  double R_min;    // ... and R there: near zero next to the critical curve
};

template <bool FAST, int KIND, bool PHI>
BHM_HD void crossing_loop(const Radial& q, const Polar& th, double r_in, double r_out, double r_seed,
                          int max_hits, double hmax, Crossings& c) {
  const Quad<FAST, KIND, PHI> Q{q, to_f32(q)};
  double seed_v[2] = {NAN, NAN};
  if (r_seed > 0.0) {
    if (KIND == 1) {
      const double s = sqrt(fmax(0.0, q.x_tp - 1.0 / r_seed));
      seed_v[0] = -s;
      seed_v[1] = s;
    } else {
      seed_v[0] = 1.0 / r_seed;
    }
  }
  double lo = q.v_obs, tlo = 0.0, plo = 0.0;
  for (int n = 0; n < 64; ++n) {
    const double T = th.tau1 + n * th.period;
    double seed = NAN;
    if (seed_v[0] > lo && seed_v[0] < q.v_end)
      seed = seed_v[0];
    else if (seed_v[1] > lo && seed_v[1] < q.v_end)
      seed = seed_v[1];
    double v, tv, pv;
    const int rc = solve_tau<FAST, KIND, PHI>(Q, T, lo, tlo, plo, q.v_end, seed, hmax, v, tv, pv);
    if (rc < 0) {
      c.status = -2;
      return;
    }
    if (rc == 0) return;  // the ray stops before this crossing
    const double r = radius_of(q, v);
    lo = v;
    tlo = tv;
    plo = pv;
    c.v_last = v;
    c.t_last = tv;
    c.p_last = pv;
    if (r >= r_in && r <= r_out) {
      // constant indices keep the per-hit records in registers
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (k == c.n_hits) {
          c.r[k] = r;
          c.tau[k] = T;
          c.phr[k] = pv;
        }
      if (++c.n_hits >= max_hits) return;
    }
  }
}

// Disk crossings (r_in <= r <= r_out) of a ray in the order the tracer finds
// them, up to max_hits (<= 3), from its radial motion q and polar motion th
// (polar_motion). r_seed > 0 is a guess of the first hit radius that starts
// the Newton iterations. FAST: FP32 quadrature (r to ~4e-6 instead of
// ~1e-8). PHI: Phi_r at each hit (set_azimuth(q, ...) first).
template <bool FAST = false, bool PHI = false>
BHM_HD Crossings crossings(const Radial& q, const Polar& th, double r_in, double r_out, double r_seed,
                           int max_hits, double hmax) {
  Crossings c{};
  c.status = 0;
  c.n_hits = 0;
  c.kind = q.kind;
  c.r_min = q.r_min;
  c.R_min = q.R_min;
  c.v_last = q.v_obs;
  c.t_last = 0.0;
  c.p_last = 0.0;
  if (q.kind < 0) {
    c.status = -1;
    return c;
  }
  if (!th.crosses) return c;
  if (q.kind == 1)
    crossing_loop<FAST, 1, PHI>(q, th, r_in, r_out, r_seed, max_hits, hmax, c);
  else
    crossing_loop<FAST, 0, PHI>(q, th, r_in, r_out, r_seed, max_hits, hmax, c);
  return c;
}

// Mino time (and, with PHI, Phi_r) at which the tracer stops (escape or
// horizon radius), from a point (v, tau(v), Phi_r(v)) of the ray.
template <bool FAST = false, bool PHI = false>
BHM_HD TauPhi tau_end(const Radial& q, double v, double tv, double pv, double hmax) {
  TauPhi d;
  if (FAST) {
    const RadialF f = to_f32(q);
    d = q.kind == 1 ? integrate_f2<1, PHI>(f, v, q.v_end, hmax) : integrate_f2<0, PHI>(f, v, q.v_end, hmax);
  } else {
    d = integrate2<16, PHI>(q, v, q.v_end, hmax);
  }
  return TauPhi{tv + d.t, pv + d.ph};
}

// First-order image-plane distance (M) from pixel (alpha, beta) to the
// critical curve: |R(r_min)| over the (alpha, beta) gradient of R at fixed
// r = r_min (the envelope of R's minimum). carter selects q_R = eta
// (textbook) instead of the reference's q_R = eta + lambda^2.
BHM_HD double critical_distance(double r_min, double R_min, double a, double lam, bool carter, double sin_o,
                                double cos_o, double alpha, double beta) {
  if (!(r_min > 0.0)) return INFINITY;
  const double r = r_min;
  const double A = r * r + a * a - a * lam;
  const double D = r * r - 2.0 * r + a * a;
  const double dC_dlam = (carter ? 0.0 : 2.0 * lam) + 2.0 * (lam - a);
  const double dR_dlam = -2.0 * a * A - D * dC_dlam;
  const double dR_deta = -D;
  const double gx = -dR_dlam * sin_o + dR_deta * 2.0 * alpha * cos_o * cos_o;
  const double gy = dR_deta * 2.0 * beta;
  return fabs(R_min) / fmax(sqrt(gx * gx + gy * gy), 1e-300);
}

}  // namespace bhmino
