// kerr_analytic.cuh - closed-form Kerr null rays in Mino time (FP64; device
// code under nvcc, plain C++ elsewhere).
//
// The image tracer integrates (r, u = cos theta, phi) in Mino time tau with
// p_r^2 = R(r) = r^4 + p2 r^2 + p1 r + p0 and p_u^2 = U(u). Here the same ray
// is written down instead of stepped:
//
// * r(tau), from the roots of R (Gralla & Lupsasca, "Null geodesics of the
//   Kerr exterior", Phys. Rev. D 101, 044032 (2020), section IV), in three
//   root configurations, roots ascending r1 <= r2 <= r3 <= r4, rij = ri - rj:
//     S   four real roots, r_hor < r4 < r_obs: the ray turns at r4.
//           X = (1/2) sqrt(r31 r42) (tau - tau_tp),
//           r = (r4 r31 - r3 r41 sn^2(X|m)) / (r31 - r41 sn^2(X|m)),
//           m = r32 r41 / (r31 r42), 1 - m = r21 r43 / (r31 r42);
//     P4  four real roots below the horizon: the same form, X decreasing
//           from X(r_obs) (r > r4 throughout);
//     P2  real r1 < r2 below the horizon and a complex pair c +- i d:
//           X = sqrt(A B) I, A = |r2 - r3|, B = |r1 - r3|,
//           r = ((B r2 - A r1) + (B r2 + A r1) cn(X|m)) / ((B - A) + (B + A) cn(X|m)),
//           m = ((A + B)^2 - r21^2) / (4 A B).
//   The complementary parameter 1 - m is formed from root differences
//   without cancellation, so rays next to the critical curve (1 - m -> 0,
//   many half-orbits) keep full precision.
// * u(tau) = sqrt(z+) sin chi, chi = am(sqrt(w) (Phi_0 + tau) | -m_th / w).
// * phi(tau) = -(Phi_r + Phi_th) (the tracer's time-reversed azimuth), with
//   Phi_r = a / (r+ - r-) sum_(+-) +-(2 r+- - a lambda) int dtau / (r - r+-) and
//   Phi_th = lambda int dtau / (1 - u^2): elliptic integrals of the third
//   kind in Carlson's form, R_J with its Cauchy principal value where the
//   characteristic crosses the path's parameter range.
//
// sn, cn, dn by Bulirsch's descending Landen sequence (negative parameters of
// the polar motion by Abramowitz & Stegun 16.10); the amplitude of every
// point the ray reports is known in closed form or from sn, cn (the
// observer's and the escape radius from the roots, an equatorial crossing at
// chi = j pi), so no inverse trigonometric recursion is needed. Carlson's
// R_F, R_C and R_J by duplication (B. C. Carlson, "Numerical computation of
// real or complex elliptic integrals", Numer. Algorithms 10 (1995) 13-26;
// R_J in that paper's form with R_C(1, 1 + e_m), and for p < 0 through the
// transformation of its section 4); complete integrals of the third kind by
// Bulirsch's cel.
#pragma once

#include "mino_solve.cuh"

// The heavy routines are calls on the device (each keeps its working set in
// its own frame instead of the caller's registers), with internal linkage:
// nvcc's host stubs of external device functions would otherwise take the
// names of the host build of this header in the same library.
#ifdef __CUDACC__
#define BHA_CALL static __device__ __noinline__
#else
#define BHA_CALL inline
#endif
// The routines that take a ray's solution (RadSol, PolSol, JPole) by
// reference: device calls as well unless BHA_INLINE_SOLUTION is defined, in
// which case they are inlined, so the solution can stay in registers instead
// of the stack frame (for kernels compiled with registers to hold it).
#ifdef BHA_INLINE_SOLUTION
#define BHA_SCALL BHM_HD
#else
#define BHA_SCALL BHA_CALL
#endif
// The azimuth's routines among them (the elliptic integrals of the third
// kind and their per-ray constants) alone: BHA_INLINE_PHI.
#if defined(BHA_INLINE_SOLUTION) || defined(BHA_INLINE_PHI)
#define BHA_PCALL BHM_HD
#else
#define BHA_PCALL BHA_CALL
#endif

namespace bhan {

using bhmino::inv_sqrt;

// Carlson's R_F as one shared device call: inlined at each of its call sites
// it made the tracer's code large enough that instruction fetch, not
// arithmetic, bounded the kernel (ncu: "no instruction" was 17 of 24 stall
// cycles per issue); as a call the image takes 17 % less time.
BHA_CALL double carlson_rf(double x, double y, double z) { return bhmino::carlson_rf<double>(x, y, z); }
#ifndef __CUDACC__
using std::isnan;
#endif

// R_C(x, y) = R_F(x, y, y) in closed form, the Cauchy principal value for
// y < 0: R_C(x, y) = R_C(1, 1 + d) / sqrt(x), d = (y - x) / x, with
// R_C(1, 1 + d) = atan(sqrt d) / sqrt d (d > 0), atanh(sqrt -d) / sqrt -d
// (d < 0), and its series 1 - d/3 + d^2/5 - ... for |d| < 1e-3.
BHM_HD double carlson_rc(double x, double y) {
  double f = 1.0;
  if (y < 0.0) {
    f = sqrt(x / (x - y));
    x = x - y;
    y = -y;
  }
  if (x == 0.0) return f * 1.5707963267948966 / sqrt(y);
  const double d = (y - x) / x;
  double g;
  if (fabs(d) < 1e-3) {
    g = 1.0 - d * (1.0 / 3.0 - d * (0.2 - d * (1.0 / 7.0 - d * (1.0 / 9.0 - d * (1.0 / 11.0)))));
  } else if (d > 0.0) {
    const double sd = sqrt(d);
    g = atan(sd) / sd;
  } else {
    const double sd = sqrt(-d);
    g = atanh(sd) / sd;
  }
  return f * g * inv_sqrt(x);
}

// R_C(1, 1 + e) (e > -1), shared with the surrogate's refinement (mino_solve.cuh).
BHM_HD double carlson_rc1(double e) { return bhmino::rc1<double>(e); }

// R_J(x, y, z, p) for p > 0 in Carlson's 1995 form (mino_solve.cuh), as one
// shared device call.
BHA_CALL double carlson_rj_pos(double x, double y, double z, double p) { return bhmino::rj_pos<double>(x, y, z, p); }
BHM_HD double rj_series(double X, double Y, double Z, double P) { return bhmino::rj_series<double>(X, Y, Z, P); }

// R_J for any p != 0 (x, y, z >= 0, at most one zero); p < 0 gives the
// Cauchy principal value via an R_J with positive fourth argument.
BHA_CALL double carlson_rj(double x, double y, double z, double p) {
  if (p > 0.0) return carlson_rj_pos(x, y, z, p);
  // sort so that x <= y <= z
  if (x > y) { const double t = x; x = y; y = t; }
  if (y > z) { const double t = y; y = z; z = t; }
  if (x > y) { const double t = x; x = y; y = t; }
  const double a = 1.0 / (y - p);
  const double b = a * (z - y) * (y - x);
  const double pt = y + b;
  const double rho = x * z / y;
  const double tau = p * pt / y;
  return a * (b * carlson_rj_pos(x, y, z, pt) + 3.0 * (carlson_rc(rho, tau) - carlson_rf(x, y, z)));
}

// R_J(x, y, z, p1) and R_J(x, y, z, p2) for p1, p2 > 0 in one duplication
// sequence (the x, y, z part of each step is shared), Carlson's 1995 form.
BHA_CALL void carlson_rj2(double x, double y, double z, double p1, double p2, double &o1, double &o2) {
  const double dxyz1 = (p1 - x) * (p1 - y) * (p1 - z), dxyz2 = (p2 - x) * (p2 - y) * (p2 - z);
  double s1 = 0.0, s2 = 0.0, fac = 1.0, f3 = 1.0;
  for (int it = 0; it < 60; ++it) {
    const double sx = sqrt(x), sy = sqrt(y), sz = sqrt(z), sp1 = sqrt(p1), sp2 = sqrt(p2);
    const double lam = sx * sy + sy * sz + sz * sx;
    const double d1 = (sp1 + sx) * (sp1 + sy) * (sp1 + sz), d2 = (sp2 + sx) * (sp2 + sy) * (sp2 + sz);
    s1 += fac * carlson_rc1(f3 * dxyz1 / (d1 * d1)) / d1;
    s2 += fac * carlson_rc1(f3 * dxyz2 / (d2 * d2)) / d2;
    fac *= 0.25;
    f3 *= 1.0 / 64.0;
    x = 0.25 * (x + lam);
    y = 0.25 * (y + lam);
    z = 0.25 * (z + lam);
    p1 = 0.25 * (p1 + lam);
    p2 = 0.25 * (p2 + lam);
    const double A1 = (x + y + z + 2.0 * p1) * 0.2, A2 = (x + y + z + 2.0 * p2) * 0.2;
    const double X1 = (A1 - x) / A1, Y1 = (A1 - y) / A1, Z1 = (A1 - z) / A1, P1 = (A1 - p1) / A1;
    const double X2 = (A2 - x) / A2, Y2 = (A2 - y) / A2, Z2 = (A2 - z) / A2, P2 = (A2 - p2) / A2;
    const double e1 = fmax(fmax(fabs(X1), fabs(Y1)), fmax(fabs(Z1), fabs(P1)));
    const double e2 = fmax(fmax(fabs(X2), fabs(Y2)), fmax(fabs(Z2), fabs(P2)));
    if (fmax(e1, e2) < 1e-3) {
      o1 = 6.0 * s1 + fac * rj_series(X1, Y1, Z1, P1) * inv_sqrt(A1) / A1;
      o2 = 6.0 * s2 + fac * rj_series(X2, Y2, Z2, P2) * inv_sqrt(A2) / A2;
      return;
    }
  }
  o1 = o2 = NAN;
}

// sn, cn, dn(u | m), m = 1 - m1 in [0, 1): R. Bulirsch, "Numerical calculation
// of elliptic integrals and elliptic functions", Numer. Math. 7 (1965)
// 78-90 -- the descending Landen sequence by the AGM, one sin and cos at its
// end, and a backward recurrence for cn/sn and dn; accurate to ~|u| eps.
BHA_CALL void sncndn(double u, double m1, double &sn, double &cn, double &dn) {
  constexpr int kMax = 14;
  double em[kMax], en[kMax];
  double a = 1.0, emc = m1, c = 1.0;
  int n = kMax;
#pragma unroll 1
  for (int k = 0; k < kMax; ++k) {
    em[k] = a;
    emc = sqrt(emc);
    en[k] = emc;
    c = 0.5 * (a + emc);
    if (fabs(a - emc) <= 1e-15 * a) {
      n = k + 1;
      break;
    }
    emc *= a;
    a = c;
  }
  const double v = u * c;
  sn = sin(v);
  cn = cos(v);
  dn = 1.0;
  if (sn != 0.0) {
    double t = cn / sn, cc = c * t;
#pragma unroll 1
    for (int k = n - 1; k >= 0; --k) {
      const double b = em[k];
      t *= cc;
      cc *= dn;
      dn = (en[k] + t) / (b + t);
      t = cc / b;
    }
    const double r = 1.0 / sqrt(cc * cc + 1.0);
    sn = sn >= 0.0 ? r : -r;
    cn = cc * sn;
  }
}

// sn, cn, dn(u | m) for m = 1 - m1 < 0 (m1 > 1): Abramowitz & Stegun 16.10.2-4,
// sn(u | m) = sd(u sqrt(m1) | mu) / sqrt(m1), cn = cd, dn = nd, mu = 1 - 1 / m1.
BHM_HD void sncndn_neg(double u, double m1, double &sn, double &cn, double &dn) {
  const double r = sqrt(m1);
  double s, c, d;
  sncndn(u * r, 1.0 / m1, s, c, d);
  sn = s / (d * r);
  cn = c / d;
  dn = 1.0 / d;
}

// Bulirsch's complete integral cel(kc, p, a, b) (mino_solve.cuh; p < 0 gives
// the Cauchy principal value), as one shared device call.
BHA_CALL double bulirsch_cel(double kc, double p, double a, double b) { return bhmino::cel<double>(kc, p, a, b); }

// The complete Q(n; pi/2 | m) = int_0^(pi/2) sin^2 / ((1 - n sin^2) dn) = cel(sqrt m1, 1 - n, 0, 1).
BHM_HD double ellip_qc(double n, double m1) { return bulirsch_cel(sqrt(m1), 1.0 - n, 0.0, 1.0); }

// Incomplete F(phi | m) for phi in [-pi/2, pi/2] from sin, cos (Carlson's form).
BHM_HD double ellip_f(double s, double c, double m1) { return s * carlson_rf(c * c, c * c + m1 * s * s, 1.0); }

// Q(n; phi | m) from the amplitude's sine s and cosine c, phi in [-pi/2, pi]
// (c < 0: phi = pi - phi' with Q(phi) = 2 Q(pi/2) - Q(phi')).
BHM_HD double q_part(double n, double s, double c, double m1) {
  return s * s * s * carlson_rj(c * c, c * c + m1 * s * s, 1.0, 1.0 - n * s * s) * (1.0 / 3.0);
}
BHA_PCALL double ellip_q_sc(double n, double s, double c, double m1, double &qc) {
  if (c >= 0.0) return q_part(n, s, c, m1);
  if (isnan(qc)) qc = ellip_qc(n, m1);
  return 2.0 * qc - q_part(n, s, -c, m1);
}
// The same with the complement nc = 1 - n given (1 - n s^2 = c^2 + nc s^2 with
// no cancellation): the polar motion's n = z+ tends to 1 as lambda -> 0, and
// 1 - z+ ~ lambda^2 drops below FP64 resolution when formed from z+.
BHM_HD double ellip_qc_nc(double nc, double m1) { return bulirsch_cel(sqrt(m1), nc, 0.0, 1.0); }
BHM_HD double q_part_nc(double nc, double s, double c, double m1) {
  return s * s * s * carlson_rj(c * c, c * c + m1 * s * s, 1.0, c * c + nc * s * s) * (1.0 / 3.0);
}
BHA_PCALL double ellip_q_sc_nc(double nc, double s, double c, double m1, double &qc) {
  if (c >= 0.0) return q_part_nc(nc, s, c, m1);
  if (isnan(qc)) qc = ellip_qc_nc(nc, m1);
  return 2.0 * qc - q_part_nc(nc, s, -c, m1);
}
// Both poles at once (the same amplitude, characteristics n1, n2; c >= 0).
BHA_PCALL void ellip_q2_sc(double n1, double n2, double s, double c, double m1, double &q1, double &q2) {
  const double x = c * c, y = c * c + m1 * s * s, s2 = s * s, s3 = s2 * s * (1.0 / 3.0);
  const double p1 = 1.0 - n1 * s2, p2 = 1.0 - n2 * s2;
  if (p1 > 0.0 && p2 > 0.0) {
    double a, b;
    carlson_rj2(x, y, 1.0, p1, p2, a, b);
    q1 = s3 * a;
    q2 = s3 * b;
  } else {
    q1 = s3 * carlson_rj(x, y, 1.0, p1);
    q2 = s3 * carlson_rj(x, y, 1.0, p2);
  }
}

// ---- radial motion ----------------------------------------------------------------

enum RadType { kUnhandled = -1, kCaptured = 0, kS = 1, kP4 = 2, kP2 = 3 };

// The amplitude of a radial point: its sine, cosine and delta (dn).
struct Amp {
  double s, c, d;
};

struct RadSol {
  int type;
  double r1, r2, r3, r4;  // S, P4: the four roots; P2: r1, r2 and (r3, r4) = (c, d)
  double m1;              // complementary parameter
  double sc;              // dX / dtau
  double A, B;            // P2
  double X0;              // X at the observer (tau = 0)
  double dir;             // dX / dtau sign: +1 (S), -1 (P4, P2)
  double tau_end;         // Mino time at which the tracer stops (escape or horizon radius)
  Amp a0;                 // amplitude at the observer
  double X_end;           // S: X at the escape radius ...
  Amp a_end;              // ... and its amplitude
};

BHM_HD double newton_root(double p2, double p1, double p0, double r) {
  for (int it = 0; it < 100; ++it) {
    const double r2 = r * r;
    const double R = (r2 + p2) * r2 + p1 * r + p0;
    const double dR = 4.0 * r2 * r + 2.0 * p2 * r + p1;
    const double dr = R / dR;
    r -= dr;
    if (fabs(dr) <= 1e-15 * fabs(r)) break;
  }
  return r;
}

// Ferrari's factorization x^4 + p2 x^2 + p1 x + p0 = (x^2 + al x + be)(x^2 - al x + ga),
// al^2 = z the largest root of the resolvent cubic z^3 + 2 p2 z^2 + (p2^2 - 4 p0) z - p1^2
// (found in closed form, then polished by Newton); false if z <= 0.
BHA_CALL bool ferrari_factor(double p2, double p1, double p0, double &al, double &be, double &ga) {
  // depressed resolvent: z = t - 2 p2 / 3, t^3 + P t + Q = 0
  const double P = -(p2 * p2) * (1.0 / 3.0) - 4.0 * p0;
  const double Q = -(2.0 / 27.0) * p2 * p2 * p2 + (8.0 / 3.0) * p2 * p0 - p1 * p1;
  const double disc = 0.25 * Q * Q + P * P * P * (1.0 / 27.0);
  double t;
  if (disc < 0.0) {
    const double rr = sqrt(-P * (1.0 / 3.0));
    const double cc = fmax(-1.0, fmin(1.0, (-0.5 * Q) / (rr * rr * rr)));
    t = 2.0 * rr * cos(acos(cc) * (1.0 / 3.0));
  } else {
    const double sd = sqrt(disc);
    t = cbrt(-0.5 * Q + sd) + cbrt(-0.5 * Q - sd);
  }
  double z = t - (2.0 / 3.0) * p2;
  for (int it = 0; it < 3; ++it) {
    const double f = ((z + 2.0 * p2) * z + (p2 * p2 - 4.0 * p0)) * z - p1 * p1;
    const double df = (3.0 * z + 4.0 * p2) * z + (p2 * p2 - 4.0 * p0);
    if (df != 0.0) z -= f / df;
  }
  if (!(z > 0.0)) return false;
  al = sqrt(z);
  be = 0.5 * (p2 + z - p1 / al);
  ga = 0.5 * (p2 + z + p1 / al);
  return true;
}

// Real roots of x^4 + p2 x^2 + p1 x + p0 from that factorization, polished
// by Newton. Returns the number of real roots (ascending in re[]); with two,
// (c, d) of the complex pair and its squared modulus c^2 + d^2 (the constant
// term of its quadratic factor).
BHA_CALL int ferrari(double p2, double p1, double p0, double re[4], double &c, double &d, double &mod2) {
  double al, be, ga;
  if (!ferrari_factor(p2, p1, p0, al, be, ga)) return -1;
  const double z = al * al;
  const double d1 = z - 4.0 * be, d2 = z - 4.0 * ga;
  int n = 0;
  if (d1 >= 0.0) {
    const double s = sqrt(d1);
    re[n++] = 0.5 * (-al - s);
    re[n++] = 0.5 * (-al + s);
  } else {
    c = -0.5 * al;
    d = 0.5 * sqrt(-d1);
    mod2 = be;
  }
  if (d2 >= 0.0) {
    const double s = sqrt(d2);
    re[n++] = 0.5 * (al - s);
    re[n++] = 0.5 * (al + s);
  } else {
    c = 0.5 * al;
    d = 0.5 * sqrt(-d2);
    mod2 = ga;
  }
  for (int k = 0; k < n; ++k) re[k] = newton_root(p2, p1, p0, re[k]);
  for (int i = 1; i < n; ++i)  // ascending
    for (int j = i; j > 0 && re[j] < re[j - 1]; --j) {
      const double tmp = re[j];
      re[j] = re[j - 1];
      re[j - 1] = tmp;
    }
  return n;
}

// X(r) = the Jacobi argument of radius r (S, P4: F(phi | m) from r4; P2:
// from r2), with its amplitude's sine, cosine and delta written without
// cancellation from the roots.
BHA_SCALL double x_of_r(const RadSol &q, double r, Amp &a) {
  if (q.type == kP2) {
    const double A = q.A, B = q.B;
    const double num = A * (r - q.r1) - B * (r - q.r2);
    const double den = A * (r - q.r1) + B * (r - q.r2);
    a.c = num / den;
    a.s = 2.0 * sqrt(A * B * (r - q.r1) * (r - q.r2)) / den;
    a.d = sqrt(a.c * a.c + q.m1 * a.s * a.s);
    const double F = ellip_f(a.s, fabs(a.c), q.m1);
    return (a.c < 0.0) ? 2.0 * carlson_rf(0.0, q.m1, 1.0) - F : F;
  }
  const double r31 = q.r3 - q.r1, r41 = q.r4 - q.r1, r43 = q.r4 - q.r3;
  const double s2 = r31 * (r - q.r4) / (r41 * (r - q.r3));
  const double c2 = r43 * (r - q.r1) / (r41 * (r - q.r3));
  a.s = sqrt(s2);
  a.c = sqrt(c2);
  a.d = sqrt(c2 + q.m1 * s2);
  return a.s * carlson_rf(c2, c2 + q.m1 * s2, 1.0);
}

// Radial solution of a ray with R = r^4 + p2 r^2 + p1 r + p0 seen from r_obs;
// the tracer stops at r_hor (captured) or r_esc (escaped). crosses: whether
// the polar motion reaches the equator (rays that do not are only classified).
BHA_SCALL RadSol radial(double p2, double p1, double p0, double r_plus, double r_hor, double r_obs, double r_esc,
                       bool crosses) {
  RadSol q{};
  q.type = kUnhandled;
  double re[4], c = 0.0, d = 0.0, mod2 = 0.0;
  if (p0 > 0.0) {  // q_R < 0: possibly several turning points above r+
    if (crosses) return q;
    const int n = ferrari(p2, p1, p0, re, c, d, mod2);
    if (n < 0) return q;
    for (int k = 0; k < n; ++k)
      if (re[k] >= r_hor) return q;
    q.type = kCaptured;
    return q;
  }
  const double rm = bhmino::largest_dR_root(p2, p1);
  const double Rm = rm > r_plus ? (rm * rm + p2) * rm * rm + p1 * rm + p0 : 1.0;
  if (rm > r_plus && Rm < 0.0) {
    const double d2 = 12.0 * rm * rm + 2.0 * p2;
    const double off = sqrt(-2.0 * Rm / fmax(d2, 1e-300));
    const double r4 = newton_root(p2, p1, p0, rm + off);
    if (!(r4 > r_hor) || !(r4 < r_obs) || !crosses) return q;
    const double r3 = newton_root(p2, p1, p0, rm - off);
    if (!(r3 < r4)) return q;
    const double sm = -(r3 + r4), pr = p0 / (r3 * r4);
    const double sq = sqrt(fmax(sm * sm - 4.0 * pr, 0.0));
    q.r1 = 0.5 * (sm - sq);
    q.r2 = 0.5 * (sm + sq);
    q.r3 = r3;
    q.r4 = r4;
    q.type = kS;
  } else {
    if (!crosses) {
      q.type = kCaptured;
      return q;
    }
    const int n = ferrari(p2, p1, p0, re, c, d, mod2);
    if (n == 4) {
      if (!(re[3] < r_hor)) return q;
      q.r1 = re[0];
      q.r2 = re[1];
      q.r3 = re[2];
      q.r4 = re[3];
      q.type = kP4;
    } else if (n == 2) {
      q.r1 = re[0];
      q.r2 = re[1];
      c = -0.5 * (q.r1 + q.r2);  // the roots sum to zero
      const double dd = mod2 - c * c;
      if (!(dd > 0.0) || !(q.r2 < r_hor)) return q;
      q.r3 = c;
      q.r4 = sqrt(dd);
      q.type = kP2;
    } else {
      return q;
    }
  }
  Amp a_h;
  if (q.type == kP2) {
    const double c_ = q.r3, d_ = q.r4;
    const double u2 = c_ - q.r2, u1 = c_ - q.r1, d2 = d_ * d_;
    const double A = sqrt(u2 * u2 + d2), B = sqrt(u1 * u1 + d2);
    const double r21 = q.r2 - q.r1;
    // 1 - m = r21^2 ((A - u2) + (B - u1)) ((A + u2) + (B + u1)) / ((A + B)^2 4 A B), each sum without cancellation
    const double amu2 = u2 > 0.0 ? d2 / (A + u2) : A - u2;
    const double bmu1 = u1 > 0.0 ? d2 / (B + u1) : B - u1;
    const double apu2 = u2 > 0.0 ? A + u2 : d2 / (A - u2);
    const double bpu1 = u1 > 0.0 ? B + u1 : d2 / (B - u1);
    q.A = A;
    q.B = B;
    q.m1 = r21 * r21 * (amu2 + bmu1) * (apu2 + bpu1) / ((A + B) * (A + B) * 4.0 * A * B);
    q.sc = sqrt(A * B);
    q.X0 = x_of_r(q, r_obs, q.a0);
    q.dir = -1.0;
    q.tau_end = (q.X0 - x_of_r(q, r_hor, a_h)) / q.sc;
  } else {
    const double r31 = q.r3 - q.r1, r42 = q.r4 - q.r2, r21 = q.r2 - q.r1, r43 = q.r4 - q.r3;
    q.m1 = r21 * r43 / (r31 * r42);
    q.sc = 0.5 * sqrt(r31 * r42);
    const double x_obs = x_of_r(q, r_obs, q.a0);
    if (q.type == kS) {  // X runs from -X(r_obs) through the turning point (X = 0) to X(r_esc)
      q.X0 = -x_obs;
      q.a0.s = -q.a0.s;
      q.dir = 1.0;
      q.X_end = x_of_r(q, r_esc, q.a_end);
      q.tau_end = (x_obs + q.X_end) / q.sc;
    } else {
      q.X0 = x_obs;
      q.dir = -1.0;
      q.tau_end = (x_obs - x_of_r(q, r_hor, a_h)) / q.sc;
    }
  }
  return q;
}

BHM_HD double x_at(const RadSol &q, double tau) { return q.X0 + q.dir * q.sc * tau; }

// r from the amplitude at X (S, P4: sn; P2: cn).
BHM_HD double r_of_amp(const RadSol &q, const Amp &a) {
  if (q.type == kP2)
    return ((q.B * q.r2 - q.A * q.r1) + (q.B * q.r2 + q.A * q.r1) * a.c) / ((q.B - q.A) + (q.B + q.A) * a.c);
  const double s2 = a.s * a.s;
  const double r31 = q.r3 - q.r1, r41 = q.r4 - q.r1;
  return (q.r4 * r31 - q.r3 * r41 * s2) / (r31 - r41 * s2);
}

BHM_HD Amp amp_at(const RadSol &q, double X) {
  Amp a;
  sncndn(X, q.m1, a.s, a.c, a.d);
  return a;
}

// int_0^tau dtau / (r - r+-) for the two poles r+ and r- of a ray: the
// constants (j_poles, once per ray) and the values at X = x_at(tau) with
// amplitude a (j_eval).
//   S, P4: 1 / (r - rpm) = (1 - n sn^2) / ((r4 - rpm)(1 - h sn^2))
//            = (n/h + (1 - n/h) / (1 - h sn^2)) / (r4 - rpm),
//          integrated over X: (dX + (h - n) dQ(h)) / (r4 - rpm), no
//          cancellation as h -> 0; the amplitude stays in [-pi/2, pi/2].
//   P2:    1 / (r - rpm) = (B + A) / D1 - 2 A B r21 / (D1 D0) / (1 + al cn),
//          al = D1 / D0, and int_0^X dX / (1 + al cn) = Pi(na; ph) / (1 - al^2)
//          - al G with Pi = X + na Q(na; ph), na = al^2 / (al^2 - 1),
//          G = int_0^X cn dX / (1 - al^2 cn^2) = int dt / (Aq + Cq t^2), t = sn / dn;
//          the amplitude stays in [0, pi].
struct JPole {
  double par;         // h (S, P4) or na (P2): the characteristic of Q
  double k1, k2;      // S, P4: dir / ((r4 - rpm) sc), h - n; P2: (B + A) / (D1 sc), -2 A B r21 / (D1 D0 sc)
  double al, Aq, Cq;  // P2
  double t0;          // the observer's term: Q(h; ph0) (S, P4) or R1(X0) (P2)
  double qc;          // complete Q(par), NaN until needed
};

BHM_HD double p2_g(const JPole &J, const Amp &a) {
  const double t = a.s / a.d;
  if (J.Aq * J.Cq > 0.0) return atan(t * sqrt(J.Cq / J.Aq)) / sqrt(J.Aq * J.Cq);
  const double p1 = sqrt(-J.Aq / J.Cq);
  return log(fabs((t - p1) / (t + p1))) / (2.0 * p1 * J.Cq);
}

BHM_HD double p2_r1(JPole &J, double m1, double X, const Amp &a) {
  return (X + J.par * ellip_q_sc(J.par, a.s, a.c, m1, J.qc)) / J.Aq - J.al * p2_g(J, a);
}

BHA_PCALL void j_poles(const RadSol &q, double r_plus, double r_minus, JPole &jp, JPole &jm) {
  for (int k = 0; k < 2; ++k) {
    JPole &J = k == 0 ? jp : jm;
    const double rpm = k == 0 ? r_plus : r_minus;
    J = JPole{};
    J.qc = NAN;
    if (q.type == kP2) {
      const double A = q.A, B = q.B, r21 = q.r2 - q.r1;
      const double D0 = B * (q.r2 - rpm) - A * (q.r1 - rpm);
      const double D1 = B * (q.r2 - rpm) + A * (q.r1 - rpm);
      J.al = D1 / D0;
      const double al2 = J.al * J.al;
      J.par = al2 / (al2 - 1.0);
      J.Aq = 1.0 - al2;
      J.Cq = J.Aq * (1.0 - q.m1) + al2;
      J.k1 = (B + A) / (D1 * q.sc);
      J.k2 = -2.0 * A * B * r21 / (D1 * D0 * q.sc);
      J.t0 = p2_r1(J, q.m1, q.X0, q.a0);
    } else {
      const double r31 = q.r3 - q.r1, r41 = q.r4 - q.r1;
      J.par = r41 * (q.r3 - rpm) / (r31 * (q.r4 - rpm));
      J.k1 = q.dir / ((q.r4 - rpm) * q.sc);
      J.k2 = J.par - r41 / r31;
    }
  }
  if (q.type != kP2) ellip_q2_sc(jp.par, jm.par, q.a0.s, q.a0.c, q.m1, jp.t0, jm.t0);
}

// The integrand of Q: sin^2 / ((1 - n sin^2) sqrt(cos^2 + m1 sin^2)).
BHM_HD double q_integrand(double n, double m1, double ph) {
  const double s = sin(ph), c = cos(ph), s2 = s * s;
  return s2 / ((1.0 - n * s2) * sqrt(c * c + m1 * s2));
}

// S rays at the escape radius: the amplitude there differs little from the
// observer's mirror image (+phi_obs), so Q(h; phi_end) = -Q(h; -phi_obs) +
// int_(phi_obs)^(phi_end) by 4-point Gauss-Legendre when that interval is
// short (< 0.05 rad: error ~ 1e-20 relative); otherwise as at any point.
BHA_PCALL void j_eval_escape(const RadSol &q, JPole &jp, JPole &jm, double &vp, double &vm);

BHA_PCALL void j_eval(const RadSol &q, JPole &jp, JPole &jm, double X, const Amp &a, double &vp, double &vm) {
  if (q.type == kP2) {
    vp = jp.k1 * (q.X0 - X) + jp.k2 * (jp.t0 - p2_r1(jp, q.m1, X, a));
    vm = jm.k1 * (q.X0 - X) + jm.k2 * (jm.t0 - p2_r1(jm, q.m1, X, a));
    return;
  }
  double qp, qm;
  ellip_q2_sc(jp.par, jm.par, a.s, a.c, q.m1, qp, qm);
  vp = jp.k1 * ((X - q.X0) + jp.k2 * (qp - jp.t0));
  vm = jm.k1 * ((X - q.X0) + jm.k2 * (qm - jm.t0));
}

BHA_PCALL void j_eval_escape(const RadSol &q, JPole &jp, JPole &jm, double &vp, double &vm) {
  const double p0 = atan2(-q.a0.s, q.a0.c), p1 = atan2(q.a_end.s, q.a_end.c);  // both in (0, pi/2)
  const double d = p1 - p0;
  if (q.type != kS || !(fabs(d) < 0.05)) {
    j_eval(q, jp, jm, q.X_end, q.a_end, vp, vm);
    return;
  }
  constexpr double x1 = 0.3399810435848563, x2 = 0.8611363115940526;  // Gauss-Legendre, 4 points
  constexpr double w1 = 0.6521451548625461, w2 = 0.3478548451374538;
  const double mid = 0.5 * (p0 + p1), hh = 0.5 * d;
  double ip = 0.0, im = 0.0;
  const double nodes[4] = {mid - hh * x2, mid - hh * x1, mid + hh * x1, mid + hh * x2};
  const double wts[4] = {w2, w1, w1, w2};
  for (int k = 0; k < 4; ++k) {
    ip += wts[k] * q_integrand(jp.par, q.m1, nodes[k]);
    im += wts[k] * q_integrand(jm.par, q.m1, nodes[k]);
  }
  const double qp = -jp.t0 + hh * ip, qm = -jm.t0 + hh * im;
  vp = jp.k1 * ((q.X_end - q.X0) + jp.k2 * (qp - jp.t0));
  vm = jm.k1 * ((q.X_end - q.X0) + jm.k2 * (qm - jm.t0));
}

// ---- polar motion -------------------------------------------------------------------
//
// u = sqrt(z+) sin chi, Phi(chi) = F(chi | -mm / w) / sqrt(w) the Mino time
// since chi = 0; the ray starts at Phi = phi_start and crosses the equator at
// chi = j pi, i.e. at tau = j period - phi_start.

struct PolSol {
  bool crosses;
  double zp, w, mm, sz;  // U = (z+ - u^2)(a^2 u^2 + w), mm = a^2 z+, sz = sqrt(z+)
  double zc;             // 1 - z+, formed without cancellation
  double m1;             // complementary parameter of -mm / w
  double sw;             // sqrt(w)
  double phi_start;      // Phi at the observer [Mino time]
  double tau1, period;   // first crossing, time between crossings
  double s0, c0;         // chi at the observer: sin, cos (chi0 in (-pi/2, 3 pi/2); cos has the sign of du/dtau)
  double q0, qc;         // Q(z+; chi0) and the complete Q(z+) (NaN until needed)
};

BHA_SCALL PolSol polar(double a2, double qTh, double lam, double u0, double pu0) {
  PolSol t{};
  const double c0 = qTh - lam * lam;
  t.crosses = c0 > 0.0;
  if (!t.crosses) return t;
  const double b2 = a2 - qTh;
  const double sq = sqrt(b2 * b2 + 4.0 * a2 * c0);
  t.zp = (b2 > 0.0) ? (b2 + sq) / (2.0 * a2) : 2.0 * c0 / (sq - b2);
  t.zc = 2.0 * lam * lam / (a2 + qTh + sq);  // (a^2 + qTh)^2 - sq^2 = 4 a^2 lambda^2
  t.w = c0 / t.zp;
  t.mm = a2 * t.zp;
  t.sz = sqrt(t.zp);
  t.m1 = 1.0 + t.mm / t.w;
  t.sw = sqrt(t.w);
  const double s0 = fmax(-1.0, fmin(1.0, u0 / t.sz));
  // cos^2 chi_obs from U(u0) = pu0^2 = (z+ - u0^2)(a^2 u0^2 + w): exact where
  // 1 - s0^2 would cancel (an observer at a polar turning point, beta ~ 0)
  const double c2 = pu0 * pu0 / ((a2 * u0 * u0 + t.w) * t.zp);
  const double phi_x = s0 * carlson_rf(t.w * c2, t.w + t.mm * s0 * s0, t.w);
  const double K = bhmino::quarter_period<double>(t.w, t.mm);
  t.phi_start = (pu0 >= 0.0) ? phi_x : 2.0 * K - phi_x;
  // |Phi(chi0)| to the next crossing when moving toward the equator, else over the turning point
  t.tau1 = ((pu0 * u0) < 0.0) ? fabs(phi_x) : 2.0 * K - fabs(phi_x);
  t.period = 2.0 * K;
  t.s0 = s0;
  t.c0 = (pu0 >= 0.0 ? 1.0 : -1.0) * sqrt(c2);  // dchi/dtau > 0: cos chi has the sign of du/dtau
  t.q0 = NAN;
  t.qc = NAN;
  return t;
}

BHM_HD void polar_q0(PolSol &t) {
  if (isnan(t.q0)) t.q0 = ellip_q_sc_nc(t.zc, t.s0, t.c0, t.m1, t.qc);
  if (isnan(t.qc)) t.qc = ellip_qc_nc(t.zc, t.m1);
}

// lambda int_0^tau dtau / (1 - u^2) at an equatorial crossing (chi = j pi,
// Q(z+; j pi) = 2 j Q(pi/2)): lambda (tau + (z+ / sqrt(w)) (2 j Q_c - Q(chi0))).
// With 1 - z+ == 0 (lambda == 0, or lambda^2 below the smallest double) the
// integral is its limit lambda -> 0 from the side of lambda's sign: a turn by
// copysign(pi, lambda) at each pass over the pole (chi = pi/2 + j pi), so
// lambda = +0 and -0 continue their two sides, which agree modulo 2 pi.
BHM_HD double pole_turns(const PolSol &t, double lam, double tau) {
  const double K = 0.5 * t.period;
  const double passes = floor((t.phi_start + tau - K) / t.period) - floor((t.phi_start - K) / t.period);
  return copysign(3.141592653589793, lam) * passes;
}

BHA_PCALL double phi_theta_crossing(PolSol &t, double lam, double tau) {
  if (!(t.zc > 0.0)) return pole_turns(t, lam, tau);
  polar_q0(t);
  const double j = rint((t.phi_start + tau) / t.period);
  return lam * (tau + t.zp / t.sw * (2.0 * j * t.qc - t.q0));
}

// u, du/dtau and lambda int_0^tau dtau / (1 - u^2) at any tau.
BHA_PCALL void polar_at(PolSol &t, double lam, double tau, double &u, double &pu, double &phi_th) {
  const double total = t.phi_start + tau;
  const double j = floor(total / t.period);
  double sa, ca, da;  // amplitude in [0, pi): sa >= 0
  sncndn_neg(t.sw * (total - j * t.period), t.m1, sa, ca, da);
  sa = fabs(sa);
  const double sg = fmod(j, 2.0) != 0.0 ? -1.0 : 1.0;
  u = sg * t.sz * sa;
  pu = sg * t.sz * ca * sqrt(t.w + t.mm * sa * sa);
  if (!(t.zc > 0.0)) {
    phi_th = pole_turns(t, lam, tau);
    return;
  }
  polar_q0(t);
  const double q = 2.0 * j * t.qc + ellip_q_sc_nc(t.zc, sa, ca, t.m1, t.qc);
  phi_th = lam * (tau + t.zp / t.sw * (q - t.q0));
}

}  // namespace bhan
