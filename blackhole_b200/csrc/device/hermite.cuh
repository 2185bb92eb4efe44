// hermite.cuh - equatorial crossing inside an accepted step, FP64.
//
// In the second-order Mino-time form each position x in {r, u} has x' = p_x
// and x'' = F_x(position) known at both ends of a step, so the quintic
// Hermite interpolant through (x, h x', h^2 x'') at t = 0 and t = 1 follows
// x(t0 + t h) to O(h^6) -- below the step's own truncation error -- with no
// further right-hand-side evaluation; phi' is known at both ends (cubic
// Hermite). The root of u on [0, 1], bracketed by u0 and u1 of opposite sign,
// is found with Illinois regula falsi on the polynomial. A lane that detects
// a crossing therefore spends ~60 FLOPs instead of re-integrating sub-steps
// while the rest of its warp waits.
//
// The evaluation order matches the CPU oracle (oracle/kerr_oracle.hpp,
// hermite_crossing), so a translation unit compiled with -fmad=false
// reproduces it bit for bit.
#pragma once

namespace bhh_dev {

struct Quintic {
  double c0, c1, c2, c3, c4, c5;
};

__device__ __forceinline__ Quintic quintic_hermite(double p0, double v0, double a0, double p1, double v1,
                                                   double a1) {
  const double A = ((p1 - p0) - v0) - 0.5 * a0;
  const double B = (v1 - v0) - a0;
  const double Cc = a1 - a0;
  Quintic q;
  q.c0 = p0;
  q.c1 = v0;
  q.c2 = 0.5 * a0;
  q.c3 = (10.0 * A - 4.0 * B) + 0.5 * Cc;
  q.c4 = (7.0 * B - 15.0 * A) - Cc;
  q.c5 = (6.0 * A - 3.0 * B) + 0.5 * Cc;
  return q;
}

__device__ __forceinline__ double eval_quintic(const Quintic &q, double t) {
  return q.c0 + t * (q.c1 + t * (q.c2 + t * (q.c3 + t * (q.c4 + t * q.c5))));
}

__device__ __forceinline__ double eval_cubic_hermite(double p0, double v0, double p1, double v1, double t) {
  const double A = (p1 - p0) - v0;
  const double B = v1 - v0;
  const double c2 = 3.0 * A - B;
  const double c3 = B - 2.0 * A;
  return p0 + t * (v0 + t * (c2 + t * c3));
}

// Step endpoints: position (r, u, phi), momenta (p_r, p_u) and the forces
// F_r = p_r', F_u = p_u' and rate phi' from the right-hand side at each end.
struct Ends {
  double r0, u0, phi0, pr0, pu0, fr0, fu0, dphi0;
  double r1, u1, phi1, pr1, pu1, fr1, fu1, dphi1;
};

__device__ __forceinline__ void hermite_crossing(const Ends &e, double h, double &r_c, double &phi_c) {
  const double h2 = h * h;
  const Quintic qu = quintic_hermite(e.u0, h * e.pu0, h2 * e.fu0, e.u1, h * e.pu1, h2 * e.fu1);
  double a = 0.0, fa = e.u0, b = 1.0, fb = e.u1;
  const double tol = 1e-15 * (fabs(fa) + fabs(fb));
  int side = 0;
  double t = 0.5;
  for (int i = 0; i < 60; ++i) {
    t = (a * fb - b * fa) / (fb - fa);
    if (!(t > a && t < b)) t = 0.5 * (a + b);
    const double fc = eval_quintic(qu, t);
    if (fabs(fc) <= tol || (b - a) <= 1e-14) break;
    if ((fc * fb) > 0.0) {
      b = t;
      fb = fc;
      if (side == -1) fa = 0.5 * fa;
      side = -1;
    } else {
      a = t;
      fa = fc;
      if (side == 1) fb = 0.5 * fb;
      side = 1;
    }
  }
  const Quintic qr = quintic_hermite(e.r0, h * e.pr0, h2 * e.fr0, e.r1, h * e.pr1, h2 * e.fr1);
  r_c = eval_quintic(qr, t);
  phi_c = eval_cubic_hermite(e.phi0, h * e.dphi0, e.phi1, h * e.dphi1, t);
}

}  // namespace bhh_dev
