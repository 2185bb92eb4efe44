// rt_oracle.hpp - CPU restatement of the along-ray radiative transfer
// (test infrastructure only): the same DP45 ray as kerr_oracle.hpp's image
// tracer, sampled along each accepted step, with the reference's physics:
//   thermal synchrotron j_nu (Mahadevan 1996, K_2 ~ 2 Theta^2) and
//   alpha_nu = j_nu / B_nu (src/physics/rte_integrator.h:291-356),
//   planckFunction (:221-230), j g^2 and alpha / g (:480-512),
//   the exact constant-coefficient segment with the tau < 1e-4 Taylor branch
//   (rteStep, :138-187), written front to back (I += T S (1 - e^-tau)).
// The medium (grid of n_e, Theta_e, |B|) and the synchrotron table (ln j) are
// inputs: the tests hand the oracle the arrays the device generated.
#pragma once

#include <cmath>
#include <cstdint>

#include "kerr_oracle.hpp"

namespace bho_rt {

struct Medium {
  const float *cells;  // float4 [n_r][n_th][n_ph]
  int n_r, n_th, n_ph;
  double r_min, r_max, inv_log_range;
  const float *lut;  // [n_lt][n_lx]
  int n_lt, n_lx;
  double lt0, lt1, lx0, lx1;
  double nu, length_cm, ds_max, min_transmit;
};

struct Result {
  double I, tau;
  int cls, steps;
};

inline constexpr double kE = 4.80320425e-10, kMe = 9.1093837015e-28, kC = 2.99792458e10, kKb = 1.380649e-16,
                        kH = 6.62607015e-27, kTwoPi = 6.283185307179586;

inline bool sample(const Medium &q, double r, double u, double phi, double &n, double &th, double &b) {
  if (!(r >= q.r_min && r <= q.r_max)) return false;
  const double fr = (std::log(r / q.r_min) * q.inv_log_range) * double(q.n_r - 1);
  int i0 = int(std::floor(fr));
  i0 = i0 < 0 ? 0 : (i0 > q.n_r - 2 ? q.n_r - 2 : i0);
  double tr = fr - double(i0);
  tr = tr < 0.0 ? 0.0 : (tr > 1.0 ? 1.0 : tr);
  const double theta = std::acos(u < -1.0 ? -1.0 : (u > 1.0 ? 1.0 : u));
  const double ft = (theta * (1.0 / 3.141592653589793)) * double(q.n_th) - 0.5;
  int j0 = int(std::floor(ft));
  j0 = j0 < 0 ? 0 : (j0 > q.n_th - 2 ? q.n_th - 2 : j0);
  double tt = ft - double(j0);
  tt = tt < 0.0 ? 0.0 : (tt > 1.0 ? 1.0 : tt);
  const double fp = (phi * (1.0 / kTwoPi)) * double(q.n_ph);
  const double fl = std::floor(fp);
  const double tp = fp - fl;
  long long k0 = (long long)fl % q.n_ph;
  if (k0 < 0) k0 += q.n_ph;
  const long long k1 = (k0 + 1) % q.n_ph;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj)
      for (int dk = 0; dk < 2; ++dk) {
        const double w = (di ? tr : 1.0 - tr) * (dj ? tt : 1.0 - tt) * (dk ? tp : 1.0 - tp);
        const long long idx = ((long long)(i0 + di) * q.n_th + (j0 + dj)) * q.n_ph + (dk ? k1 : k0);
        const float *v = q.cells + 4 * idx;
        acc[0] = acc[0] + w * double(v[0]);
        acc[1] = acc[1] + w * double(v[1]);
        acc[2] = acc[2] + w * double(v[2]);
      }
  n = acc[0];
  th = acc[1];
  b = acc[2];
  return true;
}

inline double redshift(double a, double r, double u, double lam) {
  const double u2 = u * u;
  const double s2 = (1.0 - u) * (1.0 + u);
  const double sig = r * r + a * a * u2;
  const double delta = r * r - 2.0 * r + a * a;
  const double A = (r * r + a * a) * (r * r + a * a) - a * a * delta * s2;
  const double om = 1.0 / (r * std::sqrt(r) + a);
  const double gtt = -(1.0 - 2.0 * r / sig);
  const double gtp = -2.0 * a * r * s2 / sig;
  const double gpp = A * s2 / sig;
  const double norm = -(gtt + 2.0 * gtp * om + gpp * om * om);
  if (!(norm > 0.0)) return 0.0;
  const double ut = 1.0 / std::sqrt(norm);
  const double den = ut * (1.0 - om * lam);
  return den > 0.0 ? 1.0 / den : 0.0;
}

inline double planck(double nu, double temp) {
  const double x = (kH * nu) / (kKb * temp);
  const double den = (x > 500.0) ? std::exp(x) : std::expm1(x);
  if (!(den > 0.0)) return 0.0;
  return (2.0 * kH * nu * nu * nu / (kC * kC)) / den;
}

inline void synchrotron(const Medium &q, double n, double theta_e, double b, double nu_e, double &j, double &alpha) {
  j = 0.0;
  alpha = 0.0;
  if (!(n > 0.0 && theta_e > 0.0 && b > 0.0 && nu_e > 0.0)) return;
  const double nu_b = kE * b / (kTwoPi * kMe * kC);
  const double nu_s = 1.5 * nu_b * theta_e * theta_e;
  const double lx = std::log(nu_e / nu_s);
  if (lx > q.lx1) return;
  const double lt = std::log(theta_e);
  double ft = (lt - q.lt0) / (q.lt1 - q.lt0) * double(q.n_lt - 1);
  double fx = (lx - q.lx0) / (q.lx1 - q.lx0) * double(q.n_lx - 1);
  ft = ft < 0.0 ? 0.0 : (ft > double(q.n_lt - 1) ? double(q.n_lt - 1) : ft);
  fx = fx < 0.0 ? 0.0 : (fx > double(q.n_lx - 1) ? double(q.n_lx - 1) : fx);
  int i0 = int(std::floor(ft)), k0 = int(std::floor(fx));
  i0 = i0 > q.n_lt - 2 ? q.n_lt - 2 : i0;
  k0 = k0 > q.n_lx - 2 ? q.n_lx - 2 : k0;
  const double ti = ft - double(i0), tk = fx - double(k0);
  const float *L = q.lut;
  const double v00 = L[i0 * q.n_lx + k0], v01 = L[i0 * q.n_lx + k0 + 1];
  const double v10 = L[(i0 + 1) * q.n_lx + k0], v11 = L[(i0 + 1) * q.n_lx + k0 + 1];
  const double J = ((1.0 - ti) * ((1.0 - tk) * v00 + tk * v01)) + (ti * ((1.0 - tk) * v10 + tk * v11));
  j = n * nu_b * std::exp(J);
  const double bnu = planck(nu_e, theta_e * kMe * kC * kC / kKb);
  alpha = bnu > 0.0 ? j / bnu : 0.0;
}

// One front-to-back segment of the formal solution.
inline void segment(double jo, double ao, double ds, double &I, double &T, double &tau) {
  const double ts = ao * ds;
  const double om = (ts < 1.0e-4) ? ts * (1.0 - 0.5 * ts) : -std::expm1(-ts);
  I = (ao > 0.0) ? I + T * ((jo / ao) * om) : I + T * (jo * ds);
  T = T * (1.0 - om);
  tau = tau + ts;
}

inline Result trace_pixel_rt(const bho::Scene &s, const bho::SceneDerived<double> &d, double alpha, double beta,
                             const Medium &q) {
  using namespace bho;
  Result out{0.0, 0.0, 3, 0};
  RayConsts<double> c;
  Y<double> y;
  init_ray(d, s, alpha, beta, c, y);
  const PolyRhs<double> f{c};
  f.project(y);
  const double a2 = d.a * d.a;
  double h = mino_step(s, y, d.a);
  Y<double> k1 = f(y);
  double I = 0.0, T = 1.0, tau = 0.0;
  int64_t attempts = 0;
  const int64_t max_attempts = int64_t(4) * s.max_steps + 64;
  for (;;) {
    if (out.steps >= s.max_steps || attempts >= max_attempts) { out.cls = 3; break; }
    if (y.r <= d.r_hor) { out.cls = 0; break; }
    if (y.r >= d.r_esc) { out.cls = 2; break; }
    ++attempts;
    const DPOut<double> o = img_dp45(y, h, f, k1, s.rtol, s.atol, true);
    if (o.err <= 1.0) {
      ++out.steps;
      const Y<double> &y0 = y, &k0 = k1, &y1 = o.y5, &kk = o.k7;
      const double rm = 0.5 * (y0.r + y1.r) + 0.125 * h * (k0.r - kk.r);
      const double um = 0.5 * (y0.u + y1.u) + 0.125 * h * (k0.u - kk.u);
      const double sig_m = rm * rm + a2 * um * um;
      double ns = std::ceil((sig_m * h) / q.ds_max);
      ns = ns < 1.0 ? 1.0 : (ns > 64.0 ? 64.0 : ns);
      const int nsub = int(ns);
      const double dt = h / ns;
      for (int m = 0; m < nsub; ++m) {
        const double t = (double(m) + 0.5) / ns;
        const double t2 = t * t, t3 = t2 * t;
        const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + t;
        const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
        const double r = h00 * y0.r + h10 * h * k0.r + h01 * y1.r + h11 * h * kk.r;
        const double u = h00 * y0.u + h10 * h * k0.u + h01 * y1.u + h11 * h * kk.u;
        const double psi = h00 * y0.phi + h10 * h * k0.phi + h01 * y1.phi + h11 * h * kk.phi;
        const double dl = (r * r + a2 * u * u) * dt;
        double n, th, b;
        const double phi = phi_of_psi(psi, r, s.r_obs, d.a, d.r_plus, d.r_minus);
        if (!sample(q, r, u, phi, n, th, b)) continue;
        const double g = redshift(d.a, r, u, c.lam);
        if (!(g > 0.0)) continue;
        double j, al;
        synchrotron(q, n, th, b, q.nu / g, j, al);
        segment(g * g * j, al / g, dl * q.length_cm, I, T, tau);
      }
      y = o.y5;
      k1 = o.k7;
      f.project(y);
      k1.r = y.pr;
      k1.u = y.pu;
      h = h * step_factor(o.err, true);
      if (T < q.min_transmit) { out.cls = 4; break; }
    } else {
      h = h * step_factor(o.err, false);
    }
  }
  out.I = I;
  out.tau = tau;
  return out;
}

}  // namespace bho_rt
