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

using bho::s_acos;
using bho::s_ceil;
using bho::s_exp;
using bho::s_expm1;
using bho::s_floor;
using bho::s_log;
using bho::s_sqrt;

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

// Every function is templated on the scalar: double for the oracle itself,
// bho::Counted to count the operations per accepted step (the roofline's
// FLOP constant). Integer index arithmetic runs on plain values.
template <class T>
inline bool sample(const Medium &q, T r, T u, T phi, T &n, T &th, T &b) {
  if (!(r >= T(q.r_min) && r <= T(q.r_max))) return false;
  const T fr = (s_log(r / T(q.r_min)) * T(q.inv_log_range)) * T(double(q.n_r - 1));
  int i0 = int(double(s_floor(fr)));
  i0 = i0 < 0 ? 0 : (i0 > q.n_r - 2 ? q.n_r - 2 : i0);
  T tr = fr - T(double(i0));
  tr = tr < T(0.0) ? T(0.0) : (tr > T(1.0) ? T(1.0) : tr);
  const T theta = s_acos(u < T(-1.0) ? T(-1.0) : (u > T(1.0) ? T(1.0) : u));
  const T ft = (theta * T(1.0 / 3.141592653589793)) * T(double(q.n_th)) - T(0.5);
  int j0 = int(double(s_floor(ft)));
  j0 = j0 < 0 ? 0 : (j0 > q.n_th - 2 ? q.n_th - 2 : j0);
  T tt = ft - T(double(j0));
  tt = tt < T(0.0) ? T(0.0) : (tt > T(1.0) ? T(1.0) : tt);
  const T fp = (phi * T(1.0 / kTwoPi)) * T(double(q.n_ph));
  const T fl = s_floor(fp);
  const T tp = fp - fl;
  long long k0 = (long long)double(fl) % q.n_ph;
  if (k0 < 0) k0 += q.n_ph;
  const long long k1 = (k0 + 1) % q.n_ph;
  T acc[3] = {T(0.0), T(0.0), T(0.0)};
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj)
      for (int dk = 0; dk < 2; ++dk) {
        const T w = (di ? tr : T(1.0) - tr) * (dj ? tt : T(1.0) - tt) * (dk ? tp : T(1.0) - tp);
        const long long idx = ((long long)(i0 + di) * q.n_th + (j0 + dj)) * q.n_ph + (dk ? k1 : k0);
        const float *v = q.cells + 4 * idx;
        acc[0] = acc[0] + w * T(double(v[0]));
        acc[1] = acc[1] + w * T(double(v[1]));
        acc[2] = acc[2] + w * T(double(v[2]));
      }
  n = acc[0];
  th = acc[1];
  b = acc[2];
  return true;
}

template <class T>
inline T redshift(T a, T r, T u, T lam) {
  const T u2 = u * u;
  const T s2 = (T(1.0) - u) * (T(1.0) + u);
  const T sig = r * r + a * a * u2;
  const T delta = r * r - T(2.0) * r + a * a;
  const T A = (r * r + a * a) * (r * r + a * a) - a * a * delta * s2;
  const T om = T(1.0) / (r * s_sqrt(r) + a);
  const T gtt = -(T(1.0) - T(2.0) * r / sig);
  const T gtp = -T(2.0) * a * r * s2 / sig;
  const T gpp = A * s2 / sig;
  const T norm = -(gtt + T(2.0) * gtp * om + gpp * om * om);
  if (!(norm > T(0.0))) return T(0.0);
  const T ut = T(1.0) / s_sqrt(norm);
  const T den = ut * (T(1.0) - om * lam);
  return den > T(0.0) ? T(1.0) / den : T(0.0);
}

template <class T>
inline T planck(T nu, T temp) {
  const T x = (T(kH) * nu) / (T(kKb) * temp);
  const T den = (x > T(500.0)) ? s_exp(x) : s_expm1(x);
  if (!(den > T(0.0))) return T(0.0);
  return (T(2.0) * T(kH) * nu * nu * nu / (T(kC) * T(kC))) / den;
}

template <class T>
inline void synchrotron(const Medium &q, T n, T theta_e, T b, T nu_e, T &j, T &alpha) {
  j = T(0.0);
  alpha = T(0.0);
  if (!(n > T(0.0) && theta_e > T(0.0) && b > T(0.0) && nu_e > T(0.0))) return;
  const T nu_b = T(kE) * b / (T(kTwoPi) * T(kMe) * T(kC));
  const T nu_s = T(1.5) * nu_b * theta_e * theta_e;
  const T lx = s_log(nu_e / nu_s);
  if (lx > T(q.lx1)) return;
  const T lt = s_log(theta_e);
  T ft = (lt - T(q.lt0)) / (T(q.lt1) - T(q.lt0)) * T(double(q.n_lt - 1));
  T fx = (lx - T(q.lx0)) / (T(q.lx1) - T(q.lx0)) * T(double(q.n_lx - 1));
  ft = ft < T(0.0) ? T(0.0) : (ft > T(double(q.n_lt - 1)) ? T(double(q.n_lt - 1)) : ft);
  fx = fx < T(0.0) ? T(0.0) : (fx > T(double(q.n_lx - 1)) ? T(double(q.n_lx - 1)) : fx);
  int i0 = int(double(s_floor(ft))), k0 = int(double(s_floor(fx)));
  i0 = i0 > q.n_lt - 2 ? q.n_lt - 2 : i0;
  k0 = k0 > q.n_lx - 2 ? q.n_lx - 2 : k0;
  const T ti = ft - T(double(i0)), tk = fx - T(double(k0));
  const float *L = q.lut;
  const T v00 = T(double(L[i0 * q.n_lx + k0])), v01 = T(double(L[i0 * q.n_lx + k0 + 1]));
  const T v10 = T(double(L[(i0 + 1) * q.n_lx + k0])), v11 = T(double(L[(i0 + 1) * q.n_lx + k0 + 1]));
  const T J = ((T(1.0) - ti) * ((T(1.0) - tk) * v00 + tk * v01)) + (ti * ((T(1.0) - tk) * v10 + tk * v11));
  j = n * nu_b * s_exp(J);
  const T bnu = planck(nu_e, theta_e * T(kMe) * T(kC) * T(kC) / T(kKb));
  alpha = bnu > T(0.0) ? j / bnu : T(0.0);
}

// One front-to-back segment of the formal solution.
template <class T>
inline void segment(T jo, T ao, T ds, T &I, T &Tr, T &tau) {
  const T ts = ao * ds;
  const T om = (ts < T(1.0e-4)) ? ts * (T(1.0) - T(0.5) * ts) : -s_expm1(-ts);
  I = (ao > T(0.0)) ? I + Tr * ((jo / ao) * om) : I + Tr * (jo * ds);
  Tr = Tr * (T(1.0) - om);
  tau = tau + ts;
}

template <class T>
inline Result trace_pixel_rt(const bho::Scene &s, const bho::SceneDerived<T> &d, T alpha, T beta, const Medium &q,
                             int64_t *samples = nullptr) {
  using namespace bho;
  Result out{0.0, 0.0, 3, 0};
  RayConsts<T> c;
  Y<T> y;
  init_ray(d, s, alpha, beta, c, y);
  const PolyRhs<T> f{c};
  f.project(y);
  const T a2 = d.a * d.a;
  T h = mino_step(s, y, d.a);
  Y<T> k1 = f(y);
  T I = T(0.0), Tr = T(1.0), tau = T(0.0);
  int64_t attempts = 0;
  const int64_t max_attempts = int64_t(4) * s.max_steps + 64;
  for (;;) {
    if (out.steps >= s.max_steps || attempts >= max_attempts) { out.cls = 3; break; }
    if (y.r <= d.r_hor) { out.cls = 0; break; }
    if (y.r >= d.r_esc) { out.cls = 2; break; }
    ++attempts;
    const DPOut<T> o = img_dp45(y, h, f, k1, T(s.rtol), T(s.atol), true);
    if (o.err <= T(1.0)) {
      ++out.steps;
      const Y<T> &y0 = y, &k0 = k1, &y1 = o.y5, &kk = o.k7;
      const T rm = T(0.5) * (y0.r + y1.r) + T(0.125) * h * (k0.r - kk.r);
      const T um = T(0.5) * (y0.u + y1.u) + T(0.125) * h * (k0.u - kk.u);
      const T sig_m = rm * rm + a2 * um * um;
      // A step that stays beyond r_max samples nothing: on t in [0, 1] the
      // cubic Hermite r(t) >= min(r0, r1) - (4/27) |h| (|r0'| + |r1'|).
      const T rlow = (y0.r < y1.r ? y0.r : y1.r) - T(4.0 / 27.0) * (h < T(0.0) ? -h : h) *
                                                         ((k0.r < T(0.0) ? -k0.r : k0.r) + (kk.r < T(0.0) ? -kk.r : kk.r));
      const bool outside = rlow > T(q.r_max);
      T ns = s_ceil((sig_m * h) / T(q.ds_max));
      ns = ns < T(1.0) ? T(1.0) : (ns > T(64.0) ? T(64.0) : ns);
      const int nsub = outside ? 0 : int(double(ns));
      const T dt = h / ns;
      for (int m = 0; m < nsub; ++m) {
        const T t = (T(double(m)) + T(0.5)) / ns;
        const T t2 = t * t, t3 = t2 * t;
        const T h00 = T(2.0) * t3 - T(3.0) * t2 + T(1.0), h10 = t3 - T(2.0) * t2 + t;
        const T h01 = -T(2.0) * t3 + T(3.0) * t2, h11 = t3 - t2;
        const T r = h00 * y0.r + h10 * h * k0.r + h01 * y1.r + h11 * h * kk.r;
        const T u = h00 * y0.u + h10 * h * k0.u + h01 * y1.u + h11 * h * kk.u;
        const T psi = h00 * y0.phi + h10 * h * k0.phi + h01 * y1.phi + h11 * h * kk.phi;
        const T dl = (r * r + a2 * u * u) * dt;
        T n, th, b;
        const T phi = phi_of_psi(psi, r, T(s.r_obs), d.a, d.r_plus, d.r_minus);
        if (samples) ++*samples;
        if (!sample(q, r, u, phi, n, th, b)) continue;
        const T g = redshift(d.a, r, u, c.lam);
        if (!(g > T(0.0))) continue;
        T j, al;
        synchrotron(q, n, th, b, T(q.nu) / g, j, al);
        segment(g * g * j, al / g, dl * T(q.length_cm), I, Tr, tau);
      }
      y = o.y5;
      k1 = o.k7;
      f.project(y);
      k1.r = y.pr;
      k1.u = y.pu;
      h = h * T(step_factor(double(o.err), true));
      if (Tr < T(q.min_transmit)) { out.cls = 4; break; }
    } else {
      h = h * T(step_factor(double(o.err), false));
    }
  }
  out.I = double(I);
  out.tau = double(tau);
  return out;
}

}  // namespace bho_rt
