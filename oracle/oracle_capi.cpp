// oracle_capi.cpp - extern "C" surface of the CPU oracle (test infrastructure
// only: loaded by tests/, __graft_entry__.smoke() and bench.py's CPU legs).
//
// Wraps kerr_oracle.hpp for ctypes: batched reference stepper (Part A),
// image tracer over any pixel subset with std::thread workers (Part B),
// the FLOP count per step with the counting scalar, and a __float128 run of
// the stepper.
#include <atomic>
#include <bit>
#include <cstring>
#include <thread>
#include <vector>

#include "../include/bh_kerr.h"
#include "kerr_oracle.hpp"
#include "rt_oracle.hpp"

namespace {

bho::Scene to_scene(const BH_KerrScene *s) {
  bho::Scene o{};
  o.spin = s->spin;
  o.r_obs = s->r_obs;
  o.theta_obs = s->theta_obs;
  o.alpha_min = s->alpha_min;
  o.alpha_max = s->alpha_max;
  o.beta_min = s->beta_min;
  o.beta_max = s->beta_max;
  o.width = s->width;
  o.height = s->height;
  o.integrator = s->integrator;
  o.potential_form = s->potential_form;
  o.max_crossings = s->max_crossings;
  o.max_steps = s->max_steps;
  o.step_coeff = s->step_coeff;
  o.step_rcap = s->step_rcap;
  o.rtol = s->rtol;
  o.atol = s->atol;
  o.horizon_factor = s->horizon_factor;
  o.escape_factor = s->escape_factor;
  o.disk_r_in = s->disk_r_in;
  o.disk_r_out = s->disk_r_out;
  return o;
}

template <class T>
void store(const BH_KerrImageOut *out, int64_t idx, int64_t n, int maxc, const bho::PixelResult<T> &p) {
  if (out->cls) out->cls[idx] = p.cls;
  if (out->steps) out->steps[idx] = p.steps;
  if (out->n_cross) out->n_cross[idx] = p.n_cross;
  for (int k = 0; k < maxc; ++k) {
    if (out->r_hit) out->r_hit[k * n + idx] = double(p.r_hit[k]);
    if (out->phi_hit) out->phi_hit[k * n + idx] = double(p.phi_hit[k]);
    if (out->g) out->g[k * n + idx] = double(p.g[k]);
  }
  if (out->flux) out->flux[idx] = double(p.flux);
  if (out->intensity) out->intensity[idx] = double(p.intensity);
  if (out->theta_inf) out->theta_inf[idx] = double(p.theta_inf);
  if (out->phi_inf) out->phi_inf[idx] = double(p.phi_inf);
}

template <class F> void parallel_for(int64_t n, int threads, F &&f) {
  if (threads <= 1 || n < 2) {
    for (int64_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int64_t> next{0};
  const int64_t chunk = 16;
  std::vector<std::thread> pool;
  pool.reserve(threads);
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&]() {
      for (;;) {
        const int64_t b = next.fetch_add(chunk);
        if (b >= n) break;
        const int64_t e = std::min(n, b + chunk);
        for (int64_t i = b; i < e; ++i) f(i);
      }
    });
  }
  for (auto &th : pool) th.join();
}

}  // namespace

extern "C" {

// Trace pixels [pix_index[0..n)] of the scene (or pixels 0..n-1 when pix_index
// is NULL). Output arrays are indexed 0..n-1 (crossing planes have stride n).
int bho_trace_pixels(const BH_KerrScene *scene, int64_t n, const int64_t *pix_index,
                     const BH_KerrImageOut *out, int threads) {
  const bho::Scene s = to_scene(scene);
  const auto d = bho::derive<double>(s);
  const int maxc = std::max(1, std::min(3, int(s.max_crossings)));
  parallel_for(n, threads, [&](int64_t i) {
    const int64_t pix = pix_index ? pix_index[i] : i;
    double alpha, beta;
    bho::pixel_alpha_beta(s, pix, alpha, beta);
    const auto p = bho::trace_pixel<double>(s, d, alpha, beta);
    store(out, i, n, maxc, p);
  });
  return 0;
}

// Same at explicit image-plane coordinates.
int bho_trace_alpha_beta(const BH_KerrScene *scene, int64_t n, const double *alpha, const double *beta,
                         const BH_KerrImageOut *out, int threads) {
  const bho::Scene s = to_scene(scene);
  const auto d = bho::derive<double>(s);
  const int maxc = std::max(1, std::min(3, int(s.max_crossings)));
  parallel_for(n, threads, [&](int64_t i) {
    const auto p = bho::trace_pixel<double>(s, d, alpha[i], beta[i]);
    store(out, i, n, maxc, p);
  });
  return 0;
}

// ---- background sky (restated from the OpenGL cube-map convention) ----
//
// Face of the largest |component| (ties: x, then y) in the order +X, -X, +Y,
// -Y, +Z, -Z; face coordinates +X (-z,-y), -X (z,-y), +Y (x,z), -Y (x,-z),
// +Z (x,-y), -Z (-x,-y); nearest texel of u = (s/ma + 1)/2, v = (t/ma + 1)/2.
static int64_t sky_texel(double x, double y, double z, int N) {
  const double ax = std::fabs(x), ay = std::fabs(y), az = std::fabs(z);
  int face;
  double sc, tc, ma;
  if (ax >= ay && ax >= az) {
    ma = ax;
    face = x >= 0.0 ? 0 : 1;
    sc = x >= 0.0 ? -z : z;
    tc = -y;
  } else if (ay >= az) {
    ma = ay;
    face = y >= 0.0 ? 2 : 3;
    sc = x;
    tc = y >= 0.0 ? z : -z;
  } else {
    ma = az;
    face = z >= 0.0 ? 4 : 5;
    sc = z >= 0.0 ? x : -x;
    tc = -y;
  }
  const double u = 0.5 * (sc / ma + 1.0), v = 0.5 * (tc / ma + 1.0);
  int i = int(u * double(N)), j = int(v * double(N));
  i = std::min(std::max(i, 0), N - 1);
  j = std::min(std::max(j, 0), N - 1);
  return (int64_t(face) * N + j) * N + i;
}

// Direction of motion of the ray at its escape point (the sky point it comes
// from): the Cartesian velocity of (r, theta, phi) with dr = p_r,
// du = p_u (u = cos theta) and dphi.
static void motion_dir(double r, double u, double phi, double pr, double pu, double dphi, double &x, double &y,
                       double &z) {
  const double st = std::sqrt((1.0 - u) * (1.0 + u));
  const double cp = std::cos(phi), sp = std::sin(phi);
  const double dst = st > 1e-300 ? -u * pu / st : 0.0;
  x = (pr * st + r * dst) * cp - (r * st * dphi) * sp;
  y = (pr * st + r * dst) * sp + (r * st * dphi) * cp;
  z = pr * u + r * pu;
}

static double sky_radiance(const uint16_t *tex, int N, double r, double u, double phi, double pr, double pu,
                           double dphi) {
  double x, y, z;
  motion_dir(r, u, phi, pr, pu, dphi, x, y, z);
  const _Float16 h = std::bit_cast<_Float16>(tex[sky_texel(x, y, z, N)]);
  return double(float(h));
}

// bho_trace_pixels with the sky added to escaped rays' intensity.
int bho_trace_pixels_sky(const BH_KerrScene *scene, int64_t n, const int64_t *pix_index, const BH_KerrImageOut *out,
                         int threads, const uint16_t *sky, int sky_size) {
  const bho::Scene s = to_scene(scene);
  const auto d = bho::derive<double>(s);
  const int maxc = std::max(1, std::min(3, int(s.max_crossings)));
  parallel_for(n, threads, [&](int64_t i) {
    const int64_t pix = pix_index ? pix_index[i] : i;
    double alpha, beta;
    bho::pixel_alpha_beta(s, pix, alpha, beta);
    auto p = bho::trace_pixel<double>(s, d, alpha, beta);
    if (sky && p.cls == 2)
      p.intensity = p.intensity + sky_radiance(sky, sky_size, p.r_end, p.u_inf, p.phi_inf, p.pr_end, p.pu_end,
                                               p.dphi_end);
    store(out, i, n, maxc, p);
  });
  return 0;
}

// Rays of a camera at finite distance (kerr_oracle.hpp Camera; cam_f64 =
// right[3], up[3], fwd[3], fov, aspect, shift_x, shift_y, r0, u0, cphi, sphi;
// cam_i32 = width, height). scene: spin, r_obs = r0, escape and disk radii,
// integrator and tolerances (the camera sets the initial data). esc_dir
// (3 n, may be NULL): unit direction of motion of escaped rays in the
// camera-azimuth frame, zero otherwise.
int bho_trace_camera(const BH_KerrScene *scene, const double *cam_f64, const int32_t *cam_i32, int64_t n,
                     const int64_t *pix_index, const BH_KerrImageOut *out, double *esc_dir, int threads) {
  const bho::Scene s = to_scene(scene);
  const auto d = bho::derive<double>(s);
  const int maxc = std::max(1, std::min(3, int(s.max_crossings)));
  bho::Camera cam{};
  for (int k = 0; k < 3; ++k) {
    cam.right[k] = cam_f64[k];
    cam.up[k] = cam_f64[3 + k];
    cam.fwd[k] = cam_f64[6 + k];
  }
  cam.fov = cam_f64[9];
  cam.aspect = cam_f64[10];
  cam.shift_x = cam_f64[11];
  cam.shift_y = cam_f64[12];
  cam.r0 = cam_f64[13];
  cam.u0 = cam_f64[14];
  cam.cphi = cam_f64[15];
  cam.sphi = cam_f64[16];
  cam.width = cam_i32[0];
  cam.height = cam_i32[1];
  parallel_for(n, threads, [&](int64_t i) {
    const int64_t pix = pix_index ? pix_index[i] : i;
    bho::RayConsts<double> c;
    bho::Y<double> y;
    bho::init_ray_camera(d, cam, pix, c, y);
    const auto p = bho::trace_pixel_from<double>(s, d, c, y, [](const bho::RayConsts<double> &cc) {
      return bho::PolyRhs<double>{cc};
    });
    store(out, i, n, maxc, p);
    if (esc_dir) {
      double x = 0, yy = 0, z = 0;
      if (p.cls == 2) {
        motion_dir(p.r_end, p.u_inf, p.phi_inf, p.pr_end, p.pu_end, p.dphi_end, x, yy, z);
        const double nn = std::sqrt(x * x + yy * yy + z * z);
        x /= nn;
        yy /= nn;
        z /= nn;
      }
      esc_dir[i] = x;
      esc_dir[n + i] = yy;
      esc_dir[2 * n + i] = z;
    }
  });
  return 0;
}

// Paths of image-plane rays at explicit (alpha, beta): the position (x, y, z)
// before the first step and after every classical RK4 step (affine step
// step_coeff min(r, step_rcap), Mino step over Sigma, projection after each
// step) until the horizon or escape radius or max_points; xyz [n][max][3].
int bho_trace_paths(const BH_KerrScene *scene, int64_t n, const double *alpha, const double *beta, int max_points,
                    double *xyz, int32_t *counts, int threads) {
  const bho::Scene s = to_scene(scene);
  const auto d = bho::derive<double>(s);
  parallel_for(n, threads, [&](int64_t i) {
    bho::RayConsts<double> c;
    bho::Y<double> y;
    bho::init_ray(d, s, alpha[i], beta[i], c, y);
    const bho::PolyRhs<double> f{c};
    f.project(y);
    double *o = xyz + i * int64_t(max_points) * 3;
    int m = 0;
    for (;;) {
      const double st = std::sqrt(std::max(0.0, (1.0 - y.u) * (1.0 + y.u)));
      const double ph = bho::phi_of_psi(y.phi, y.r, s.r_obs, d.a, d.r_plus, d.r_minus);
      o[3 * m + 0] = y.r * st * std::cos(ph);
      o[3 * m + 1] = y.r * st * std::sin(ph);
      o[3 * m + 2] = y.r * y.u;
      ++m;
      if (m >= max_points || y.r <= d.r_hor || y.r >= d.r_esc) break;
      const double h = bho::mino_step(s, y, d.a);
      y = bho::img_rk4(y, h, f, f(y));
      f.project(y);
    }
    counts[i] = m;
  });
  return 0;
}

// Texel indices of directions (tests of the addressing).
int bho_sky_texels(int64_t n, const double *x, const double *y, const double *z, int N, int64_t *out) {
  for (int64_t i = 0; i < n; ++i) out[i] = sky_texel(x[i], y[i], z[i], N);
  return 0;
}

// ---- along-ray radiative transfer (rt_oracle.hpp) ----

// Operation counts of the transfer of the given pixels with the counting
// scalar (single thread): counts[0..6] as bho_count_ops summed over the
// pixels, counts[7] accepted steps, counts[8] medium samples.
int bho_count_rt_ops(const BH_KerrScene *scene, int64_t n, const int64_t *pix_index, const float *cells, int n_r,
                     int n_th, int n_ph, double r_min, double r_max, const float *lut, int n_lt, int n_lx, double lt0,
                     double lt1, double lx0, double lx1, double nu, double length_cm, double ds_max,
                     double min_transmit, int64_t *counts) {
  const bho::Scene s = to_scene(scene);
  const auto d = bho::derive<bho::Counted>(s);
  const bho_rt::Medium q{cells, n_r, n_th, n_ph, r_min, r_max, 1.0 / std::log(r_max / r_min), lut, n_lt, n_lx,
                         lt0, lt1, lx0, lx1, nu, length_cm, ds_max, min_transmit};
  for (int k = 0; k < 9; ++k) counts[k] = 0;
  for (int64_t i = 0; i < n; ++i) {
    double alpha, beta;
    bho::pixel_alpha_beta(s, pix_index[i], alpha, beta);
    bho::g_counts = bho::OpCounts{};
    int64_t samples = 0;
    const bho_rt::Result r =
        bho_rt::trace_pixel_rt(s, d, bho::Counted(alpha), bho::Counted(beta), q, &samples);
    const bho::OpCounts c = bho::g_counts;
    counts[0] += c.add;
    counts[1] += c.mul;
    counts[2] += c.div;
    counts[3] += c.sqrt;
    counts[4] += c.trig;
    counts[5] += c.pow;
    counts[6] += c.cmp;
    counts[7] += r.steps;
    counts[8] += samples;
  }
  return 0;
}
int bho_trace_rt(const BH_KerrScene *scene, int64_t n, const int64_t *pix_index, const float *cells, int n_r,
                 int n_th, int n_ph, double r_min, double r_max, const float *lut, int n_lt, int n_lx, double lt0,
                 double lt1, double lx0, double lx1, double nu, double length_cm, double ds_max, double min_transmit,
                 double *i_nu, double *tau, int32_t *cls, int32_t *steps, int threads) {
  const bho::Scene s = to_scene(scene);
  const auto d = bho::derive<double>(s);
  const bho_rt::Medium q{cells, n_r, n_th, n_ph, r_min, r_max, 1.0 / std::log(r_max / r_min), lut, n_lt, n_lx,
                         lt0, lt1, lx0, lx1, nu, length_cm, ds_max, min_transmit};
  parallel_for(n, threads, [&](int64_t i) {
    const int64_t pix = pix_index ? pix_index[i] : i;
    double alpha, beta;
    bho::pixel_alpha_beta(s, pix, alpha, beta);
    const bho_rt::Result r = bho_rt::trace_pixel_rt(s, d, alpha, beta, q);
    i_nu[i] = r.I;
    tau[i] = r.tau;
    cls[i] = r.cls;
    steps[i] = r.steps;
  });
  return 0;
}

// Front-to-back formal solution over segments given near to far.
double bho_rt_path(int64_t n, const double *j, const double *alpha, const double *ds) {
  double I = 0.0, T = 1.0, tau = 0.0;
  for (int64_t i = 0; i < n; ++i) bho_rt::segment(j[i], alpha[i], ds[i], I, T, tau);
  return I;
}

// Same in long double (x87 80-bit) for rounding checks.
int bho_trace_alpha_beta_ld(const BH_KerrScene *scene, int64_t n, const double *alpha, const double *beta,
                            const BH_KerrImageOut *out, int threads) {
  const bho::Scene s = to_scene(scene);
  const auto d = bho::derive<long double>(s);
  const int maxc = std::max(1, std::min(3, int(s.max_crossings)));
  parallel_for(n, threads, [&](int64_t i) {
    const auto p = bho::trace_pixel<long double>(s, d, (long double)alpha[i], (long double)beta[i]);
    store(out, i, n, maxc, p);
  });
  return 0;
}

// FLOPs of one traced pixel with the counting scalar. counts[0..6] receive
// add, mul, div, sqrt, trig, pow, cmp; steps[0] the accepted steps.
int bho_count_ops(const BH_KerrScene *scene, double alpha, double beta, int64_t *counts, int32_t *steps) {
  const bho::Scene s = to_scene(scene);
  const auto d = bho::derive<bho::Counted>(s);
  bho::g_counts = bho::OpCounts{};
  const auto p = bho::trace_pixel<bho::Counted>(s, d, bho::Counted(alpha), bho::Counted(beta));
  const bho::OpCounts c = bho::g_counts;
  counts[0] = c.add;
  counts[1] = c.mul;
  counts[2] = c.div;
  counts[3] = c.sqrt;
  counts[4] = c.trig;
  counts[5] = c.pow;
  counts[6] = c.cmp;
  steps[0] = p.steps;
  return p.cls;
}

// FLOPs of one right-hand-side evaluation and one RK4 step (no bisection):
// out[0..6] for the RHS, out[7..13] for the step.
int bho_count_step_ops(double spin, double alpha, double beta, int64_t *out) {
  bho::RayConsts<bho::Counted> c{};
  c.a = spin;
  c.lam = alpha;
  c.qTh = beta * beta + alpha * alpha;
  c.qR = c.qTh;
  c.K = c.qR + (c.lam - c.a) * (c.lam - c.a);
  bho::Y<bho::Counted> y{bho::Counted(10.0), bho::Counted(0.3), bho::Counted(0.0), bho::Counted(-50.0),
                         bho::Counted(1.0)};
  auto dump = [&](int64_t *o) {
    o[0] = bho::g_counts.add; o[1] = bho::g_counts.mul; o[2] = bho::g_counts.div; o[3] = bho::g_counts.sqrt;
    o[4] = bho::g_counts.trig; o[5] = bho::g_counts.pow; o[6] = bho::g_counts.cmp;
  };
  bho::g_counts = bho::OpCounts{};
  (void)bho::img_rhs(y, c);
  dump(out);
  bho::Scene s{};
  s.step_coeff = 0.02;
  s.step_rcap = 20.0;
  bho::g_counts = bho::OpCounts{};
  const bho::Counted h = bho::mino_step(s, y, c.a);
  const bho::PolyRhs<bho::Counted> f{c};
  (void)bho::img_rk4(y, h, f, f(y));
  (void)(y.r <= bho::Counted(1.0));  // horizon, escape and crossing tests
  (void)(y.r >= bho::Counted(1.0));
  (void)(y.u * y.u < bho::Counted(0.0));
  dump(out + 7);
  return 0;
}

// ----- Part A: batched reference stepper -----------------------------------

int bho_kerr_potentials(int64_t n, const double *r, const double *theta, double mass, double a,
                        const double *e, const double *lz, const double *q, double *rpot, double *drpot,
                        double *thpot, double *dthpot) {
  for (int64_t i = 0; i < n; ++i) {
    const bho::Consts<double> c{e[i], lz[i], q[i]};
    const auto p = bho::kerr_potentials<double>(r[i], theta[i], mass, a, c);
    if (rpot) rpot[i] = p.rPot;
    if (drpot) drpot[i] = p.dRdr;
    if (thpot) thpot[i] = p.thetaPot;
    if (dthpot) dthpot[i] = p.dThetadtheta;
  }
  return 0;
}

// state arrays are updated in place: r, theta, phi, t, sign_r, sign_theta.
int bho_kerr_step_mino(int64_t n, double *r, double *theta, double *phi, double *t, double *sr, double *sth,
                       double mass, double a, const double *e, const double *lz, const double *q,
                       const double *dlam, double dlam_scalar, int32_t nsteps) {
  for (int64_t i = 0; i < n; ++i) {
    bho::State<double> s{r[i], theta[i], phi[i], t[i], sr[i], sth[i]};
    const bho::Consts<double> c{e[i], lz[i], q[i]};
    const double h = dlam ? dlam[i] : dlam_scalar;
    for (int32_t k = 0; k < nsteps; ++k) s = bho::kerr_step_mino<double>(s, mass, a, c, h);
    r[i] = s.r; theta[i] = s.theta; phi[i] = s.phi; t[i] = s.t; sr[i] = s.signR; sth[i] = s.signTheta;
  }
  return 0;
}

// Same stepper in __float128; inputs/outputs in double.
int bho_kerr_step_mino_f128(int64_t n, double *r, double *theta, double *phi, double *t, const double *sr,
                            const double *sth, double mass, double a, const double *e, const double *lz,
                            const double *q, double dlam, int32_t nsteps) {
  using F = bho::f128;
  for (int64_t i = 0; i < n; ++i) {
    bho::State<F> s{F(r[i]), F(theta[i]), F(phi[i]), F(t[i]), F(sr[i]), F(sth[i])};
    const bho::Consts<F> c{F(e[i]), F(lz[i]), F(q[i])};
    for (int32_t k = 0; k < nsteps; ++k) s = bho::kerr_step_mino<F>(s, F(mass), F(a), c, F(dlam));
    r[i] = double(s.r); theta[i] = double(s.theta); phi[i] = double(s.phi); t[i] = double(s.t);
  }
  return 0;
}

int bho_kerr_trace_rays(int64_t n, const double *r, const double *theta, const double *phi, const double *t,
                        const double *sr, const double *sth, const double *e, const double *lz,
                        const double *q, double mass, double a, double r_horizon, double r_escape,
                        double step, int32_t max_steps, int32_t *status, int32_t *steps, double *dist,
                        double *rf, double *thf, double *phf, double *redshift, int threads) {
  parallel_for(n, threads, [&](int64_t i) {
    const bho::State<double> s{r[i], theta[i], phi[i], t[i], sr[i], sth[i]};
    const bho::Consts<double> c{e[i], lz[i], q[i]};
    const auto res = bho::kerr_trace<double>(s, c, mass, a, r_horizon, r_escape, step, max_steps);
    if (status) status[i] = res.status;
    if (steps) steps[i] = res.steps;
    if (dist) dist[i] = res.totalDistance;
    if (rf) rf[i] = res.r;
    if (thf) thf[i] = res.theta;
    if (phf) phf[i] = res.phi;
    if (redshift) redshift[i] = res.redshift;
  });
  return 0;
}

// Known answers of kerr.h for geometric mass m: out = {r_plus, r_minus,
// isco_pro, isco_retro, r_ph_pro, r_ph_retro, nt_isco, nt_eta_flux_peak}.
int bho_kerr_radii(double m, double a, double *out) {
  out[0] = bho::outer_horizon_geom(m, a);
  const double disc = m * m - a * a;
  out[1] = disc < 0 ? NAN : m - std::sqrt(disc);
  out[2] = bho::isco_geom(m, a, true);
  out[3] = bho::isco_geom(m, a, false);
  out[4] = bho::photon_orbit_prograde_geom(m, a);
  out[5] = bho::photon_orbit_retrograde_geom(m, a);
  out[6] = bho::nt_isco(a / m);
  out[7] = bho::nt_normalized_flux(1.5 * bho::nt_isco(a / m), a / m);
  return 0;
}

double bho_nt_normalized_flux(double r, double a_star) { return bho::nt_normalized_flux(r, a_star); }
double bho_nt_radiative_efficiency(double a_star) { return bho::nt_radiative_efficiency(a_star); }
double bho_disk_g(double r, double a, double lam) { return bho::disk_g<double>(r, a, lam); }
double bho_unit_mass(void) { return bho::kUnitMass; }

}  // extern "C"
