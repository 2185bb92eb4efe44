// ref_shim.cpp - extern "C" wrappers around the reference's own compiled
// Kerr code (test infrastructure only).
//
// Built by oracle/Makefile against the reference's unmodified
// src/physics/kerr.cpp and schwarzschild.cpp into oracle/_ref/libbh_ref.so.
// It lets the tests pin the oracle restatement bit for bit against the
// reference, and gives bench.py's CPU baseline the reference's own compiled
// potentials:
//   ref_kerr_potentials  -> physics::kerrPotentials (src/physics/kerr.cpp:69-97)
//   ref_kerr_step_mino   -> physics::kerrStepMino   (src/physics/kerr.cpp:99-134)
//   ref_kerr_trace_rays  -> the loop of physics::KerrRaytracer::trace
//                           (src/physics/raytracer.h:324-378; raytracer.h itself
//                           needs glm/Eigen, so its 40-line loop is restated here
//                           around the reference's compiled functions)
//   ref_trace_pixels     -> the image tracer of kerr_oracle.hpp with every
//                           potential and potential derivative taken from the
//                           compiled physics::kerrPotentials.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <vector>

#include "physics/constants.h"
#include "physics/kerr.h"
#include "physics/novikov_thorne.h"
#include "physics/rte_integrator.h"

#include "../include/bh_kerr.h"
#include "kerr_oracle.hpp"

namespace {

template <class F> void parallel_for(int64_t n, int threads, F &&f) {
  if (threads <= 1 || n < 2) {
    for (int64_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int64_t> next{0};
  const int64_t chunk = 16;
  std::vector<std::thread> pool;
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

// Right-hand side of the second-order u = cos(theta) system, built from the
// reference's compiled kerrPotentials: p_r' = dRdr/2 and
// p_u' = dU/du / 2 = -u Theta - sin(theta) dTheta/dtheta / 2 (U = sin^2 Theta).
// The azimuth rate is kerr.cpp:61 with E = 1, negated for the backward ray.
struct RefRhs {
  double mass, a;
  physics::KerrGeodesicConsts cR, cTh;
  bool same;
  bho::Y<double> operator()(const bho::Y<double> &y) const {
    const double u = std::clamp(y.u, -1.0, 1.0);
    const double th = std::acos(u);
    const physics::KerrPotentials pR = physics::kerrPotentials(y.r, th, mass, a, cR);
    const physics::KerrPotentials pT = same ? pR : physics::kerrPotentials(y.r, th, mass, a, cTh);
    const double sinTheta = std::sin(th);
    const double sin2 = std::max(sinTheta * sinTheta, 1e-12);
    const double delta = (y.r * y.r) - (2.0 * y.r) + (a * a);
    const double aFactor = ((y.r * y.r) + (a * a)) - (a * cR.lz);
    const double deltaSafe = std::max(delta, 1e-12);
    bho::Y<double> d;
    d.r = y.pr;
    d.u = y.pu;
    d.pr = 0.5 * pR.dRdr;
    d.pu = -(y.u * pT.thetaPot) - (0.5 * sinTheta * pT.dThetadtheta);
    // horizon-regular azimuth psi (kerr_oracle.hpp, img_rhs): the forward
    // rate kerr.cpp:61 with a A / Delta replaced by a (A + p_r) / Delta, in
    // its rationalized form K / (A - p_r) for ingoing rays
    const double K = cR.q + (cR.lz - a) * (cR.lz - a);
    const bool in = y.pr < 0.0;
    const double num = in ? K : (aFactor + y.pr);
    const double den = in ? (aFactor - y.pr) : deltaSafe;
    d.phi = (a - (cR.lz / sin2)) - (a * (num / den));
    return d;
  }
  // First-integral projection with R from kerrPotentials and U = sin^2 Theta.
  void project(bho::Y<double> &y) const {
    const double u = std::clamp(y.u, -1.0, 1.0);
    const double th = std::acos(u);
    const double Rv = physics::kerrPotentials(y.r, th, mass, a, cR).rPot;
    const double r2 = y.r * y.r;
    if (Rv > bho::kProjTau * (r2 * r2)) y.pr = bho::with_sign_of(std::sqrt(Rv), y.pr);
    const double sinTheta = std::sin(th);
    const double Uv = sinTheta * sinTheta * physics::kerrPotentials(y.r, th, mass, a, cTh).thetaPot;
    if (Uv > bho::kProjTau * (std::fabs(cTh.q) + a * a)) y.pu = bho::with_sign_of(std::sqrt(Uv), y.pu);
  }
};

}  // namespace

extern "C" {

int ref_kerr_potentials(int64_t n, const double *r, const double *theta, double mass, double a,
                        const double *e, const double *lz, const double *q, double *rpot, double *drpot,
                        double *thpot, double *dthpot) {
  for (int64_t i = 0; i < n; ++i) {
    const physics::KerrGeodesicConsts c{e[i], lz[i], q[i]};
    const physics::KerrPotentials p = physics::kerrPotentials(r[i], theta[i], mass, a, c);
    if (rpot) rpot[i] = p.rPot;
    if (drpot) drpot[i] = p.dRdr;
    if (thpot) thpot[i] = p.thetaPot;
    if (dthpot) dthpot[i] = p.dThetadtheta;
  }
  return 0;
}

int ref_kerr_step_mino(int64_t n, double *r, double *theta, double *phi, double *t, double *sr, double *sth,
                       double mass, double a, const double *e, const double *lz, const double *q,
                       const double *dlam, double dlam_scalar, int32_t nsteps) {
  for (int64_t i = 0; i < n; ++i) {
    physics::KerrGeodesicState s{r[i], theta[i], phi[i], t[i], sr[i], sth[i]};
    const physics::KerrGeodesicConsts c{e[i], lz[i], q[i]};
    const double h = dlam ? dlam[i] : dlam_scalar;
    for (int32_t k = 0; k < nsteps; ++k) s = physics::kerrStepMino(s, mass, a, c, h);
    r[i] = s.r; theta[i] = s.theta; phi[i] = s.phi; t[i] = s.t; sr[i] = s.signR; sth[i] = s.signTheta;
  }
  return 0;
}

// KerrRaytracer constructor values (raytracer.h:311-318): horizon, escape, step.
int ref_kerr_raytracer_defaults(double mass, double spin_param, double *out) {
  const physics::Kerr kerr(mass, spin_param);
  const double rS = physics::schwarzschildRadius(mass);
  double rH = kerr.outerHorizon();
  if (!std::isfinite(rH) || rH <= 0.0) rH = rS;
  out[0] = kerr.spin();
  out[1] = rH;
  out[2] = 1000.0 * rS;
  out[3] = 0.02 * rS;
  return 0;
}

int ref_kerr_trace_rays(int64_t n, const double *r, const double *theta, const double *phi, const double *t,
                        const double *sr, const double *sth, const double *e, const double *lz,
                        const double *q, double mass, double a, double r_horizon, double r_escape,
                        double step, int32_t max_steps, int32_t *status, int32_t *steps, double *dist,
                        double *rf, double *thf, double *phf, double *redshift, int threads) {
  const physics::Kerr kerr(mass, a);
  parallel_for(n, threads, [&](int64_t i) {
    physics::KerrGeodesicState state{r[i], theta[i], phi[i], t[i], sr[i], sth[i]};
    const physics::KerrGeodesicConsts c{e[i], lz[i], q[i]};
    int32_t st = 0, taken = 0;
    double total = 0.0, red = 1.0;
    for (int32_t k = 0; k < max_steps; ++k) {
      if (state.r <= (r_horizon * 1.001)) { st = 2; break; }
      if (state.r >= r_escape) { st = 1; break; }
      const physics::KerrPotentials p = kerr.potentials(state.r, state.theta, c);
      physics::KerrGeodesicState next = state;
      if (p.rPot < 0.0) next.signR = -next.signR;
      if (p.thetaPot < 0.0) next.signTheta = -next.signTheta;
      next = kerr.stepMino(next, c, step);
      state = next;
      total += step;
      ++taken;
    }
    if (st == 0) st = (taken >= max_steps) ? 4 : 1;
    if (state.r > (r_horizon * 1.001)) red = 1.0 + kerr.redshift(state.r, state.theta);
    if (status) status[i] = st;
    if (steps) steps[i] = taken;
    if (dist) dist[i] = total;
    if (rf) rf[i] = state.r;
    if (thf) thf[i] = state.theta;
    if (phf) phf[i] = state.phi;
    if (redshift) redshift[i] = red;
  });
  return 0;
}

// Known answers straight from the reference headers for mass [g] and spin
// parameter a [cm]: out = {r_plus, r_minus, isco_pro, isco_retro, r_ph_pro,
// r_ph_retro} (src/physics/kerr.h:132-274), then for a* = a / M the
// NovikovThorneDisk ISCO, radiative efficiency and normalised flux at 1.5 r_isco
// and at 10 M (src/physics/novikov_thorne.h:50-190).
int ref_kerr_radii(double mass, double a, double *out) {
  out[0] = physics::kerrOuterHorizon(mass, a);
  out[1] = physics::kerrInnerHorizon(mass, a);
  out[2] = physics::kerrIscoRadius(mass, a, true);
  out[3] = physics::kerrIscoRadius(mass, a, false);
  out[4] = physics::kerrPhotonOrbitPrograde(mass, a);
  out[5] = physics::kerrPhotonOrbitRetrograde(mass, a);
  const double aStar = physics::dimensionlessSpin(a, mass);
  using NT = blackhole::physics::NovikovThorneDisk;
  out[6] = NT::iscoRadius(aStar);
  out[7] = NT::radiativeEfficiency(aStar);
  out[8] = NT::normalizedFlux(1.5 * NT::iscoRadius(aStar), aStar);
  out[9] = NT::normalizedFlux(10.0, aStar);
  return 0;
}

double ref_nt_normalized_flux(double r, double a_star) {
  return blackhole::physics::NovikovThorneDisk::normalizedFlux(r, a_star);
}

// Image tracer with the reference's compiled potentials; same pixel and
// output conventions as bho_trace_pixels (oracle_capi.cpp).
int ref_trace_pixels(const BH_KerrScene *scene, int64_t n, const int64_t *pix_index,
                     const BH_KerrImageOut *out, int threads) {
  bho::Scene s{};
  s.spin = scene->spin; s.r_obs = scene->r_obs; s.theta_obs = scene->theta_obs;
  s.alpha_min = scene->alpha_min; s.alpha_max = scene->alpha_max;
  s.beta_min = scene->beta_min; s.beta_max = scene->beta_max;
  s.width = scene->width; s.height = scene->height;
  s.integrator = scene->integrator; s.potential_form = scene->potential_form;
  s.max_crossings = scene->max_crossings; s.max_steps = scene->max_steps;
  s.step_coeff = scene->step_coeff; s.step_rcap = scene->step_rcap;
  s.rtol = scene->rtol; s.atol = scene->atol;
  s.horizon_factor = scene->horizon_factor; s.escape_factor = scene->escape_factor;
  s.disk_r_in = scene->disk_r_in; s.disk_r_out = scene->disk_r_out;
  const auto d = bho::derive<double>(s);
  const int maxc = std::max(1, std::min(3, int(s.max_crossings)));
  const double mass = physics::C2 / physics::G;  // G * mass / C2 == 1 exactly
  parallel_for(n, threads, [&](int64_t i) {
    const int64_t pix = pix_index ? pix_index[i] : i;
    double alpha, beta;
    bho::pixel_alpha_beta(s, pix, alpha, beta);
    const auto make = [&](const bho::RayConsts<double> &c) {
      return RefRhs{mass, c.a, physics::KerrGeodesicConsts{1.0, c.lam, c.qR},
                    physics::KerrGeodesicConsts{1.0, c.lam, c.qTh}, c.qR == c.qTh};
    };
    const auto p = bho::trace_pixel<double>(s, d, alpha, beta, make);
    if (out->cls) out->cls[i] = p.cls;
    if (out->steps) out->steps[i] = p.steps;
    if (out->n_cross) out->n_cross[i] = p.n_cross;
    for (int k = 0; k < maxc; ++k) {
      if (out->r_hit) out->r_hit[k * n + i] = p.r_hit[k];
      if (out->phi_hit) out->phi_hit[k * n + i] = p.phi_hit[k];
      if (out->g) out->g[k * n + i] = p.g[k];
    }
    if (out->flux) out->flux[i] = p.flux;
    if (out->intensity) out->intensity[i] = p.intensity;
    if (out->theta_inf) out->theta_inf[i] = p.theta_inf;
    if (out->phi_inf) out->phi_inf[i] = p.phi_inf;
  });
  return 0;
}

// The reference's own radiative-transfer physics (src/physics/rte_integrator.h).
double ref_synchrotron_j(double nu, double b, double n, double theta) {
  return physics::synchrotronThermalEmissivity(nu, b, n, theta);
}
double ref_synchrotron_alpha(double nu, double b, double n, double theta) {
  return physics::synchrotronThermalAbsorption(nu, b, n, theta);
}
double ref_planck(double nu, double temp) { return physics::planckFunction(nu, temp); }

// rteStep over segments given near to far, applied far to near as the
// reference's integrateRtePath orders them.
double ref_rte_path(int64_t n, const double *j, const double *alpha, const double *ds) {
  physics::RteState st{};
  for (int64_t i = n - 1; i >= 0; --i) st = physics::rteStep(st, j[i], alpha[i], ds[i]);
  return st.iNu;
}

}  // extern "C"
