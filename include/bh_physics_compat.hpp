/*
 * bh_physics_compat.hpp -- the reference's scalar Kerr API of src/physics
 * (namespace physics: KerrGeodesicConsts, KerrGeodesicState, KerrPotentials,
 * kerrEquatorialConsts, kerrEquatorialState, kerrPotentials, kerrStepMino,
 * RayStatus, RayTraceResult, KerrRaytracer) with the reference's names,
 * signatures, units (CGS) and results, implemented over this library's C ABI
 * (bh_kerr.h), so that a C++ caller of the reference recompiles against this
 * header and links libblackhole_b200.so instead of the reference's
 * src/physics. Header-only C++23; the caller needs no CUDA headers or
 * libraries.
 *
 *   reference                                   here
 *   kerr.h:362-366  KerrGeodesicConsts          same fields
 *   kerr.h:381-388  KerrGeodesicState           same fields
 *   kerr.h:396-404  kerrEquatorialConsts        same
 *   kerr.h:428-437  kerrEquatorialState         same
 *   kerr.h:439-450  kerrPotentials              bh_kerr_potentials_host (n = 1)
 *   kerr.h:452-453  kerrStepMino                bh_kerr_step_mino_host (n = 1)
 *   raytracer.h:46-79  RayStatus, RayTraceResult  same (finalPosition / path
 *                                               as a plain {x, y, z} triple)
 *   raytracer.h:309-399 KerrRaytracer           bh_kerr_raytracer_defaults +
 *                                               bh_kerr_trace_rays_host
 *
 * Every call runs the library's GPU kernels: one launch and a round trip per
 * call. KerrRaytracer::trace of many rays at once (the span overload, not in
 * the reference) traces them in one launch. With setRecordPath(true) the
 * trace steps through kerrPotentials / kerrStepMino one step per round trip,
 * as the reference's loop does (raytracer.h:338-363), to record every point:
 * correct, but slow. Errors throw std::runtime_error with bh_last_error().
 */
#ifndef BH_PHYSICS_COMPAT_HPP
#define BH_PHYSICS_COMPAT_HPP

#include <numbers>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "bh_kerr.h"

namespace physics {

namespace math {
/** (r, theta, phi) triple of RayTraceResult (the reference's math::Vec3d). */
struct Vec3d {
  double x = 0.0, y = 0.0, z = 0.0;
  constexpr Vec3d() = default;
  constexpr Vec3d(double a, double b, double c) : x(a), y(b), z(c) {}
};
}  // namespace math

struct KerrGeodesicConsts {
  double e;   // energy per unit mass
  double lz;  // angular momentum
  double q;   // Carter constant
};

struct KerrGeodesicState {
  double r;
  double theta;
  double phi;
  double t;
  double signR;      // +1 or -1
  double signTheta;  // +1 or -1
};

struct KerrPotentials {
  double rPot;
  double dRdr;
  double thetaPot;
  double dThetadtheta;
};

enum class RayStatus { PROPAGATING, ESCAPED, CAPTURED, HitDisk, MaxSteps };

struct RayTraceResult {
  math::Vec3d finalPosition{};
  double totalDistance = 0.0;
  double redshift = 0.0;
  int stepsTaken = 0;
  RayStatus status = RayStatus::PROPAGATING;
  std::vector<math::Vec3d> path;
};

namespace detail {
inline void check(int rc) {
  if (rc != 0) throw std::runtime_error(std::string("blackhole_b200: ") + bh_last_error());
}
inline BH_KerrConstsSoA consts_view(const KerrGeodesicConsts& c) { return BH_KerrConstsSoA{&c.e, &c.lz, &c.q}; }
}  // namespace detail

/** Constants of an equatorial null ray of impact parameter b = lz / e (q = 0). */
[[nodiscard]] inline KerrGeodesicConsts kerrEquatorialConsts(double impactParam, double energy = 1.0) {
  return KerrGeodesicConsts{energy, impactParam * energy, 0.0};
}

/** An equatorial state at (r, phi) moving with the sign of signR. */
[[nodiscard]] inline KerrGeodesicState kerrEquatorialState(double r, double phi, double signR) {
  return KerrGeodesicState{r, 0.5 * std::numbers::pi, phi, 0.0, signR >= 0.0 ? 1.0 : -1.0, 1.0};
}

[[nodiscard]] inline KerrPotentials kerrPotentials(double r, double theta, double mass, double a,
                                                   const KerrGeodesicConsts& c) {
  KerrPotentials p{};
  detail::check(bh_kerr_potentials_host(1, &r, &theta, mass, a, detail::consts_view(c), &p.rPot, &p.dRdr,
                                        &p.thetaPot, &p.dThetadtheta));
  return p;
}

[[nodiscard]] inline KerrGeodesicState kerrStepMino(const KerrGeodesicState& state, double mass, double a,
                                                    const KerrGeodesicConsts& c, double dlam) {
  KerrGeodesicState s = state;
  const BH_KerrStateSoA v{&s.r, &s.theta, &s.phi, &s.t, &s.signR, &s.signTheta};
  detail::check(bh_kerr_step_mino_host(1, v, mass, a, detail::consts_view(c), nullptr, dlam));
  return s;
}

class KerrRaytracer {
 public:
  /** mass [g], spinParam a [cm]: the reference's defaults (horizon, escape at
   *  1000 r_s, step 0.02 r_s, 10000 steps). */
  KerrRaytracer(double mass, double spinParam) { detail::check(bh_kerr_raytracer_defaults(mass, spinParam, &p_)); }

  void setStepSize(double h) { p_.step_size = h; }
  void setMaxSteps(int n) { p_.max_steps = n; }
  void setEscapeRadius(double r) { p_.r_escape = r; }
  void setRecordPath(bool record) { record_ = record; }

  [[nodiscard]] RayTraceResult trace(const KerrGeodesicState& initial, const KerrGeodesicConsts& c) const {
    if (record_) return trace_recorded(initial, c);
    std::vector<RayTraceResult> out = trace(std::span<const KerrGeodesicState>(&initial, 1),
                                            std::span<const KerrGeodesicConsts>(&c, 1));
    return std::move(out.front());
  }

  [[nodiscard]] RayTraceResult traceEquatorial(double r, double phi, double impactParam, double signR,
                                               double energy = 1.0) const {
    return trace(kerrEquatorialState(r, phi, signR), kerrEquatorialConsts(impactParam, energy));
  }

  /** Many rays in one GPU launch (no path recording): states[i] with consts[i]. */
  [[nodiscard]] std::vector<RayTraceResult> trace(std::span<const KerrGeodesicState> states,
                                                  std::span<const KerrGeodesicConsts> consts) const {
    if (states.size() != consts.size()) throw std::invalid_argument("states and consts differ in length");
    const size_t n = states.size();
    std::vector<double> f(9 * n), o(5 * n);
    std::vector<int32_t> st(n), steps(n);
    for (size_t i = 0; i < n; ++i) {
      const KerrGeodesicState& s = states[i];
      const double row[9] = {s.r, s.theta, s.phi, s.t, s.signR, s.signTheta, consts[i].e, consts[i].lz, consts[i].q};
      for (int k = 0; k < 9; ++k) f[k * n + i] = row[k];
    }
    const BH_KerrStateSoA sv{&f[0], &f[n], &f[2 * n], &f[3 * n], &f[4 * n], &f[5 * n]};
    const BH_KerrConstsSoA cv{&f[6 * n], &f[7 * n], &f[8 * n]};
    detail::check(bh_kerr_trace_rays_host(int64_t(n), sv, cv, &p_, st.data(), steps.data(), &o[0], &o[n], &o[2 * n],
                                          &o[3 * n], &o[4 * n]));
    std::vector<RayTraceResult> res(n);
    for (size_t i = 0; i < n; ++i) {
      res[i].status = static_cast<RayStatus>(st[i]);
      res[i].stepsTaken = steps[i];
      res[i].totalDistance = o[i];
      res[i].finalPosition = math::Vec3d(o[n + i], o[2 * n + i], o[3 * n + i]);
      res[i].redshift = o[4 * n + i];
    }
    return res;
  }

 private:
  // The per-step form that records the path (the reference's loop order:
  // horizon, escape, sign flips from the potentials, one Mino-time step).
  RayTraceResult trace_recorded(const KerrGeodesicState& initial, const KerrGeodesicConsts& c) const {
    RayTraceResult res;
    res.redshift = 1.0;
    KerrGeodesicState s = initial;
    res.path.emplace_back(s.r, s.theta, s.phi);
    for (int step = 0; step < p_.max_steps; ++step) {
      if (s.r <= p_.r_horizon * 1.001) {
        res.status = RayStatus::CAPTURED;
        break;
      }
      if (s.r >= p_.r_escape) {
        res.status = RayStatus::ESCAPED;
        break;
      }
      const KerrPotentials pot = kerrPotentials(s.r, s.theta, p_.mass, p_.a, c);
      if (pot.rPot < 0.0) s.signR = -s.signR;
      if (pot.thetaPot < 0.0) s.signTheta = -s.signTheta;
      s = kerrStepMino(s, p_.mass, p_.a, c, p_.step_size);
      res.totalDistance += p_.step_size;
      ++res.stepsTaken;
      res.path.emplace_back(s.r, s.theta, s.phi);
    }
    if (res.status == RayStatus::PROPAGATING)
      res.status = res.stepsTaken >= p_.max_steps ? RayStatus::MaxSteps : RayStatus::ESCAPED;
    res.finalPosition = math::Vec3d(s.r, s.theta, s.phi);
    // the final redshift as the library computes it: a trace of no steps from the final state
    KerrRaytracer at_end = *this;
    at_end.record_ = false;
    at_end.p_.max_steps = 0;
    res.redshift = at_end.trace(s, c).redshift;
    return res;
  }

  BH_KerrRaytracerParams p_{};
  bool record_ = false;
};

}  // namespace physics

#endif /* BH_PHYSICS_COMPAT_HPP */
