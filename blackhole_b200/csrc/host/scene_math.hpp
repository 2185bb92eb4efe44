// scene_math.hpp - host-side per-scene constants (C++23).
//
// Every libm-derived quantity the kernels need is computed here, once per
// scene, with the same formulas and evaluation order as the reference:
//   outer horizon      src/physics/kerr.h:132-141
//   prograde ISCO      src/physics/kerr.h:203-225 (cbrt form, disk inner edge)
//   NT ISCO and peak   src/physics/novikov_thorne.h:81-90, 170-190 (pow form)
//   KerrRaytracer      src/physics/raytracer.h:311-318 with physics::Kerr's
//                      spin clamp (src/physics/kerr.h:446-456)
#pragma once

#include <algorithm>
#include <cmath>

#include "../../../include/bh_kerr.h"

namespace bhh {

inline constexpr double kC = 2.99792458e10;  // src/physics/constants.h:23
inline constexpr double kC2 = kC * kC;
inline constexpr double kG = 6.67430e-8;     // src/physics/constants.h:29
inline constexpr double kGOverC2 = kG / kC2;
inline constexpr double kTwoGOverC2 = 2.0 * kGOverC2;

inline double outer_horizon(double m, double a) {
  const double disc = (m * m) - (a * a);
  if (disc < 0) return std::nan("");
  return m + std::sqrt(disc);
}

inline double isco_prograde(double m, double a) {
  const double aStar = a / m;
  if (std::abs(aStar) > 1.0) return std::nan("");
  const double oneMinusA2 = 1.0 - (aStar * aStar);
  const double cbrtFactor = std::cbrt(oneMinusA2);
  const double cbrtPlus = std::cbrt(1.0 + aStar);
  const double cbrtMinus = std::cbrt(1.0 - aStar);
  const double z1 = 1.0 + (cbrtFactor * (cbrtPlus + cbrtMinus));
  const double z2 = std::sqrt((3.0 * aStar * aStar) + (z1 * z1));
  const double sq = std::sqrt((3.0 - z1) * (3.0 + z1 + (2.0 * z2)));
  return (3.0 + z2 - sq) * m;
}

inline double nt_isco(double aStar) {
  aStar = std::clamp(aStar, -0.9999, 0.9999);
  const double z1 = 1.0 + (std::pow(1.0 - (aStar * aStar), 1.0 / 3.0) *
                           (std::pow(1.0 + aStar, 1.0 / 3.0) + std::pow(1.0 - aStar, 1.0 / 3.0)));
  const double z2 = std::sqrt((3.0 * aStar * aStar) + (z1 * z1));
  return 3.0 + z2 - std::copysign(std::sqrt((3.0 - z1) * (3.0 + z1 + (2.0 * z2))), aStar);
}

struct SceneConstants {
  double r_plus, r_minus, r_hor, r_esc, r_in, sin_o, cos_o, nt_isco, nt_flux_peak;
};

inline SceneConstants scene_constants(const BH_KerrScene &s) {
  SceneConstants k{};
  k.r_plus = outer_horizon(1.0, s.spin);
  k.r_minus = 1.0 - std::sqrt(1.0 - s.spin * s.spin);
  k.r_hor = s.horizon_factor * k.r_plus;
  k.r_esc = s.escape_factor * s.r_obs;
  k.r_in = (s.disk_r_in > 0) ? s.disk_r_in : isco_prograde(1.0, s.spin);
  k.sin_o = std::sin(s.theta_obs);
  k.cos_o = std::cos(s.theta_obs);
  k.nt_isco = nt_isco(s.spin);
  const double rPeak = 1.5 * k.nt_isco;
  const double fPeak = std::max(0.0, 1.0 - std::sqrt(k.nt_isco / rPeak));
  k.nt_flux_peak = fPeak / (rPeak * rPeak * rPeak);
  return k;
}

struct RaytracerDefaults {
  double a, r_horizon, r_escape, step;
};

// physics::KerrRaytracer(mass, spinParam): Kerr clamps |a*| > 1 to 0.998 of
// the same sign; horizon = outer horizon (r_s if not finite or not > 0);
// escape = 1000 r_s; step = 0.02 r_s.
inline RaytracerDefaults raytracer_defaults(double mass, double spin_param) {
  const double mGeom = kG * mass / kC2;
  double a = spin_param;
  double aStar = spin_param / (kG * mass / kC2);
  if (std::abs(aStar) > 1.0) {
    aStar = (aStar > 0) ? 0.998 : -0.998;
    a = aStar * mGeom;
  }
  const double rS = kTwoGOverC2 * mass;
  const double disc = (mGeom * mGeom) - (a * a);
  double rH = disc < 0 ? std::nan("") : mGeom + std::sqrt(disc);
  if (!std::isfinite(rH) || rH <= 0.0) rH = rS;
  return RaytracerDefaults{a, rH, 1000.0 * rS, 0.02 * rS};
}

}  // namespace bhh
