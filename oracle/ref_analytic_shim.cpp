// Test infrastructure: C entry points over the reference's own
// src/physics/analytic_kerr_geodesic.h (compiled unmodified from where it lies
// by oracle/Makefile into _ref/libbh_ref_analytic.so), so that tests can pin
// the analytic helpers of include/bh_analytic.h against it. The Boost-only
// parts of that header (rAnalytic, radialHalfPeriod) are not built here.
#include <complex>

#include "physics/analytic_kerr_geodesic.h"

extern "C" {

double ref_radial_potential(double r, double a, double xi, double eta) {
  return physics::radialPotential(r, a, xi, eta);
}

void ref_quartic_coeffs(double a, double xi, double eta, double out[3]) {
  const physics::QuarticCoeffs c = physics::radialQuarticCoeffs(a, xi, eta);
  out[0] = c.c2;
  out[1] = c.c1;
  out[2] = c.c0;
}

// roots as (re, im) pairs in the reference's order; returns nReal, type in *type.
int ref_radial_roots(double c2, double c1, double c0, double re[4], double im[4], int *type) {
  physics::QuarticCoeffs c;
  c.c2 = c2;
  c.c1 = c1;
  c.c0 = c0;
  const physics::RadialRoots r = physics::findRadialRoots(c);
  for (int k = 0; k < 4; ++k) {
    re[k] = r.roots[k].real();
    im[k] = r.roots[k].imag();
  }
  *type = static_cast<int>(r.type);
  return r.nReal;
}

void ref_critical_impact_params(double r_ph, double a, double out[2]) {
  const physics::ImpactParams p = physics::criticalImpactParams(r_ph, a);
  out[0] = p.xi;
  out[1] = p.eta;
}

double ref_prograde_photon_orbit(double a) { return physics::progradePhotonOrbit(a); }
double ref_retrograde_photon_orbit(double a) { return physics::retrogradePhotonOrbit(a); }

}  // extern "C"
