/*
 * bh_analytic.h - closed-form Kerr null-geodesic helpers (host, FP64).
 *
 * The reference's analytic helpers as C entry points: src/physics/
 * analytic_kerr_geodesic.h (FP64, CPU) and src/cuda/device_analytic_kerr.cuh
 * (FP32 device functions its tests exercise). They run the same code as the
 * image tracer's closed-form integrator (BH_INTEGRATOR_ANALYTIC in
 * bh_kerr.h; blackhole_b200/csrc/device/kerr_analytic.cuh compiled for the
 * host). M = 1 throughout; xi = L/E, eta = Q/E^2; "lambda" below is Mino
 * time (dr/dlambda = +-sqrt(R(r))).
 */
#ifndef BH_ANALYTIC_H
#define BH_ANALYTIC_H

#ifdef __cplusplus
extern "C" {
#endif

/* R(r) = (r^2 + a^2 - a xi)^2 - Delta (eta + (xi - a)^2), Delta = r^2 - 2r + a^2
 * (analytic_kerr_geodesic.h:119 radialPotential). */
double bh_analytic_radial_potential(double r, double a, double xi, double eta);

/* R(r) = r^4 + c2 r^2 + c1 r + c0: out = {c2, c1, c0}
 * (analytic_kerr_geodesic.h:154 radialQuarticCoeffs). */
void bh_analytic_quartic_coeffs(double a, double xi, double eta, double out[3]);

/* Motion type labels of analytic_kerr_geodesic.h:66 (RadialMotionType), which
 * label a root set by its number of real roots: 4 TRANSIT, 2 SCATTER, 0 PLUNGE. */
enum BH_AnalyticMotion {
    BH_MOTION_TRANSIT = 0,
    BH_MOTION_PLUNGE = 1,
    BH_MOTION_SCATTER = 2,
    BH_MOTION_ORBIT = 3,
    BH_MOTION_INVALID = 4
};

/* Roots of r^4 + c2 r^2 + c1 r + c0 (Ferrari's factorization, real roots
 * polished by Newton): re/im receive the four roots, real ones first in
 * descending order, then complex pairs (+im first). Returns the number of
 * real roots (0, 2 or 4; -1 if the resolvent has no positive root), and the
 * motion label in *motion (may be NULL). Replaces findRadialRoots
 * (analytic_kerr_geodesic.h:180), whose resolvent uses 4/3 where
 * d_quartic_real_roots (device_analytic_kerr.cuh:198-213) has the correct
 * 8/3 -- the reference's CPU version returns no real roots for the quartic
 * with roots 4, 2, 1, -7 that tests/cuda_analytic_kerr_test.cu:224-255
 * checks; this one returns the device version's roots. */
int bh_analytic_radial_roots(double c2, double c1, double c0, double re[4], double im[4], int *motion);

/* r(lambda) in the allowed band [r3, r2] between the middle roots of four
 * real roots r1 >= r2 >= r3 >= r4 (roots[] descending):
 *   r = (r3 (r2 - r4) - r4 (r2 - r3) sn^2) / ((r2 - r4) - (r2 - r3) sn^2),
 *   sn = sn((1/2) sqrt((r1 - r3)(r2 - r4)) (lambda - lambda0) | m),
 *   m = (r2 - r3)(r1 - r4) / ((r1 - r3)(r2 - r4)),
 * so r(lambda0) = r3 and r(lambda0 + T/2) = r2 (device_analytic_kerr.cuh:340
 * d_kerr_r_analytic; the CPU rAnalytic, analytic_kerr_geodesic.h:314, anchors
 * the Moebius map on r1 and leaves the band). NaN unless the roots are
 * ordered and distinct enough to define m in [0, 1]. */
double bh_analytic_r_bound(double lambda, const double roots[4], double lambda0);

/* Half-period T/2 = K(m) / ((1/2) sqrt((r1 - r3)(r2 - r4))) of that motion
 * (device_analytic_kerr.cuh:385, analytic_kerr_geodesic.h:361). */
double bh_analytic_radial_half_period(const double roots[4]);

/* Critical impact parameters of the spherical photon orbit at r_ph:
 * xi = (r^2 + a^2)/a - 4 r Delta / (a Delta'), eta = 16 r^2 Delta / Delta'^2 - (xi - a)^2
 * (analytic_kerr_geodesic.h:410 criticalImpactParams): out = {xi, eta};
 * a = 0 gives {0, 27}, Delta' = 0 gives {0, 0}. (The device version,
 * device_analytic_kerr.cuh:418-449, has 2 r Delta / (a Delta') and drops a
 * factor r from eta; R = R' = 0 holds for this one.) */
void bh_analytic_critical_impact_params(double r_ph, double a, double out[2]);

/* Equatorial photon orbit radii 2 (1 + cos(2/3 acos(-+|a|)))
 * (analytic_kerr_geodesic.h:454, :465). */
double bh_analytic_prograde_photon_orbit(double a);
double bh_analytic_retrograde_photon_orbit(double a);

/* Jacobi sn, cn, dn(u | m) for m <= 1 (device_analytic_kerr.cuh:50 d_ellpj):
 * Bulirsch's descending Landen sequence, negative m by A&S 16.10, m = 1 by
 * sn = tanh, cn = dn = sech. out = {sn, cn, dn}. */
void bh_analytic_ellpj(double u, double m, double out[3]);

/* Complete elliptic integral of the first kind K(k), k the modulus (m = k^2)
 * (device_analytic_kerr.cuh:124 d_ellint_K); +inf at |k| = 1. */
double bh_analytic_ellint_k(double k);

#ifdef __cplusplus
}
#endif

#endif /* BH_ANALYTIC_H */
