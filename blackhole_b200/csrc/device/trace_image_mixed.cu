// trace_image_mixed.cu - mixed-precision image-plane Kerr tracer (sm_100a).
//
// Same persistent warp-refill structure and trace-loop order as the FP64
// kernel (trace_image_fp64.cu), with the integration in FP32:
//   * FP64: per-ray set-up (lambda, eta, q, K, initial momenta from R(r_obs)),
//     the first-integral projection's R(r) and U(u) (the Carter/energy
//     constraint check of every accepted step), the crossing radius and
//     azimuth handed to the outputs, the redshift g, the Novikov-Thorne flux
//     and the intensity.
//   * FP32: every right-hand side, the Dormand-Prince / RK4 stages, the error
//     estimate and the step controller. A detected equatorial crossing is
//     located by the FP64 Hermite interpolation of hermite.cuh from the
//     compensated step endpoints.
//   * Compensated FP32 (hi + lo with TwoSum) for the positions r, u, phi, so
//     that thousands of small FP32 increments accumulate without drift.
// The DP45 error estimate is formed from the stage derivatives (h sum e_j k_j),
// never as a difference of two positions, so its FP32 rounding noise is
// ~1e-7 of the step increment rather than of the position: rtol = 1e-8 is
// honoured by the controller.
#include <cuda_runtime.h>

#include <cstdio>

#include "frame_source.cuh"
#include "sky.cuh"
#include "hermite.cuh"
#include "image_mixed.cuh"
#include "launch.h"
#include "rt.cuh"
#include "vol.cuh"

namespace bhm {

constexpr unsigned kFull = 0xffffffffu;

struct RayMx {
  RayCf c;
  Yf y;
  Lof lo;
  Yf k1;       // DP45 FSAL stage
  float h;     // DP45 trial step / unused for RK4
  RayCd cd;    // FP64 constants: projection and g
  double inten;
  float r_hor, r_esc, rtol, atol;  // frame constants used every iteration
  long long pix;
  int f;  // frame of the current ray (batch launches)
  int steps;
  int attempts;
  int ncross;
  float cl_r, cl_u, cl_psi;  // closest approach so far (camera rays only)
  float drift;               // largest Carter-constant residual the projection removed
  bhvol::Accum va;           // disk slab seen so far (camera rays of the volumetric modes)
};

__device__ __forceinline__ void split(double v, float &hi, float &lo) {
  hi = (float)v;
  lo = (float)(v - (double)hi);
}

__device__ __forceinline__ void init_ray(const BhkImageParams &p, long long pix, RayMx &R) {
  const long long i = pix % p.width, j = pix / p.width;
  const double alpha = p.alpha_min + ((double)i + 0.5) * p.dalpha;
  const double beta = p.beta_min + ((double)j + 0.5) * p.dbeta;
  const double a = p.a;
  const double lam = -alpha * p.sin_o;
  const double eta = beta * beta + (alpha * alpha - a * a) * p.cos_o * p.cos_o;
  const double qTh = eta + lam * lam;
  const double qR = (p.form == 1) ? eta : qTh;
  const double K = qR + (lam - a) * (lam - a);
  const double r0 = p.r_obs;
  const double A = r0 * r0 + a * a - a * lam;
  const double D = r0 * r0 - 2.0 * r0 + a * a;
  const double Rv = A * A - D * K;
  R.c.a = (float)a;
  R.c.a2 = (float)(a * a);
  R.c.lam = (float)lam;
  R.c.qTh = (float)qTh;
  R.c.K = (float)K;
  R.c.a2_minus_alam = (float)(a * a - a * lam);
  R.c.c_pu = (float)(a * a - qTh);
  R.cd.a = a;
  R.cd.lam = lam;
  R.cd.qTh = qTh;
  R.cd.K = K;
  split(r0, R.y.r, R.lo.r);
  split(p.cos_o, R.y.u, R.lo.u);
  R.y.phi = 0.0f;
  R.lo.phi = 0.0f;
  R.y.pr = (float)(-sqrt(Rv < 0.0 ? 0.0 : Rv));
  R.y.pu = (float)(beta * p.sin_o);
  R.inten = 0.0;
  R.pix = pix;
  R.steps = 0;
  R.attempts = 0;
  R.ncross = 0;
  R.r_hor = (float)p.r_hor;
  R.r_esc = (float)p.r_esc;
  R.rtol = (float)p.rtol;
  R.atol = (float)p.atol;
  project(R.y, R.lo, R.cd);  // idempotent from here on (see iterate)
  R.drift = 0.0f;
  const float hh = (float)p.step_coeff * fminf(R.y.r, (float)p.step_rcap);
  R.h = hh / fmaf(R.c.a2 * R.y.u, R.y.u, R.y.r * R.y.r);
  R.k1 = rhs(R.y, R.c);
}

// A ray of a camera at finite distance (BhkCamera): the pixel's direction d
// in the world frame, taken as the direction in the camera's locally
// non-rotating frame (Bardeen, Press & Teukolsky 1972) at (r0, theta0). The
// photon the pixel sees arrives moving along -d; with the frame's lapse
// alpha_L = sqrt(Sigma Delta / A), rotation omega = 2 a r / A and cylindrical
// radius varpi = sqrt(A / Sigma) sin(theta) its constants per unit energy are
//   lambda = varpi v_phi / (alpha_L + omega varpi v_phi),
//   Theta(theta0) = (sqrt(Sigma) v_theta / (alpha_L + omega varpi v_phi))^2,
// v = -d in the (r, theta, phi) frame; eta = Theta - a^2 cos^2 + lambda^2 cot^2
// (textbook Carter potentials: q_R = eta, q_Th = eta + lambda^2). The traced
// (past-directed) ray moves along d: p_r has the sign of d_r, p_u the sign of
// -d_theta. Azimuths are measured from the camera's.
__device__ __forceinline__ void init_ray_camera(const BhkImageParams &p, const BhkCamera &cam, long long pix,
                                                RayMx &R) {
  const long long i = pix % cam.width, j = pix / cam.width;
  const double uu = (2.0 * ((double)i + 0.5) / (double)cam.width - 1.0) * cam.fov * cam.aspect + cam.shift_x;
  const double vv = (2.0 * ((double)j + 0.5) / (double)cam.height - 1.0) * cam.fov + cam.shift_y;
  double d[3];
  for (int k = 0; k < 3; ++k) d[k] = -uu * cam.right[k] - vv * cam.up[k] + cam.fwd[k];
  const double dn = 1.0 / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  for (int k = 0; k < 3; ++k) d[k] *= dn;
  // local spherical frame at the camera (azimuth phi0 = 0 after rotating by the camera's azimuth)
  const double u0 = cam.u0, s0 = sqrt(fmax(0.0, (1.0 - u0) * (1.0 + u0)));
  const double dx = cam.cphi * d[0] + cam.sphi * d[1], dy = -cam.sphi * d[0] + cam.cphi * d[1], dz = d[2];
  const double n_r = s0 * dx + u0 * dz;
  const double n_th = u0 * dx - s0 * dz;
  const double n_ph = dy;
  const double a = p.a, a2 = p.a2, r = cam.r0;
  const double sig = r * r + a2 * u0 * u0;
  const double del = r * r - 2.0 * r + a2;
  const double AA = (r * r + a2) * (r * r + a2) - a2 * del * s0 * s0;
  const double lapse = sqrt(sig * del / AA);
  const double omega = 2.0 * a * r / AA;
  const double varpi = sqrt(AA / sig) * s0;
  const double v_ph = -n_ph, v_th = -n_th;
  const double e = lapse + omega * varpi * v_ph;  // E / E_local
  const double lam = varpi * v_ph / e;
  const double pth = sqrt(sig) * v_th / e;
  const double cot2 = s0 > 1e-12 ? (u0 * u0) / (s0 * s0) : 0.0;
  const double eta = pth * pth - a2 * u0 * u0 + lam * lam * cot2;
  const double qTh = eta + lam * lam;
  const double K = eta + (lam - a) * (lam - a);
  const double A = r * r + a2 - a * lam;
  const double Rv = A * A - del * K;
  const double Uv = (qTh + a2 * u0 * u0) * (1.0 - u0 * u0) - lam * lam;
  R.c.a = (float)a;
  R.c.a2 = (float)a2;
  R.c.lam = (float)lam;
  R.c.qTh = (float)qTh;
  R.c.K = (float)K;
  R.c.a2_minus_alam = (float)(a2 - a * lam);
  R.c.c_pu = (float)(a2 - qTh);
  R.cd.a = a;
  R.cd.lam = lam;
  R.cd.qTh = qTh;
  R.cd.K = K;
  split(r, R.y.r, R.lo.r);
  split(u0, R.y.u, R.lo.u);
  R.y.phi = 0.0f;
  R.lo.phi = 0.0f;
  const double mr = sqrt(Rv < 0.0 ? 0.0 : Rv), mu = sqrt(Uv < 0.0 ? 0.0 : Uv);
  R.y.pr = (float)(n_r < 0.0 ? -mr : mr);
  R.y.pu = (float)(n_th > 0.0 ? -mu : mu);
  R.inten = 0.0;
  R.pix = pix;
  R.steps = 0;
  R.attempts = 0;
  R.ncross = 0;
  R.r_hor = (float)p.r_hor;
  R.r_esc = (float)p.r_esc;
  R.rtol = (float)p.rtol;
  R.atol = (float)p.atol;
  project(R.y, R.lo, R.cd);
  R.drift = 0.0f;
  const float hh = (float)p.step_coeff * fminf(R.y.r, (float)p.step_rcap);
  R.h = hh / fmaf(R.c.a2 * R.y.u, R.y.u, R.y.r * R.y.r);
  R.k1 = rhs(R.y, R.c);
}

// phi = psi + a (G(r) - G(r_obs)) at the outputs (image_fp64.cuh).
__device__ __forceinline__ double phi_of_psi(double psi, double r, const BhkImageParams &p) {
  if (p.a == 0.0) return psi;
  const double q = ((r - p.r_plus) * (p.r_obs - p.r_minus)) / ((r - p.r_minus) * (p.r_obs - p.r_plus));
  return psi + p.a * (log(q) / (p.r_plus - p.r_minus));
}

__device__ __forceinline__ double disk_g(double r, double a, double lam) {
  const double x = sqrt(r);
  const double x3 = x * x * x;
  const double v = x3 * (x3 - 3.0 * x + 2.0 * a);
  if (v <= 0.0) return 0.0;
  return sqrt(v) / (x3 + a - lam);
}

__device__ __forceinline__ bool on_crossing(const BhkImageParams &p, const BhkImageOut &o, RayMx &R, double r_c,
                                            double phi_c) {
  if (!(r_c >= p.r_in && r_c <= p.r_out)) return false;
  const int k = R.ncross;
  const long long off = (long long)k * p.n_pix + R.pix;
  const double g = disk_g(r_c, p.a, R.cd.lam);
  if (o.r_hit) o.r_hit[off] = r_c;
  if (o.phi_hit) o.phi_hit[off] = phi_of_psi(phi_c, r_c, p);
  if (o.g) o.g[off] = g;
  const double q = p.r_in / r_c;
  const double g2 = g * g;
  R.inten += g2 * g2 * q * q * q;
  if (k == 0 && o.flux) {
    double f = 0.0;
    if (r_c >= p.nt_isco) {
      const double t = 1.0 - sqrt(p.nt_isco / r_c);
      f = fmin(1.0, (t > 0.0 ? t : 0.0) / (r_c * r_c * r_c) / p.nt_flux_peak);
    }
    o.flux[R.pix] = f;
  }
  R.ncross = k + 1;
  return R.ncross >= p.max_cross;
}

// The escaping ray's direction of motion (bhsky::direction_of_motion) in
// FP32: the mixed tracer's own state is FP32, and a texel of the sky spans
// 2e-3 rad. The azimuth is reduced to [-pi, pi] in FP64 first, so the fast
// sine and cosine keep their accuracy. A finishing lane runs this while the
// rest of its warp waits, so its cost counts once per ray for the whole warp.
__device__ __forceinline__ void direction_of_motion_f(double r, double u, double phi, float pr, float pu, double dphi,
                                                      float &x, float &y, float &z) {
  const double two_pi = 6.283185307179586;
  float sp, cp;
  __sincosf((float)(phi - two_pi * rint(phi / two_pi)), &sp, &cp);
  const float uc = fminf(1.0f, fmaxf(-1.0f, (float)u));
  const float st = sqrtf((1.0f - uc) * (1.0f + uc));
  const float rf = (float)r;
  const float dst = st > 1e-30f ? -uc * pu / st : 0.0f;  // d(sin theta)
  const float a = pr * st + rf * dst, b = rf * st * (float)dphi;
  x = a * cp - b * sp;
  y = a * sp + b * cp;
  z = pr * uc + rf * pu;
}

__device__ __forceinline__ void finish(const BhkImageParams &p, const BhkImageOut &o, const RayMx &R, int cls) {
  const long long pix = R.pix;
  if (o.cls) o.cls[pix] = cls;
  if (o.steps) o.steps[pix] = R.steps;
  if (o.n_cross) o.n_cross[pix] = R.ncross;
  if (R.ncross == 0 && o.flux) o.flux[pix] = 0.0;
  for (int k = R.ncross; k < p.max_cross; ++k) {
    const long long off = (long long)k * p.n_pix + pix;
    if (o.r_hit) o.r_hit[off] = 0.0;
    if (o.phi_hit) o.phi_hit[off] = 0.0;
    if (o.g) o.g[off] = 0.0;
  }
  double th = 0.0, ph = 0.0, inten = R.inten;
  float dir[3] = {0.0f, 0.0f, 0.0f};
  if (cls == 2) {
    const double u = to_f64(R.y.u, R.lo.u);
    th = acos(fmin(1.0, fmax(-1.0, u)));
    ph = phi_of_psi(to_f64(R.y.phi, R.lo.phi), to_f64(R.y.r, R.lo.r), p);
    if (p.sky || o.esc_dir) {  // dphi/dtau = dpsi/dtau + a p_r / Delta  (phi = psi + a G(r), G' = 1 / Delta)
      const Yf k = rhs(R.y, R.c);
      const double r = to_f64(R.y.r, R.lo.r);
      const double delta = r * r - 2.0 * r + p.a2;
      const double dphi = (double)k.phi + p.a * (double)R.y.pr / delta;
      float fx, fy, fz;  // one direction of motion for the sky and the caller
      direction_of_motion_f(r, u, ph, R.y.pr, R.y.pu, dphi, fx, fy, fz);
      if (p.sky) inten += bhsky::radiance_dir(p.sky, p.sky_size, (double)fx, (double)fy, (double)fz);
      if (o.esc_dir) {
        const float nn = sqrtf(fx * fx + fy * fy + fz * fz);
        if (nn > 0.0f) {
          const float inv = 1.0f / nn;
          dir[0] = fx * inv;
          dir[1] = fy * inv;
          dir[2] = fz * inv;
        }
      }
    }
  }
  if (o.esc_dir) {
    o.esc_dir[pix] = dir[0];
    o.esc_dir[p.n_pix + pix] = dir[1];
    o.esc_dir[2 * p.n_pix + pix] = dir[2];
  }
  if (o.intensity) o.intensity[pix] = inten;
  if (o.theta_inf) o.theta_inf[pix] = th;
  if (o.phi_inf) o.phi_inf[pix] = ph;
  if (o.carter_drift) o.carter_drift[pix] = (double)R.drift;
}

// The disk slab along one accepted step (camera rays of the RTE and Stokes
// modes), from the step's start y0 + lo0, end R.y + R.lo, their derivatives k0,
// k1 and Mino-time length h. Only the part of the step within 5 slab heights
// of the equatorial plane is sampled: with z = r u taken linear over the step
// that part is an interval of step fraction, widened by a tenth at either end;
// a step whose ends lie on one side of the slab is skipped unless the cubic
// Hermite bound on z lets it dip into it, and then sampled whole. The
// interval's midpoints (16, or one per M of radius crossed if more, at most
// 128) lie on the cubic Hermite interpolant of (r, u, psi). Each is a segment
// of the reference's path length |d tau| / m. Returns true once the slab has
// made the ray opaque.
__device__ __forceinline__ bool vol_step(const BhkImageParams &p, const BhkVolume &v, RayMx &R, const Yf &y0,
                                         const Lof &lo0, const Yf &k0, const Yf &k1, float h) {
  if (!v.emit) return false;
  const float r0 = y0.r + lo0.r, r1 = R.y.r + R.lo.r;
  const float u0 = y0.u + lo0.u, u1 = R.y.u + R.lo.u;
  const float inv_m = 1.0f / v.m;
  const float rin = v.r_in * inv_m, rout = v.r_out * inv_m, zw = 5.0f * v.h * inv_m;
  const float ah = fabsf(h);
  const float slack_r = (4.0f / 27.0f) * ah * (fabsf(k0.r) + fabsf(k1.r));
  if (fminf(r0, r1) - slack_r > 1.02f * rout || fmaxf(r0, r1) + slack_r < rin) return false;
  const float z0 = r0 * u0, z1 = r1 * u1, dz = z1 - z0;
  float fa = 0.0f, fb = 1.0f;
  if (z0 * z1 > 0.0f && fminf(fabsf(z0), fabsf(z1)) > zw) {
    const float dz0 = k0.r * u0 + r0 * k0.u, dz1 = k1.r * u1 + r1 * k1.u;
    if (fminf(fabsf(z0), fabsf(z1)) - (4.0f / 27.0f) * ah * (fabsf(dz0) + fabsf(dz1)) > zw) return false;
  } else if (fabsf(dz) > 1e-6f * zw) {
    float f1 = (-zw - z0) / dz, f2 = (zw - z0) / dz;
    if (f1 > f2) {
      const float t = f1;
      f1 = f2;
      f2 = t;
    }
    const float pad = 0.1f * (f2 - f1);
    fa = fmaxf(0.0f, f1 - pad);
    fb = fminf(1.0f, f2 + pad);
    if (!(fb > fa)) return false;
  }
  const int n = min(128, max(16, (int)ceilf(fabsf(r1 - r0) * (fb - fa))));
  const float ds = ah * (fb - fa) / (float)n * inv_m;
  const float psi0 = y0.phi + lo0.phi, psi1 = R.y.phi + R.lo.phi;
  const float rp = (float)p.r_plus, rmn = (float)p.r_minus, ro = (float)p.r_obs;
  const float gscale = p.a == 0.0 ? 0.0f : (float)p.a / (rp - rmn);
  const float g_obs = (ro - rmn) / (ro - rp);
  float c2b, s2b;
  __sincosf(2.0f * v.b_angle, &s2b, &c2b);
  for (int m = 0; m < n; ++m) {
    const float t = fa + (fb - fa) * ((float)m + 0.5f) / (float)n;
    const float t2 = t * t, t3 = t2 * t;
    const float h00 = 2.0f * t3 - 3.0f * t2 + 1.0f, h10 = (t3 - 2.0f * t2 + t) * h;
    const float h01 = 3.0f * t2 - 2.0f * t3, h11 = (t3 - t2) * h;
    const float r = h00 * r0 + h10 * k0.r + h01 * r1 + h11 * k1.r;
    if (!(r > rp)) continue;
    const float u = fmaxf(-1.0f, fminf(1.0f, h00 * u0 + h10 * k0.u + h01 * u1 + h11 * k1.u));
    const float psi = h00 * psi0 + h10 * k0.phi + h01 * psi1 + h11 * k1.phi;
    const float phi = psi + gscale * __logf(__fdividef(r - rp, r - rmn) * g_obs);  // phi = psi + a (G(r) - G(r_obs))
    float sp, cp;
    __sincosf(phi, &sp, &cp);
    const float rw = r * v.m, sw = rw * sqrtf(fmaxf(0.0f, (1.0f - u) * (1.0f + u)));
    const float x = sw * (cp * v.cphi - sp * v.sphi), y = sw * (sp * v.cphi + cp * v.sphi), z = rw * u;
    float col[3], rho;
    const float j = bhvol::slab_emission(x, y, z, v.rs, v.r_in, v.r_out, v.h, col, rho);
    if (j < 0.0f) continue;
    if (bhvol::accum_segment(R.va, j, col, rho, ds, v.opacity, v.mode, c2b, s2b, v.ne_scale)) return true;
  }
  return false;
}

// Applies the increment d of an accepted step (acc) to the ray: compensated
// positions, crossing test and record, projection; returns true if the ray
// stops. A rejected attempt (acc false) runs the same instructions with a
// zero increment -- adding 0 leaves a compensated pair unchanged and the
// projection is idempotent on a projected state -- so accepted and rejected
// lanes of a warp never diverge. k0 = rhs(y0); k1 = rhs(y1) when the caller
// has it (DP45's FSAL stage), else NULL and evaluated only at a crossing.
// TRACK: also keep the ray's closest approach (camera rays): the smallest r
// of the step ends, and inside a step where p_r turns from negative to
// positive the radial turning point, with p_r linear over the step: at the
// fraction s = -p_r0 / (p_r1 - p_r0) of it, r = r0 + p_r0 s h / 2, u and psi
// interpolated linearly.
// VOL: also integrate the disk slab of vol over the step (needs k1).
// DRIFT: keep the largest Carter-constant residual the projection removes (a
// separate instantiation, so the plain kernels carry none of it).
template <bool TRACK = false, bool VOL = false, bool DRIFT = false>
__device__ __forceinline__ bool accept(const BhkImageParams &p, const BhkImageOut &o, RayMx &R, const Yf &d,
                                       bool acc, float h, const Yf &k0, const Yf *k1,
                                       const BhkVolume *vol = nullptr) {
  const Yf y0 = R.y;
  const Lof lo0 = R.lo;
  comp_add(R.y.r, R.lo.r, acc ? d.r : 0.0f);
  comp_add(R.y.u, R.lo.u, acc ? d.u : 0.0f);
  comp_add(R.y.phi, R.lo.phi, acc ? d.phi : 0.0f);
  R.y.pr += acc ? d.pr : 0.0f;
  R.y.pu += acc ? d.pu : 0.0f;
  R.steps += acc ? 1 : 0;
  if (TRACK && acc) {
    const float r1 = R.y.r + R.lo.r;
    if (r1 < R.cl_r) {
      R.cl_r = r1;
      R.cl_u = R.y.u;
      R.cl_psi = R.y.phi;
    }
    if (y0.pr < 0.0f && R.y.pr >= 0.0f) {
      const float s = -y0.pr / (R.y.pr - y0.pr);
      const float r_tp = (y0.r + lo0.r) + 0.5f * y0.pr * s * h;
      if (r_tp < R.cl_r) {
        R.cl_r = r_tp;
        R.cl_u = y0.u + s * (R.y.u - y0.u);
        R.cl_psi = y0.phi + s * (R.y.phi - y0.phi);
      }
    }
  }
  bool stop = false;
  if (VOL && acc && k1) stop = vol_step(p, *vol, R, y0, lo0, k0, *k1, h);
  if (acc && (y0.u + lo0.u) * (R.y.u + R.lo.u) < 0.0f) {
    const Yf kk = k1 ? *k1 : rhs(R.y, R.c);
    const bhh_dev::Ends e{to_f64(y0.r, lo0.r),   to_f64(y0.u, lo0.u),   to_f64(y0.phi, lo0.phi),
                          (double)y0.pr,         (double)y0.pu,         (double)k0.pr,
                          (double)k0.pu,         (double)k0.phi,        to_f64(R.y.r, R.lo.r),
                          to_f64(R.y.u, R.lo.u), to_f64(R.y.phi, R.lo.phi), (double)R.y.pr,
                          (double)R.y.pu,        (double)kk.pr,         (double)kk.pu,
                          (double)kk.phi};
    double r_c, phi_c;
    bhh_dev::hermite_crossing(e, (double)h, r_c, phi_c);
    stop = on_crossing(p, o, R, r_c, phi_c) || stop;
  }
  const float drift = project(R.y, R.lo, R.cd, DRIFT);
  if (DRIFT && acc) R.drift = fmaxf(R.drift, drift);
  return stop;
}

template <int INTEG, bool TRACK = false, bool VOL = false, bool DRIFT = false>
__device__ __forceinline__ int iterate(const BhkImageParams &p, const BhkImageOut &o, RayMx &R,
                                       const BhkVolume *vol = nullptr) {
  const float r_hor = R.r_hor, r_esc = R.r_esc;
  if (INTEG == 0) {
    if (R.steps >= p.max_steps) return 3;
    if (R.y.r <= r_hor) return 0;
    if (R.y.r >= r_esc) return 2;
    const float hh = (float)p.step_coeff * fminf(R.y.r, (float)p.step_rcap);
    const float h = __fdividef(hh, fmaf(R.c.a2 * R.y.u, R.y.u, R.y.r * R.y.r));
    const Yf k0 = rhs(R.y, R.c);
    const Yf d = rk4_inc(R.y, h, R.c, k0);
    return accept<TRACK, VOL, DRIFT>(p, o, R, d, true, h, k0, nullptr, vol) ? 1 : -1;
  } else {
    const long long max_attempts = 4LL * p.max_steps + 64;
    if (R.steps >= p.max_steps || R.attempts >= max_attempts) return 3;
    if (R.y.r <= r_hor) return 0;
    if (R.y.r >= r_esc) return 2;
    ++R.attempts;
    const DPf d = dp45(R.y, R.h, R.c, R.k1, R.rtol, R.atol, true);
    const bool acc = d.err <= 1.0f;
    const float h = R.h;
    const bool stop = accept<TRACK, VOL, DRIFT>(p, o, R, d.d, acc, h, R.k1, &d.k7, vol);
    R.k1 = acc ? d.k7 : R.k1;
    R.k1.r = R.y.pr;  // projection moved only the momenta
    R.k1.u = R.y.pu;
    R.h = h * step_factor(d.err, acc);
    return stop ? 1 : -1;
  }
}

// The pixels of one camera frame.
struct CameraSrc {
  const BhkImageParams &p;
  const BhkCamera &cam;
  const BhkImageOut &o;
  __device__ __forceinline__ long long total() const { return p.n_pix; }
  __device__ __forceinline__ int frame_of(long long w, long long &pix) const {
    pix = w;
    return 0;
  }
  __device__ __forceinline__ const BhkImageParams &params(int) const { return p; }
  __device__ __forceinline__ const BhkImageOut &out(int) const { return o; }
  __device__ __forceinline__ void pixel_done(int) const {}
};

// Sources whose rays keep their closest approach (for the reference look of
// the render launch ABI): the camera's.
template <class Src>
struct tracks_closest {
  static constexpr bool value = false;
};
template <>
struct tracks_closest<CameraSrc> {
  static constexpr bool value = true;
};

// A camera frame whose rays also integrate the disk slab (RTE and Stokes modes).
struct CameraVolSrc : CameraSrc {
  const BhkVolume &vol;
};
template <>
struct tracks_closest<CameraVolSrc> {
  static constexpr bool value = true;
};
template <class Src>
struct has_volume {
  static constexpr bool value = false;
};
template <>
struct has_volume<CameraVolSrc> {
  static constexpr bool value = true;
};
template <class Src>
__device__ __forceinline__ const BhkVolume *volume_of(const Src &) {
  return nullptr;
}
__device__ __forceinline__ const BhkVolume *volume_of(const CameraVolSrc &src) { return &src.vol; }

// The slab's totals of a finished ray: [8][n] r, g, b, transmittance, Q, U, V,
// 1 if the slab made it opaque.
__device__ __forceinline__ void write_vol(const BhkImageParams &p, const BhkImageOut &o, const RayMx &R, bool opaque) {
  if (!o.vol) return;
  const long long n = p.n_pix, i = R.pix;
  o.vol[i] = R.va.rgb[0];
  o.vol[n + i] = R.va.rgb[1];
  o.vol[2 * n + i] = R.va.rgb[2];
  o.vol[3 * n + i] = R.va.T;
  o.vol[4 * n + i] = R.va.s.q;
  o.vol[5 * n + i] = R.va.s.u;
  o.vol[6 * n + i] = R.va.s.v;
  o.vol[7 * n + i] = opaque ? 1.0f : 0.0f;
}

__device__ __forceinline__ void write_closest(const BhkImageParams &p, const BhkImageOut &o, const RayMx &R) {
  if (!o.closest) return;
  o.closest[R.pix] = R.cl_r;
  o.closest[p.n_pix + R.pix] = R.cl_u;
  o.closest[2 * p.n_pix + R.pix] = (float)phi_of_psi((double)R.cl_psi, (double)R.cl_r, p);
}

// A ray's initial state: image-plane pixels for every source but the camera.
template <class Src>
__device__ __forceinline__ void init_from(const Src &src, int f, long long pix, RayMx &R) {
  init_ray(src.params(f), pix, R);
}
__device__ __forceinline__ void init_from(const CameraSrc &src, int, long long pix, RayMx &R) {
  init_ray_camera(src.p, src.cam, pix, R);
  R.cl_r = R.y.r + R.lo.r;
  R.cl_u = R.y.u;
  R.cl_psi = 0.0f;
}
__device__ __forceinline__ void init_from(const CameraVolSrc &src, int f, long long pix, RayMx &R) {
  init_from(static_cast<const CameraSrc &>(src), f, pix, R);
  bhvol::accum_init(R.va);
}

// The persistent loop shared by the single-frame and batch kernels (see
// trace_image_fp64.cu).
template <int INTEG, bool DRIFT = false, class Src>
__device__ __forceinline__ void trace_loop(const Src &src, unsigned long long *__restrict__ counter, int refill) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  const unsigned long long total = (unsigned long long)src.total();
  RayMx R;
  bool active = false;
  bool exhausted = false;
  for (;;) {
    const unsigned need = __ballot_sync(kFull, !active && !exhausted);
    if (need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if ((int)lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(need));
      base = __shfl_sync(kFull, base, leader);
      if (!active && !exhausted) {
        const unsigned long long mine = base + (unsigned long long)__popc(need & lanemask_lt);
        if (mine < total) {
          long long pix;
          const int f = src.frame_of((long long)mine, pix);
          init_from(src, f, pix, R);
          R.f = f;
          active = true;
        } else {
          exhausted = true;
        }
      }
    }
    if (!__any_sync(kFull, active)) break;
    for (int k = 0; k < refill; ++k) {
      if (active) {
        const BhkImageParams &P = src.params(R.f);
        const int cls =
            iterate<INTEG, tracks_closest<Src>::value, has_volume<Src>::value, DRIFT>(P, src.out(R.f), R,
                                                                                     volume_of(src));
        if (cls >= 0) {
          if (tracks_closest<Src>::value) write_closest(P, src.out(R.f), R);
          if (has_volume<Src>::value) write_vol(P, src.out(R.f), R, cls == 1);
          finish(P, src.out(R.f), R, cls);
          src.pixel_done(R.f);
          active = false;
        }
      }
    }
  }
}

template <int INTEG, bool DRIFT>
__global__ void __launch_bounds__(128, 4) k_trace_image_mixed(const __grid_constant__ BhkImageParams p,
                                                           const __grid_constant__ BhkImageOut o,
                                                           unsigned long long *__restrict__ counter, int refill) {
  trace_loop<INTEG, DRIFT>(bhsrc::SingleSrc{p, o}, counter, refill);
}

template <int INTEG, bool DRIFT>
__global__ void __launch_bounds__(128, 4) k_trace_list_mixed(const __grid_constant__ BhkImageParams p,
                                                          const __grid_constant__ BhkImageOut o,
                                                          const int *__restrict__ list,
                                                          const unsigned int *__restrict__ count,
                                                          unsigned long long *__restrict__ counter, int refill) {
  trace_loop<INTEG, DRIFT>(bhsrc::ListSrc{p, o, list, count}, counter, refill);
}

__global__ void __launch_bounds__(128) k_trace_camera_mixed(const __grid_constant__ BhkImageParams p,
                                                            const __grid_constant__ BhkCamera cam,
                                                            const __grid_constant__ BhkImageOut o,
                                                            unsigned long long *__restrict__ counter, int refill) {
  trace_loop<1>(CameraSrc{p, cam, o}, counter, refill);
}

__global__ void __launch_bounds__(128) k_trace_camera_vol_mixed(const __grid_constant__ BhkImageParams p,
                                                                const __grid_constant__ BhkCamera cam,
                                                                const __grid_constant__ BhkVolume vol,
                                                                const __grid_constant__ BhkImageOut o,
                                                                unsigned long long *__restrict__ counter, int refill) {
  trace_loop<1>(CameraVolSrc{{p, cam, o}, vol}, counter, refill);
}

template <int INTEG, bool DRIFT>
__global__ void __launch_bounds__(128) k_trace_batch_mixed(const __grid_constant__ BhkBatchDev b,
                                                           unsigned long long *__restrict__ counter, int refill) {
  if (threadIdx.x == 0) atomicMin(b.start_ns, bhsrc::globaltimer_ns());
  trace_loop<INTEG, DRIFT>(bhsrc::BatchSrc{b}, counter, refill);
}

// ---- along-ray transfer on the mixed tracer ---------------------------------------
//
// The FP64 transfer kernel (trace_image_fp64.cu, k_trace_rt_fp64) with the
// geodesic from the mixed tracer and every sample in FP32 (rt.cuh, FP32
// variants): positions by cubic Hermite interpolation of the accepted step,
// at most ds_max apart in affine length; intensity and optical depth summed
// in FP64.
__device__ __forceinline__ void rt_segment_f(const BhkImageParams &p, const bhrt::MediumF &q, const RayCf &c,
                                             const Yf &y0, const Yf &k0, const Yf &y1, const Yf &k1, float h,
                                             double &I, float &T, double &tau) {
  const float a2 = c.a2;
  const float rm = fmaf(0.125f * h, k0.r - k1.r, 0.5f * (y0.r + y1.r));
  const float um = fmaf(0.125f * h, k0.u - k1.u, 0.5f * (y0.u + y1.u));
  // a step that stays beyond r_max samples nothing (see the FP64 transfer)
  const float rlow = fminf(y0.r, y1.r) - (4.0f / 27.0f) * fabsf(h) * (fabsf(k0.r) + fabsf(k1.r));
  if (rlow > q.r_max) return;
  const float sig_m = fmaf(rm, rm, a2 * um * um);
  const float ns = fminf(fmaxf(ceilf(__fdividef(sig_m * h, q.ds_max)), 1.0f), 64.0f);
  const int nsub = (int)ns;
  const float dt = __fdividef(h, ns);
  const float rp = (float)p.r_plus, rmn = (float)p.r_minus, ro = (float)p.r_obs;
  const float gscale = c.a == 0.0f ? 0.0f : __fdividef(c.a, rp - rmn);
  const float g_obs = __fdividef(ro - rmn, ro - rp);
  for (int m = 0; m < nsub; ++m) {
    const float t = __fdividef((float)m + 0.5f, ns);
    const float t2 = t * t, t3 = t2 * t;
    const float h00 = 2.0f * t3 - 3.0f * t2 + 1.0f, h10 = t3 - 2.0f * t2 + t;
    const float h01 = -2.0f * t3 + 3.0f * t2, h11 = t3 - t2;
    const float r = h00 * y0.r + h10 * h * k0.r + h01 * y1.r + h11 * h * k1.r;
    const float u = h00 * y0.u + h10 * h * k0.u + h01 * y1.u + h11 * h * k1.u;
    const float psi = h00 * y0.phi + h10 * h * k0.phi + h01 * y1.phi + h11 * h * k1.phi;
    const float phi = psi + gscale * __logf(__fdividef(r - rp, r - rmn) * g_obs);  // phi = psi + a (G(r) - G(r_obs))
    float n, th, b;
    if (!bhrt::sample_f(q, r, u, phi, n, th, b)) continue;
    const float g = bhrt::redshift_f(c.a, r, u, c.lam);
    float ln_alpha, ln_s;
    if (!bhrt::ln_emission_f(q, n, th, b, g, ln_alpha, ln_s)) continue;
    const float dl = fmaf(r, r, a2 * u * u) * dt;  // affine length of the sample, M
    const float ts = __expf(ln_alpha + __logf(dl) + q.ln_len);
    const float om = ts < 1.0e-4f ? ts * (1.0f - 0.5f * ts) : -expm1f(-ts);
    I += (double)(T * __expf(ln_s) * om);
    T *= 1.0f - om;
    tau += (double)ts;
  }
}

__global__ void __launch_bounds__(128) k_trace_rt_mixed(const __grid_constant__ BhkImageParams p,
                                                        const __grid_constant__ bhrt::MediumF q,
                                                        double *__restrict__ i_nu, double *__restrict__ tau_out,
                                                        int *__restrict__ cls_out, int *__restrict__ steps_out,
                                                        unsigned long long *__restrict__ counter) {
  const unsigned lane = threadIdx.x & 31u;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(counter, 32ull);
    base = __shfl_sync(kFull, base, 0);
    if (base >= (unsigned long long)p.n_pix) break;
    const long long pix = (long long)base + lane;
    if (pix >= p.n_pix) continue;
    RayMx R;
    init_ray(p, pix, R);
    double I = 0.0, tau = 0.0;
    float T = 1.0f;
    int cls = 3;
    const long long max_attempts = 4LL * p.max_steps + 64;
    for (;;) {
      if (R.steps >= p.max_steps || R.attempts >= max_attempts) {
        cls = 3;
        break;
      }
      if (R.y.r <= R.r_hor) {
        cls = 0;
        break;
      }
      if (R.y.r >= R.r_esc) {
        cls = 2;
        break;
      }
      ++R.attempts;
      const float h = R.h;
      const DPf d = dp45(R.y, h, R.c, R.k1, R.rtol, R.atol, true);
      if (d.err <= 1.0f) {
        ++R.steps;
        const Yf y0 = R.y, k0 = R.k1;
        comp_add(R.y.r, R.lo.r, d.d.r);
        comp_add(R.y.u, R.lo.u, d.d.u);
        comp_add(R.y.phi, R.lo.phi, d.d.phi);
        R.y.pr += d.d.pr;
        R.y.pu += d.d.pu;
        rt_segment_f(p, q, R.c, y0, k0, R.y, d.k7, h, I, T, tau);
        project(R.y, R.lo, R.cd);
        R.k1 = d.k7;
        R.k1.r = R.y.pr;
        R.k1.u = R.y.pu;
        R.h = h * step_factor(d.err, true);
        if (T < q.min_transmit) {
          cls = 4;
          break;
        }
      } else {
        R.h = h * step_factor(d.err, false);
      }
    }
    if (i_nu) i_nu[pix] = I;
    if (tau_out) tau_out[pix] = tau;
    if (cls_out) cls_out[pix] = cls;
    if (steps_out) steps_out[pix] = R.steps;
  }
}

}  // namespace bhm

extern "C" int bhk_trace_rt_mixed(const BhkImageParams *p, const BhkRtParams *q, double *i_nu, double *tau,
                                  int32_t *cls, int32_t *steps, unsigned long long *counter, void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s) != cudaSuccess) return -1;
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bhm::k_trace_rt_mixed, 128, 0) != cudaSuccess)
    return -1;
  const long long need = (p->n_pix + 127) / 128;
  const int grid = (int)(need < (long long)sms * per_sm ? need : (long long)sms * per_sm);
  const bhrt::MediumF m = bhrt::medium_f(*q);
  bhm::k_trace_rt_mixed<<<grid > 0 ? grid : 1, 128, 0, s>>>(*p, m, i_nu, tau, cls, steps, counter);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_image_mixed(const BhkImageParams *p, const BhkImageOut *o, unsigned long long *counter,
                                     BhkLaunch launch, void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s) != cudaSuccess) return -1;
  const bool drift = o->carter_drift != nullptr;
  auto k = p->integrator == 0 ? (drift ? bhm::k_trace_image_mixed<0, true> : bhm::k_trace_image_mixed<0, false>)
                              : (drift ? bhm::k_trace_image_mixed<1, true> : bhm::k_trace_image_mixed<1, false>);
  k<<<launch.grid, launch.block, 0, s>>>(*p, *o, counter, launch.refill);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_image_mixed_occupancy(int integrator, int block, int *blocks_per_sm) {
  const cudaError_t e =
      (integrator == 0)
          ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhm::k_trace_image_mixed<0, false>, block, 0)
          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhm::k_trace_image_mixed<1, false>, block, 0);
  return e == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_list_mixed(const BhkImageParams *p, const BhkImageOut *o, const int *list,
                                    const unsigned int *count, unsigned long long *counter, BhkLaunch L,
                                    void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s) != cudaSuccess) return -1;
  const bool drift = o->carter_drift != nullptr;
  auto k = p->integrator == 0 ? (drift ? bhm::k_trace_list_mixed<0, true> : bhm::k_trace_list_mixed<0, false>)
                              : (drift ? bhm::k_trace_list_mixed<1, true> : bhm::k_trace_list_mixed<1, false>);
  k<<<L.grid, L.block, 0, s>>>(*p, *o, list, count, counter, L.refill);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_camera_mixed(const BhkImageParams *p, const BhkCamera *cam, const BhkImageOut *o,
                                      unsigned long long *counter, BhkLaunch L, void *stream, const BhkVolume *vol) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s) != cudaSuccess) return -1;
  if (vol && (vol->mode == 1 || vol->mode == 2))
    bhm::k_trace_camera_vol_mixed<<<L.grid, L.block, 0, s>>>(*p, *cam, *vol, *o, counter, L.refill);
  else
    bhm::k_trace_camera_mixed<<<L.grid, L.block, 0, s>>>(*p, *cam, *o, counter, L.refill);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_camera_mixed_occupancy(int block, int *blocks_per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhm::k_trace_camera_mixed, block, 0) ==
                 cudaSuccess
             ? 0
             : -1;
}

extern "C" int bhk_trace_batch_mixed(const BhkBatchDev *b, int integrator, unsigned long long *counter, BhkLaunch L,
                                     void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s) != cudaSuccess) return -1;
  auto k = integrator == 0 ? (b->drift ? bhm::k_trace_batch_mixed<0, true> : bhm::k_trace_batch_mixed<0, false>)
                           : (b->drift ? bhm::k_trace_batch_mixed<1, true> : bhm::k_trace_batch_mixed<1, false>);
  k<<<L.grid, L.block, 0, s>>>(*b, counter, L.refill);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_batch_mixed_occupancy(int integrator, int block, int *blocks_per_sm) {
  const cudaError_t e =
      (integrator == 0)
          ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhm::k_trace_batch_mixed<0, false>, block, 0)
          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhm::k_trace_batch_mixed<1, false>, block, 0);
  return e == cudaSuccess ? 0 : -1;
}
