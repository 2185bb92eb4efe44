// ref_stepper.cu - the reference's src/physics Kerr API batched on the GPU.
//
//   k_kerr_potentials  <- physics::kerrPotentials       (src/physics/kerr.cpp:69-97)
//   k_kerr_step_mino   <- physics::kerrStepMino         (src/physics/kerr.cpp:99-134)
//   k_kerr_trace_rays  <- physics::KerrRaytracer::trace (src/physics/raytracer.h:324-378)
//
// First-order Mino-time form with sign flips, CGS units, exactly the
// reference's expression order; compiled with -fmad=false so every FP64
// operation rounds once as on the CPU. The only device/host difference left
// is CUDA's sin/cos against glibc's (at most an ulp or two). One thread per
// state; inputs and outputs are structure-of-arrays.
#include <cuda_runtime.h>

#include "launch.h"

namespace {

constexpr double kC = 2.99792458e10;
constexpr double kC2 = kC * kC;
constexpr double kG = 6.67430e-8;
constexpr double kPI = 3.141592653589793;

struct Pot {
  double rPot, dRdr, thetaPot, dThetadtheta;
};
struct St {
  double r, theta, phi, t, signR, signTheta;
};
struct Cs {
  double e, lz, q;
};
struct Dv {
  double dr, dtheta, dphi, dt;
};

__device__ __forceinline__ double mx(double a, double b) { return (a < b) ? b : a; }

__device__ __forceinline__ Pot potentials(double r, double theta, double mass, double a, const Cs &c) {
  const double mGeom = kG * mass / kC2;
  const double rr = r * r;
  const double aa = a * a;
  double sinTheta, cosTheta;
  sincos(theta, &sinTheta, &cosTheta);
  const double sin2 = mx(sinTheta * sinTheta, 1e-12);
  const double cos2 = cosTheta * cosTheta;
  const double delta = rr - (2.0 * mGeom * r) + aa;
  const double aFactor = ((rr + aa) * c.e) - (a * c.lz);
  const double lzMinusAe = c.lz - (a * c.e);
  Pot p;
  p.rPot = (aFactor * aFactor) - (delta * (c.q + (lzMinusAe * lzMinusAe)));
  const double dAdR = 2.0 * r * c.e;
  const double dDeltaDr = (2.0 * r) - (2.0 * mGeom);
  p.dRdr = (2.0 * aFactor * dAdR) - (dDeltaDr * (c.q + (lzMinusAe * lzMinusAe)));
  p.thetaPot = c.q + (aa * c.e * c.e * cos2) - (c.lz * c.lz / sin2);
  p.dThetadtheta = -(2.0 * aa * c.e * c.e * cosTheta * sinTheta) + (2.0 * c.lz * c.lz * cosTheta / (sin2 * sinTheta));
  return p;
}

// kerrMinoDerivatives (kerr.cpp:40-66). The reference recomputes the full
// potentials (including the unused derivatives) and sin(theta) twice; the
// values that feed the result are identical here.
__device__ __forceinline__ Dv mino_derivs(const St &s, double mass, double a, const Cs &c) {
  const double mGeom = kG * mass / kC2;
  const double r = s.r;
  const double rr = r * r;
  const double aa = a * a;
  double sinTheta, cosTheta;
  sincos(s.theta, &sinTheta, &cosTheta);
  const double sin2 = mx(sinTheta * sinTheta, 1e-12);
  const double cos2 = cosTheta * cosTheta;
  const double delta = rr - (2.0 * mGeom * r) + aa;
  const double aFactor = ((rr + aa) * c.e) - (a * c.lz);
  const double lzMinusAe = c.lz - (a * c.e);
  const double rPotRaw = (aFactor * aFactor) - (delta * (c.q + (lzMinusAe * lzMinusAe)));
  const double thetaPotRaw = c.q + (aa * c.e * c.e * cos2) - (c.lz * c.lz / sin2);
  const double rPot = mx(rPotRaw, 0.0);
  const double thetaPot = mx(thetaPotRaw, 0.0);
  const double deltaSafe = mx(delta, 1e-12);
  Dv d;
  d.dr = s.signR * sqrt(rPot);
  d.dtheta = s.signTheta * sqrt(thetaPot);
  d.dphi = (c.lz / sin2) - (a * c.e) + (a * aFactor / deltaSafe);
  d.dt = (((rr + aa) * aFactor) / deltaSafe) + (a * (c.lz - (a * c.e * sin2)));
  return d;
}

__device__ __forceinline__ St step_mino(const St &state, double mass, double a, const Cs &c, double dlam) {
  St next = state;
  const Dv k1 = mino_derivs(state, mass, a, c);
  St s2 = state;
  s2.r += 0.5 * dlam * k1.dr;
  s2.theta += 0.5 * dlam * k1.dtheta;
  s2.phi += 0.5 * dlam * k1.dphi;
  s2.t += 0.5 * dlam * k1.dt;
  const Dv k2 = mino_derivs(s2, mass, a, c);
  St s3 = state;
  s3.r += 0.5 * dlam * k2.dr;
  s3.theta += 0.5 * dlam * k2.dtheta;
  s3.phi += 0.5 * dlam * k2.dphi;
  s3.t += 0.5 * dlam * k2.dt;
  const Dv k3 = mino_derivs(s3, mass, a, c);
  St s4 = state;
  s4.r += dlam * k3.dr;
  s4.theta += dlam * k3.dtheta;
  s4.phi += dlam * k3.dphi;
  s4.t += dlam * k3.dt;
  const Dv k4 = mino_derivs(s4, mass, a, c);
  next.r += dlam * (k1.dr + (2.0 * k2.dr) + (2.0 * k3.dr) + k4.dr) / 6.0;
  next.theta += dlam * (k1.dtheta + (2.0 * k2.dtheta) + (2.0 * k3.dtheta) + k4.dtheta) / 6.0;
  next.phi += dlam * (k1.dphi + (2.0 * k2.dphi) + (2.0 * k3.dphi) + k4.dphi) / 6.0;
  next.t += dlam * (k1.dt + (2.0 * k2.dt) + (2.0 * k3.dt) + k4.dt) / 6.0;
  const double lo = 1e-6, hi = kPI - 1e-6;
  next.theta = (next.theta < lo) ? lo : ((hi < next.theta) ? hi : next.theta);
  return next;
}

__global__ void k_kerr_potentials(int64_t n, const double *__restrict__ r, const double *__restrict__ th,
                                  double mass, double a, BhkConstsSoA c, double *rp, double *drp, double *tp,
                                  double *dtp) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const Cs cs{c.e[i], c.lz[i], c.q[i]};
    const Pot p = potentials(r[i], th[i], mass, a, cs);
    if (rp) rp[i] = p.rPot;
    if (drp) drp[i] = p.dRdr;
    if (tp) tp[i] = p.thetaPot;
    if (dtp) dtp[i] = p.dThetadtheta;
  }
}

__global__ void k_kerr_step_mino(int64_t n, BhkStateSoA s, double mass, double a, BhkConstsSoA c,
                                 const double *__restrict__ dlam, double dlam_scalar) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const St st{s.r[i], s.theta[i], s.phi[i], s.t[i], s.sr[i], s.sth[i]};
    const Cs cs{c.e[i], c.lz[i], c.q[i]};
    const St nx = step_mino(st, mass, a, cs, dlam ? dlam[i] : dlam_scalar);
    s.r[i] = nx.r;
    s.theta[i] = nx.theta;
    s.phi[i] = nx.phi;
    s.t[i] = nx.t;
    s.sr[i] = nx.signR;
    s.sth[i] = nx.signTheta;
  }
}

// kerrRedshift (src/physics/kerr.h:361-378) for geometric mass m.
__device__ __forceinline__ double redshift_z(double r, double theta, double m, double a) {
  const double rS = 2.0 * m;
  const double cosTheta = cos(theta);
  const double sigma = (r * r) + (a * a * cosTheta * cosTheta);
  const double factor = 1.0 - ((rS * r) / sigma);
  if (factor <= 0.0) return __longlong_as_double(0x7ff0000000000000LL);
  return (1.0 / sqrt(factor)) - 1.0;
}

__global__ void k_kerr_trace_rays(int64_t n, BhkStateSoA init, BhkConstsSoA c, double mass, double a,
                                  double rH, double rEsc, double step, int32_t maxSteps, int32_t *status,
                                  int32_t *steps, double *dist, double *rf, double *thf, double *phf,
                                  double *red) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    St state{init.r[i], init.theta[i], init.phi[i], init.t[i], init.sr[i], init.sth[i]};
    const Cs cs{c.e[i], c.lz[i], c.q[i]};
    int32_t st = 0, taken = 0;
    double total = 0.0;
    for (int32_t k = 0; k < maxSteps; ++k) {
      if (state.r <= (rH * 1.001)) { st = 2; break; }
      if (state.r >= rEsc) { st = 1; break; }
      const Pot p = potentials(state.r, state.theta, mass, a, cs);
      St next = state;
      if (p.rPot < 0.0) next.signR = -next.signR;
      if (p.thetaPot < 0.0) next.signTheta = -next.signTheta;
      state = step_mino(next, mass, a, cs, step);
      total += step;
      ++taken;
    }
    if (st == 0) st = (taken >= maxSteps) ? 4 : 1;
    double rs = 1.0;
    if (state.r > (rH * 1.001)) rs = 1.0 + redshift_z(state.r, state.theta, kG * mass / kC2, a);
    if (status) status[i] = st;
    if (steps) steps[i] = taken;
    if (dist) dist[i] = total;
    if (rf) rf[i] = state.r;
    if (thf) thf[i] = state.theta;
    if (phf) phf[i] = state.phi;
    if (red) red[i] = rs;
  }
}

int grid_for(int64_t n, int block) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (n + block - 1) / block;
  const int64_t cap = (int64_t)sms * 16;
  return (int)((want < cap) ? (want > 0 ? want : 1) : cap);
}

}  // namespace

extern "C" int bhk_kerr_potentials(int64_t n, const double *r, const double *theta, double mass, double a,
                                   BhkConstsSoA c, double *rp, double *drp, double *tp, double *dtp,
                                   void *stream) {
  if (n <= 0) return 0;
  k_kerr_potentials<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, r, theta, mass, a, c, rp, drp, tp, dtp);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_kerr_step_mino(int64_t n, BhkStateSoA s, double mass, double a, BhkConstsSoA c,
                                  const double *dlam, double dlam_scalar, void *stream) {
  if (n <= 0) return 0;
  k_kerr_step_mino<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, s, mass, a, c, dlam, dlam_scalar);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_kerr_trace_rays(int64_t n, BhkStateSoA init, BhkConstsSoA c, double mass, double a,
                                   double r_horizon, double r_escape, double step, int32_t max_steps,
                                   int32_t *status, int32_t *steps, double *dist, double *rf, double *thf,
                                   double *phf, double *redshift, void *stream) {
  if (n <= 0) return 0;
  k_kerr_trace_rays<<<grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(
      n, init, c, mass, a, r_horizon, r_escape, step, max_steps, status, steps, dist, rf, thf, phf, redshift);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
