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
  if (cls == 2) {
    const double u = to_f64(R.y.u, R.lo.u);
    th = acos(fmin(1.0, fmax(-1.0, u)));
    ph = phi_of_psi(to_f64(R.y.phi, R.lo.phi), to_f64(R.y.r, R.lo.r), p);
    if (p.sky) {  // dphi/dtau = dpsi/dtau + a p_r / Delta  (phi = psi + a G(r), G' = 1 / Delta)
      const Yf k = rhs(R.y, R.c);
      const double r = to_f64(R.y.r, R.lo.r);
      const double delta = r * r - 2.0 * r + p.a2;
      const double dphi = (double)k.phi + p.a * (double)R.y.pr / delta;
      inten += bhsky::radiance(p.sky, p.sky_size, r, u, ph, (double)R.y.pr, (double)R.y.pu, dphi);
    }
  }
  if (o.intensity) o.intensity[pix] = inten;
  if (o.theta_inf) o.theta_inf[pix] = th;
  if (o.phi_inf) o.phi_inf[pix] = ph;
}

// Applies the increment d of an accepted step (acc) to the ray: compensated
// positions, crossing test and record, projection; returns true if the ray
// stops. A rejected attempt (acc false) runs the same instructions with a
// zero increment -- adding 0 leaves a compensated pair unchanged and the
// projection is idempotent on a projected state -- so accepted and rejected
// lanes of a warp never diverge. k0 = rhs(y0); k1 = rhs(y1) when the caller
// has it (DP45's FSAL stage), else NULL and evaluated only at a crossing.
__device__ __forceinline__ bool accept(const BhkImageParams &p, const BhkImageOut &o, RayMx &R, const Yf &d,
                                       bool acc, float h, const Yf &k0, const Yf *k1) {
  const Yf y0 = R.y;
  const Lof lo0 = R.lo;
  comp_add(R.y.r, R.lo.r, acc ? d.r : 0.0f);
  comp_add(R.y.u, R.lo.u, acc ? d.u : 0.0f);
  comp_add(R.y.phi, R.lo.phi, acc ? d.phi : 0.0f);
  R.y.pr += acc ? d.pr : 0.0f;
  R.y.pu += acc ? d.pu : 0.0f;
  R.steps += acc ? 1 : 0;
  bool stop = false;
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
    stop = on_crossing(p, o, R, r_c, phi_c);
  }
  project(R.y, R.lo, R.cd);
  return stop;
}

template <int INTEG>
__device__ __forceinline__ int iterate(const BhkImageParams &p, const BhkImageOut &o, RayMx &R) {
  const float r_hor = R.r_hor, r_esc = R.r_esc;
  if (INTEG == 0) {
    if (R.steps >= p.max_steps) return 3;
    if (R.y.r <= r_hor) return 0;
    if (R.y.r >= r_esc) return 2;
    const float hh = (float)p.step_coeff * fminf(R.y.r, (float)p.step_rcap);
    const float h = __fdividef(hh, fmaf(R.c.a2 * R.y.u, R.y.u, R.y.r * R.y.r));
    const Yf k0 = rhs(R.y, R.c);
    const Yf d = rk4_inc(R.y, h, R.c, k0);
    return accept(p, o, R, d, true, h, k0, nullptr) ? 1 : -1;
  } else {
    const long long max_attempts = 4LL * p.max_steps + 64;
    if (R.steps >= p.max_steps || R.attempts >= max_attempts) return 3;
    if (R.y.r <= r_hor) return 0;
    if (R.y.r >= r_esc) return 2;
    ++R.attempts;
    const DPf d = dp45(R.y, R.h, R.c, R.k1, R.rtol, R.atol, true);
    const bool acc = d.err <= 1.0f;
    const float h = R.h;
    const bool stop = accept(p, o, R, d.d, acc, h, R.k1, &d.k7);
    R.k1 = acc ? d.k7 : R.k1;
    R.k1.r = R.y.pr;  // projection moved only the momenta
    R.k1.u = R.y.pu;
    R.h = h * step_factor(d.err, acc);
    return stop ? 1 : -1;
  }
}

// The persistent loop shared by the single-frame and batch kernels (see
// trace_image_fp64.cu).
template <int INTEG, class Src>
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
          init_ray(src.params(f), pix, R);
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
        const int cls = iterate<INTEG>(P, src.out(R.f), R);
        if (cls >= 0) {
          finish(P, src.out(R.f), R, cls);
          src.pixel_done(R.f);
          active = false;
        }
      }
    }
  }
}

template <int INTEG>
__global__ void __launch_bounds__(128) k_trace_image_mixed(const __grid_constant__ BhkImageParams p,
                                                           const __grid_constant__ BhkImageOut o,
                                                           unsigned long long *__restrict__ counter, int refill) {
  trace_loop<INTEG>(bhsrc::SingleSrc{p, o}, counter, refill);
}

template <int INTEG>
__global__ void __launch_bounds__(128) k_trace_list_mixed(const __grid_constant__ BhkImageParams p,
                                                          const __grid_constant__ BhkImageOut o,
                                                          const int *__restrict__ list,
                                                          const unsigned int *__restrict__ count,
                                                          unsigned long long *__restrict__ counter, int refill) {
  trace_loop<INTEG>(bhsrc::ListSrc{p, o, list, count}, counter, refill);
}

template <int INTEG>
__global__ void __launch_bounds__(128) k_trace_batch_mixed(const __grid_constant__ BhkBatchDev b,
                                                           unsigned long long *__restrict__ counter, int refill) {
  if (threadIdx.x == 0) atomicMin(b.start_ns, bhsrc::globaltimer_ns());
  trace_loop<INTEG>(bhsrc::BatchSrc{b}, counter, refill);
}

}  // namespace bhm

extern "C" int bhk_trace_image_mixed(const BhkImageParams *p, const BhkImageOut *o, unsigned long long *counter,
                                     BhkLaunch launch, void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s) != cudaSuccess) return -1;
  if (p->integrator == 0)
    bhm::k_trace_image_mixed<0><<<launch.grid, launch.block, 0, s>>>(*p, *o, counter, launch.refill);
  else
    bhm::k_trace_image_mixed<1><<<launch.grid, launch.block, 0, s>>>(*p, *o, counter, launch.refill);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_image_mixed_occupancy(int integrator, int block, int *blocks_per_sm) {
  const cudaError_t e =
      (integrator == 0)
          ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhm::k_trace_image_mixed<0>, block, 0)
          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhm::k_trace_image_mixed<1>, block, 0);
  return e == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_list_mixed(const BhkImageParams *p, const BhkImageOut *o, const int *list,
                                    const unsigned int *count, unsigned long long *counter, BhkLaunch L,
                                    void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s) != cudaSuccess) return -1;
  if (p->integrator == 0)
    bhm::k_trace_list_mixed<0><<<L.grid, L.block, 0, s>>>(*p, *o, list, count, counter, L.refill);
  else
    bhm::k_trace_list_mixed<1><<<L.grid, L.block, 0, s>>>(*p, *o, list, count, counter, L.refill);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_batch_mixed(const BhkBatchDev *b, int integrator, unsigned long long *counter, BhkLaunch L,
                                     void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s) != cudaSuccess) return -1;
  if (integrator == 0)
    bhm::k_trace_batch_mixed<0><<<L.grid, L.block, 0, s>>>(*b, counter, L.refill);
  else
    bhm::k_trace_batch_mixed<1><<<L.grid, L.block, 0, s>>>(*b, counter, L.refill);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_batch_mixed_occupancy(int integrator, int block, int *blocks_per_sm) {
  const cudaError_t e =
      (integrator == 0)
          ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhm::k_trace_batch_mixed<0>, block, 0)
          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhm::k_trace_batch_mixed<1>, block, 0);
  return e == cudaSuccess ? 0 : -1;
}
