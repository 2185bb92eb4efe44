// trace_image_fp64.cu - FP64 image-plane Kerr tracer (sm_100a).
//
// One ray per lane in a persistent grid: each warp keeps 32 rays in
// registers and, whenever rays terminate (horizon, disk, escape, step
// budget), refills exactly those lanes from a global work counter with one
// warp-aggregated atomicAdd (ballot + popc), so finished rays never idle a
// lane while work remains. The integration follows the reference trace loop
// order (src/physics/raytracer.h:338-365): step budget, horizon test, escape
// test, step; then the equatorial-crossing test, located inside the step by
// Hermite interpolation (hermite.cuh) on the bracket of the
// src/physics/event_detection.h:127-180 pattern.
//
// Built with -fmad=false: bit-identical to the FP64 CPU oracle.
#include <cuda_runtime.h>

#include <cstdio>

#include "frame_source.cuh"
#include "rt.cuh"
#include "sky.cuh"
#include "hermite.cuh"
#include "image_fp64.cuh"
#include "launch.h"

namespace bhk {

constexpr unsigned kFull = 0xffffffffu;

struct RayFp64 {
  RayC c;
  Yd y;
  Yd k1;        // DP45: FSAL stage of y
  double h;     // DP45: next trial step
  double inten;
  long long pix;
  int f;  // frame of the current ray (batch launches)
  int steps;
  int attempts;
  int ncross;
  double drift;  // largest Carter-constant residual the projection removed
};

__device__ __forceinline__ void init_ray(const BhkImageParams &p, long long pix, RayFp64 &R) {
  const long long i = pix % p.width, j = pix / p.width;
  const double alpha = p.alpha_min + ((double)i + 0.5) * p.dalpha;
  const double beta = p.beta_min + ((double)j + 0.5) * p.dbeta;
  R.c.a = p.a;
  R.c.a2 = p.a2;
  R.c.lam = -alpha * p.sin_o;
  const double eta = (beta * beta) + (((alpha * alpha) - (p.a * p.a)) * p.cos_o) * p.cos_o;
  R.c.qTh = eta + (R.c.lam * R.c.lam);
  const double qR = (p.form == 1) ? eta : R.c.qTh;
  R.c.K = qR + ((R.c.lam - R.c.a) * (R.c.lam - R.c.a));
  R.y.r = p.r_obs;
  R.y.u = p.cos_o;
  R.y.phi = 0.0;
  const double Rv = pot_R(R.y.r, R.c);
  R.y.pr = -sqrt((Rv < 0.0) ? 0.0 : Rv);
  R.y.pu = beta * p.sin_o;
  R.steps = 0;
  R.attempts = 0;
  R.ncross = 0;
  R.inten = 0.0;
  R.pix = pix;
  project(R.y, R.c);  // idempotent from here on (see iterate)
  R.drift = 0.0;
  if (p.integrator == 1) {
    const double hh = p.step_coeff * dmin_(R.y.r, p.step_rcap);
    const double sigma = (R.y.r * R.y.r) + ((p.a2 * R.y.u) * R.y.u);
    R.h = hh / sigma;
    R.k1 = rhs(R.y, R.c);
  }
}

// Crossing of u = 0 inside the accepted step y0 -> y1 (y1 before the
// projection) with k0 = rhs(y0), k1 = rhs(y1): Hermite interpolation.
__device__ __forceinline__ void step_crossing(const Yd &y0, const Yd &k0, const Yd &y1, const Yd &k1, double h,
                                              double &r_c, double &phi_c) {
  const bhh_dev::Ends e{y0.r, y0.u, y0.phi, y0.pr, y0.pu, k0.pr, k0.pu, k0.phi,
                        y1.r, y1.u, y1.phi, y1.pr, y1.pu, k1.pr, k1.pu, k1.phi};
  bhh_dev::hermite_crossing(e, h, r_c, phi_c);
}

// Records a crossing at (r_c, phi_c) when it lies on the disk; returns true
// when the ray stops there (last allowed crossing).
__device__ __forceinline__ bool on_crossing(const BhkImageParams &p, const BhkImageOut &o, RayFp64 &R,
                                            double r_c, double phi_c) {
  if (!(r_c >= p.r_in && r_c <= p.r_out)) return false;
  const int k = R.ncross;
  const long long off = (long long)k * p.n_pix + R.pix;
  const double g = disk_g(r_c, p.a, R.c.lam);
  if (o.r_hit) o.r_hit[off] = r_c;
  if (o.phi_hit) o.phi_hit[off] = phi_of_psi(phi_c, r_c, p);
  if (o.g) o.g[off] = g;
  const double q = p.r_in / r_c;
  const double g2 = g * g;
  R.inten = R.inten + ((((g2 * g2) * q) * q) * q);
  if (k == 0 && o.flux) o.flux[R.pix] = nt_flux(r_c, p.nt_isco, p.nt_flux_peak);
  R.ncross = k + 1;
  return R.ncross >= p.max_cross;
}

__device__ __forceinline__ void finish(const BhkImageParams &p, const BhkImageOut &o, const RayFp64 &R,
                                       int cls) {
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
    const double u = R.y.u;
    th = acos((u < -1.0) ? -1.0 : ((1.0 < u) ? 1.0 : u));
    ph = phi_of_psi(R.y.phi, R.y.r, p);
    if (p.sky) {  // dphi/dtau = dpsi/dtau + a p_r / Delta  (phi = psi + a G(r), G' = 1 / Delta)
      const Yd k = rhs(R.y, R.c);
      const double delta = ((R.y.r * R.y.r) - (2.0 * R.y.r)) + p.a2;
      const double dphi = k.phi + (p.a * R.y.pr) / delta;
      inten = inten + bhsky::radiance(p.sky, p.sky_size, R.y.r, u, ph, R.y.pr, R.y.pu, dphi);
    }
  }
  if (o.intensity) o.intensity[pix] = inten;
  if (o.theta_inf) o.theta_inf[pix] = th;
  if (o.phi_inf) o.phi_inf[pix] = ph;
  if (o.carter_drift) o.carter_drift[pix] = R.drift;
}

// One iteration of the trace loop for an active ray; returns the class when
// the ray terminates, -1 otherwise.
// DRIFT: keep the largest Carter-constant residual the projection removes (a
// separate instantiation, so the plain kernels carry none of it).
template <int INTEG, bool DRIFT = false>
__device__ __forceinline__ int iterate(const BhkImageParams &p, const BhkImageOut &o, RayFp64 &R) {
  if (INTEG == 0) {
    if (R.steps >= p.max_steps) return 3;
    if (R.y.r <= p.r_hor) return 0;
    if (R.y.r >= p.r_esc) return 2;
    const double hh = p.step_coeff * dmin_(R.y.r, p.step_rcap);
    const double sigma = (R.y.r * R.y.r) + ((p.a2 * R.y.u) * R.y.u);
    const double h = hh / sigma;
    const Yd k0 = rhs(R.y, R.c);
    Yd yn = rk4(R.y, h, R.c, k0);
    ++R.steps;
    if ((R.y.u * yn.u) < 0.0) {
      double r_c, phi_c;
      step_crossing(R.y, k0, yn, rhs(yn, R.c), h, r_c, phi_c);
      if (on_crossing(p, o, R, r_c, phi_c)) return 1;
    }
    if (DRIFT)
      R.drift = dmax_(R.drift, project(yn, R.c, true));
    else
      project(yn, R.c);
    R.y = yn;
    return -1;
  } else {
    const long long max_attempts = 4LL * p.max_steps + 64;
    if (R.steps >= p.max_steps || R.attempts >= max_attempts) return 3;
    if (R.y.r <= p.r_hor) return 0;
    if (R.y.r >= p.r_esc) return 2;
    ++R.attempts;
    const DPRes d = dp45(R.y, R.h, R.c, R.k1, p.rtol, p.atol, true);
    // Accepted and rejected lanes run the same instructions: a rejected lane
    // keeps its state and re-projects it, which is exact no-op because every
    // state is already on its first integrals (projected at set-up).
    const bool acc = d.err <= 1.0;
    bool stop = false;
    if (acc) {
      ++R.steps;
      if ((R.y.u * d.y5.u) < 0.0) {
        double r_c, phi_c;
        step_crossing(R.y, R.k1, d.y5, d.k7, R.h, r_c, phi_c);
        stop = on_crossing(p, o, R, r_c, phi_c);
      }
    }
    R.y = acc ? d.y5 : R.y;
    R.k1 = acc ? d.k7 : R.k1;
    const double drift = project(R.y, R.c, DRIFT);
    if (DRIFT && acc) R.drift = dmax_(R.drift, drift);
    R.k1.r = R.y.pr;  // projection moves only the momenta
    R.k1.u = R.y.pu;
    R.h = R.h * step_factor(d.err, acc);
    return stop ? 1 : -1;
  }
}

// The persistent loop shared by the single-frame and batch kernels. Every
// `refill` integration steps, the lanes whose ray finished take new work
// items with one warp-aggregated atomicAdd on the counter (ballot + popc).
template <int INTEG, bool DRIFT = false, class Src>
__device__ __forceinline__ void trace_loop(const Src &src, unsigned long long *__restrict__ counter, int refill) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  const unsigned long long total = (unsigned long long)src.total();
  RayFp64 R;
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
        const int cls = iterate<INTEG, DRIFT>(P, src.out(R.f), R);
        if (cls >= 0) {
          finish(P, src.out(R.f), R, cls);
          src.pixel_done(R.f);
          active = false;
        }
      }
    }
  }
}

template <int INTEG, bool DRIFT>
__global__ void __launch_bounds__(128, 4) k_trace_image_fp64(const __grid_constant__ BhkImageParams p,
                                                          const __grid_constant__ BhkImageOut o,
                                                          unsigned long long *__restrict__ counter, int refill) {
  trace_loop<INTEG, DRIFT>(bhsrc::SingleSrc{p, o}, counter, refill);
}

template <int INTEG, bool DRIFT>
__global__ void __launch_bounds__(128, 4) k_trace_list_fp64(const __grid_constant__ BhkImageParams p,
                                                         const __grid_constant__ BhkImageOut o,
                                                         const int *__restrict__ list,
                                                         const unsigned int *__restrict__ count,
                                                         unsigned long long *__restrict__ counter, int refill) {
  trace_loop<INTEG, DRIFT>(bhsrc::ListSrc{p, o, list, count}, counter, refill);
}

template <int INTEG, bool DRIFT>
__global__ void __launch_bounds__(128, 4) k_trace_batch_fp64(const __grid_constant__ BhkBatchDev b,
                                                          unsigned long long *__restrict__ counter, int refill) {
  if (threadIdx.x == 0) atomicMin(b.start_ns, bhsrc::globaltimer_ns());
  trace_loop<INTEG, DRIFT>(bhsrc::BatchSrc{b}, counter, refill);
}

// ---- along-ray radiative transfer -------------------------------------------

// Transfer over one accepted step y0 -> y1 (derivatives k0, k1 at its ends):
// samples at most ds_max apart in affine length, positions by cubic Hermite
// interpolation in Mino time.
__device__ __forceinline__ void rt_segment(const BhkImageParams &p, const BhkRtParams &q, const RayC &c,
                                           const Yd &y0, const Yd &k0, const Yd &y1, const Yd &k1, double h,
                                           double &I, double &T, double &tau) {
  const double rm = 0.5 * (y0.r + y1.r) + 0.125 * h * (k0.r - k1.r);
  const double um = 0.5 * (y0.u + y1.u) + 0.125 * h * (k0.u - k1.u);
  const double sig_m = rm * rm + p.a2 * um * um;
  // a step that stays beyond r_max samples nothing: on t in [0, 1] the cubic
  // Hermite r(t) >= min(r0, r1) - (4/27) |h| (|r0'| + |r1'|)
  const double rlow = (y0.r < y1.r ? y0.r : y1.r) - (4.0 / 27.0) * fabs(h) * (fabs(k0.r) + fabs(k1.r));
  if (rlow > q.r_max) return;
  double ns = ceil((sig_m * h) / q.ds_max);
  ns = ns < 1.0 ? 1.0 : (ns > 64.0 ? 64.0 : ns);
  const int nsub = (int)ns;
  const double dt = h / ns;
  for (int m = 0; m < nsub; ++m) {
    const double t = ((double)m + 0.5) / ns;
    const double t2 = t * t, t3 = t2 * t;
    const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + t;
    const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
    const double r = h00 * y0.r + h10 * h * k0.r + h01 * y1.r + h11 * h * k1.r;
    const double u = h00 * y0.u + h10 * h * k0.u + h01 * y1.u + h11 * h * k1.u;
    const double psi = h00 * y0.phi + h10 * h * k0.phi + h01 * y1.phi + h11 * h * k1.phi;
    const double dl = (r * r + p.a2 * u * u) * dt;  // affine length of the sample, M
    double n, th, b;
    if (!bhrt::sample(q, r, u, phi_of_psi(psi, r, p), n, th, b)) continue;
    const double g = bhrt::redshift(p.a, r, u, c.lam);
    if (!(g > 0.0)) continue;
    double j, al;
    bhrt::synchrotron(q, n, th, b, q.nu / g, j, al);
    const double jo = g * g * j, ao = al / g;
    const double ds = dl * q.length_cm;
    const double ts = ao * ds;
    const double om = (ts < 1.0e-4) ? ts * (1.0 - 0.5 * ts) : -expm1(-ts);
    I = (ao > 0.0) ? I + T * ((jo / ao) * om) : I + T * (jo * ds);
    T = T * (1.0 - om);
    tau = tau + ts;
  }
}

__global__ void __launch_bounds__(128) k_trace_rt_fp64(const __grid_constant__ BhkImageParams p,
                                                       const __grid_constant__ BhkRtParams q,
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
    RayFp64 R;
    init_ray(p, pix, R);
    double I = 0.0, T = 1.0, tau = 0.0;
    int cls = 3;
    const long long max_attempts = 4LL * p.max_steps + 64;
    for (;;) {
      if (R.steps >= p.max_steps || R.attempts >= max_attempts) {
        cls = 3;
        break;
      }
      if (R.y.r <= p.r_hor) {
        cls = 0;
        break;
      }
      if (R.y.r >= p.r_esc) {
        cls = 2;
        break;
      }
      ++R.attempts;
      const DPRes d = dp45(R.y, R.h, R.c, R.k1, p.rtol, p.atol, true);
      if (d.err <= 1.0) {
        ++R.steps;
        rt_segment(p, q, R.c, R.y, R.k1, d.y5, d.k7, R.h, I, T, tau);
        R.y = d.y5;
        R.k1 = d.k7;
        project(R.y, R.c);
        R.k1.r = R.y.pr;
        R.k1.u = R.y.pu;
        R.h = R.h * step_factor(d.err, true);
        if (T < q.min_transmit) {
          cls = 4;
          break;
        }
      } else {
        R.h = R.h * step_factor(d.err, false);
      }
    }
    if (i_nu) i_nu[pix] = I;
    if (tau_out) tau_out[pix] = tau;
    if (cls_out) cls_out[pix] = cls;
    if (steps_out) steps_out[pix] = R.steps;
  }
}

}  // namespace bhk

namespace {
thread_local char g_err[256] = {0};
int set_err(cudaError_t e, const char *what) {
  snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
  return -1;
}
}  // namespace

extern "C" const char *bhk_last_error(void) { return g_err; }

extern "C" int bhk_trace_image_fp64(const BhkImageParams *p, const BhkImageOut *o, unsigned long long *counter,
                                    BhkLaunch launch, void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return set_err(e, "work-counter reset");
  const bool drift = o->carter_drift != nullptr;
  auto k = p->integrator == 0 ? (drift ? bhk::k_trace_image_fp64<0, true> : bhk::k_trace_image_fp64<0, false>)
                              : (drift ? bhk::k_trace_image_fp64<1, true> : bhk::k_trace_image_fp64<1, false>);
  k<<<launch.grid, launch.block, 0, s>>>(*p, *o, counter, launch.refill);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(e, "k_trace_image_fp64 launch");
  return 0;
}

extern "C" int bhk_trace_list_fp64(const BhkImageParams *p, const BhkImageOut *o, const int *list,
                                   const unsigned int *count, unsigned long long *counter, BhkLaunch L,
                                   void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return set_err(e, "work-counter reset");
  const bool drift = o->carter_drift != nullptr;
  auto k = p->integrator == 0 ? (drift ? bhk::k_trace_list_fp64<0, true> : bhk::k_trace_list_fp64<0, false>)
                              : (drift ? bhk::k_trace_list_fp64<1, true> : bhk::k_trace_list_fp64<1, false>);
  k<<<L.grid, L.block, 0, s>>>(*p, *o, list, count, counter, L.refill);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(e, "k_trace_list_fp64 launch");
  return 0;
}

extern "C" int bhk_trace_image_fp64_occupancy(int integrator, int block, int *blocks_per_sm) {
  cudaError_t e = (integrator == 0)
                      ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhk::k_trace_image_fp64<0, false>,
                                                                      block, 0)
                      : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhk::k_trace_image_fp64<1, false>,
                                                                      block, 0);
  if (e != cudaSuccess) return set_err(e, "occupancy query");
  return 0;
}

extern "C" int bhk_trace_batch_fp64(const BhkBatchDev *b, int integrator, unsigned long long *counter, BhkLaunch L,
                                    void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return set_err(e, "work-counter reset");
  auto k = integrator == 0 ? (b->drift ? bhk::k_trace_batch_fp64<0, true> : bhk::k_trace_batch_fp64<0, false>)
                           : (b->drift ? bhk::k_trace_batch_fp64<1, true> : bhk::k_trace_batch_fp64<1, false>);
  k<<<L.grid, L.block, 0, s>>>(*b, counter, L.refill);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(e, "k_trace_batch_fp64 launch");
  return 0;
}

extern "C" int bhk_trace_batch_fp64_occupancy(int integrator, int block, int *blocks_per_sm) {
  cudaError_t e = (integrator == 0)
                      ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhk::k_trace_batch_fp64<0, false>,
                                                                      block, 0)
                      : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, bhk::k_trace_batch_fp64<1, false>,
                                                                      block, 0);
  if (e != cudaSuccess) return set_err(e, "occupancy query");
  return 0;
}

extern "C" int bhk_trace_rt_fp64(const BhkImageParams *p, const BhkRtParams *q, double *i_nu, double *tau,
                                 int32_t *cls, int32_t *steps, unsigned long long *counter, int grid, int block,
                                 void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return set_err(e, "work-counter reset");
  bhk::k_trace_rt_fp64<<<grid, block, 0, s>>>(*p, *q, i_nu, tau, cls, steps, counter);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(e, "k_trace_rt_fp64 launch");
  return 0;
}

namespace bhk {

// Paths of image-plane rays (the Blender bridge's geodesic export): one
// thread per ray, classical RK4 with the image tracer's affine step rule,
// the position written before the first step and after every step until the
// ray reaches the horizon or escape radius or max_points are written.
__global__ void __launch_bounds__(128) k_trace_paths_fp64(const __grid_constant__ BhkImageParams p,
                                                          float *__restrict__ xyz, int32_t *__restrict__ counts,
                                                          int max_points) {
  const long long pix = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= p.n_pix) return;
  RayFp64 R;
  init_ray(p, pix, R);
  float *out = xyz + pix * (long long)max_points * 3;
  int n = 0;
  for (;;) {
    const double s = sqrt(dmax_(0.0, (1.0 - R.y.u) * (1.0 + R.y.u)));
    const double ph = phi_of_psi(R.y.phi, R.y.r, p);
    out[3 * n + 0] = (float)(R.y.r * s * cos(ph));
    out[3 * n + 1] = (float)(R.y.r * s * sin(ph));
    out[3 * n + 2] = (float)(R.y.r * R.y.u);
    ++n;
    if (n >= max_points || R.y.r <= p.r_hor || R.y.r >= p.r_esc) break;
    const double hh = p.step_coeff * dmin_(R.y.r, p.step_rcap);
    const double h = hh / ((R.y.r * R.y.r) + ((p.a2 * R.y.u) * R.y.u));
    R.y = rk4(R.y, h, R.c, rhs(R.y, R.c));
    project(R.y, R.c);
  }
  counts[pix] = n;
}

}  // namespace bhk

extern "C" int bhk_trace_paths_fp64(const BhkImageParams *p, float *xyz, int32_t *counts, int max_points,
                                    void *stream) {
  if (p->n_pix <= 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long blocks = (p->n_pix + 127) / 128;
  bhk::k_trace_paths_fp64<<<(unsigned)blocks, 128, 0, s>>>(*p, xyz, counts, max_points);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(e, "k_trace_paths_fp64 launch");
  return 0;
}
