// trace_image_analytic.cu - the image tracer without stepping
// (BH_INTEGRATOR_ANALYTIC): every pixel's equatorial crossings, their radius,
// redshift and azimuth, and the escape direction, in closed form
// (kerr_analytic.cuh), FP64. O(1) work per crossing whatever the number of
// half-orbits, so the photon-ring band costs what the rest of the image does.
//
// Pixels whose ray the closed form does not cover -- a turning point between
// the horizon cut and r+, rays with q_R < 0 that reach the equator or do not
// fall in, four complex roots with equator crossings -- are appended to a
// list that the DP45 tracer finishes (launched by the host after this kernel).
// Outputs follow the tracer's conventions (trace_image_fp64.cu finish and
// on_crossing); steps = 0. Escaped rays report theta, phi and, with a sky,
// its radiance exactly at r_esc, where the tracer reports them after its
// last step's overshoot past r_esc.
#include <cuda_runtime.h>

// The routines that take a ray's solution structs are inlined, so that the
// structs live in registers rather than in each thread's stack frame (the
// kernel is compiled with 168 registers per thread: 384-thread CTAs).
#ifndef BHA_INLINE_SOLUTION
#define BHA_INLINE_SOLUTION 1
#endif

#include "image_fp64.cuh"
#include "kerr_analytic.cuh"
#include "launch.h"
#include "sky.cuh"

namespace {

struct Ray {
  double a, lam, qTh;
};

// The azimuth's constants of one ray: the two poles r+- of its radial part.
struct PhiCtx {
  bhan::JPole jp, jm;
  bool ready;
};

// The radial part of phi, a (r+ - r-)^-1 sum_(+-) +-(2 r+- - a lambda) int dtau / (r - r+-),
// at X with amplitude am (escape: at the escape radius of an S ray).
__device__ __forceinline__ double phi_radial(const BhkImageParams &p, const Ray &c, const bhan::RadSol &rs, PhiCtx &f,
                                             double X, const bhan::Amp &am, bool escape) {
  if (c.a == 0.0) return 0.0;
  if (!f.ready) {
    bhan::j_poles(rs, p.r_plus, p.r_minus, f.jp, f.jm);
    f.ready = true;
  }
  double jp, jm;
  if (escape)
    bhan::j_eval_escape(rs, f.jp, f.jm, jp, jm);
  else
    bhan::j_eval(rs, f.jp, f.jm, X, am, jp, jm);
  return c.a / (p.r_plus - p.r_minus) * ((2.0 * p.r_plus - c.a * c.lam) * jp - (2.0 * p.r_minus - c.a * c.lam) * jm);
}

// Traces one pixel in four phases with a CTA barrier after each: set-up,
// the crossing search, the azimuths of the hits, the escape. Every thread of
// the CTA calls it and reaches every barrier (live: the thread has a pixel).
// The kernel's code is longer than the instruction cache holds, and warps at
// different points of it kept evicting each other's instructions (47 % of
// fetches hit); aligned by the barriers, the CTA's warps run each phase's
// code at about the same time. Measured on the 2048^2 a = 0.9, 60 deg frame
// with all outputs: 9.56 ms unaligned in 128-thread CTAs, 6.85 ms with one
// barrier per pixel, 4.62 ms with that in 512-thread CTAs, 4.34 ms phased
// in 512-thread CTAs (outputs bit-identical). Returns false when the closed
// form does not cover the ray.
__device__ __forceinline__ bool trace_pixel(const BhkImageParams &p, const BhkImageOut &o, long long pix,
                                            bool live) {
  Ray c{};
  bhan::PolSol th{};
  bhan::RadSol rs{};
  rs.type = bhan::kUnhandled;
  double K = 0.0;
  if (live) {
    const long long i = pix % p.width, j = pix / p.width;
    const double alpha = p.alpha_min + ((double)i + 0.5) * p.dalpha;
    const double beta = p.beta_min + ((double)j + 0.5) * p.dbeta;
    c.a = p.a;
    c.lam = -alpha * p.sin_o;
    const double eta = beta * beta + (alpha * alpha - p.a2) * p.cos_o * p.cos_o;
    c.qTh = eta + c.lam * c.lam;
    const double qR = (p.form == 1) ? eta : c.qTh;
    K = qR + (c.lam - c.a) * (c.lam - c.a);
    const double a2l = p.a2 - c.a * c.lam;
    const double pu0 = beta * p.sin_o;
    th = bhan::polar(p.a2, c.qTh, c.lam, p.cos_o, pu0);
    rs = bhan::radial(2.0 * a2l - K, 2.0 * K, a2l * a2l - p.a2 * K, p.r_plus, p.r_hor, p.r_obs, p.r_esc,
                      th.crosses);
  }
  bool ok = live && rs.type != bhan::kUnhandled;
  const bool search = ok && rs.type != bhan::kCaptured;
  __syncthreads();

  int cls = 0, nhit = 0;
  double rh[3] = {0.0, 0.0, 0.0}, gh[3] = {0.0, 0.0, 0.0}, fh[3] = {0.0, 0.0, 0.0};
  double Th[3], Xh[3];
  bhan::Amp Ah[3];
  double inten = 0.0, th_inf = 0.0, ph_inf = 0.0;
  if (search) {
    bool done = false;
    for (int n = 0; n < 4096; ++n) {
      const double T = th.tau1 + n * th.period;
      if (!(T < rs.tau_end)) {
        done = true;
        break;
      }
      const double X = bhan::x_at(rs, T);
      const bhan::Amp am = bhan::amp_at(rs, X);
      const double r = bhan::r_of_amp(rs, am);
      if (r >= p.r_in && r <= p.r_out) {
        rh[nhit] = r;
        const double g = bhk::disk_g(r, c.a, c.lam);
        gh[nhit] = g;
        const double q = p.r_in / r, g2 = g * g;
        inten = inten + ((((g2 * g2) * q) * q) * q);
        Th[nhit] = T;
        Xh[nhit] = X;
        Ah[nhit] = am;
        if (++nhit >= p.max_cross) {
          done = true;
          break;
        }
      }
    }
    if (!done) ok = false;  // more crossings than the loop allows: leave it to the integrator
  }
  __syncthreads();

  PhiCtx f;
  f.ready = false;
  if (search && ok && o.phi_hit)
    for (int k = 0; k < nhit; ++k)
      fh[k] = -(phi_radial(p, c, rs, f, Xh[k], Ah[k], false) + bhan::phi_theta_crossing(th, c.lam, Th[k]));
  __syncthreads();

  if (search && ok) {
    cls = nhit >= p.max_cross ? 1 : (rs.type == bhan::kS ? 2 : 0);
    if (cls == 2) {
      const double T = rs.tau_end;
      double u, pu, phth;
      bhan::polar_at(th, c.lam, T, u, pu, phth);
      th_inf = acos(fmin(1.0, fmax(-1.0, u)));
      if (o.phi_inf || p.sky) ph_inf = -(phi_radial(p, c, rs, f, rs.X_end, rs.a_end, true) + phth);
      if (p.sky) {
        const double r = p.r_esc, r2 = r * r;
        const double A = (r2 + p.a2) - c.a * c.lam;
        const double D = (r2 - 2.0 * r) + p.a2;
        const double pr = sqrt(fmax(0.0, A * A - D * K));
        const double dphi = -(c.a * (2.0 * r - c.a * c.lam) / D + c.lam / fmax(1.0 - u * u, 1e-12));
        inten = inten + bhsky::radiance(p.sky, p.sky_size, r, u, ph_inf, pr, pu, dphi);
      }
    }
  }
  __syncthreads();
  if (!ok) return false;
  if (o.cls) o.cls[pix] = cls;
  if (o.steps) o.steps[pix] = 0;
  if (o.n_cross) o.n_cross[pix] = nhit;
  if (o.flux) o.flux[pix] = nhit > 0 ? bhk::nt_flux(rh[0], p.nt_isco, p.nt_flux_peak) : 0.0;
  for (int k = 0; k < p.max_cross; ++k) {
    const long long off = (long long)k * p.n_pix + pix;
    if (o.r_hit) o.r_hit[off] = rh[k];
    if (o.phi_hit) o.phi_hit[off] = fh[k];
    if (o.g) o.g[off] = gh[k];
  }
  if (o.intensity) o.intensity[pix] = inten;
  if (o.theta_inf) o.theta_inf[pix] = th_inf;
  if (o.phi_inf) o.phi_inf[pix] = ph_inf;
  if (o.carter_drift) o.carter_drift[pix] = 0.0;  // no stepping: nothing to project
  return true;
}

// Threads per CTA and resident CTAs per SM the closed form is compiled for:
// one CTA per SM, whose warps the phases of trace_pixel keep together. 384
// threads at 168 registers (the solution structs in registers, a ~690-byte
// frame) ran the 2048^2 a = 0.9, 60 deg frame in 4.06 ms with all outputs
// and 1.61 ms with the disk fields, against 4.33 and 1.69 ms for 512
// threads at 128 registers (1 KB frames that overflow L1); 320 threads
// (168 registers, more spills) and 256 threads (246 registers) were slower.
#ifndef BH_ANALYTIC_MIN_CTAS
#define BH_ANALYTIC_MIN_CTAS 1
#endif
#ifndef BH_ANALYTIC_THREADS
#define BH_ANALYTIC_THREADS 384
#endif

__global__ void __launch_bounds__(BH_ANALYTIC_THREADS, BH_ANALYTIC_MIN_CTAS) k_trace_image_analytic(const __grid_constant__ BhkImageParams p,
                                                              const __grid_constant__ BhkImageOut o,
                                                              int *__restrict__ list,
                                                              unsigned int *__restrict__ count) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  // every thread of the CTA takes the same trips through the phases' barriers
  for (long long base = (long long)blockIdx.x * blockDim.x; base < p.n_pix; base += stride) {
    const long long pix = base + threadIdx.x;
    const bool live = pix < p.n_pix;
    if (!trace_pixel(p, o, pix, live) && live) list[atomicAdd(count, 1u)] = (int)pix;
  }
}

// The same over a list of pixels (the surrogate renderer's rejected pixels);
// those it does not cover go on to list2.
__global__ void __launch_bounds__(BH_ANALYTIC_THREADS, BH_ANALYTIC_MIN_CTAS)
    k_trace_list_analytic(const __grid_constant__ BhkImageParams p, const __grid_constant__ BhkImageOut o,
                          const int *__restrict__ list, const unsigned int *__restrict__ count,
                          int *__restrict__ list2, unsigned int *__restrict__ count2) {
  const unsigned int total = *count;  // the same for every thread: uniform trips through the barriers
  // A short list (the renderer's ~1 % of a frame) is spread over every CTA
  // in whole warps of consecutive entries, not packed into the first few
  // CTAs: per CTA at most blockDim.x, at least a warp.
  const unsigned int per =
      min(blockDim.x, ((total + gridDim.x - 1) / gridDim.x + 31u) & ~31u);
  const unsigned int stride = gridDim.x * per;
  for (unsigned int base = blockIdx.x * per; base < total; base += stride) {
    const unsigned int w = base + threadIdx.x;
    const bool live = threadIdx.x < per && w < total;
    const int pix = live ? list[w] : 0;
    if (!trace_pixel(p, o, pix, live) && live) list2[atomicAdd(count2, 1u)] = pix;
  }
}

}  // namespace

extern "C" int bhk_trace_list_analytic(const BhkImageParams *p, const BhkImageOut *o, const int *list,
                                       const unsigned int *count, int *list2, unsigned int *count2, BhkLaunch L,
                                       void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(count2, 0, sizeof(unsigned int), s) != cudaSuccess) return -1;
  k_trace_list_analytic<<<L.grid, L.block, 0, s>>>(*p, *o, list, count, list2, count2);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_image_analytic(const BhkImageParams *p, const BhkImageOut *o, int *list,
                                        unsigned int *count, BhkLaunch L, void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(count, 0, sizeof(unsigned int), s) != cudaSuccess) return -1;
  k_trace_image_analytic<<<L.grid, L.block, 0, s>>>(*p, *o, list, count);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_trace_image_analytic_block(void) { return BH_ANALYTIC_THREADS; }

extern "C" int bhk_trace_image_analytic_occupancy(int block, int *blocks_per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_trace_image_analytic, block, 0) ==
                 cudaSuccess
             ? 0
             : -1;
}
