// surrogate_render.cu - per-pixel decision of the surrogate renderer.
//
// Input: the network's head outputs for every pixel of a frame. Each pixel
// either takes the network's answer -- refined exactly where the answer is a
// disk hit -- or joins the list of pixels the integrator retraces:
//   1. class confidence below the threshold          -> integrator
//   2. within the stated image-plane distance of the
//      critical curve (first-order, from the minimum
//      of the radial potential)                       -> integrator
//   3. radial potential of a form not handled, or the
//      exact solve does not converge                  -> integrator
//   4. the exact solve disagrees with the network's
//      class (verify 1, 2; with verify 3 the solved
//      class stands)                                  -> integrator
// Accepted disk pixels get r_hit from the Mino-time solve seeded with the
// network's radius (FP32 quadrature and elliptic integrals by default, all
// FP64 on request), and g, flux and intensity from r_hit exactly as the
// tracer computes them; escaped pixels get theta_inf from the exact polar
// motion at the escape radius. When the caller asks for azimuths, phi_hit
// and phi_inf are solved too: the radial part on the Mino-time quadrature's
// own nodes, the polar part in closed form (R_J, cel), so no output of an
// accepted pixel is the network's. Escaped rays whose polar motion stays on
// one side of the equator go to the integrator.
#include <cuda_runtime.h>

#include <algorithm>

#include "image_fp64.cuh"
#include "launch.h"
#include "mino_solve.cuh"

namespace {

constexpr unsigned kFull = 0xffffffffu;
// Gauss-Legendre-16 panel width of the Mino-time quadrature: 0.125 for the
// FP64 solve (r to ~1e-8); the FP32 fast path, limited to ~4e-6 in r by its
// integrand, gets the same accuracy from panels twice as wide.
template <bool FAST>
constexpr double kPanel = FAST ? 0.25 : 0.125;

__device__ __forceinline__ void warp_count(unsigned *stats, int slot, bool pred) {
  const unsigned m = __ballot_sync(kFull, pred);
  if ((threadIdx.x & 31u) == 0 && m) atomicAdd(stats + slot, (unsigned)__popc(m));
}

// Resident 128-thread CTAs per SM the refinement is compiled for: 6 caps it
// at 80 registers, so that one CTA fits beside the inference kernel's
// persistent CTA (576 threads x 96 registers leave 10,240 of the SM's 65,536)
// and refines chunk k while the network infers chunk k + 1. The all-FP64
// solve (refine_fp64) would spill at 80 and keeps 2.
#ifndef BH_REFINE_MIN_CTAS
#define BH_REFINE_MIN_CTAS 6
#endif
#ifndef BH_REFINE_PHASED
#define BH_REFINE_PHASED 1
#endif

template <bool FAST, bool PHI>
__global__ void __launch_bounds__(128, FAST ? BH_REFINE_MIN_CTAS : 2) k_surrogate_refine(const __grid_constant__ BhkImageParams p,
                                                          const __grid_constant__ BhkImageOut o,
                                                          const float *__restrict__ head, float min_conf,
                                                          double band, int verify, int *__restrict__ list,
                                                          unsigned int *__restrict__ count,
                                                          unsigned int *__restrict__ stats, long long p0,
                                                          long long p1) {
  const long long pix = p0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = pix < p1;
  int reason = 0;  // 0 accepted, 1 confidence, 2 critical band, 3 solve, 4 disagreement
  if (live) {
    const long long i = pix % p.width, j = pix / p.width;
    const double alpha = p.alpha_min + ((double)i + 0.5) * p.dalpha;
    const double beta = p.beta_min + ((double)j + 0.5) * p.dbeta;
    const double a = p.a;
    const double lam = -alpha * p.sin_o;
    const double eta = beta * beta + (alpha * alpha - a * a) * p.cos_o * p.cos_o;
    const double qTh = eta + lam * lam;
    const double qR = (p.form == 1) ? eta : qTh;
    const double C = qR + (lam - a) * (lam - a);
    const double pu0 = beta * p.sin_o;

    const float *h = head + pix * 16;
    const float m = fmaxf(h[0], fmaxf(h[1], h[2]));
    const float e0 = __expf(h[0] - m), e1 = __expf(h[1] - m), e2 = __expf(h[2] - m);
    const float Z = e0 + e1 + e2;
    const int nn_cls = (e1 >= e0 && e1 >= e2) ? 1 : ((e2 >= e0) ? 2 : 0);
    const float conf = fmaxf(e0, fmaxf(e1, e2)) / Z;

    if (!(conf >= min_conf)) {
      reason = 1;
    } else {
      bhmino::Radial q = bhmino::radial_motion(p.a2, p.a2 - a * lam, C, p.r_obs, p.r_plus, p.r_hor, p.r_esc);
      if (PHI) bhmino::set_azimuth(q, a, lam);
      const double d = bhmino::critical_distance(q.r_min, q.R_min, a, lam, p.form == 1, p.sin_o, p.cos_o, alpha,
                                                 beta);
      if (q.kind < 0) {
        reason = 3;
      } else if (d < band) {
        reason = 2;
      } else {
        int cls = q.kind == 1 ? 2 : 0;  // radial kind: escapes or falls in
        const bool search = nn_cls == 1 || verify >= 2;
        bhmino::Polar th{};
        if (search || cls == 2)
          th = FAST ? bhmino::polar_motion<float>(p.a2, qTh, lam, p.cos_o, pu0, PHI)
                    : bhmino::polar_motion<double>(p.a2, qTh, lam, p.cos_o, pu0, PHI);
        int nhit = 0;
        bool solved = true;
        bhmino::Crossings c{};
        c.v_last = q.v_obs;
        c.t_last = 0.0;
        c.p_last = 0.0;
        if (search) {
          const double r_seed = (double)__expf(h[3] + 2.0f);
          c = bhmino::crossings<FAST, PHI>(q, th, p.r_in, p.r_out, r_seed, p.max_cross, kPanel<FAST>);
          solved = c.status == 0;
          nhit = c.n_hits;
          if (nhit >= p.max_cross) cls = 1;
        }
        const int opaque_cls = nhit > 0 ? 1 : cls;
        if (!solved) {
          reason = 3;
        } else if (verify <= 2 && opaque_cls != nn_cls) {
          reason = 4;  // verify 3: the solved class stands
        } else if (nhit > 0 && cls == 2) {
          reason = 4;  // passed the disk and escaped: left to the integrator
        } else if (cls == 2 && !th.crosses) {
          reason = 3;  // polar motion on one side of the equator (vortical): left to the integrator
        } else {
          double th_inf = 0.0, ph_inf = 0.0;
          if (cls == 2) {
            const bhmino::TauPhi te = bhmino::tau_end<FAST, PHI>(q, c.v_last, c.t_last, c.p_last, kPanel<FAST>);
            double phth = 0.0;
            const double u = FAST ? bhmino::polar_at<float>(th, lam, te.t, PHI, phth)
                                  : bhmino::polar_at<double>(th, lam, te.t, PHI, phth);
            th_inf = acos(fmin(1.0, fmax(-1.0, u)));
            if (PHI) ph_inf = -(te.ph + phth);
          }
          double inten = 0.0;
#pragma unroll
          for (int k = 0; k < 3; ++k) {  // max_cross <= 3; constant k keeps c's records in registers
            if (k >= p.max_cross) break;
            const long long off = (long long)k * p.n_pix + pix;
            double r = 0.0, g = 0.0, ph = 0.0;
            if (k < nhit) {
              r = c.r[k];
              g = bhk::disk_g(r, a, lam);
              const double qq = p.r_in / r;
              inten += g * g * g * g * qq * qq * qq;
              if (PHI) ph = -(c.phr[k] + bhmino::phi_theta_crossing(th, lam, c.tau[k]));
            }
            if (o.r_hit) o.r_hit[off] = r;
            if (o.g) o.g[off] = g;
            if (o.phi_hit) o.phi_hit[off] = ph;
          }
          if (o.cls) o.cls[pix] = cls;
          if (o.steps) o.steps[pix] = 0;
          if (o.n_cross) o.n_cross[pix] = nhit;
          if (o.flux) o.flux[pix] = nhit > 0 ? bhk::nt_flux(c.r[0], p.nt_isco, p.nt_flux_peak) : 0.0;
          if (o.intensity) o.intensity[pix] = inten;
          if (o.theta_inf) o.theta_inf[pix] = th_inf;
          if (o.phi_inf) o.phi_inf[pix] = ph_inf;
          if (o.carter_drift) o.carter_drift[pix] = 0.0;  // solved, not stepped
        }
      }
    }
  }
  // Append the pixels the integrator must retrace (one atomic per warp).
  const bool fb = live && reason != 0;
  const unsigned mask = __ballot_sync(kFull, fb);
  const unsigned lane = threadIdx.x & 31u;
  unsigned base = 0;
  if (lane == 0 && mask) base = atomicAdd(count, (unsigned)__popc(mask));
  base = __shfl_sync(kFull, base, 0);
  if (fb) list[base + __popc(mask & ((1u << lane) - 1u))] = (int)pix;
  for (int r = 0; r < 5; ++r) warp_count(stats, r, live && reason == r);
}

#if BH_REFINE_PHASED
// The same decision in phases with a CTA barrier after each (set-up and
// gate; polar motion and crossings; decisions and escape direction;
// outputs), in large CTAs, so that a CTA's warps run each phase's code
// together.
#ifndef BH_REFINE_THREADS
#define BH_REFINE_THREADS 256
#endif
template <bool FAST, bool PHI>
__global__ void __launch_bounds__(BH_REFINE_THREADS, 1)
    k_surrogate_refine_phased(const __grid_constant__ BhkImageParams p, const __grid_constant__ BhkImageOut o,
                              const float *__restrict__ head, float min_conf, double band, int verify,
                              int *__restrict__ list, unsigned int *__restrict__ count,
                              unsigned int *__restrict__ stats, long long p0, long long p1) {
  const long long pix = p0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = pix < p1;
  int reason = 0;  // 0 accepted, 1 confidence, 2 critical band, 3 solve, 4 disagreement
  const double a = p.a;
  double lam = 0.0, qTh = 0.0, pu0 = 0.0;
  int nn_cls = 0;
  float h3 = 0.0f;
  bool go = false;
  bhmino::Radial q{};
  if (live) {
    const long long i = pix % p.width, j = pix / p.width;
    const double alpha = p.alpha_min + ((double)i + 0.5) * p.dalpha;
    const double beta = p.beta_min + ((double)j + 0.5) * p.dbeta;
    lam = -alpha * p.sin_o;
    const double eta = beta * beta + (alpha * alpha - a * a) * p.cos_o * p.cos_o;
    qTh = eta + lam * lam;
    const double qR = (p.form == 1) ? eta : qTh;
    const double C = qR + (lam - a) * (lam - a);
    pu0 = beta * p.sin_o;
    const float *h = head + pix * 16;
    const float m = fmaxf(h[0], fmaxf(h[1], h[2]));
    const float e0 = __expf(h[0] - m), e1 = __expf(h[1] - m), e2 = __expf(h[2] - m);
    const float Z = e0 + e1 + e2;
    nn_cls = (e1 >= e0 && e1 >= e2) ? 1 : ((e2 >= e0) ? 2 : 0);
    const float conf = fmaxf(e0, fmaxf(e1, e2)) / Z;
    h3 = h[3];
    if (!(conf >= min_conf)) {
      reason = 1;
    } else {
      q = bhmino::radial_motion(p.a2, p.a2 - a * lam, C, p.r_obs, p.r_plus, p.r_hor, p.r_esc);
      if (PHI) bhmino::set_azimuth(q, a, lam);
      const double d = bhmino::critical_distance(q.r_min, q.R_min, a, lam, p.form == 1, p.sin_o, p.cos_o, alpha,
                                                 beta);
      if (q.kind < 0)
        reason = 3;
      else if (d < band)
        reason = 2;
      else
        go = true;
    }
  }
  __syncthreads();

  int cls = q.kind == 1 ? 2 : 0;  // radial kind: escapes or falls in
  const bool search = go && (nn_cls == 1 || verify >= 2);
  bhmino::Polar th{};
  if (go && (search || cls == 2))
    th = FAST ? bhmino::polar_motion<float>(p.a2, qTh, lam, p.cos_o, pu0, PHI)
              : bhmino::polar_motion<double>(p.a2, qTh, lam, p.cos_o, pu0, PHI);
  int nhit = 0;
  bool solved = true;
  bhmino::Crossings c{};
  c.v_last = q.v_obs;
  c.t_last = 0.0;
  c.p_last = 0.0;
  if (search) {
    const double r_seed = (double)__expf(h3 + 2.0f);
    c = bhmino::crossings<FAST, PHI>(q, th, p.r_in, p.r_out, r_seed, p.max_cross, kPanel<FAST>);
    solved = c.status == 0;
    nhit = c.n_hits;
    if (nhit >= p.max_cross) cls = 1;
  }
  __syncthreads();

  bool write = false;
  double th_inf = 0.0, ph_inf = 0.0;
  if (go) {
    const int opaque_cls = nhit > 0 ? 1 : cls;
    if (!solved)
      reason = 3;
    else if (verify <= 2 && opaque_cls != nn_cls)
      reason = 4;  // verify 3: the solved class stands
    else if (nhit > 0 && cls == 2)
      reason = 4;  // passed the disk and escaped: left to the integrator
    else if (cls == 2 && !th.crosses)
      reason = 3;  // polar motion on one side of the equator (vortical): left to the integrator
    else
      write = true;
    if (write && cls == 2) {
      const bhmino::TauPhi te = bhmino::tau_end<FAST, PHI>(q, c.v_last, c.t_last, c.p_last, kPanel<FAST>);
      double phth = 0.0;
      const double u = FAST ? bhmino::polar_at<float>(th, lam, te.t, PHI, phth)
                            : bhmino::polar_at<double>(th, lam, te.t, PHI, phth);
      th_inf = acos(fmin(1.0, fmax(-1.0, u)));
      if (PHI) ph_inf = -(te.ph + phth);
    }
  }
  __syncthreads();

  if (write) {
    double inten = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {  // max_cross <= 3; constant k keeps c's records in registers
      if (k >= p.max_cross) break;
      const long long off = (long long)k * p.n_pix + pix;
      double r = 0.0, g = 0.0, ph = 0.0;
      if (k < nhit) {
        r = c.r[k];
        g = bhk::disk_g(r, a, lam);
        const double qq = p.r_in / r;
        inten += g * g * g * g * qq * qq * qq;
        if (PHI) ph = -(c.phr[k] + bhmino::phi_theta_crossing(th, lam, c.tau[k]));
      }
      if (o.r_hit) o.r_hit[off] = r;
      if (o.g) o.g[off] = g;
      if (o.phi_hit) o.phi_hit[off] = ph;
    }
    if (o.cls) o.cls[pix] = cls;
    if (o.steps) o.steps[pix] = 0;
    if (o.n_cross) o.n_cross[pix] = nhit;
    if (o.flux) o.flux[pix] = nhit > 0 ? bhk::nt_flux(c.r[0], p.nt_isco, p.nt_flux_peak) : 0.0;
    if (o.intensity) o.intensity[pix] = inten;
    if (o.theta_inf) o.theta_inf[pix] = th_inf;
    if (o.phi_inf) o.phi_inf[pix] = ph_inf;
    if (o.carter_drift) o.carter_drift[pix] = 0.0;  // solved, not stepped
  }
  // Append the pixels the integrator must retrace (one atomic per warp).
  const bool fb = live && reason != 0;
  const unsigned mask = __ballot_sync(kFull, fb);
  const unsigned lane = threadIdx.x & 31u;
  unsigned base = 0;
  if (lane == 0 && mask) base = atomicAdd(count, (unsigned)__popc(mask));
  base = __shfl_sync(kFull, base, 0);
  if (fb) list[base + __popc(mask & ((1u << lane) - 1u))] = (int)pix;
  for (int r = 0; r < 5; ++r) warp_count(stats, r, live && reason == r);
}
#endif

// Copies the outputs of the first min(*count, cap) pixels of `list` into
// compact arrays: field f's entry w (plane c) goes to dst[f][c * cap + w].
__global__ void k_gather_pixels(BhkGather g, const int *__restrict__ list, const unsigned int *__restrict__ count,
                                long long n_pix, int cap) {
  const unsigned int total = *count, m = min(total, (unsigned int)cap);
  if (blockIdx.x == 0 && threadIdx.x == 0) *g.count_out = total;
  for (unsigned int w = blockIdx.x * blockDim.x + threadIdx.x; w < m; w += gridDim.x * blockDim.x) {
    const long long pix = list[w];
    g.list_out[w] = (int)pix;
    for (int f = 0; f < 10; ++f) {
      if (!g.src[f]) continue;
      for (int c = 0; c < g.planes[f]; ++c) {
        const long long from = (long long)c * n_pix + pix, to = (long long)c * cap + w;
        if (g.size[f] == 4)
          static_cast<int *>(g.dst[f])[to] = static_cast<const int *>(g.src[f])[from];
        else
          static_cast<double *>(g.dst[f])[to] = static_cast<const double *>(g.src[f])[from];
      }
    }
  }
  __threadfence_system();
}

}  // namespace

extern "C" int bhk_gather_pixels(const BhkGather *g, const int *list, const unsigned int *count, long long n_pix,
                                 int cap, void *stream) {
  if (cap <= 0) return 0;
  const unsigned blocks = (unsigned)std::min<long long>(1184, (cap + 255) / 256);
  k_gather_pixels<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(*g, list, count, n_pix, cap);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_surrogate_refine(const BhkImageParams *p, const BhkImageOut *o, const float *head, float min_conf,
                                    double band, int verify, int refine_fp64, long long p0, long long p1, int *list,
                                    unsigned int *count, unsigned int *stats, void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p1 = p1 < p->n_pix ? p1 : p->n_pix;
  if (p1 <= p0) return 0;
  const unsigned blocks = (unsigned)((p1 - p0 + 127) / 128);
  const bool phi = o->phi_hit != nullptr || o->phi_inf != nullptr;
#if BH_REFINE_PHASED
  // With azimuths the phased kernel is faster (2048^2 frame, serialised:
  // 1.01 against 1.13 ms per render); without them its body is short enough
  // that the unphased kernel wins (0.70 against 0.82 ms).
  if (!refine_fp64 && phi) {
    const unsigned pb = (unsigned)((p1 - p0 + BH_REFINE_THREADS - 1) / BH_REFINE_THREADS);
    k_surrogate_refine_phased<true, true><<<pb, BH_REFINE_THREADS, 0, s>>>(*p, *o, head, min_conf, band, verify,
                                                                         list, count, stats, p0, p1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }
#endif
  if (refine_fp64) {
    if (phi)
      k_surrogate_refine<false, true><<<blocks, 128, 0, s>>>(*p, *o, head, min_conf, band, verify, list, count,
                                                             stats, p0, p1);
    else
      k_surrogate_refine<false, false><<<blocks, 128, 0, s>>>(*p, *o, head, min_conf, band, verify, list, count,
                                                              stats, p0, p1);
  } else {
    if (phi)
      k_surrogate_refine<true, true><<<blocks, 128, 0, s>>>(*p, *o, head, min_conf, band, verify, list, count,
                                                            stats, p0, p1);
    else
      k_surrogate_refine<true, false><<<blocks, 128, 0, s>>>(*p, *o, head, min_conf, band, verify, list, count,
                                                             stats, p0, p1);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
