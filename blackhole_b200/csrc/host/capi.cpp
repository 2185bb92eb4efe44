// capi.cpp - C++23 host implementation of include/bh_kerr.h.
//
// Validates parameters, precomputes every per-scene constant on the host
// (so device code needs no libm transcendental), owns the small per-device
// scratch (the persistent kernels' work counter) and the grow-only device
// buffers of the _host entry points, sizes persistent grids from the
// occupancy calculator, and dispatches to the CUDA translation units through
// the internal C ABI in csrc/device/launch.h.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numbers>

#include "../../../include/bh_kerr.h"
#include "../device/launch.h"
#include "scene_math.hpp"
#include "dalloc.hpp"

namespace {

thread_local char g_last_error[512] = "";

int fail(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return -1;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

// ---- per-device scratch -----------------------------------------------------
constexpr int kMaxDevices = 64;
struct DeviceScratch {
  unsigned long long *counter = nullptr;  // persistent-kernel work counter (+ list count in word 1)
  int sms = 0;
  int *list = nullptr;  // pixels the analytic integrator leaves to DP45 (grow-only)
  int64_t list_cap = 0;
};
std::array<DeviceScratch, kMaxDevices> g_scratch{};
std::mutex g_scratch_mu;

int device_scratch(DeviceScratch **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail("device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  DeviceScratch &s = g_scratch[dev];
  if (!s.counter) {
    e = bhh_malloc((&s.counter), 256);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(work counter)");
    e = cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
  }
  *out = &s;
  return 0;
}

int g_block_override = 0;
int g_ctas_per_sm_override = 0;

}  // namespace

extern "C" {

const char *bh_last_error(void) { return g_last_error; }
int bh_abi_version(void) { return BH_KERR_ABI_VERSION; }

int bh_kerr_set_launch(int32_t block_threads, int32_t ctas_per_sm) {
  if (block_threads < 0 || block_threads > 1024 || (block_threads % 32) != 0)
    return fail("block_threads must be 0 or a multiple of 32 up to 1024, got %d", block_threads);
  if (block_threads > 128) return fail("the image kernels are compiled for at most 128 threads per CTA");
  if (ctas_per_sm < 0 || ctas_per_sm > 64) return fail("ctas_per_sm must be in [0, 64], got %d", ctas_per_sm);
  g_block_override = block_threads;
  g_ctas_per_sm_override = ctas_per_sm;
  return 0;
}

void bh_kerr_scene_defaults(BH_KerrScene *s) {
  if (!s) return;
  std::memset(s, 0, sizeof(*s));
  s->spin = 0.9;
  s->r_obs = 1000.0;
  s->theta_obs = 60.0 * std::numbers::pi / 180.0;
  s->alpha_min = -12.0;
  s->alpha_max = 12.0;
  s->beta_min = -12.0;
  s->beta_max = 12.0;
  s->width = 256;
  s->height = 256;
  s->integrator = BH_INTEGRATOR_RK4;
  s->precision = BH_PRECISION_FP64;
  s->potential_form = BH_POTENTIAL_REFERENCE;
  s->max_crossings = 1;
  s->max_steps = 20000;
  s->step_coeff = 0.02;
  s->step_rcap = 20.0;
  s->rtol = 1e-8;
  s->atol = 1e-10;
  s->horizon_factor = 1.001;
  s->escape_factor = 1.01;
  s->disk_r_in = 0.0;
  s->disk_r_out = 30.0;
}

int bh_kerr_scene_validate(const BH_KerrScene *s) {
  if (!s) return fail("scene is NULL");
  if (!(std::fabs(s->spin) < 1.0)) return fail("spin must satisfy |spin| < 1, got %g", s->spin);
  if (!(s->r_obs > 2.0 && std::isfinite(s->r_obs))) return fail("r_obs must be finite and > 2, got %g", s->r_obs);
  if (!(s->theta_obs > 0.0 && s->theta_obs < std::numbers::pi))
    return fail("theta_obs must lie in (0, pi), got %g", s->theta_obs);
  if (!(s->alpha_max > s->alpha_min) || !(s->beta_max > s->beta_min)) return fail("empty image-plane window");
  if (s->width < 0 || s->height < 0) return fail("negative image size %dx%d", s->width, s->height);
  if ((int64_t)s->width * s->height > (int64_t(1) << 31))
    return fail("image of %lld pixels exceeds 2^31", (long long)s->width * s->height);
  if (s->integrator != BH_INTEGRATOR_RK4 && s->integrator != BH_INTEGRATOR_DP45 &&
      s->integrator != BH_INTEGRATOR_ANALYTIC)
    return fail("unknown integrator %d", s->integrator);
  if (s->precision != BH_PRECISION_FP64 && s->precision != BH_PRECISION_MIXED)
    return fail("unknown precision %d", s->precision);
  if (s->potential_form != BH_POTENTIAL_REFERENCE && s->potential_form != BH_POTENTIAL_CARTER)
    return fail("unknown potential form %d", s->potential_form);
  if (s->max_crossings < 1 || s->max_crossings > BH_MAX_CROSSINGS)
    return fail("max_crossings must be in [1, %d], got %d", BH_MAX_CROSSINGS, s->max_crossings);
  if (s->max_steps < 0) return fail("max_steps must be >= 0");
  if (!(s->step_coeff > 0.0) || !(s->step_rcap > 0.0)) return fail("step_coeff and step_rcap must be > 0");
  if (s->integrator != BH_INTEGRATOR_RK4 && (!(s->rtol > 0.0) || !(s->atol > 0.0)))
    return fail("DP45 (and the analytic integrator's DP45 fallback) needs rtol > 0 and atol > 0");
  if (!(s->horizon_factor >= 1.0) || !(s->escape_factor > 0.0)) return fail("bad horizon/escape factor");
  if (!(s->disk_r_out > 0.0)) return fail("disk_r_out must be > 0");
  return 0;
}

// Host-side constants of one scene (scene_math.hpp).
static BhkImageParams make_params(const BH_KerrScene *s) {
  BhkImageParams p{};
  const bhh::SceneConstants k = bhh::scene_constants(*s);
  p.a = s->spin;
  p.a2 = s->spin * s->spin;
  p.r_obs = s->r_obs;
  p.r_plus = k.r_plus;
  p.r_minus = k.r_minus;
  p.r_hor = k.r_hor;
  p.r_esc = k.r_esc;
  p.r_in = k.r_in;
  p.r_out = s->disk_r_out;
  p.sin_o = k.sin_o;
  p.cos_o = k.cos_o;
  p.alpha_min = s->alpha_min;
  p.dalpha = (s->alpha_max - s->alpha_min) / double(s->width);
  p.beta_min = s->beta_min;
  p.dbeta = (s->beta_max - s->beta_min) / double(s->height);
  p.step_coeff = s->step_coeff;
  p.step_rcap = s->step_rcap;
  p.rtol = s->rtol;
  p.atol = s->atol;
  p.nt_isco = k.nt_isco;
  p.nt_flux_peak = k.nt_flux_peak;
  p.n_pix = int64_t(s->width) * s->height;
  p.width = s->width;
  p.max_steps = s->max_steps;
  p.max_cross = s->max_crossings;
  p.form = s->potential_form;
  p.integrator = s->integrator;
  p.precision = s->precision;
  return p;
}

int bhh_make_params(const BH_KerrScene *scene, BhkImageParams *p) {
  if (bh_kerr_scene_validate(scene) != 0) return -1;
  *p = make_params(scene);
  return 0;
}

// Validates the scene and fills the kernel parameters and the persistent
// grid shape (SM count x resident CTAs per SM, capped by the pixel count).
// Allocates nothing. Returns 0, or -1 with the error message set.
int bhh_prepare_image_launch(const BH_KerrScene *scene, BhkImageParams *p, BhkLaunch *L) {
  if (bh_kerr_scene_validate(scene) != 0) return -1;
  *p = make_params(scene);
  *L = BhkLaunch{0, 0, 1, 0};
  if (p->n_pix == 0) return 0;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
  const bool analytic = p->integrator == BH_INTEGRATOR_ANALYTIC;
  const int block = analytic ? bhk_trace_image_analytic_block() : (g_block_override ? g_block_override : 128);
  int per_sm = 0;
  const int occ_rc = analytic ? bhk_trace_image_analytic_occupancy(block, &per_sm)
                     : (p->precision == BH_PRECISION_MIXED)
                         ? bhk_trace_image_mixed_occupancy(p->integrator, block, &per_sm)
                         : bhk_trace_image_fp64_occupancy(p->integrator, block, &per_sm);
  if (occ_rc != 0) return cuda_fail(cudaGetLastError(), "occupancy query");
  if (g_ctas_per_sm_override) per_sm = std::min(per_sm, g_ctas_per_sm_override);
  if (per_sm < 1) return fail("kernel does not fit on an SM at %d threads per CTA", block);
  const int64_t full = int64_t(sms) * per_sm;
  const int64_t need = (p->n_pix + block - 1) / block;
  *L = BhkLaunch{int32_t(std::max<int64_t>(1, std::min(full, need))), block, 1, 0};
  return 0;
}

// Records an error message from the device layer (noalloc.cu).
int bhh_fail(const char *msg) { return fail("%s", msg); }

// ---- device allocations -------------------------------------------------------
namespace {
std::atomic<int64_t> g_device_allocs{0};  // successful bhh_malloc calls
std::atomic<int64_t> g_fail_in{0};        // > 0: the g_fail_in-th allocation from now fails
}  // namespace

// The current device's persistent-kernel work counter.
int bhh_work_counter(unsigned long long **counter) {
  DeviceScratch *ds = nullptr;
  if (device_scratch(&ds) != 0) return -1;
  *counter = ds->counter;
  return 0;
}

// The analytic integrator: the closed-form kernel, then DP45 (at the scene's
// precision) on the pixels it listed, over a persistent grid of that kernel.
static int launch_analytic(const BhkImageParams *p, const BhkImageOut *o, unsigned long long *counter, BhkLaunch L,
                           void *stream, int *list) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (!list) {
    DeviceScratch *ds = nullptr;
    if (device_scratch(&ds) != 0) return -1;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (ds->list_cap < p->n_pix) {
      if (ds->list) cudaFree(ds->list);
      ds->list = nullptr;
      ds->list_cap = 0;
      e = bhh_malloc((&ds->list), size_t(p->n_pix) * sizeof(int));
      if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(analytic fallback list)");
      ds->list_cap = p->n_pix;
    }
    list = ds->list;
  }
  unsigned int *count = reinterpret_cast<unsigned int *>(counter + 1);
  if (bhk_trace_image_analytic(p, o, list, count, L, stream) != 0)
    return cuda_fail(cudaGetLastError(), "k_trace_image_analytic launch");
  BhkImageParams q = *p;
  q.integrator = BH_INTEGRATOR_DP45;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
  int per_sm = 0;
  const int block = 128;
  const int occ_rc = (q.precision == BH_PRECISION_MIXED) ? bhk_trace_image_mixed_occupancy(1, block, &per_sm)
                                                         : bhk_trace_image_fp64_occupancy(1, block, &per_sm);
  if (occ_rc != 0 || per_sm < 1) return cuda_fail(cudaGetLastError(), "occupancy query");
  const BhkLaunch LL{int32_t(std::max<int64_t>(1, std::min<int64_t>(int64_t(sms) * per_sm, (q.n_pix + block - 1) / block))),
                     block, 1, 0};
  if (q.precision == BH_PRECISION_MIXED) {
    if (bhk_trace_list_mixed(&q, o, list, count, counter, LL, stream) != 0)
      return cuda_fail(cudaGetLastError(), "k_trace_list_mixed launch");
    return 0;
  }
  if (bhk_trace_list_fp64(&q, o, list, count, counter, LL, stream) != 0) return fail("%s", bhk_last_error());
  return 0;
}

int bhh_launch_image(const BhkImageParams *p, const BhkImageOut *o, unsigned long long *counter, BhkLaunch L,
                     void *stream, int *list) {
  if (p->integrator == BH_INTEGRATOR_ANALYTIC) return launch_analytic(p, o, counter, L, stream, list);
  if (p->precision == BH_PRECISION_MIXED) {
    if (bhk_trace_image_mixed(p, o, counter, L, stream) != 0)
      return cuda_fail(cudaGetLastError(), "k_trace_image_mixed launch");
    return 0;
  }
  if (bhk_trace_image_fp64(p, o, counter, L, stream) != 0) return fail("%s", bhk_last_error());
  return 0;
}

int bh_kerr_trace_image(const BH_KerrScene *scene, const BH_KerrImageOut *out, void *stream) {
  if (!out) return fail("output descriptor is NULL");
  BhkImageParams p;
  BhkLaunch L;
  if (bhh_prepare_image_launch(scene, &p, &L) != 0) return -1;
  if (p.n_pix == 0) return 0;
  DeviceScratch *ds = nullptr;
  if (device_scratch(&ds) != 0) return -1;
  const BhkImageOut o{out->cls,   out->steps,     out->n_cross,   out->r_hit,     out->phi_hit,
                      out->g,     out->flux,      out->intensity, out->theta_inf, out->phi_inf, nullptr, nullptr, out->carter_drift, nullptr};
  return bhh_launch_image(&p, &o, ds->counter, L, stream, nullptr);
}

// ---- host-buffer entry point ---------------------------------------------------
namespace {
struct HostCallBuffers {
  void *dev = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  int device = -1;
};
thread_local HostCallBuffers g_hb;

static int ensure_host_buffers(size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (g_hb.device != dev) {
    g_hb = HostCallBuffers{};
    g_hb.device = dev;
  }
  if (!g_hb.stream) {
    e = cudaStreamCreateWithFlags(&g_hb.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
  }
  if (g_hb.bytes < bytes) {
    if (g_hb.dev) cudaFree(g_hb.dev);
    g_hb.dev = nullptr;
    g_hb.bytes = 0;
    e = bhh_malloc(&g_hb.dev, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(output buffers)");
    g_hb.bytes = bytes;
  }
  return 0;
}
}  // namespace

int bh_kerr_trace_image_host(const BH_KerrScene *scene, const BH_KerrImageOut *h) {
  if (bh_kerr_scene_validate(scene) != 0) return -1;
  if (!h) return fail("output descriptor is NULL");
  const size_t n = size_t(scene->width) * size_t(scene->height);
  if (n == 0) return 0;
  const size_t mc = size_t(scene->max_crossings);
  struct F { void *host; size_t bytes; };
  const F fields[10] = {
      {h->cls, 4 * n},          {h->steps, 4 * n},          {h->n_cross, 4 * n},    {h->r_hit, 8 * n * mc},
      {h->phi_hit, 8 * n * mc}, {h->g, 8 * n * mc},         {h->flux, 8 * n},       {h->intensity, 8 * n},
      {h->theta_inf, 8 * n},    {h->phi_inf, 8 * n}};
  size_t total = 0;
  size_t off[10];
  for (int i = 0; i < 10; ++i) {
    off[i] = total;
    if (fields[i].host) total += (fields[i].bytes + 255) & ~size_t(255);
  }
  if (total == 0) return 0;
  if (ensure_host_buffers(total) != 0) return -1;
  char *base = static_cast<char *>(g_hb.dev);
  void *d[10];
  for (int i = 0; i < 10; ++i) d[i] = fields[i].host ? base + off[i] : nullptr;
  BH_KerrImageOut dev_out{static_cast<int32_t *>(d[0]), static_cast<int32_t *>(d[1]), static_cast<int32_t *>(d[2]),
                          static_cast<double *>(d[3]),  static_cast<double *>(d[4]),  static_cast<double *>(d[5]),
                          static_cast<double *>(d[6]),  static_cast<double *>(d[7]),  static_cast<double *>(d[8]),
                          static_cast<double *>(d[9]), nullptr};  // the drift diagnostic is not staged
  if (bh_kerr_trace_image(scene, &dev_out, g_hb.stream) != 0) return -1;
  for (int i = 0; i < 10; ++i) {
    if (!fields[i].host) continue;
    cudaError_t e = cudaMemcpyAsync(fields[i].host, d[i], fields[i].bytes, cudaMemcpyDeviceToHost, g_hb.stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(D2H)");
  }
  cudaError_t e = cudaStreamSynchronize(g_hb.stream);
  if (e != cudaSuccess) return cuda_fail(e, "bh_kerr_trace_image_host");
  return 0;
}

// ---- reference src/physics API ---------------------------------------------------

int bh_kerr_potentials(int64_t n, const double *r, const double *theta, double mass, double a,
                       BH_KerrConstsSoA c, double *rp, double *drp, double *tp, double *dtp, void *stream) {
  if (n < 0) return fail("negative count");
  if (n > 0 && (!r || !theta || !c.e || !c.lz || !c.q)) return fail("NULL input array");
  const BhkConstsSoA cc{c.e, c.lz, c.q};
  if (bhk_kerr_potentials(n, r, theta, mass, a, cc, rp, drp, tp, dtp, stream) != 0)
    return cuda_fail(cudaGetLastError(), "k_kerr_potentials launch");
  return 0;
}

int bh_kerr_step_mino(int64_t n, BH_KerrStateSoA s, double mass, double a, BH_KerrConstsSoA c, const double *dlam,
                      double dlam_scalar, void *stream) {
  if (n < 0) return fail("negative count");
  if (n > 0 && (!s.r || !s.theta || !s.phi || !s.t || !s.sign_r || !s.sign_theta || !c.e || !c.lz || !c.q))
    return fail("NULL state or constant array");
  const BhkStateSoA ss{s.r, s.theta, s.phi, s.t, s.sign_r, s.sign_theta};
  const BhkConstsSoA cc{c.e, c.lz, c.q};
  if (bhk_kerr_step_mino(n, ss, mass, a, cc, dlam, dlam_scalar, stream) != 0)
    return cuda_fail(cudaGetLastError(), "k_kerr_step_mino launch");
  return 0;
}

int bh_kerr_raytracer_defaults(double mass, double spin_param, BH_KerrRaytracerParams *out) {
  if (!out) return fail("params is NULL");
  const bhh::RaytracerDefaults d = bhh::raytracer_defaults(mass, spin_param);
  out->mass = mass;
  out->a = d.a;
  out->r_horizon = d.r_horizon;
  out->r_escape = d.r_escape;
  out->step_size = d.step;
  out->max_steps = 10000;
  out->reserved = 0;
  return 0;
}

int bh_kerr_trace_rays(int64_t n, BH_KerrStateSoA s, BH_KerrConstsSoA c, const BH_KerrRaytracerParams *p,
                       int32_t *status, int32_t *steps, double *dist, double *rf, double *thf, double *phf,
                       double *redshift, void *stream) {
  if (!p) return fail("params is NULL");
  if (n < 0) return fail("negative count");
  if (p->max_steps < 0) return fail("max_steps must be >= 0");
  if (n > 0 && (!s.r || !s.theta || !s.phi || !s.t || !s.sign_r || !s.sign_theta || !c.e || !c.lz || !c.q))
    return fail("NULL state or constant array");
  const BhkStateSoA ss{s.r, s.theta, s.phi, s.t, s.sign_r, s.sign_theta};
  const BhkConstsSoA cc{c.e, c.lz, c.q};
  if (bhk_kerr_trace_rays(n, ss, cc, p->mass, p->a, p->r_horizon, p->r_escape, p->step_size, p->max_steps, status,
                          steps, dist, rf, thf, phf, redshift, stream) != 0)
    return cuda_fail(cudaGetLastError(), "k_kerr_trace_rays launch");
  return 0;
}

}  // extern "C"

cudaError_t bhh_malloc(void **p, size_t bytes) {
  int64_t k = g_fail_in.load();
  while (k > 0 && !g_fail_in.compare_exchange_weak(k, k - 1)) {
  }
  if (k == 1) return cudaErrorMemoryAllocation;  // injected: as if the device were out of memory
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) g_device_allocs.fetch_add(1);
  return e;
}

extern "C" int64_t bh_debug_device_allocations(void) { return g_device_allocs.load(); }

extern "C" int bh_debug_fail_device_allocation(int64_t nth) {
  if (nth < 0) return fail("bh_debug_fail_device_allocation: nth must be >= 0, got %lld", (long long)nth);
  g_fail_in.store(nth);
  return 0;
}
