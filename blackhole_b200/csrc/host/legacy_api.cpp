// legacy_api.cpp - C++23 host side of include/bh_legacy.h: the reference
// renderer's launch ABI (BH_LaunchParams, bhCuda*, bhbCuda*) on the
// mixed-precision camera tracer and the RGBA shading of legacy.cu.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numbers>
#include <vector>

#include "../../../include/bh_kerr.h"
#include "../../../include/bh_legacy.h"
#include "../device/launch.h"
#include "scene_math.hpp"
#include "dalloc.hpp"

namespace {

int fail_msg(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
int fail_msg(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return bhh_fail(buf);
}

int cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return 0;
  return fail_msg("%s: %s", what, cudaGetErrorString(e));
}

// ---- blackbody colour table ---------------------------------------------------
//
// Linear-sRGB chromaticity (Y = 1) of a blackbody at temperature T: the
// Planck spectrum integrated against the CIE 1931 colour-matching functions
// in the multi-lobe Gaussian fit of Wyman, Sloan & Shirley (JCGT 2(2), 2013),
// 360-830 nm in 1 nm steps, converted with the sRGB (IEC 61966-2-1) matrix
// and clamped at 0. 256 entries, log2 T evenly spaced over [log2 400, log2 50000].

constexpr int kBbEntries = 256;
constexpr float kBbLog2T0 = 8.643856189774724f;   // log2(400)
constexpr float kBbLog2T1 = 15.609640474436812f;  // log2(50000)

double lobe(double x, double mu, double s1, double s2) {
  const double t = (x - mu) / (x < mu ? s1 : s2);
  return std::exp(-0.5 * t * t);
}

std::array<float, 3 * kBbEntries> blackbody_table() {
  std::array<float, 3 * kBbEntries> tab{};
  constexpr double c2 = 1.438776877e7;  // h c / k [nm K]
  for (int i = 0; i < kBbEntries; ++i) {
    const double l2 = kBbLog2T0 + (kBbLog2T1 - kBbLog2T0) * i / (kBbEntries - 1);
    const double T = std::exp2(l2);
    double X = 0, Y = 0, Z = 0;
    for (int w = 360; w <= 830; ++w) {
      const double lam = w;
      const double B = 1.0 / (std::pow(lam, 5.0) * std::expm1(c2 / (lam * T)));
      X += B * (1.056 * lobe(lam, 599.8, 37.9, 31.0) + 0.362 * lobe(lam, 442.0, 16.0, 26.7) -
                0.065 * lobe(lam, 501.1, 20.4, 26.2));
      Y += B * (0.821 * lobe(lam, 568.8, 46.9, 40.5) + 0.286 * lobe(lam, 530.9, 16.3, 31.1));
      Z += B * (1.217 * lobe(lam, 437.0, 11.8, 36.0) + 0.681 * lobe(lam, 459.0, 26.0, 13.8));
    }
    X /= Y;
    Z /= Y;
    Y = 1.0;
    const double r = 3.2406 * X - 1.5372 * Y - 0.4986 * Z;
    const double g = -0.9689 * X + 1.8758 * Y + 0.0415 * Z;
    const double b = 0.0557 * X - 0.2040 * Y + 1.0570 * Z;
    tab[3 * i] = float(std::max(r, 0.0));
    tab[3 * i + 1] = float(std::max(g, 0.0));
    tab[3 * i + 2] = float(std::max(b, 0.0));
  }
  return tab;
}

constexpr float kDiskPeakTemperature = 10000.0f;  // K at the Novikov-Thorne flux peak (colour only)

// ---- process state (the reference keeps these in __constant__ memory) ---------

std::mutex g_mu;
unsigned long long g_lut[8] = {};
unsigned long long g_equirect = 0;

constexpr int kMaxDevices = 64;

// Per-device scratch of the legacy renders (grow-only, one allocation).
struct Scratch {
  void *base = nullptr;
  int64_t cap = 0;
  int32_t *cls = nullptr;
  double *r_hit = nullptr, *g = nullptr, *flux = nullptr;
  double *phi_hit = nullptr, *theta_inf = nullptr, *phi_inf = nullptr;
  float *esc_dir = nullptr;
  float *closest = nullptr;
  float *vol = nullptr;  // [8][n] the slab of the RTE and Stokes modes
  unsigned long long *counter = nullptr;
  float *post = nullptr;  // bloom planes and composite of bhb_cuda_postprocess
  int64_t post_cap = 0;
  bool blackbody = false;
  int sms = 0;
};
std::array<Scratch, kMaxDevices> g_scratch{};

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

int scratch(int64_t n, Scratch **out) {
  int dev = 0;
  if (int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
  if (dev < 0 || dev >= kMaxDevices) return fail_msg("device ordinal %d out of range", dev);
  Scratch &s = g_scratch[dev];
  if (!s.blackbody) {
    const auto tab = blackbody_table();
    if (bhk_legacy_set_blackbody(tab.data(), kBbEntries, kBbLog2T0, kBbLog2T1) != 0)
      return fail_msg("legacy: blackbody table upload failed");
    if (int rc = cuda_check(cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev), "SM count"))
      return rc;
    s.blackbody = true;
  }
  if (n > s.cap) {
    if (s.base) cudaFree(s.base);
    s.base = nullptr;
    s.cap = 0;
    const size_t b_cls = up256(size_t(n) * 4), b_d = up256(size_t(n) * 8), b_dir = up256(size_t(n) * 12);
    const size_t b_vol = up256(size_t(n) * 32);
    char *p = nullptr;
    if (int rc = cuda_check(bhh_malloc((&p), b_cls + 6 * b_d + 2 * b_dir + b_vol + 256),
                            "cudaMalloc(legacy scratch)"))
      return rc;
    s.base = p;
    s.cls = reinterpret_cast<int32_t *>(p);
    double *d = reinterpret_cast<double *>(p + b_cls);
    const size_t nd = b_d / 8;
    s.r_hit = d;
    s.g = d + nd;
    s.flux = d + 2 * nd;
    s.phi_hit = d + 3 * nd;
    s.theta_inf = d + 4 * nd;
    s.phi_inf = d + 5 * nd;
    s.esc_dir = reinterpret_cast<float *>(p + b_cls + 6 * b_d);
    s.closest = reinterpret_cast<float *>(p + b_cls + 6 * b_d + b_dir);
    s.vol = reinterpret_cast<float *>(p + b_cls + 6 * b_d + 2 * b_dir);
    s.counter = reinterpret_cast<unsigned long long *>(p + b_cls + 6 * b_d + 2 * b_dir + b_vol);
    s.cap = n;
  }
  *out = &s;
  return 0;
}

// ---- shading: the reference's look (default) or physical -----------------------

int g_shading = -1;  // BH_SHADING_*, -1 until first read from BLACKHOLE_SHADING

int shading_mode() {
  if (g_shading < 0) {
    const char *v = std::getenv("BLACKHOLE_SHADING");
    g_shading = (v && std::strcmp(v, "physical") == 0) ? BH_SHADING_PHYSICAL : BH_SHADING_REFERENCE;
  }
  return g_shading;
}

// ---- BH_LaunchParams -> camera and tracer parameters --------------------------

struct CameraJob {
  BhkImageParams p;
  BhkCamera cam;
};

int camera_job(const BH_LaunchParams *lp, CameraJob *job) {
  if (!(lp->width > 0 && lp->height > 0)) return fail_msg("legacy: image size %dx%d", lp->width, lp->height);
  if ((int64_t)lp->width * lp->height > (int64_t(1) << 31)) return fail_msg("legacy: image exceeds 2^31 pixels");
  if (!(lp->rs > 0.0f) || !std::isfinite(lp->rs)) return fail_msg("legacy: rs must be finite and > 0");
  if (!(std::fabs(lp->spin) < 1.0f)) return fail_msg("legacy: spin must satisfy |spin| < 1, got %g", lp->spin);
  if (!(lp->fov_scale > 0.0f) || !std::isfinite(lp->fov_scale)) return fail_msg("legacy: fov_scale must be > 0");
  if (!(lp->max_dist > 0.0f)) return fail_msg("legacy: max_dist must be > 0");
  if (lp->max_steps < 1) return fail_msg("legacy: max_steps must be >= 1");
  for (float v : lp->cam_pos)
    if (!std::isfinite(v)) return fail_msg("legacy: camera position not finite");
  for (float v : lp->cam_basis)
    if (!std::isfinite(v)) return fail_msg("legacy: camera basis not finite");
  const double m = 0.5 * double(lp->rs);  // world units per M
  const double x = lp->cam_pos[0] / m, y = lp->cam_pos[1] / m, z = lp->cam_pos[2] / m;
  const double r0 = std::sqrt(x * x + y * y + z * z);
  const double spin = lp->kerr_enabled ? double(lp->spin) : 0.0;
  BH_KerrScene s;
  bh_kerr_scene_defaults(&s);
  const double r_plus = 1.0 + std::sqrt(1.0 - spin * spin);
  if (!(r0 > 2.0 && r0 > 1.01 * r_plus))
    return fail_msg("legacy: camera at r = %g M is not outside the horizon (r+ = %g M) and 2 M", r0, r_plus);
  const double u0 = z / r0;
  s.spin = spin;
  s.r_obs = r0;
  s.theta_obs = std::clamp(std::acos(std::clamp(u0, -1.0, 1.0)), 1e-9, std::numbers::pi - 1e-9);
  s.alpha_min = -1.0;
  s.alpha_max = 1.0;
  s.beta_min = -1.0;
  s.beta_max = 1.0;
  s.width = lp->width;
  s.height = lp->height;
  s.integrator = BH_INTEGRATOR_DP45;
  s.precision = BH_PRECISION_MIXED;
  s.potential_form = BH_POTENTIAL_CARTER;
  s.max_crossings = 1;
  s.max_steps = lp->max_steps;
  s.escape_factor = std::max(double(lp->max_dist) / m, 1.01 * r0) / r0;
  s.disk_r_in = lp->isco > 0.0f ? double(lp->isco) / m : 0.0;
  s.disk_r_out = lp->adisk_enabled ? 30.0 * double(lp->rs) / m : 1e-9;  // 30 rs; else nothing is a hit
  if (bhh_make_params(&s, &job->p) != 0) return -1;
  BhkCamera &c = job->cam;
  for (int k = 0; k < 3; ++k) {
    c.right[k] = lp->cam_basis[k];
    c.up[k] = lp->cam_basis[3 + k];
    c.fwd[k] = lp->cam_basis[6 + k];
  }
  c.fov = lp->fov_scale;
  c.aspect = double(lp->width) / double(lp->height);
  c.shift_x = lp->frame_shift_x;
  c.shift_y = lp->frame_shift_y;
  c.r0 = r0;
  c.u0 = u0;
  const double rho = std::sqrt(x * x + y * y);
  c.cphi = rho > 0.0 ? x / rho : 1.0;
  c.sphi = rho > 0.0 ? y / rho : 0.0;
  c.width = lp->width;
  c.height = lp->height;
  return 0;
}

int launch_shape(const Scratch &sc, int64_t n, BhkLaunch *L) {
  int per_sm = 0;
  if (bhk_trace_camera_mixed_occupancy(128, &per_sm) != 0 || per_sm < 1)
    return fail_msg("legacy: occupancy query failed");
  const int64_t need = (n + 127) / 128;
  *L = BhkLaunch{int32_t(std::max<int64_t>(1, std::min<int64_t>(int64_t(sc.sms) * per_sm, need))), 128, 1, 0};
  return 0;
}

// Trace and shade one frame into the device framebuffer.
int render(void *fb, const BH_LaunchParams *lp, int variant, cudaStream_t st) {
  if (!fb) return fail_msg("legacy: framebuffer is NULL");
  if (!lp) return fail_msg("legacy: params is NULL");
  if (variant >= BH_KERNEL_COUNT) return fail_msg("legacy: unknown kernel variant %d", variant);
  CameraJob job{};
  if (camera_job(lp, &job) != 0) return -1;
  const int64_t n = job.p.n_pix;
  Scratch *sc = nullptr;
  std::lock_guard<std::mutex> lock(g_mu);
  if (scratch(n, &sc) != 0) return -1;
  BhkLaunch L;
  if (launch_shape(*sc, n, &L) != 0) return -1;
  const bool look = shading_mode() == BH_SHADING_REFERENCE;
  // The reference's RTE and Stokes modes (Stokes first), which it traces only
  // for a spinning hole; otherwise its single-scatter look
  // (src/cuda/kernels_fp32.cu:47-70, device_physics.cuh:2037-2046).
  BhkVolume vol{};
  const bool kerr = lp->kerr_enabled && std::fabs(0.5f * lp->spin * lp->rs) >= 1e-6f;
  vol.mode = (look && kerr) ? (lp->stokes_enabled ? 2 : (lp->rte_enabled ? 1 : 0)) : 0;
  if (vol.mode) {
    vol.emit = lp->adisk_enabled;
    vol.m = 0.5f * lp->rs;
    vol.rs = lp->rs;
    vol.r_in = lp->isco;
    vol.r_out = 100.0f * lp->rs;
    vol.h = std::max(0.1f * lp->rs, 1e-6f);
    vol.opacity = lp->rte_opacity_scale;
    vol.b_angle = lp->stokes_b_field_angle;
    vol.ne_scale = lp->stokes_ne_scale;
    vol.cphi = float(job.cam.cphi);
    vol.sphi = float(job.cam.sphi);
    job.p.r_out = 0.0;  // the disk is the slab: no opaque crossing
    job.p.r_in = 1.0;
  }
  BhkImageOut o{};
  o.cls = sc->cls;
  o.r_hit = sc->r_hit;
  if (look) {
    o.phi_hit = sc->phi_hit;
    o.theta_inf = sc->theta_inf;
    o.phi_inf = sc->phi_inf;
    o.closest = sc->closest;
    if (vol.mode) o.vol = sc->vol;
  } else {
    o.g = sc->g;
    o.flux = sc->flux;
    o.esc_dir = sc->esc_dir;
  }
  if (bhk_trace_camera_mixed(&job.p, &job.cam, &o, sc->counter, L, st, vol.mode ? &vol : nullptr) != 0)
    return cuda_check(cudaGetLastError(), "k_trace_camera_mixed launch");
  if (look) {
    BhkLook lk{};
    lk.n = n;
    lk.m = 0.5f * lp->rs;
    lk.rs = lp->rs;
    lk.isco = lp->isco;
    lk.spin = lp->spin;
    lk.r_esc = job.p.r_esc;
    for (int k = 0; k < 3; ++k) {
      lk.cam_pos[k] = lp->cam_pos[k];
      lk.cam_right[k] = lp->cam_basis[k];
    }
    lk.cphi = float(job.cam.cphi);
    lk.sphi = float(job.cam.sphi);
    lk.redshift_enabled = lp->redshift_enabled;
    lk.use_luts = lp->use_luts;
    lk.background_enabled = lp->background_enabled;
    lk.vol_mode = vol.mode;
    lk.adisk_lit = lp->adisk_lit;
    lk.doppler_strength = lp->doppler_strength;
    lk.bg_intensity = lp->background_intensity;
    lk.time_sec = lp->time_sec;
    lk.glow_strength = lp->photon_glow_strength;
    lk.bg_yaw = lp->background_yaw_rad;
    lk.bg_pitch = lp->background_pitch_rad;
    lk.bg_filter = lp->background_filter_radius;
    for (int k = 0; k < 12; ++k) lk.bg_layers[k] = lp->background_layer_params[k];
    for (int k = 0; k < 3; ++k) lk.bg_lod_bias[k] = lp->background_layer_lod_bias[k];
    lk.lut_r_min = lp->lut_radius_min;
    lk.lut_r_max = lp->lut_radius_max;
    lk.z_r_min = lp->redshift_radius_min;
    lk.z_r_max = lp->redshift_radius_max;
    lk.spec_r_min = lp->spectral_radius_min;
    lk.spec_r_max = lp->spectral_radius_max;
    lk.grmhd_r_min = lp->grmhd_r_min;
    lk.grmhd_r_max = lp->grmhd_r_max;
    lk.grmhd_alpha = lp->grmhd_alpha;
    lk.tex_emissivity = g_lut[0];
    lk.tex_redshift = g_lut[1];
    lk.tex_spectral = g_lut[2];
    lk.tex_galaxy = g_lut[4];
    lk.tex_grmhd = g_lut[5];
    lk.tex_grmhd_right = g_lut[7];
    lk.tex_equirect = g_equirect;
    if (bhk_legacy_look(&lk, sc->cls, sc->r_hit, sc->phi_hit, sc->theta_inf, sc->phi_inf, sc->closest, sc->vol,
                        static_cast<float *>(fb), st) != 0)
      return cuda_check(cudaGetLastError(), "k_legacy_look launch");
    return 0;
  }
  BhkShade sh{};
  sh.n = n;
  sh.width = lp->width;
  sh.redshift_enabled = lp->redshift_enabled;
  sh.background_enabled = lp->background_enabled;
  sh.use_luts = lp->use_luts;
  sh.adisk_lit = lp->adisk_lit;
  sh.background_intensity = lp->background_intensity;
  sh.t_peak = kDiskPeakTemperature;
  sh.lut_r_min = lp->lut_radius_min;
  sh.lut_r_max = lp->lut_radius_max;
  sh.spec_r_min = lp->spectral_radius_min;
  sh.spec_r_max = lp->spectral_radius_max;
  sh.cphi = float(job.cam.cphi);
  sh.sphi = float(job.cam.sphi);
  sh.tex_emissivity = g_lut[0];
  sh.tex_spectral = g_lut[2];
  sh.tex_galaxy = g_lut[4];
  sh.tex_equirect = g_equirect;
  if (bhk_legacy_shade(&sh, sc->cls, sc->r_hit, sc->g, sc->flux, sc->esc_dir, static_cast<float *>(fb), st) != 0)
    return cuda_check(cudaGetLastError(), "k_legacy_shade launch");
  return 0;
}

// ---- bridge defaults and environment overrides -----------------------------------
//
// The bridge reads its render settings from BLACKHOLE_BRIDGE_* variables
// (src/blender_bridge/cuda_renderer.cu:28-68): an empty or unparsable value
// keeps the default; a flag is off for "0", "false", "FALSE", "off", "OFF".

float env_float(const char *name, float fallback) {
  const char *raw = std::getenv(name);
  if (!raw || !*raw) return fallback;
  char *end = nullptr;
  const float v = std::strtof(raw, &end);
  return end != raw ? v : fallback;
}

int env_int(const char *name, int fallback) {
  const char *raw = std::getenv(name);
  if (!raw || !*raw) return fallback;
  char *end = nullptr;
  const long v = std::strtol(raw, &end, 10);
  return end != raw ? int(v) : fallback;
}

int env_flag(const char *name, int fallback) {
  const char *raw = std::getenv(name);
  if (!raw || !*raw) return fallback;
  for (const char *off : {"0", "false", "FALSE", "off", "OFF"})
    if (std::strcmp(raw, off) == 0) return 0;
  return 1;
}

// Bardeen-Press-Teukolsky prograde ISCO in rs (= 2 M), in float as the
// bridge evaluates it (cuda_renderer.cu:433-439).
float bridge_isco_rs(float a) {
  const float z1 = 1.0f + std::pow(1.0f - a * a, 1.0f / 3.0f) *
                              (std::pow(1.0f + a, 1.0f / 3.0f) + std::pow(1.0f - a, 1.0f / 3.0f));
  const float z2 = std::sqrt(3.0f * a * a + z1 * z1);
  return 0.5f * (3.0f + z2 - std::sqrt((3.0f - z1) * (3.0f + z1 + 2.0f * z2)));
}

// Everything but the camera (cuda_renderer.cu:425-447, 520-522).
void bridge_common(BH_LaunchParams *p, float spin, float fov, int w, int h) {
  std::memset(p, 0, sizeof(*p));
  p->rs = 1.0f;
  p->spin = spin;
  p->isco = bridge_isco_rs(spin);
  p->step_size = env_float("BLACKHOLE_BRIDGE_STEP_SIZE", 0.08f);
  p->fov_scale = std::max(fov, 0.05f);
  p->max_dist = env_float("BLACKHOLE_BRIDGE_MAX_DIST", 500.0f);
  p->max_steps = env_int("BLACKHOLE_BRIDGE_MAX_STEPS", 600);
  p->width = w;
  p->height = h;
}

// Feature switches and the background layers, after the camera is placed
// (cuda_renderer.cu:500-552; the layer offsets follow the camera position).
void bridge_features(BH_LaunchParams *p) {
  p->frame_shift_x = env_float("BLACKHOLE_BRIDGE_FRAME_SHIFT_X", 0.0f);
  p->frame_shift_y = env_float("BLACKHOLE_BRIDGE_FRAME_SHIFT_Y", 0.0f);
  p->adisk_enabled = env_flag("BLACKHOLE_BRIDGE_ADISK_ENABLED", 1);
  p->redshift_enabled = env_flag("BLACKHOLE_BRIDGE_REDSHIFT_ENABLED", 1);
  p->kerr_enabled = std::fabs(p->spin) > 1e-6f ? 1 : 0;
  p->use_luts = 0;
  p->time_sec = 0.0f;
  p->doppler_strength = env_float("BLACKHOLE_BRIDGE_DOPPLER_STRENGTH", 1.0f);
  p->background_intensity = env_float("BLACKHOLE_BRIDGE_BACKGROUND_INTENSITY", 0.8f);
  p->background_enabled = env_flag("BLACKHOLE_BRIDGE_BACKGROUND_ENABLED", 1);
  p->photon_glow_strength = env_float("BLACKHOLE_BRIDGE_PHOTON_GLOW_STRENGTH", 1.0f);
  constexpr float deg = std::numbers::pi_v<float> / 180.0f;
  p->background_yaw_rad = env_float("BLACKHOLE_BRIDGE_BACKGROUND_YAW_DEG", 0.0f) * deg;
  p->background_pitch_rad = env_float("BLACKHOLE_BRIDGE_BACKGROUND_PITCH_DEG", 0.0f) * deg;
  p->background_filter_radius = env_float("BLACKHOLE_BRIDGE_BACKGROUND_FILTER_RADIUS", 0.0f);
  const float parallax = env_float("BLACKHOLE_BRIDGE_BACKGROUND_PARALLAX_STRENGTH", 0.0006f);
  const float drift = env_float("BLACKHOLE_BRIDGE_BACKGROUND_DRIFT_STRENGTH", 0.01f);
  static const char *const kVar[3][4] = {
      {"BLACKHOLE_BRIDGE_BACKGROUND_LAYER0_DEPTH", "BLACKHOLE_BRIDGE_BACKGROUND_LAYER0_SCALE",
       "BLACKHOLE_BRIDGE_BACKGROUND_LAYER0_INTENSITY", "BLACKHOLE_BRIDGE_BACKGROUND_LAYER0_LOD_BIAS"},
      {"BLACKHOLE_BRIDGE_BACKGROUND_LAYER1_DEPTH", "BLACKHOLE_BRIDGE_BACKGROUND_LAYER1_SCALE",
       "BLACKHOLE_BRIDGE_BACKGROUND_LAYER1_INTENSITY", "BLACKHOLE_BRIDGE_BACKGROUND_LAYER1_LOD_BIAS"},
      {"BLACKHOLE_BRIDGE_BACKGROUND_LAYER2_DEPTH", "BLACKHOLE_BRIDGE_BACKGROUND_LAYER2_SCALE",
       "BLACKHOLE_BRIDGE_BACKGROUND_LAYER2_INTENSITY", "BLACKHOLE_BRIDGE_BACKGROUND_LAYER2_LOD_BIAS"}};
  static const float kDefault[3][4] = {{0.2f, 1.0f, 1.0f, 0.0f}, {0.5f, 1.08f, 0.6f, 1.0f}, {0.9f, 1.16f, 0.35f, 2.0f}};
  const float px = p->cam_pos[0] * parallax, py = p->cam_pos[1] * parallax;
  const float dx = std::cos(p->time_sec * 0.02f) * drift, dy = std::sin(p->time_sec * 0.02f) * drift;
  for (int i = 0; i < 3; ++i) {
    const float depth = env_float(kVar[i][0], kDefault[i][0]);
    p->background_layer_params[4 * i + 0] = dx + px * depth;
    p->background_layer_params[4 * i + 1] = dy + py * depth;
    p->background_layer_params[4 * i + 2] = env_float(kVar[i][1], kDefault[i][1]);
    p->background_layer_params[4 * i + 3] = env_float(kVar[i][2], kDefault[i][2]);
    p->background_layer_lod_bias[i] = std::max(env_float(kVar[i][3], kDefault[i][3]), 0.0f);
  }
  p->adisk_lit = env_float("BLACKHOLE_BRIDGE_ADISK_LIT", 0.35f);
}

// The Blender bridge's camera: on the (y, z) circle of radius observer_r
// [rs] at the inclination from +z, looking at the origin; right = forward x
// (0, 1, 0), up = right x forward (cuda_renderer.cu:452-492).
void bridge_params(BH_LaunchParams *p, float spin, float observer_r, float incl, float fov, int w, int h) {
  bridge_common(p, spin, fov, w, h);
  const float ci = std::cos(incl), si = std::sin(incl);
  p->cam_pos[0] = 0.0f;
  p->cam_pos[1] = observer_r * si;
  p->cam_pos[2] = observer_r * ci;
  float f[3] = {0.0f, -si, -ci};
  float r[3] = {-f[2], 0.0f, f[0]};  // forward x (0, 1, 0)
  float rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  if (rl < 1e-6f) {
    r[0] = 1.0f;
    r[1] = r[2] = 0.0f;
    rl = 1.0f;
  }
  for (float &v : r) v /= rl;
  const float u[3] = {r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0]};
  for (int k = 0; k < 3; ++k) {
    p->cam_basis[k] = r[k];
    p->cam_basis[3 + k] = u[k];
    p->cam_basis[6 + k] = f[k];
  }
  bridge_features(p);
}

// ---- bloom and tone mapping -------------------------------------------------------

// The normalized Gaussian taps of half-width 4, 8, 16, 32 with sigma = r / 2,
// evaluated in float as the reference's blur passes do
// (cuda_postprocess.cu:42-64): g = exp(-dx^2 / (2 sigma^2)), divided by their sum.
BhkPostTaps post_taps() {
  BhkPostTaps t{};
  int off = 0;
  for (int r : {4, 8, 16, 32}) {
    const float sigma = float(r) * 0.5f, inv2s2 = 1.0f / (2.0f * sigma * sigma);
    float wt = 0.0f;
    for (int dx = -r; dx <= r; ++dx) wt += std::exp(-float(dx * dx) * inv2s2);
    const float inv = 1.0f / wt;
    for (int dx = -r; dx <= r; ++dx) t.w[off + dx + r] = std::exp(-float(dx * dx) * inv2s2) * inv;
    off += 2 * r + 1;
  }
  return t;
}

// Bloom (bright-pass over the threshold, four blur scales, added with the
// strength), then exposure, vignette, ACES and gamma, in place on the
// float4 framebuffer. Caller holds g_mu.
int postprocess_locked(float *fb, int w, int h, float threshold, float strength, float exposure, cudaStream_t st) {
  if (!fb) return fail_msg("postprocess: framebuffer is NULL");
  if (w <= 0 || h <= 0) return fail_msg("postprocess: image size %dx%d", w, h);
  if ((int64_t)w * h > (int64_t(1) << 31)) return fail_msg("postprocess: image exceeds 2^31 pixels");
  Scratch *sc = nullptr;
  if (scratch(0, &sc) != 0) return -1;
  const int64_t need = bhk_post_scratch_floats(w, h);
  if (need > sc->post_cap) {
    if (sc->post) cudaFree(sc->post);
    sc->post = nullptr;
    sc->post_cap = 0;
    if (int rc = cuda_check(bhh_malloc((&sc->post), size_t(need) * 4),
                            "cudaMalloc(postprocess scratch)"))
      return rc;
    sc->post_cap = need;
  }
  static const BhkPostTaps taps = post_taps();
  if (bhk_post_process(fb, w, h, &taps, threshold, strength, exposure, sc->post, st) != 0)
    return cuda_check(cudaGetLastError(), "postprocess launch");
  return 0;
}

// Render to a temporary device framebuffer, post-process as the bridge does
// (bloom threshold 1, strength 0, exposure 12 unless overridden:
// cuda_renderer.cu:665-673), copy to the host buffer.
int render_to_host(const BH_LaunchParams *lp, float *out_rgba) {
  if (!out_rgba) return fail_msg("bridge: output buffer is NULL");
  if (!(lp->width > 0 && lp->height > 0)) return fail_msg("bridge: image size %dx%d", lp->width, lp->height);
  const size_t bytes = size_t(lp->width) * size_t(lp->height) * 16;
  void *fb = nullptr;
  if (int rc = cuda_check(bhh_malloc(&fb, bytes), "cudaMalloc(bridge framebuffer)")) return rc;
  int rc = render(fb, lp, BH_KERNEL_FP32_BASELINE, nullptr);
  if (rc == 0) {
    std::lock_guard<std::mutex> lock(g_mu);
    rc = postprocess_locked(static_cast<float *>(fb), lp->width, lp->height,
                            env_float("BLACKHOLE_BRIDGE_BLOOM_THRESHOLD", 1.0f),
                            env_float("BLACKHOLE_BRIDGE_BLOOM_STRENGTH", 0.0f),
                            env_float("BLACKHOLE_BRIDGE_EXPOSURE", 12.0f), nullptr);
  }
  if (rc == 0) rc = cuda_check(cudaMemcpy(out_rgba, fb, bytes, cudaMemcpyDeviceToHost), "bridge copy-out");
  cudaFree(fb);
  return rc;
}

}  // namespace

// ---- kernel launch ABI ----------------------------------------------------------

int bh_launch_geodesic_kernel(void *framebuffer, const BH_LaunchParams *params, int variant, void *stream) {
  return render(framebuffer, params, variant, static_cast<cudaStream_t>(stream));
}

int bh_select_kernel_variant(void) { return BH_KERNEL_FP32_BASELINE; }

int bh_legacy_set_shading(int mode) {
  if (mode != BH_SHADING_REFERENCE && mode != BH_SHADING_PHYSICAL)
    return fail_msg("bh_legacy_set_shading: mode must be BH_SHADING_REFERENCE (0) or BH_SHADING_PHYSICAL (1), got %d",
                    mode);
  std::lock_guard<std::mutex> lock(g_mu);
  g_shading = mode;
  return 0;
}

int bh_stokes_steps(long long n, const float *state, const float *coef, float *out, void *stream) {
  if (n < 0) return fail_msg("bh_stokes_steps: n must be >= 0, got %lld", (long long)n);
  if (n > 0 && (!state || !coef || !out)) return fail_msg("bh_stokes_steps: state, coef and out must be non-NULL");
  if (reinterpret_cast<uintptr_t>(state) % 16 || reinterpret_cast<uintptr_t>(out) % 16)
    return fail_msg("bh_stokes_steps: state and out must be 16-byte aligned");
  if (bhk_stokes_steps(n, state, coef, out, stream) != 0) return cuda_check(cudaGetLastError(), "k_stokes_steps launch");
  return 0;
}

int bh_legacy_get_shading(void) {
  std::lock_guard<std::mutex> lock(g_mu);
  return shading_mode();
}

void bh_upload_lut_textures(unsigned long long emissivity, unsigned long long redshift, unsigned long long spectral,
                            unsigned long long grb, unsigned long long galaxy, unsigned long long grmhd,
                            unsigned long long synch_g, unsigned long long grmhd_right) {
  std::lock_guard<std::mutex> lock(g_mu);
  const unsigned long long v[8] = {emissivity, redshift, spectral, grb, galaxy, grmhd, synch_g, grmhd_right};
  std::memcpy(g_lut, v, sizeof(v));
}

void bh_upload_bridge_background_texture(unsigned long long background_equirect) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_equirect = background_equirect;
}

// ---- backend ----------------------------------------------------------------------

struct BhCudaBackend {
  int device = 0;
  int width = 0, height = 0;
  void *fb = nullptr;
  cudaStream_t stream = nullptr;
  int variant = -1;
};

BH_CudaBackend *bhCudaInit(unsigned int /*gl_texture*/, int width, int height) {
  if (width <= 0 || height <= 0) {
    fail_msg("backend: image size %dx%d", width, height);
    return nullptr;
  }
  auto *b = new BhCudaBackend;
  if (cuda_check(cudaGetDevice(&b->device), "cudaGetDevice") ||
      cuda_check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate") ||
      cuda_check(bhh_malloc(&b->fb, size_t(width) * size_t(height) * 16), "cudaMalloc(framebuffer)")) {
    bhCudaShutdown(b);
    return nullptr;
  }
  b->width = width;
  b->height = height;
  return b;
}

int bhCudaRenderFrame(BH_CudaBackend *b, const BH_LaunchParams *params) {
  if (!b || !params) return fail_msg("backend: NULL argument");
  if (params->width != b->width || params->height != b->height)
    return fail_msg("backend: params are %dx%d, framebuffer %dx%d (bhCudaResize first)", params->width,
                    params->height, b->width, b->height);
  if (render(b->fb, params, b->variant, b->stream) != 0) return -1;
  return cuda_check(cudaStreamSynchronize(b->stream), "bhCudaRenderFrame");
}

int bhCudaResize(BH_CudaBackend *b, unsigned int /*gl_texture*/, int width, int height) {
  if (!b) return fail_msg("backend: NULL handle");
  if (width <= 0 || height <= 0) return fail_msg("backend: image size %dx%d", width, height);
  if (width == b->width && height == b->height) return 0;
  if (int rc = cuda_check(cudaStreamSynchronize(b->stream), "bhCudaResize")) return rc;
  cudaFree(b->fb);
  b->fb = nullptr;
  b->width = b->height = 0;
  if (int rc = cuda_check(bhh_malloc(&b->fb, size_t(width) * size_t(height) * 16), "cudaMalloc(framebuffer)"))
    return rc;
  b->width = width;
  b->height = height;
  return 0;
}

int bhCudaRegisterLut(BH_CudaBackend * /*b*/, int /*slot*/, unsigned int /*gl_texture*/, unsigned int /*target*/) {
  return fail_msg("backend: OpenGL textures cannot be registered (no graphics stack); pass CUDA texture objects "
                  "to bh_upload_lut_textures");
}

int bhCudaRegisterBackgroundTexture(BH_CudaBackend * /*b*/, unsigned int /*gl_texture*/, unsigned int /*target*/) {
  return fail_msg("backend: OpenGL textures cannot be registered (no graphics stack); pass a CUDA texture object "
                  "to bh_upload_bridge_background_texture");
}

int bhCudaSetVariant(BH_CudaBackend *b, int variant) {
  if (!b) return fail_msg("backend: NULL handle");
  if (variant >= BH_KERNEL_COUNT) return fail_msg("backend: unknown kernel variant %d", variant);
  b->variant = variant < 0 ? -1 : variant;
  return b->variant;
}

int bhCudaGetVariant(BH_CudaBackend *b) {
  if (!b) return fail_msg("backend: NULL handle");
  return b->variant;
}

void bhCudaShutdown(BH_CudaBackend *b) {
  if (!b) return;
  int cur = -1;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->fb) cudaFree(b->fb);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (cur >= 0) cudaSetDevice(cur);
  delete b;
}

void *bhCudaFramebuffer(BH_CudaBackend *b) { return b ? b->fb : nullptr; }

// ---- Blender bridge -------------------------------------------------------------

int bhbHasCuda(void) { return 1; }

int bhbCudaResetDevice(void) {
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  if (int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
  if (int rc = cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize")) return rc;
  if (dev >= 0 && dev < kMaxDevices) {
    Scratch &s = g_scratch[dev];
    if (s.base) cudaFree(s.base);
    if (s.post) cudaFree(s.post);
    s.base = nullptr;
    s.cap = 0;
    s.post = nullptr;
    s.post_cap = 0;
  }
  return 0;
}

int bhbCudaRenderRaytracedCamera(float spin, float observerR, float inclinationRad, float fovScale, int width,
                                 int height, float *outRgba) {
  BH_LaunchParams p;
  bridge_params(&p, spin, observerR, inclinationRad, fovScale, width, height);
  return render_to_host(&p, outRgba);
}

int bhbCudaRenderRaytraced(float spin, float observerR, float inclinationRad, int width, int height,
                           float *outRgba) {
  return bhbCudaRenderRaytracedCamera(spin, observerR, inclinationRad, 1.0f, width, height, outRgba);
}

int bhbCudaRenderRaytracedView(float spin, const float *camPos, const float *camBasis, float fovScale, int width,
                               int height, float *outRgba) {
  if (!camPos || !camBasis) return fail_msg("bridge: camera position or basis is NULL");
  BH_LaunchParams p;
  bridge_common(&p, spin, fovScale, width, height);  // cuda_renderer.cu:557-585
  std::memcpy(p.cam_pos, camPos, sizeof(p.cam_pos));
  std::memcpy(p.cam_basis, camBasis, sizeof(p.cam_basis));
  bridge_features(&p);
  return render_to_host(&p, outRgba);
}

int bhbCudaRenderLensingMap(double aStar, double observerRRg, double inclinationRad, int width, int height,
                            float *outRgba) {
  if (!outRgba || width <= 0 || height <= 0) return fail_msg("lensing map: bad arguments");
  BH_KerrScene s;
  bh_kerr_scene_defaults(&s);
  s.spin = aStar;
  s.r_obs = observerRRg;
  s.theta_obs = std::clamp(inclinationRad, 1e-9, std::numbers::pi - 1e-9);
  s.width = width;
  s.height = height;
  s.alpha_min = -15.0;  // replaced below: corner-anchored grid of the reference
  s.alpha_max = 15.0;
  s.integrator = BH_INTEGRATOR_DP45;
  s.precision = BH_PRECISION_MIXED;
  s.potential_form = BH_POTENTIAL_CARTER;
  s.disk_r_out = 100.0;
  BhkImageParams p;
  if (bhh_make_params(&s, &p) != 0) return -1;
  p.dalpha = 30.0 / width;  // alpha_i = 30 (i / width - 1/2): pixel i's left edge in the reference
  p.alpha_min = -15.0 - 0.5 * p.dalpha;
  p.dbeta = -30.0 / height;  // beta_j = 30 (1/2 - j / height)
  p.beta_min = 15.0 - 0.5 * p.dbeta;
  const int64_t n = p.n_pix;
  std::lock_guard<std::mutex> lock(g_mu);
  Scratch *sc = nullptr;
  if (scratch(n, &sc) != 0) return -1;
  int per_sm = 0;
  if (bhk_trace_image_mixed_occupancy(1, 128, &per_sm) != 0 || per_sm < 1)
    return fail_msg("lensing map: occupancy query failed");
  const BhkLaunch L{int32_t(std::max<int64_t>(1, std::min<int64_t>(int64_t(sc->sms) * per_sm, (n + 127) / 128))),
                    128, 1, 0};
  BhkImageOut o{};
  o.cls = sc->cls;
  o.r_hit = sc->r_hit;
  o.g = sc->g;
  const size_t bytes = size_t(n) * 16;
  void *fb = nullptr;
  if (int rc = cuda_check(bhh_malloc(&fb, bytes), "cudaMalloc(lensing map)")) return rc;
  int rc = 0;
  if (bhk_trace_image_mixed(&p, &o, sc->counter, L, nullptr) != 0 ||
      bhk_legacy_lensing(n, sc->cls, sc->r_hit, sc->g, static_cast<float *>(fb), nullptr) != 0)
    rc = cuda_check(cudaGetLastError(), "lensing map launch");
  if (rc == 0) rc = cuda_check(cudaMemcpy(outRgba, fb, bytes, cudaMemcpyDeviceToHost), "lensing map copy-out");
  cudaFree(fb);
  return rc;
}

int bhbCudaRenderDiskTexture(const BhbDiskParams *params, int width, int height, float *outRgba) {
  if (!params || !outRgba || width <= 0 || height <= 0) return fail_msg("disk texture: bad arguments");
  if (!(std::fabs(params->aStar) < 1.0)) return fail_msg("disk texture: |aStar| must be < 1");
  BH_KerrScene s;
  bh_kerr_scene_defaults(&s);
  s.spin = params->aStar;
  const bhh::SceneConstants k = bhh::scene_constants(s);
  if (!(params->rOutRg > k.r_in)) return fail_msg("disk texture: rOutRg must exceed the ISCO (%g)", k.r_in);
  const size_t bytes = size_t(width) * size_t(height) * 16;
  void *fb = nullptr;
  std::lock_guard<std::mutex> lock(g_mu);
  Scratch *sc = nullptr;
  if (scratch(0, &sc) != 0) return -1;  // colour table
  if (int rc = cuda_check(bhh_malloc(&fb, bytes), "cudaMalloc(disk texture)")) return rc;
  int rc = 0;
  if (bhk_legacy_disk_texture(s.spin, k.r_in, params->rOutRg, k.nt_flux_peak, params->inclinationRad,
                              kDiskPeakTemperature, width, height, static_cast<float *>(fb), nullptr) != 0)
    rc = cuda_check(cudaGetLastError(), "disk texture launch");
  if (rc == 0) rc = cuda_check(cudaMemcpy(outRgba, fb, bytes, cudaMemcpyDeviceToHost), "disk texture copy-out");
  cudaFree(fb);
  return rc;
}

int bhbCudaTraceGeodesics(double aStar, double observerRRg, double inclinationRad, double alphaMin, double alphaMax,
                          int nAlpha, double betaMin, double betaMax, int nBeta, int maxSteps, double stepSize,
                          float *outXyz, int *outCounts) {
  if (!outXyz || !outCounts || nAlpha < 1 || nBeta < 1 || maxSteps < 1 || !(stepSize > 0.0))
    return fail_msg("trace geodesics: bad arguments");
  BH_KerrScene s;
  bh_kerr_scene_defaults(&s);
  s.spin = aStar;
  s.r_obs = observerRRg;
  s.theta_obs = std::clamp(inclinationRad, 1e-9, std::numbers::pi - 1e-9);
  s.width = nAlpha;
  s.height = nBeta;
  s.integrator = BH_INTEGRATOR_RK4;
  s.precision = BH_PRECISION_FP64;
  s.potential_form = BH_POTENTIAL_CARTER;
  s.step_coeff = stepSize / 20.0;
  s.step_rcap = 20.0;
  BhkImageParams p;
  if (bhh_make_params(&s, &p) != 0) return -1;
  p.dalpha = nAlpha > 1 ? (alphaMax - alphaMin) / (nAlpha - 1) : 0.0;  // endpoints included
  p.alpha_min = nAlpha > 1 ? alphaMin - 0.5 * p.dalpha : 0.5 * (alphaMin + alphaMax);
  p.dbeta = nBeta > 1 ? (betaMax - betaMin) / (nBeta - 1) : 0.0;
  p.beta_min = nBeta > 1 ? betaMin - 0.5 * p.dbeta : 0.5 * (betaMin + betaMax);
  const int64_t n = p.n_pix;
  const size_t b_xyz = size_t(n) * size_t(maxSteps) * 12, b_cnt = size_t(n) * 4;
  char *d = nullptr;
  if (int rc = cuda_check(bhh_malloc((&d), b_xyz + b_cnt + 256), "cudaMalloc(geodesic paths)"))
    return rc;
  int32_t *cnt = reinterpret_cast<int32_t *>(d + ((b_xyz + 255) & ~size_t(255)));
  int rc = 0;
  if (bhk_trace_paths_fp64(&p, reinterpret_cast<float *>(d), cnt, maxSteps, nullptr) != 0)
    rc = fail_msg("trace geodesics: %s", bhk_last_error());
  if (rc == 0) rc = cuda_check(cudaMemcpy(outXyz, d, b_xyz, cudaMemcpyDeviceToHost), "paths copy-out");
  if (rc == 0) rc = cuda_check(cudaMemcpy(outCounts, cnt, b_cnt, cudaMemcpyDeviceToHost), "counts copy-out");
  cudaFree(d);
  return rc;
}

int bhb_cuda_postprocess(float *d_framebuffer, int width, int height, float bloom_threshold, float bloom_strength,
                         float exposure_gain, float /*time_sec: the reference's film grain is not implemented*/) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (int rc = postprocess_locked(d_framebuffer, width, height, bloom_threshold, bloom_strength, exposure_gain,
                                  nullptr))
    return rc;
  return cuda_check(cudaStreamSynchronize(nullptr), "bhb_cuda_postprocess");
}

int bhb_cuda_render_raytraced(float spin, float observer_r, float inclination_rad, int width, int height,
                              float *out_rgba) {
  return bhbCudaRenderRaytraced(spin, observer_r, inclination_rad, width, height, out_rgba);
}

int bhb_cuda_render_raytraced_camera(float spin, float observer_r, float inclination_rad, float fov_scale, int width,
                                     int height, float *out_rgba) {
  return bhbCudaRenderRaytracedCamera(spin, observer_r, inclination_rad, fov_scale, width, height, out_rgba);
}

int bhb_cuda_render_raytraced_view(float spin, const float *cam_pos, const float *cam_basis, float fov_scale,
                                   int width, int height, float *out_rgba) {
  return bhbCudaRenderRaytracedView(spin, cam_pos, cam_basis, fov_scale, width, height, out_rgba);
}

int bhb_cuda_render_lensing_map(float a_star, float obs_r, float inc_rad, int width, int height, float *out_rgba) {
  return bhbCudaRenderLensingMap(a_star, obs_r, inc_rad, width, height, out_rgba);
}

int bhb_cuda_render_disk_texture(float a_star, float r_out_rg, float inc_rad, int width, int height,
                                 float *out_rgba) {
  const BhbDiskParams p{a_star, 1.0, 0.1, r_out_rg, inc_rad};
  return bhbCudaRenderDiskTexture(&p, width, height, out_rgba);
}
