// rt_api.cpp - C++23 host side of include/bh_rt.h: the synthetic medium's
// random Fourier modes, the thermal-synchrotron table, and the traced
// radiative-transfer image.
#include <cuda_runtime_api.h>

#include <cmath>
#include <vector>

#include "../../../include/bh_rt.h"
#include "../device/launch.h"
#include "../device/sky.cuh"
#include "dalloc.hpp"

namespace {

constexpr int kModes = 256;
constexpr double kE = 4.80320425e-10, kMe = 9.1093837015e-28, kC = 2.99792458e10;

// Mahadevan (1996) Eq. A2 spectral function, as the reference evaluates it
// (src/physics/rte_integrator.h:304-309).
double mahadevan_im(double x) {
  return 4.0505 * std::pow(x, -1.0 / 6.0) * (1.0 + 0.40 * std::pow(x, -1.0 / 4.0) + 0.5316 * std::pow(x, -1.0 / 2.0)) *
         std::exp(-1.8899 * std::pow(x, 1.0 / 3.0));
}

struct Uniforms {
  uint64_t base, n = 0;
  double next() { return (double)(bhsky::splitmix64(base + n++) >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace

extern "C" {

void bh_torus_defaults(BH_TorusParams *t) {
  if (!t) return;
  *t = BH_TorusParams{6.0, 12.0, 3.0, 1.0e5, 20.0, 30.0, 0.5, 2.0, 1};
}

void bh_rt_defaults(BH_RtParams *rt) {
  if (!rt) return;
  *rt = BH_RtParams{230.0e9, 1.4766250e6, 0.25, 1.0e-6};
}

int bh_grmhd_synthetic(const BH_GrmhdGrid *g, const BH_TorusParams *t, void *stream) {
  if (!g || !t || !g->cells) return bhh_fail("bh_grmhd_synthetic: NULL argument");
  if (g->n_r < 2 || g->n_theta < 2 || g->n_phi < 2) return bhh_fail("bh_grmhd_synthetic: grid needs >= 2 nodes per axis");
  if (!(g->r_min > 0.0 && g->r_max > g->r_min)) return bhh_fail("bh_grmhd_synthetic: need 0 < r_min < r_max");
  if (!(t->corr_len > 0.0 && t->width > 0.0 && t->n0 > 0.0)) return bhh_fail("bh_grmhd_synthetic: bad torus parameters");
  // Gaussian correlation sigma^2 exp(-d^2 / (2 l^2)): wave vectors ~ N(0, I / l^2),
  // phases ~ U[0, 2 pi), amplitude sigma sqrt(2 / M) (random Fourier features).
  Uniforms u{t->seed ^ 0x4752464D4F444553ull};
  std::vector<double> modes(4 * kModes);
  for (int m = 0; m < kModes; ++m) {
    double z[4];
    for (int p = 0; p < 2; ++p) {
      const double u1 = 1.0 - u.next(), u2 = u.next();  // u1 in (0, 1]
      const double rad = std::sqrt(-2.0 * std::log(u1));
      z[2 * p] = rad * std::cos(6.283185307179586 * u2);
      z[2 * p + 1] = rad * std::sin(6.283185307179586 * u2);
    }
    modes[4 * m + 0] = z[0] / t->corr_len;
    modes[4 * m + 1] = z[1] / t->corr_len;
    modes[4 * m + 2] = z[2] / t->corr_len;
    modes[4 * m + 3] = 6.283185307179586 * u.next();
  }
  double *d_modes = nullptr;
  if (bhh_malloc((&d_modes), modes.size() * sizeof(double)) != cudaSuccess)
    return bhh_fail("bh_grmhd_synthetic: cudaMalloc failed");
  cudaMemcpy(d_modes, modes.data(), modes.size() * sizeof(double), cudaMemcpyHostToDevice);
  const int rc = bhk_grmhd_fill(static_cast<float *>(const_cast<void *>(g->cells)), g->n_r, g->n_theta, g->n_phi,
                                g->r_min, g->r_max, t->r_in, t->r_peak, t->width, t->n0, t->theta0, t->b0,
                                t->sigma * std::sqrt(2.0 / kModes), d_modes, kModes, stream);
  cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  cudaFree(d_modes);
  if (rc != 0) return bhh_fail("bh_grmhd_synthetic: launch failed");
  return 0;
}

int bh_synchrotron_lut_host(const BH_SynchrotronLut *lut, float *out) {
  if (!lut || !out || lut->n_theta < 2 || lut->n_x < 2) return bhh_fail("bh_synchrotron_lut: bad table");
  if (!(lut->log_theta_max > lut->log_theta_min && lut->log_x_max > lut->log_x_min))
    return bhh_fail("bh_synchrotron_lut: empty range");
  const double pref = std::sqrt(3.0) * kE * kE * kE / (kMe * kC * kC);
  for (int i = 0; i < lut->n_theta; ++i) {
    const double th = std::exp(lut->log_theta_min + (lut->log_theta_max - lut->log_theta_min) * i / (lut->n_theta - 1));
    const double k2 = 2.0 * th * th;
    for (int k = 0; k < lut->n_x; ++k) {
      const double x = std::exp(lut->log_x_min + (lut->log_x_max - lut->log_x_min) * k / (lut->n_x - 1));
      out[(size_t)i * lut->n_x + k] = (float)std::log(pref / k2 * th * th * mahadevan_im(x));
    }
  }
  return 0;
}

int bh_synchrotron_lut(const BH_SynchrotronLut *lut, void *stream) {
  if (!lut || !lut->table || lut->n_theta < 2 || lut->n_x < 2) return bhh_fail("bh_synchrotron_lut: bad table");
  if (!(lut->log_theta_max > lut->log_theta_min && lut->log_x_max > lut->log_x_min))
    return bhh_fail("bh_synchrotron_lut: empty range");
  // ln of j_nu / (n_e nu_B) = sqrt(3) e^3 / (m_e c^2) * Theta^2 / K_2(1/Theta) * I_M(x),
  // K_2(1/Theta) ~ 2 Theta^2 (src/physics/rte_integrator.h:311-325).
  std::vector<float> tab((size_t)lut->n_theta * lut->n_x);
  if (int rc = bh_synchrotron_lut_host(lut, tab.data())) return rc;
  if (cudaMemcpyAsync(const_cast<void *>(lut->table), tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice,
                      static_cast<cudaStream_t>(stream)) != cudaSuccess ||
      cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess)
    return bhh_fail("bh_synchrotron_lut: copy failed");
  return 0;
}

int bh_kerr_trace_rt(const BH_KerrScene *scene, const BH_GrmhdGrid *grid, const BH_SynchrotronLut *lut,
                     const BH_RtParams *rt, double *i_nu, double *tau, int32_t *cls, int32_t *steps, void *stream) {
  if (!scene || !grid || !lut || !grid->cells || !lut->table) return bhh_fail("bh_kerr_trace_rt: NULL argument");
  if (scene->integrator != BH_INTEGRATOR_DP45) return bhh_fail("bh_kerr_trace_rt: the transfer needs the DP45 integrator");
  BH_RtParams r;
  bh_rt_defaults(&r);
  if (rt) r = *rt;
  if (!(r.nu_hz > 0.0 && r.length_cm > 0.0 && r.ds_max > 0.0)) return bhh_fail("bh_kerr_trace_rt: bad transfer parameters");
  BH_KerrScene sc = *scene;
  const bool mixed = scene->precision == BH_PRECISION_MIXED;
  sc.precision = BH_PRECISION_FP64;  // launch shape of the FP64 kernel; the mixed one sizes its own grid
  BhkImageParams p;
  BhkLaunch L;
  if (bhh_prepare_image_launch(&sc, &p, &L) != 0) return -1;
  if (p.n_pix == 0) return 0;
  BhkRtParams q{};
  q.cells = static_cast<const float *>(grid->cells);
  q.n_r = grid->n_r;
  q.n_th = grid->n_theta;
  q.n_ph = grid->n_phi;
  q.r_min = grid->r_min;
  q.r_max = grid->r_max;
  q.inv_log_range = 1.0 / std::log(grid->r_max / grid->r_min);
  q.lut = static_cast<const float *>(lut->table);
  q.n_lt = lut->n_theta;
  q.n_lx = lut->n_x;
  q.lt0 = lut->log_theta_min;
  q.lt1 = lut->log_theta_max;
  q.lx0 = lut->log_x_min;
  q.lx1 = lut->log_x_max;
  q.nu = r.nu_hz;
  q.length_cm = r.length_cm;
  q.ds_max = r.ds_max;
  q.min_transmit = r.min_transmit;
  unsigned long long *counter = nullptr;
  if (bhh_work_counter(&counter) != 0) return -1;
  if (mixed) {
    if (bhk_trace_rt_mixed(&p, &q, i_nu, tau, cls, steps, counter, stream) != 0)
      return bhh_fail("bh_kerr_trace_rt: k_trace_rt_mixed launch failed");
    return 0;
  }
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (bhk_trace_rt_fp64(&p, &q, i_nu, tau, cls, steps, counter, sms * 4, 128, stream) != 0)
    return bhh_fail(bhk_last_error());
  return 0;
}

}  // extern "C"
