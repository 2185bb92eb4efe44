// physics_host.cpp - HOST-buffer forms of the batched src/physics drop-ins
// (bh_kerr_potentials_host, bh_kerr_step_mino_host, bh_kerr_trace_rays_host).
//
// Callers that hold their states in host memory -- the reference's own
// physics::KerrRaytracer callers, through include/bh_physics_compat.hpp --
// get the same GPU kernels without touching CUDA: inputs are staged into a
// grow-only device buffer of the calling thread, the kernel runs on that
// thread's stream, and the call returns once the outputs are back in host
// memory.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "../../../include/bh_kerr.h"
#include "../device/launch.h"
#include "dalloc.hpp"

namespace {

struct Staging {
  char *dev = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  int device = -1;
};
thread_local Staging g_stage;

int cuda_fail(cudaError_t e, const char *what) {
  char msg[256];
  std::snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
  return bhh_fail(msg);
}

// A device buffer of at least `bytes` and a stream, both of the calling thread
// on the current device.
int stage(size_t bytes, char **base, cudaStream_t *st) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (g_stage.device != dev) {
    g_stage = Staging{};
    g_stage.device = dev;
  }
  if (!g_stage.stream) {
    e = cudaStreamCreateWithFlags(&g_stage.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
  }
  if (g_stage.bytes < bytes) {
    if (g_stage.dev) cudaFree(g_stage.dev);
    g_stage.dev = nullptr;
    g_stage.bytes = 0;
    e = bhh_malloc(&g_stage.dev, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(physics staging)");
    g_stage.bytes = bytes;
  }
  *base = g_stage.dev;
  *st = g_stage.stream;
  return 0;
}

// Consecutive slices of the staging buffer, 256-byte aligned.
struct Carver {
  char *base;
  size_t off = 0;
  template <class T>
  T *take(int64_t n) {
    T *p = reinterpret_cast<T *>(base + off);
    off += (size_t(n) * sizeof(T) + 255) & ~size_t(255);
    return p;
  }
};

size_t slice(int64_t n, size_t elem) { return (size_t(n) * elem + 255) & ~size_t(255); }

int h2d(void *d, const void *h, int64_t n, size_t elem, cudaStream_t st) {
  const cudaError_t e = cudaMemcpyAsync(d, h, size_t(n) * elem, cudaMemcpyHostToDevice, st);
  return e == cudaSuccess ? 0 : cuda_fail(e, "cudaMemcpyAsync(H2D)");
}

int d2h(void *h, const void *d, int64_t n, size_t elem, cudaStream_t st) {
  if (!h) return 0;
  const cudaError_t e = cudaMemcpyAsync(h, d, size_t(n) * elem, cudaMemcpyDeviceToHost, st);
  return e == cudaSuccess ? 0 : cuda_fail(e, "cudaMemcpyAsync(D2H)");
}

int finish(cudaStream_t st, const char *what) {
  const cudaError_t e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? 0 : cuda_fail(e, what);
}

}  // namespace

extern "C" {

int bh_kerr_potentials_host(int64_t n, const double *r, const double *theta, double mass, double a,
                            BH_KerrConstsSoA c, double *rp, double *drp, double *tp, double *dtp) {
  if (n < 0) return bhh_fail("negative count");
  if (n == 0) return 0;
  if (!r || !theta || !c.e || !c.lz || !c.q) return bhh_fail("NULL input array");
  char *base = nullptr;
  cudaStream_t st = nullptr;
  if (stage(9 * slice(n, sizeof(double)), &base, &st) != 0) return -1;
  Carver cv{base};
  double *dr = cv.take<double>(n), *dth = cv.take<double>(n);
  double *de = cv.take<double>(n), *dlz = cv.take<double>(n), *dq = cv.take<double>(n);
  double *o[4] = {cv.take<double>(n), cv.take<double>(n), cv.take<double>(n), cv.take<double>(n)};
  double *host_out[4] = {rp, drp, tp, dtp};
  if (h2d(dr, r, n, 8, st) || h2d(dth, theta, n, 8, st) || h2d(de, c.e, n, 8, st) || h2d(dlz, c.lz, n, 8, st) ||
      h2d(dq, c.q, n, 8, st))
    return -1;
  const BH_KerrConstsSoA dc{de, dlz, dq};
  if (bh_kerr_potentials(n, dr, dth, mass, a, dc, rp ? o[0] : nullptr, drp ? o[1] : nullptr, tp ? o[2] : nullptr,
                         dtp ? o[3] : nullptr, st) != 0)
    return -1;
  for (int k = 0; k < 4; ++k)
    if (d2h(host_out[k], o[k], n, 8, st)) return -1;
  return finish(st, "bh_kerr_potentials_host");
}

int bh_kerr_step_mino_host(int64_t n, BH_KerrStateSoA s, double mass, double a, BH_KerrConstsSoA c,
                           const double *dlam, double dlam_scalar) {
  if (n < 0) return bhh_fail("negative count");
  if (n == 0) return 0;
  if (!s.r || !s.theta || !s.phi || !s.t || !s.sign_r || !s.sign_theta || !c.e || !c.lz || !c.q)
    return bhh_fail("NULL state or constant array");
  char *base = nullptr;
  cudaStream_t st = nullptr;
  if (stage(10 * slice(n, sizeof(double)), &base, &st) != 0) return -1;
  Carver cv{base};
  double *f[6];
  double *const hf[6] = {s.r, s.theta, s.phi, s.t, s.sign_r, s.sign_theta};
  for (int k = 0; k < 6; ++k) f[k] = cv.take<double>(n);
  double *de = cv.take<double>(n), *dlz = cv.take<double>(n), *dq = cv.take<double>(n);
  double *dl = cv.take<double>(n);
  for (int k = 0; k < 6; ++k)
    if (h2d(f[k], hf[k], n, 8, st)) return -1;
  if (h2d(de, c.e, n, 8, st) || h2d(dlz, c.lz, n, 8, st) || h2d(dq, c.q, n, 8, st)) return -1;
  if (dlam && h2d(dl, dlam, n, 8, st)) return -1;
  const BH_KerrStateSoA ds{f[0], f[1], f[2], f[3], f[4], f[5]};
  const BH_KerrConstsSoA dc{de, dlz, dq};
  if (bh_kerr_step_mino(n, ds, mass, a, dc, dlam ? dl : nullptr, dlam_scalar, st) != 0) return -1;
  for (int k = 0; k < 6; ++k)
    if (d2h(hf[k], f[k], n, 8, st)) return -1;
  return finish(st, "bh_kerr_step_mino_host");
}

int bh_kerr_trace_rays_host(int64_t n, BH_KerrStateSoA s, BH_KerrConstsSoA c, const BH_KerrRaytracerParams *p,
                            int32_t *status, int32_t *steps, double *dist, double *rf, double *thf, double *phf,
                            double *redshift) {
  if (!p) return bhh_fail("params is NULL");
  if (n < 0) return bhh_fail("negative count");
  if (n == 0) return 0;
  if (!s.r || !s.theta || !s.phi || !s.t || !s.sign_r || !s.sign_theta || !c.e || !c.lz || !c.q)
    return bhh_fail("NULL state or constant array");
  char *base = nullptr;
  cudaStream_t st = nullptr;
  if (stage(14 * slice(n, sizeof(double)) + 2 * slice(n, sizeof(int32_t)), &base, &st) != 0) return -1;
  Carver cv{base};
  double *f[6];
  const double *const hf[6] = {s.r, s.theta, s.phi, s.t, s.sign_r, s.sign_theta};
  for (int k = 0; k < 6; ++k) f[k] = cv.take<double>(n);
  double *de = cv.take<double>(n), *dlz = cv.take<double>(n), *dq = cv.take<double>(n);
  double *od[5];
  for (int k = 0; k < 5; ++k) od[k] = cv.take<double>(n);
  int32_t *oi[2] = {cv.take<int32_t>(n), cv.take<int32_t>(n)};
  for (int k = 0; k < 6; ++k)
    if (h2d(f[k], hf[k], n, 8, st)) return -1;
  if (h2d(de, c.e, n, 8, st) || h2d(dlz, c.lz, n, 8, st) || h2d(dq, c.q, n, 8, st)) return -1;
  const BH_KerrStateSoA ds{f[0], f[1], f[2], f[3], f[4], f[5]};
  const BH_KerrConstsSoA dc{de, dlz, dq};
  double *const hd[5] = {dist, rf, thf, phf, redshift};
  int32_t *const hi[2] = {status, steps};
  if (bh_kerr_trace_rays(n, ds, dc, p, status ? oi[0] : nullptr, steps ? oi[1] : nullptr, dist ? od[0] : nullptr,
                         rf ? od[1] : nullptr, thf ? od[2] : nullptr, phf ? od[3] : nullptr,
                         redshift ? od[4] : nullptr, st) != 0)
    return -1;
  for (int k = 0; k < 2; ++k)
    if (d2h(hi[k], oi[k], n, 4, st)) return -1;
  for (int k = 0; k < 5; ++k)
    if (d2h(hd[k], od[k], n, 8, st)) return -1;
  return finish(st, "bh_kerr_trace_rays_host");
}

}  // extern "C"
