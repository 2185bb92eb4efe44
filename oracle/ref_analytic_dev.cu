// Test infrastructure: the reference's own FP32 device helpers
// (src/cuda/device_analytic_kerr.cuh, included unmodified) evaluated over
// arrays on the GPU, so that tests can pin include/bh_analytic.h against
// them. Built by oracle/Makefile into _ref/libbh_ref_analytic_dev.so.
#include <cuda_runtime.h>

#include "cuda/device_analytic_kerr.cuh"

namespace {

__global__ void k_ellpj(int n, const float *u, const float *m, float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d_ellpj(u[i], m[i], out + 3 * i, out + 3 * i + 1, out + 3 * i + 2);
}

__global__ void k_ellint_k(int n, const float *k, float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = d_ellint_K(k[i]);
}

__global__ void k_roots(int n, const float *c, float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float r[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  const int nr = d_quartic_real_roots(c[3 * i], c[3 * i + 1], c[3 * i + 2], r);
  out[5 * i] = (float)nr;
  for (int k = 0; k < 4; ++k) out[5 * i + 1 + k] = r[k];
}

__global__ void k_r_analytic(int n, const float *lam, const float *roots, float lam0, float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = d_kerr_r_analytic(lam[i], roots[4 * i], roots[4 * i + 1], roots[4 * i + 2], roots[4 * i + 3], lam0);
}

__global__ void k_half_period(int n, const float *roots, float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = d_kerr_radial_half_period(roots[4 * i], roots[4 * i + 1], roots[4 * i + 2], roots[4 * i + 3]);
}

__global__ void k_critical(int n, const float *rph, const float *a, float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d_critical_impact_params(rph[i], a[i], out + 2 * i, out + 2 * i + 1);
}

__global__ void k_photon(int n, const float *a, float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[2 * i] = d_prograde_photon_orbit(a[i]);
  out[2 * i + 1] = d_retrograde_photon_orbit(a[i]);
}

// Device copies of host arrays, freed on destruction.
struct Dev {
  float *p = nullptr;
  Dev(const float *h, size_t n) {
    cudaMalloc(&p, n * sizeof(float) + 16);
    if (h) cudaMemcpy(p, h, n * sizeof(float), cudaMemcpyHostToDevice);
  }
  ~Dev() { cudaFree(p); }
};

int finish(float *out_h, const Dev &out, size_t n) {
  if (cudaMemcpy(out_h, out.p, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

unsigned blocks(int n) { return (unsigned)((n + 127) / 128); }

}  // namespace

extern "C" {

int ref_dev_ellpj(int n, const float *u, const float *m, float *out) {
  Dev du(u, n), dm(m, n), o(nullptr, 3 * (size_t)n);
  k_ellpj<<<blocks(n), 128>>>(n, du.p, dm.p, o.p);
  return finish(out, o, 3 * (size_t)n);
}

int ref_dev_ellint_k(int n, const float *k, float *out) {
  Dev dk(k, n), o(nullptr, n);
  k_ellint_k<<<blocks(n), 128>>>(n, dk.p, o.p);
  return finish(out, o, n);
}

int ref_dev_roots(int n, const float *c, float *out) {
  Dev dc(c, 3 * (size_t)n), o(nullptr, 5 * (size_t)n);
  k_roots<<<blocks(n), 128>>>(n, dc.p, o.p);
  return finish(out, o, 5 * (size_t)n);
}

int ref_dev_r_analytic(int n, const float *lam, const float *roots, float lam0, float *out) {
  Dev dl(lam, n), dr(roots, 4 * (size_t)n), o(nullptr, n);
  k_r_analytic<<<blocks(n), 128>>>(n, dl.p, dr.p, lam0, o.p);
  return finish(out, o, n);
}

int ref_dev_half_period(int n, const float *roots, float *out) {
  Dev dr(roots, 4 * (size_t)n), o(nullptr, n);
  k_half_period<<<blocks(n), 128>>>(n, dr.p, o.p);
  return finish(out, o, n);
}

int ref_dev_critical(int n, const float *rph, const float *a, float *out) {
  Dev dr(rph, n), da(a, n), o(nullptr, 2 * (size_t)n);
  k_critical<<<blocks(n), 128>>>(n, dr.p, da.p, o.p);
  return finish(out, o, 2 * (size_t)n);
}

int ref_dev_photon(int n, const float *a, float *out) {
  Dev da(a, n), o(nullptr, 2 * (size_t)n);
  k_photon<<<blocks(n), 128>>>(n, da.p, o.p);
  return finish(out, o, 2 * (size_t)n);
}

}  // extern "C"
