// grmhd.cu - fills the synthetic volumetric medium (include/bh_rt.h):
// a Gaussian torus times exp of a Gaussian random field given as a sum of
// random Fourier modes, one thread per grid node, FP64 arithmetic.
#include <cuda_runtime.h>

#include "launch.h"

namespace {

__global__ void k_grmhd_fill(float4 *__restrict__ cells, int n_r, int n_th, int n_ph, double r_min, double log_range,
                             double r_in, double r_peak, double width, double n0, double theta0, double b0,
                             double amp, const double4 *__restrict__ modes, int n_modes) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)n_r * n_th * n_ph;
  if (idx >= total) return;
  const int k = (int)(idx % n_ph);
  const int j = (int)((idx / n_ph) % n_th);
  const int i = (int)(idx / ((long long)n_ph * n_th));
  const double r = r_min * exp(log_range * (double)i / (double)(n_r - 1));
  const double th = ((double)j + 0.5) * (3.141592653589793 / (double)n_th);
  const double ph = (double)k * (6.283185307179586 / (double)n_ph);
  const double st = sin(th), ct = cos(th);
  const double x = r * st * cos(ph), y = r * st * sin(ph), z = r * ct;
  double f = 0.0;
  for (int m = 0; m < n_modes; ++m) {
    const double4 md = modes[m];
    f += cos(md.x * x + md.y * y + md.z * z + md.w);
  }
  f *= amp;
  const double R = r * st;
  double t = exp(-((R - r_peak) * (R - r_peak) + z * z) / (2.0 * width * width));
  if (r < r_in) t *= exp(-(r_in - r) * (r_in - r));
  const double n = n0 * t * exp(f);
  cells[idx] = make_float4((float)n, (float)(theta0 * r_peak / r), (float)(b0 * sqrt(n / n0)), 0.0f);
}

}  // namespace

extern "C" int bhk_grmhd_fill(float *cells, int n_r, int n_th, int n_ph, double r_min, double r_max, double r_in,
                              double r_peak, double width, double n0, double theta0, double b0, double amp,
                              const double *modes, int n_modes, void *stream) {
  const long long total = (long long)n_r * n_th * n_ph;
  if (total <= 0) return 0;
  k_grmhd_fill<<<(unsigned)((total + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<float4 *>(cells), n_r, n_th, n_ph, r_min, log(r_max / r_min), r_in, r_peak, width, n0, theta0,
      b0, amp, reinterpret_cast<const double4 *>(modes), n_modes);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
