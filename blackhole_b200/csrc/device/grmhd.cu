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

// One packed frame sampled at (r, theta, phi) the way the reference renderer's
// 3-D texture is (linear filtering, texel centres at +1/2): r clamped to the
// packed range, theta clamped, phi periodic. FP64 weights, float samples.
__device__ __forceinline__ void packed_sample(const float4 *__restrict__ f, int nr, int nt, int np, double fr,
                                              double ft, double fp, double (&acc)[2]) {
  fr = fmin(fmax(fr, 0.0), (double)(nr - 1));
  ft = fmin(fmax(ft, 0.0), (double)(nt - 1));
  const int i0 = min((int)floor(fr), max(nr - 2, 0)), j0 = min((int)floor(ft), max(nt - 2, 0));
  const int i1 = min(i0 + 1, nr - 1), j1 = min(j0 + 1, nt - 1);
  const double tr = fr - (double)i0, tt = ft - (double)j0;
  const double fl = floor(fp);
  const double tp = fp - fl;
  int k0 = (int)fmod(fl, (double)np);
  if (k0 < 0) k0 += np;
  const int k1 = (k0 + 1) % np;
  acc[0] = acc[1] = 0.0;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        const double w = (di ? tr : 1.0 - tr) * (dj ? tt : 1.0 - tt) * (dk ? tp : 1.0 - tp);
        const float4 v = __ldg(f + ((long long)(di ? i1 : i0) * nt + (dj ? j1 : j0)) * np + (dk ? k1 : k0));
        acc[0] += w * (double)v.x;
        acc[1] += w * (double)v.y;
      }
}

// Grid node (i, j, k) of the emitting medium from one or two packed frames:
// rho and u sampled, blended, converted (include/bh_rt.h, BH_PackedConversion).
__global__ void k_grmhd_from_packed(float4 *__restrict__ cells, int n_r, int n_th, int n_ph, double r_min,
                                    double log_range, const float4 *__restrict__ left,
                                    const float4 *__restrict__ right, double alpha, int pnr, int pnt, int pnp,
                                    double pr_min, double pr_max, double n_scale, double theta_scale,
                                    double b_scale) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)n_r * n_th * n_ph;
  if (idx >= total) return;
  const int k = (int)(idx % n_ph);
  const int j = (int)((idx / n_ph) % n_th);
  const int i = (int)(idx / ((long long)n_ph * n_th));
  const double r = r_min * exp(log_range * (double)i / (double)(n_r - 1));
  const double th = ((double)j + 0.5) * (3.141592653589793 / (double)n_th);
  const double ph = (double)k * (6.283185307179586 / (double)n_ph);
  const double fr = (r - pr_min) / (pr_max - pr_min) * (double)pnr - 0.5;
  const double ft = th * (1.0 / 3.141592653589793) * (double)pnt - 0.5;
  const double fp = ph * (1.0 / 6.283185307179586) * (double)pnp - 0.5;
  double a[2];
  packed_sample(left, pnr, pnt, pnp, fr, ft, fp, a);
  if (right) {
    double b[2];
    packed_sample(right, pnr, pnt, pnp, fr, ft, fp, b);
    a[0] += alpha * (b[0] - a[0]);
    a[1] += alpha * (b[1] - a[1]);
  }
  const double rho = a[0], u = a[1];
  const double n = rho > 0.0 ? n_scale * rho : 0.0;
  const double te = rho > 0.0 ? theta_scale * u / rho : 0.0;
  const double bb = b_scale * sqrt(u > 0.0 ? u : 0.0);
  cells[idx] = make_float4((float)n, (float)te, (float)bb, 0.0f);
}

}  // namespace

extern "C" int bhk_grmhd_from_packed(float *cells, int n_r, int n_th, int n_ph, double r_min, double r_max,
                                     const float *left, const float *right, double alpha, int pnr, int pnt, int pnp,
                                     double pr_min, double pr_max, double n_scale, double theta_scale,
                                     double b_scale, void *stream) {
  const long long total = (long long)n_r * n_th * n_ph;
  if (total <= 0) return 0;
  k_grmhd_from_packed<<<(unsigned)((total + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<float4 *>(cells), n_r, n_th, n_ph, r_min, log(r_max / r_min),
      reinterpret_cast<const float4 *>(left), reinterpret_cast<const float4 *>(right), alpha, pnr, pnt, pnp, pr_min,
      pr_max, n_scale, theta_scale, b_scale);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

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
