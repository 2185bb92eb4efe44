// legacy.cu - RGBA shading behind the reference renderer's launch ABI
// (include/bh_legacy.h): per-pixel colour from the tracer's outputs, the
// lensing map and the disk emission texture of the Blender bridge.
//
// Colour of thermal emission: a table of the linear-sRGB chromaticity
// (luminance Y = 1) of a blackbody against log2 T, filled by the host
// (legacy_api.cpp) and held in constant memory; linear interpolation in
// log2 T, clamped to the table's ends.
#include <cuda_runtime.h>

#include <cstdint>

#include "image_fp64.cuh"
#include "launch.h"

namespace {

constexpr int kBbMax = 256;
__constant__ float c_bb_rgb[kBbMax * 3];
__constant__ float c_bb_range[3];  // log2 T0, log2 T1, entries

__device__ __forceinline__ float3 blackbody(float t_kelvin) {
  const float n = c_bb_range[2];
  float x = (log2f(fmaxf(t_kelvin, 1.0f)) - c_bb_range[0]) / (c_bb_range[1] - c_bb_range[0]) * (n - 1.0f);
  x = fminf(fmaxf(x, 0.0f), n - 1.0f);
  const int i = min((int)x, (int)n - 2);
  const float w = x - (float)i;
  return make_float3(c_bb_rgb[3 * i] * (1.0f - w) + c_bb_rgb[3 * i + 3] * w,
                     c_bb_rgb[3 * i + 1] * (1.0f - w) + c_bb_rgb[3 * i + 4] * w,
                     c_bb_rgb[3 * i + 2] * (1.0f - w) + c_bb_rgb[3 * i + 5] * w);
}

// ACES filmic curve, the fit of K. Narkowicz (2015), clamped to [0, 1].
__device__ __forceinline__ float aces(float x) {
  const float y = (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
  return fminf(fmaxf(y, 0.0f), 1.0f);
}

__device__ __forceinline__ float lut_u(float r_rs, float lo, float hi) {
  return fminf(fmaxf((r_rs - lo) / fmaxf(hi - lo, 1e-4f), 0.0f), 1.0f);
}

// Disk pixels: observed temperature g T_peak F^(1/4) (F the flux normalized
// to its peak), bolometric intensity adisk_lit g^4 F. Escaped pixels: the
// caller's galaxy cube map, else its equirectangular background, in the
// escape direction, times background_intensity. Captured: black.
__global__ void __launch_bounds__(256) k_legacy_shade(const __grid_constant__ BhkShade s,
                                                      const int32_t *__restrict__ cls,
                                                      const double *__restrict__ r_hit, const double *__restrict__ g,
                                                      const double *__restrict__ flux,
                                                      const float *__restrict__ esc_dir, float4 *__restrict__ rgba) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  const int c = cls[i];
  float3 col = make_float3(0.0f, 0.0f, 0.0f);
  if (c == 1) {
    const float r_rs = 0.5f * (float)r_hit[i];
    float F = (float)flux[i];
    if (s.use_luts && s.tex_emissivity)
      F = fmaxf(0.0f, tex2D<float>((cudaTextureObject_t)s.tex_emissivity, lut_u(r_rs, s.lut_r_min, s.lut_r_max), 0.5f));
    float spectral = 1.0f;
    if (s.use_luts && s.tex_spectral)
      spectral =
          fmaxf(0.0f, tex2D<float>((cudaTextureObject_t)s.tex_spectral, lut_u(r_rs, s.spec_r_min, s.spec_r_max), 0.5f));
    const float gg = s.redshift_enabled ? (float)g[i] : 1.0f;
    const float t = s.t_peak * gg * sqrtf(sqrtf(F));
    const float inten = s.adisk_lit * spectral * (gg * gg) * (gg * gg) * F;
    const float3 bb = blackbody(t);
    col = make_float3(bb.x * inten, bb.y * inten, bb.z * inten);
  } else if (c != 0 && s.background_enabled) {
    const float x0 = esc_dir[i], y0 = esc_dir[s.n + i], z = esc_dir[2 * s.n + i];
    const float x = s.cphi * x0 - s.sphi * y0, y = s.sphi * x0 + s.cphi * y0;  // into the world frame
    float4 b = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (s.tex_galaxy) {
      b = texCubemap<float4>((cudaTextureObject_t)s.tex_galaxy, x, y, z);
    } else if (s.tex_equirect) {
      const float u = atan2f(y, x) * (0.5f / 3.14159265f) + 0.5f;
      const float v = acosf(fminf(fmaxf(z, -1.0f), 1.0f)) * (1.0f / 3.14159265f);
      b = tex2D<float4>((cudaTextureObject_t)s.tex_equirect, u, v);
    }
    col = make_float3(b.x * s.background_intensity, b.y * s.background_intensity, b.z * s.background_intensity);
  }
  rgba[i] = make_float4(col.x, col.y, col.z, 1.0f);
}

// Lensing map channels: R = sqrt(1 - 2 / r_hit) on the disk, 1 escaped, 0
// captured; G = g on the disk, else 1; B = disk hit; A = 1.
__global__ void __launch_bounds__(256) k_legacy_lensing(long long n, const int32_t *__restrict__ cls,
                                                        const double *__restrict__ r_hit,
                                                        const double *__restrict__ g, float4 *__restrict__ rgba) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = cls[i];
  float R = 0.0f, G = 1.0f, B = 0.0f;
  if (c == 1) {
    const double r = r_hit[i];
    R = r > 2.0 ? (float)sqrt(1.0 - 2.0 / r) : 0.0f;
    G = (float)g[i];
    B = 1.0f;
  } else if (c != 0) {
    R = 1.0f;
  }
  rgba[i] = make_float4(R, G, B, 1.0f);
}

// Disk emission texture: row iy at r = r_isco + (r_out - r_isco) iy / height,
// column ix at azimuth phi = 2 pi ix / width. A Keplerian emitter there seen
// by a distant observer at inclination incl in the (x, z) plane emits its
// photon with lambda = -r sin(phi) sin(incl) (straight-line impact
// parameter); g = 1 / (u^t (1 - Omega lambda)) exact for that lambda.
__global__ void __launch_bounds__(256) k_legacy_disk_texture(double a, double r_isco, double r_out,
                                                             double nt_flux_peak, double incl, float t_peak,
                                                             int width, int height, float4 *__restrict__ rgba) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)width * height) return;
  const int ix = (int)(i % width), iy = (int)(i / width);
  const double r = r_isco + (r_out - r_isco) * (double)iy / (double)height;
  const double phi = 6.283185307179586 * (double)ix / (double)width;
  const double F = bhk::nt_flux(r, r_isco, nt_flux_peak);
  const double lam = -r * sin(phi) * sin(incl);
  const double gg = bhk::disk_g(r, a, lam);
  const float tn = (float)sqrt(sqrt(F));
  const float3 bb = blackbody(t_peak * (float)gg * tn);
  const float inten = (float)(gg * gg * gg * gg * F);
  rgba[i] = make_float4(bb.x * inten, bb.y * inten, bb.z * inten, tn);
}

unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

extern "C" int bhk_legacy_set_blackbody(const float *rgb_table, int n, float log2_t0, float log2_t1) {
  if (n < 2 || n > kBbMax || !(log2_t1 > log2_t0)) return -1;
  const float range[3] = {log2_t0, log2_t1, (float)n};
  if (cudaMemcpyToSymbol(c_bb_rgb, rgb_table, sizeof(float) * 3 * n) != cudaSuccess) return -1;
  return cudaMemcpyToSymbol(c_bb_range, range, sizeof(range)) == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_legacy_shade(const BhkShade *s, const int32_t *cls, const double *r_hit, const double *g,
                                const double *flux, const float *esc_dir, float *rgba, void *stream) {
  if (s->n <= 0) return 0;
  k_legacy_shade<<<blocks_for(s->n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      *s, cls, r_hit, g, flux, esc_dir, reinterpret_cast<float4 *>(rgba));
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_legacy_lensing(int64_t n, const int32_t *cls, const double *r_hit, const double *g, float *rgba,
                                  void *stream) {
  if (n <= 0) return 0;
  k_legacy_lensing<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      n, cls, r_hit, g, reinterpret_cast<float4 *>(rgba));
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_legacy_disk_texture(double a, double r_isco, double r_out, double nt_flux_peak, double incl,
                                       float t_peak, int width, int height, float *rgba, void *stream) {
  const long long n = (long long)width * height;
  if (n <= 0) return 0;
  k_legacy_disk_texture<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      a, r_isco, r_out, nt_flux_peak, incl, t_peak, width, height, reinterpret_cast<float4 *>(rgba));
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
