// sky.cuh - the background sky of escaping rays: a cubemap of FP16 texels.
//
// Face order and texel addressing follow the OpenGL cube-map convention:
// faces +X, -X, +Y, -Y, +Z, -Z; for a direction (x, y, z) the face is that of
// the largest |component| (ties go to x, then y), and with ma that magnitude
// the face coordinates (s, t) are
//   +X (-z, -y)   -X (z, -y)   +Y (x, z)   -Y (x, -z)   +Z (x, -y)   -Z (-x, -y),
// u = (s / ma + 1) / 2, v = (t / ma + 1) / 2, texel (floor(u N), floor(v N))
// clamped to [0, N-1]; the texel index is (face N + row) N + column. The
// lookup is nearest-texel, in the escaping ray's direction of motion.
//
// The generated sky (bh_sky_generate) is seeded uniform noise in [0, 1):
// texel k gets the top 24 bits of splitmix64(seed * 0x100000001B3 + k)
// (Steele, Lea & Flood 2014) scaled by 2^-24, rounded to FP16; point stars add
// their brightness to single texels.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#include <cuda_fp16.h>
#define BHSKY_HD __host__ __device__ __forceinline__
#else
#define BHSKY_HD inline
#include <cmath>
#endif

namespace bhsky {

BHSKY_HD uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Noise value of texel k in [0, 1) (exact in FP32: 24 bits).
BHSKY_HD float noise(uint64_t seed, uint64_t k) {
  return (float)(splitmix64(seed * 0x100000001B3ull + k) >> 40) * (1.0f / 16777216.0f);
}

// Texel index of direction (x, y, z) in an N x N-per-face cubemap.
BHSKY_HD long long texel_of(double x, double y, double z, int N) {
  const double ax = fabs(x), ay = fabs(y), az = fabs(z);
  int face;
  double sc, tc, ma;
  if (ax >= ay && ax >= az) {
    ma = ax;
    if (x >= 0.0) {
      face = 0;
      sc = -z;
      tc = -y;
    } else {
      face = 1;
      sc = z;
      tc = -y;
    }
  } else if (ay >= az) {
    ma = ay;
    if (y >= 0.0) {
      face = 2;
      sc = x;
      tc = z;
    } else {
      face = 3;
      sc = x;
      tc = -z;
    }
  } else {
    ma = az;
    if (z >= 0.0) {
      face = 4;
      sc = x;
      tc = -y;
    } else {
      face = 5;
      sc = -x;
      tc = -y;
    }
  }
  const double u = 0.5 * (sc / ma + 1.0);
  const double v = 0.5 * (tc / ma + 1.0);
  int i = (int)(u * (double)N), j = (int)(v * (double)N);
  i = i < 0 ? 0 : (i > N - 1 ? N - 1 : i);
  j = j < 0 ? 0 : (j > N - 1 ? N - 1 : j);
  return ((long long)face * N + j) * N + i;
}

// Cartesian direction of motion of a ray at (r, u = cos theta, phi) moving
// with dr = p_r, du = p_u, dphi (derivatives in any common parameter): the
// sky point it comes from. Unlike the position angles, it changes only at
// O(M b / r^3) along an escaping ray, so where the integrator stopped past
// the escape radius does not matter.
BHSKY_HD void direction_of_motion(double r, double u, double phi, double pr, double pu, double dphi, double& x,
                                  double& y, double& z) {
  const double uc = u < -1.0 ? -1.0 : (u > 1.0 ? 1.0 : u);
  const double st = sqrt((1.0 - uc) * (1.0 + uc));
  const double cp = cos(phi), sp = sin(phi);
  const double dst = st > 1e-300 ? -uc * pu / st : 0.0;  // d(sin theta)
  x = (pr * st + r * dst) * cp - (r * st * dphi) * sp;
  y = (pr * st + r * dst) * sp + (r * st * dphi) * cp;
  z = pr * uc + r * pu;
}

#ifdef __CUDACC__
// Radiance of the nearest texel in the direction of motion (see above).
// Radiance of the texel in direction (x, y, z) (need not be unit).
__device__ __forceinline__ double radiance_dir(const uint16_t* tex, int N, double x, double y, double z) {
  const unsigned short bits = tex[texel_of(x, y, z, N)];
  return (double)__half2float(__ushort_as_half(bits));
}

__device__ __forceinline__ double radiance(const uint16_t* tex, int N, double r, double u, double phi, double pr,
                                           double pu, double dphi) {
  double x, y, z;
  direction_of_motion(r, u, phi, pr, pu, dphi, x, y, z);
  return radiance_dir(tex, N, x, y, z);
}
#endif

}  // namespace bhsky
