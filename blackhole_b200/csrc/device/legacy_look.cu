// legacy_look.cu - the reference renderer's own look behind its launch ABI
// (include/bh_legacy.h, BH_SHADING_REFERENCE): the colour of each pixel from
// this library's trace of it, computed the way the reference's shader
// computes it from its own (src/cuda/device_physics.cuh: d_shade_hit
// :1841-1928, d_disk_color :1079-1239, d_background_color :1522-1565,
// d_shape_escaped_background :1634-1763, d_sample_grmhd :1789-1829). Existing
// callers of bh_launch_geodesic_kernel / bhCuda* / bhbCuda* get the picture
// they were tuned for; the geometry under it -- where a ray meets the disk,
// how far it passes from the hole, where it leaves -- is the Kerr geodesic of
// the mixed-precision tracer instead of the reference's FP32 Euler steps.
//
// The reference's world frame: Cartesian (x, y, z) = r (sin t cos p, sin t
// sin p, cos t) of the Boyer-Lindquist (r, t, p) in the caller's length unit
// (rs = 2 M of them), spin axis +z, the disk in z = 0. Its shader mixes in a
// y-up convention (velocity, flow and sector directions about the y axis,
// grazing and mid-plane terms from y); those terms are kept as they are,
// because they are part of the look. Per pixel the tracer gives: the class,
// the first disk crossing (r, phi), the escape position (theta, phi at the
// escape radius) and the closest approach (r, cos theta, phi); azimuths are
// measured from the camera's, rotated here into the world frame.
#include <cuda_runtime.h>

#include <cstdint>

#include "launch.h"
#include "vol.cuh"

namespace {

constexpr float kEps = 1.0e-6f;  // the reference shader's guard value
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kInvTwoPi = 0.15915494309189533577f;

struct V {
  float x, y, z;
};
__device__ __forceinline__ V v3(float x, float y, float z) { return V{x, y, z}; }
__device__ __forceinline__ V add(V a, V b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V sub(V a, V b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V mul(V a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V hadamard(V a, V b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V cross(V a, V b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V unit(V a) { return mul(a, rsqrtf(fmaxf(dot(a, a), 1.0e-12f))); }
__device__ __forceinline__ V mix(V a, V b, float t) {
  return v3(fmaf(t, b.x - a.x, a.x), fmaf(t, b.y - a.y, a.y), fmaf(t, b.z - a.z, a.z));
}
__device__ __forceinline__ float clamp01(float x) { return fmaxf(0.0f, fminf(x, 1.0f)); }
// Hermite smoothstep of x from e0 to e1 (a reversed pair degenerates to a
// step at e0, as in the reference shader).
__device__ __forceinline__ float smooth(float e0, float e1, float x) {
  const float t = clamp01((x - e0) / fmaxf(e1 - e0, kEps));
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ float luma(V c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

// sRGB-encoded texel channel to linear light (IEC 61966-2-1).
__device__ __forceinline__ float srgb_linear(float c) {
  c = clamp01(c);
  return c <= 0.04045f ? c * (1.0f / 12.92f) : powf((c + 0.055f) * (1.0f / 1.055f), 2.4f);
}
__device__ __forceinline__ V srgb_linear(float4 s) { return v3(srgb_linear(s.x), srgb_linear(s.y), srgb_linear(s.z)); }

// Rodrigues rotation of v about `axis` by `angle`.
__device__ __forceinline__ V rotate(V v, V axis, float angle) {
  const V n = unit(axis);
  const float c = cosf(angle), s = sinf(angle);
  return add(add(mul(v, c), mul(cross(n, v), s)), mul(n, dot(n, v) * (1.0f - c)));
}

// A radial lookup table of 1 x N texels over [lo, hi] (in rs), sampled at r / rs.
__device__ __forceinline__ float table(unsigned long long tex, float r_rs, float lo, float hi, float min_span) {
  const float u = clamp01((r_rs - lo) / fmaxf(hi - lo, min_span));
  return tex2D<float>((cudaTextureObject_t)tex, u, 0.5f);
}

// Integer hash of a cell of the directional star grid, in [0, 1): the
// reference's multiply-xorshift mix, so the same cells hold stars.
__device__ __forceinline__ float cell_hash(V p) {
  const unsigned ix = (unsigned)((int)p.x + 16384), iy = (unsigned)((int)p.y + 16384),
                 iz = (unsigned)((int)p.z + 16384);
  unsigned h = ix * 1664525u ^ iy * 22695477u ^ iz * 1013904223u;
  h ^= h >> 16;
  h *= 0x45d9f3bu;
  h ^= h >> 16;
  return (float)(h >> 9) * (1.0f / 8388608.0f);
}

// The background's yaw about +y and pitch about the camera's right axis.
__device__ __forceinline__ V background_frame(const BhkLook &L, V d) {
  if (fabsf(L.bg_yaw) > kEps) d = rotate(d, v3(0.0f, 1.0f, 0.0f), L.bg_yaw);
  if (fabsf(L.bg_pitch) > kEps) d = rotate(d, v3(L.cam_right[0], L.cam_right[1], L.cam_right[2]), L.bg_pitch);
  return d;
}

// One texel of the galaxy cube map stored as a 6-layer 2D texture (layers
// +X, -X, +Y, -Y, +Z, -Z; OpenGL's face selection and (s, t)). The
// reference turns the direction by the background's yaw and pitch here a
// second time (its caller already did); kept, since the image depends on it.
__device__ V galaxy_texel(const BhkLook &L, V d) {
  if (fabsf(L.bg_yaw) > kEps) {
    const float cy = cosf(L.bg_yaw), sy = sinf(L.bg_yaw);
    d = v3(d.x * cy + d.z * sy, d.y, -d.x * sy + d.z * cy);
  }
  if (fabsf(L.bg_pitch) > kEps) {
    const float cp = cosf(L.bg_pitch), sp = sinf(L.bg_pitch);
    d = v3(d.x, d.y * cp - d.z * sp, d.y * sp + d.z * cp);
  }
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  float u, w;
  int layer;
  if (ax >= ay && ax >= az) {
    const float sc = 1.0f / fmaxf(ax, kEps);
    layer = d.x > 0.0f ? 0 : 1;
    u = (d.x > 0.0f ? -d.z : d.z) * sc;
    w = -d.y * sc;
  } else if (ay >= ax && ay >= az) {
    const float sc = 1.0f / fmaxf(ay, kEps);
    layer = d.y > 0.0f ? 2 : 3;
    u = d.x * sc;
    w = (d.y > 0.0f ? d.z : -d.z) * sc;
  } else {
    const float sc = 1.0f / fmaxf(az, kEps);
    layer = d.z > 0.0f ? 4 : 5;
    u = (d.z > 0.0f ? d.x : -d.x) * sc;
    w = -d.y * sc;
  }
  const float4 s = tex2DLayered<float4>((cudaTextureObject_t)L.tex_galaxy, 0.5f * (u + 1.0f), 0.5f * (w + 1.0f), layer);
  return srgb_linear(s);
}

// The galaxy, box-filtered over five directions within the filter radius.
__device__ V galaxy(const BhkLook &L, V n) {
  const float rad = fmaxf(L.bg_filter, 0.0f);
  V sum = galaxy_texel(L, background_frame(L, n));
  if (rad <= kEps) return sum;
  const V up = fabsf(n.y) < 0.9f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
  const V t = unit(cross(up, n)), b = unit(cross(n, t));
  const V offs[4] = {mul(t, rad), mul(t, -rad), mul(b, rad), mul(b, -rad)};
  for (int k = 0; k < 4; ++k) sum = add(sum, galaxy_texel(L, background_frame(L, unit(add(n, offs[k])))));
  return mul(sum, 0.2f);
}

__device__ __forceinline__ float fract(float x) { return x - floorf(x); }

// Equirectangular (u = atan2(z, x) / 2 pi + 1/2, v = asin(y) / pi + 1/2) at
// level 0, or the caller's weighted layers of it (offset, scale, weight,
// level bias, each with a 9-tap tent filter within the filter radius);
// `weight` returns the layers' total weight (0: no layer).
__device__ V equirect(const BhkLook &L, V n0, bool layered, float &weight) {
  weight = 0.0f;
  const V n = unit(background_frame(L, unit(n0)));
  const float bu = atan2f(n.z, n.x) * kInvTwoPi + 0.5f;
  const float bv = asinf(fmaxf(-1.0f, fminf(n.y, 1.0f))) * kInvPi + 0.5f;
  const cudaTextureObject_t tex = (cudaTextureObject_t)L.tex_equirect;
  if (!layered) return srgb_linear(tex2DLod<float4>(tex, bu, bv, 0.0f));
  const float rad = fmaxf(L.bg_filter, 0.0f);
  V acc = v3(0.0f, 0.0f, 0.0f);
  for (int i = 0; i < 3; ++i) {
    const float ox = L.bg_layers[4 * i], oy = L.bg_layers[4 * i + 1], sc = L.bg_layers[4 * i + 2];
    const float wt = L.bg_layers[4 * i + 3];
    if (wt <= 0.0f || sc <= kEps) continue;
    const float u = fract((bu - 0.5f) * sc + 0.5f + ox), v = fract((bv - 0.5f) * sc + 0.5f + oy);
    const float lod = fmaxf(L.bg_lod_bias[i], 0.0f);
    const float lr = rad * (1.0f + 1.5f * lod);
    float4 s = tex2DLod<float4>(tex, u, v, lod);
    if (lr > kEps) {
      const float dr = lr * 0.70710678f;
      const float4 a0 = tex2DLod<float4>(tex, fract(u + lr), v, lod), a1 = tex2DLod<float4>(tex, fract(u - lr), v, lod);
      const float4 b0 = tex2DLod<float4>(tex, u, fminf(v + lr, 1.0f), lod);
      const float4 b1 = tex2DLod<float4>(tex, u, fmaxf(v - lr, 0.0f), lod);
      const float4 c0 = tex2DLod<float4>(tex, fract(u + dr), fminf(v + dr, 1.0f), lod);
      const float4 c1 = tex2DLod<float4>(tex, fract(u + dr), fmaxf(v - dr, 0.0f), lod);
      const float4 c2 = tex2DLod<float4>(tex, fract(u - dr), fminf(v + dr, 1.0f), lod);
      const float4 c3 = tex2DLod<float4>(tex, fract(u - dr), fmaxf(v - dr, 0.0f), lod);
      s.x = (4.0f * s.x + 2.0f * (a0.x + a1.x + b0.x + b1.x) + c0.x + c1.x + c2.x + c3.x) * (1.0f / 16.0f);
      s.y = (4.0f * s.y + 2.0f * (a0.y + a1.y + b0.y + b1.y) + c0.y + c1.y + c2.y + c3.y) * (1.0f / 16.0f);
      s.z = (4.0f * s.z + 2.0f * (a0.z + a1.z + b0.z + b1.z) + c0.z + c1.z + c2.z + c3.z) * (1.0f / 16.0f);
    }
    acc = add(acc, mul(srgb_linear(s), wt));
    weight += wt;
  }
  return weight > 0.0f ? mul(acc, 1.0f / weight) : acc;
}

// The sky in world direction `dir`: turned about +y by the scene time, then
// the equirectangular texture (its layers, else the plain lookup), else the
// galaxy cube map, else the procedural field of point stars plus a faint
// ambient glow, times the background intensity.
__device__ V sky_color(const BhkLook &L, V dir) {
  if (!L.background_enabled) return v3(0.0f, 0.0f, 0.0f);
  const V n = rotate(unit(dir), v3(0.0f, 1.0f, 0.0f), L.time_sec);
  if (L.tex_equirect) {
    float w = 0.0f;
    V s = equirect(L, n, true, w);
    if (w <= 0.0f) s = equirect(L, n, false, w);
    return mul(s, L.bg_intensity);
  }
  if (L.tex_galaxy) return mul(galaxy(L, n), L.bg_intensity);
  const V cell = v3(floorf(n.x * 300.0f), floorf(n.y * 300.0f), floorf(n.z * 300.0f));
  const float h = cell_hash(cell);
  float star = 0.0f;
  if (h > 0.978f) {
    const float s = (h - 0.978f) * (1.0f / 0.022f), s2 = s * s, s4 = s2 * s2;
    star = s4 * s4;
  }
  const float temp = cell_hash(add(cell, v3(1.0f, 2.0f, 3.0f)));
  const V col = temp > 0.7f ? v3(0.8f, 0.85f, 1.0f) : (temp > 0.3f ? v3(1.0f, 0.95f, 0.85f) : v3(1.0f, 0.7f, 0.5f));
  return add(mul(col, star * L.bg_intensity), mul(v3(0.002f, 0.002f, 0.008f), L.bg_intensity));
}

// sqrt(1 - rs / r): the shader's static-observer redshift factor.
__device__ __forceinline__ float static_factor(float r, float rs) {
  if (r <= rs) return 0.0f;
  const float f = 1.0f - rs / r;
  return f <= 0.0f ? 0.0f : sqrtf(f);
}

// Redshift z at radius r: the caller's table, else 1 / static_factor - 1.
__device__ __forceinline__ float redshift_z(const BhkLook &L, float r) {
  if (L.use_luts && L.tex_redshift)
    return table(L.tex_redshift, r / fmaxf(L.rs, kEps), L.z_r_min, L.z_r_max, 1e-4f);
  return 1.0f / fmaxf(static_factor(r, L.rs), kEps) - 1.0f;
}

// Alignment, mapped to [0, 1], of `toward` with the flow about the spin (the
// shader's y axis) at point p; and the weight of the spin's effect.
__device__ __forceinline__ float flow_alignment(const BhkLook &L, V p, V toward) {
  const V axis = v3(0.0f, L.spin >= 0.0f ? 1.0f : -1.0f, 0.0f);
  return 0.5f + 0.5f * dot(unit(cross(axis, unit(p))), toward);
}
__device__ __forceinline__ float spin_weight(const BhkLook &L) {
  const float t = clamp01((fabsf(L.spin) - 0.05f) / fmaxf(0.85f - 0.05f, kEps));
  return t * t * (3.0f - 2.0f * t);
}

// The escaped sky darkened by the redshift of the closest approach and, for
// rays that passed within 5 rs, the shader's sector shaping about the hole.
__device__ V shape_sky(const BhkLook &L, V sky, float r_min, V closest) {
  const float rs = L.rs;
  if (L.redshift_enabled && r_min < 10.0f * rs) {
    const float opz = 1.0f + redshift_z(L, r_min);
    sky = mul(sky, 1.0f / fmaxf(opz * opz * opz, kEps));
  }
  if (!(r_min < 5.0f * rs)) return sky;
  const V cam = v3(L.cam_pos[0], L.cam_pos[1], L.cam_pos[2]);
  const float flow = flow_alignment(L, closest, unit(sub(cam, closest)));
  const float near = powf(clamp01(1.0f - (r_min - rs) / fmaxf(3.0f * rs, kEps)), 1.55f);
  const float bright = smooth(0.83f, 0.985f, flow), rim = smooth(0.91f, 0.995f, flow);
  const float adjacent = smooth(0.76f, 0.95f, flow) * (1.0f - bright);
  const float broad = smooth(0.46f, 0.84f, flow) * (1.0f - adjacent) * (1.0f - bright);
  const float base_luma = luma(sky);
  sky = mul(sky, (1.0f + (0.08f - 1.0f) * near * (1.0f - bright * 0.95f)) *
                     (1.0f + near * (0.40f * bright + 0.06f * rim)));
  const float l1 = luma(sky);
  const float gain = fmaxf(l1 - base_luma, 0.0f);
  sky = add(sky, mul(sky, near * (-0.50f + 0.70f * bright) * fmaxf(fminf(l1 - 0.03f, 1.0f), 0.0f)));
  const V tint = mix(v3(0.84f, 0.80f, 0.96f), v3(1.06f, 0.98f, 0.88f), rim);
  sky = mix(sky, hadamard(sky, tint), near * (0.012f + 0.05f * rim));
  sky = mul(sky, 1.0f - 0.28f * near * (1.0f - bright) * smooth(0.025f, 0.18f, l1));
  sky = mul(sky, 1.0f - 0.24f * near * (1.0f - bright) * smooth(0.01f, 0.08f, l1));
  sky = mul(sky, 1.0f - 0.16f * near * (1.0f - bright) * smooth(0.018f, 0.12f, l1));
  const float arc_gain = smooth(0.008f, 0.045f, gain);
  sky = mul(sky, 1.0f - 0.27f * near * adjacent * smooth(0.016f, 0.13f, l1) * (1.0f + 0.35f * arc_gain));
  sky = mul(sky, 1.0f - 0.13f * near * broad * smooth(0.014f, 0.10f, l1));
  return sky;
}

// The ring glow of rays that passed near the photon sphere (1.5 rs).
__device__ V ring_glow(const BhkLook &L, V sky, float r_min, V closest) {
  const float rs = L.rs;
  const float dist = fabsf(r_min - 1.5f * rs);
  const float x = fmaxf(0.0f, 1.0f - dist / fmaxf(0.5f * rs, kEps));
  const float glow = x * x * x;
  if (!(glow > 0.0f)) return sky;
  const V cam = v3(L.cam_pos[0], L.cam_pos[1], L.cam_pos[2]);
  const float flow = flow_alignment(L, closest, unit(sub(cam, closest)));
  const float aniso = 1.0f + ((0.72f + (1.65f - 0.72f) * flow) - 1.0f) * spin_weight(L);
  const float inten = powf(glow * 0.22f * fmaxf(L.glow_strength, 0.0f), 1.08f) * aniso;
  const V col = mix(v3(1.06f, 0.86f, 0.58f), v3(1.22f, 1.0f, 0.78f), smooth(0.09f * rs, 0.0f, dist));
  return v3(fminf(sky.x + col.x * inten, 100.0f), fminf(sky.y + col.y * inten, 100.0f),
            fminf(sky.z + col.z * inten, 100.0f));
}

// The disk at world point hp: the shader's temperature ramp, tints,
// approximate Doppler beaming and colour shift, sector shaping, static
// redshift dimming, and the GRMHD emissivity where a grid is registered.
__device__ V disk_color(const BhkLook &L, V hp, float &inten) {
  const float rs = L.rs;
  const float r = sqrtf(fmaf(hp.x, hp.x, hp.y * hp.y));
  const float r_in = L.isco, r_out = 4.0f * L.isco;
  const float radial = clamp01((r - r_in) / fmaxf(r_out - r_in, kEps));
  float flux;
  if (L.use_luts && L.tex_emissivity) {
    flux = fmaxf(0.0f, table(L.tex_emissivity, r / fmaxf(rs, kEps), L.lut_r_min, L.lut_r_max, 1e-4f));
  } else {
    const float x = r_in / fmaxf(r, kEps);
    flux = fmaxf(0.0f, x * x * x * (1.0f - sqrtf(x)));
  }
  const float tn = sqrtf(sqrtf(flux));
  // temperature ramp: linear between six knots
  V c;
  if (tn > 0.85f) {
    c = mix(v3(1.0f, 0.90f, 0.60f), v3(1.0f, 0.97f, 0.90f), (tn - 0.85f) / 0.15f);
  } else if (tn > 0.65f) {
    c = mix(v3(1.0f, 0.70f, 0.20f), v3(1.0f, 0.90f, 0.60f), (tn - 0.65f) / 0.20f);
  } else if (tn > 0.45f) {
    c = mix(v3(1.0f, 0.45f, 0.04f), v3(1.0f, 0.70f, 0.20f), (tn - 0.45f) / 0.20f);
  } else if (tn > 0.25f) {
    c = mix(v3(0.90f, 0.15f, 0.00f), v3(1.0f, 0.45f, 0.04f), (tn - 0.25f) / 0.20f);
  } else if (tn > 0.10f) {
    c = mix(v3(0.50f, 0.03f, 0.00f), v3(0.90f, 0.15f, 0.00f), (tn - 0.10f) / 0.15f);
  } else {
    c = mix(v3(0.10f, 0.00f, 0.00f), v3(0.50f, 0.03f, 0.00f), tn / 0.10f);
  }
  float spectral = 1.0f;
  if (L.use_luts && L.tex_spectral)
    spectral = fmaxf(0.0f, table(L.tex_spectral, r / fmaxf(rs, kEps), L.spec_r_min, L.spec_r_max, 1e-4f));
  c = hadamard(c, mix(v3(1.35f, 0.78f, 0.28f), v3(0.92f, 0.86f, 0.78f), sqrtf(radial)));

  const V cam = v3(L.cam_pos[0], L.cam_pos[1], L.cam_pos[2]);
  const V ray = unit(sub(hp, cam)), view = mul(ray, -1.0f);
  const V vel = unit(v3(-hp.z, 0.0f, hp.x));
  inten = flux * 2.0f * L.adisk_lit * spectral;
  const float doppler = 1.0f + dot(vel, unit(ray)) * 0.65f * L.doppler_strength;
  inten *= doppler * doppler * doppler;

  const float sv = flow_alignment(L, hp, view);
  c = mul(c, 1.0f + ((0.82f + (1.55f - 0.82f) * sv) - 1.0f) * spin_weight(L));
  const float inner = powf(fmaxf(0.0f, 1.0f - radial), 0.72f);
  const float bright = smooth(0.83f, 0.985f, sv), rim = smooth(0.91f, 0.997f, sv);
  const float counter = smooth(0.20f, 0.54f, sv);
  inten *= (1.0f + (0.18f - 1.0f) * inner * (1.0f - bright * 0.94f)) *
           (1.0f + inner * (0.92f * bright + 0.22f * rim + 0.04f * counter));
  c = mul(c, 1.0f + (1.55f - 1.0f) * powf(clamp01(1.0f - fabsf(ray.y)), 1.5f));
  const float mid = powf(clamp01(1.0f - fabsf(hp.y) / fmaxf(0.42f, kEps)), 0.45f);
  c = mul(c, 1.0f + (1.8f - 1.0f) * (mid * (1.0f - radial)));
  const float l = luma(c);
  c = add(c, mul(c, inner * (-0.36f + (0.26f + 0.36f) * bright) * fmaxf(fminf(l - 0.05f, 1.0f), 0.0f)));
  c = mul(c, 1.0f - 0.22f * (inner * (1.0f - bright) * smooth(0.05f, 0.25f, l)));
  if (doppler > 1.0f)
    c = mix(c, v3(0.7f, 0.85f, 1.0f), fminf((doppler - 1.0f) * 1.5f, 0.6f));
  else
    c = mix(c, v3(0.6f, 0.05f, 0.0f), fminf((1.0f - doppler) * 2.0f, 0.7f));
  if (L.redshift_enabled) {
    float z;
    if (L.use_luts && L.tex_redshift)
      z = table(L.tex_redshift, r / fmaxf(rs, kEps), L.z_r_min, L.z_r_max, 1e-4f);
    else
      z = 1.0f / fmaxf(static_factor(sqrtf(dot(hp, hp)), rs), kEps) - 1.0f;
    const float opz = 1.0f + z;
    c = mul(c, 1.0f / (opz * opz * opz));
  }
  inten *= 1.8f + (0.85f - 1.8f) * powf(radial, 0.65f);
  if (L.use_luts && L.tex_grmhd && L.grmhd_r_max - L.grmhd_r_min > kEps) {
    // emissivity ~ rho u of the caller's grid at the hit (two frames blended by alpha)
    const float rr = sqrtf(dot(hp, hp));
    const float th = rr > kEps ? acosf(hp.z / rr) : 0.0f;
    float ph = atan2f(hp.y, hp.x);
    if (ph < 0.0f) ph += 6.28318530717958647692f;
    const float u = (rr - L.grmhd_r_min) / (L.grmhd_r_max - L.grmhd_r_min), v = th * kInvPi, w = ph * kInvTwoPi;
    float4 g = tex3D<float4>((cudaTextureObject_t)L.tex_grmhd, u, v, w);
    if (L.tex_grmhd_right && L.grmhd_alpha > kEps) {
      const float4 g1 = tex3D<float4>((cudaTextureObject_t)L.tex_grmhd_right, u, v, w);
      g.x += L.grmhd_alpha * (g1.x - g.x);
      g.y += L.grmhd_alpha * (g1.y - g.y);
    }
    inten *= fmaxf(g.x, 0.0f) * fmaxf(g.y, 0.0f);
  }
  return c;
}

// World point of Boyer-Lindquist (r [M], cos theta, phi from the camera's azimuth).
__device__ __forceinline__ V world(const BhkLook &L, double r, double u, double phi) {
  const double s = sqrt(fmax(0.0, 1.0 - u * u));
  const double cp = cos(phi), sp = sin(phi);
  const double x = s * cp, y = s * sp;
  const double rw = r * (double)L.m;
  return v3((float)(rw * ((double)L.cphi * x - (double)L.sphi * y)),
            (float)(rw * ((double)L.sphi * x + (double)L.cphi * y)), (float)(rw * u));
}

__global__ void __launch_bounds__(256) k_legacy_look(const __grid_constant__ BhkLook L,
                                                     const int32_t *__restrict__ cls,
                                                     const double *__restrict__ r_hit,
                                                     const double *__restrict__ phi_hit,
                                                     const double *__restrict__ theta_inf,
                                                     const double *__restrict__ phi_inf,
                                                     const float *__restrict__ closest,
                                                     const float *__restrict__ vol, float4 *__restrict__ rgba) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  const int c = cls[i];
  float4 out = make_float4(0.0f, 0.0f, 0.0f, 1.0f);  // captured: black
  if (L.vol_mode) {
    // The slab's emission in front of the ray's end; an escaped ray adds the
    // shaped sky (no ring glow) times the transmittance left. The Stokes
    // mode tints every pixel but those the horizon ended.
    const long long n = L.n;
    float rgb[3] = {vol[i], vol[n + i], vol[2 * n + i]};
    if (c == 2) {
      const V cam = v3(L.cam_pos[0], L.cam_pos[1], L.cam_pos[2]);
      const V esc = world(L, L.r_esc, cos(theta_inf[i]), phi_inf[i]);
      const float rmin_m = closest[i];
      const V cp = world(L, (double)rmin_m, (double)closest[L.n + i], (double)closest[2 * L.n + i]);
      const V sky = shape_sky(L, sky_color(L, unit(sub(esc, cam))), rmin_m * L.m, cp);
      const float T = vol[3 * n + i];
      rgb[0] += T * sky.x;
      rgb[1] += T * sky.y;
      rgb[2] += T * sky.z;
    }
    if (L.vol_mode == 2 && c != 0) bhvol::stokes_tint(rgb, vol[4 * n + i], vol[5 * n + i], vol[6 * n + i]);
    rgba[i] = make_float4(rgb[0], rgb[1], rgb[2], 1.0f);
    return;
  }
  if (c == 1) {
    float inten = 0.0f;
    const V col = disk_color(L, world(L, r_hit[i], 0.0, phi_hit[i]), inten);
    out = make_float4(col.x * inten, col.y * inten, col.z * inten, 1.0f);
  } else if (c != 0) {
    const V cam = v3(L.cam_pos[0], L.cam_pos[1], L.cam_pos[2]);
    const V esc = world(L, L.r_esc, cos(theta_inf[i]), phi_inf[i]);
    const float rmin_m = closest[i];
    const V cp = world(L, (double)rmin_m, (double)closest[L.n + i], (double)closest[2 * L.n + i]);
    const float r_min = rmin_m * L.m;
    V sky = sky_color(L, unit(sub(esc, cam)));
    sky = shape_sky(L, sky, r_min, cp);
    sky = ring_glow(L, sky, r_min, cp);
    out = make_float4(sky.x, sky.y, sky.z, 1.0f);
  }
  rgba[i] = out;
}

__global__ void k_stokes_steps(long long n, const float4 *__restrict__ state, const float *__restrict__ coef,
                               float4 *__restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 s = state[i];
  const float *c = coef + 7 * i;
  const bhvol::Stokes o = bhvol::stokes_step(bhvol::Stokes{s.x, s.y, s.z, s.w}, c[0], c[1], c[2], c[3], c[4], c[5], c[6]);
  out[i] = make_float4(o.i, o.q, o.u, o.v);
}

}  // namespace

extern "C" int bhk_stokes_steps(long long n, const float *state, const float *coef, float *out, void *stream) {
  if (n <= 0) return 0;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  k_stokes_steps<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      n, reinterpret_cast<const float4 *>(state), coef, reinterpret_cast<float4 *>(out));
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhk_legacy_look(const BhkLook *L, const int32_t *cls, const double *r_hit, const double *phi_hit,
                               const double *theta_inf, const double *phi_inf, const float *closest, const float *vol,
                               float *rgba, void *stream) {
  if (L->n <= 0) return 0;
  const unsigned blocks = (unsigned)((L->n + 255) / 256);
  k_legacy_look<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(*L, cls, r_hit, phi_hit, theta_inf, phi_inf,
                                                                        closest, vol, reinterpret_cast<float4 *>(rgba));
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
