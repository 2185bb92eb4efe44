// vol.cuh - the volumetric disk of the render launch ABI's RTE and Stokes
// modes: emission of a Gaussian slab about the equatorial plane, front-to-back
// compositing, and the exact step of polarized transfer with absorption and
// Faraday rotation. Host and device (the host build serves the C entry point
// that tests the Stokes step against its analytic limits).
//
// The model is the reference renderer's (src/cuda/device_physics.cuh:
// d_rte_step :1988-2014, d_trace_geodesic_rte :2037-2173, d_stokes_step
// :2216-2284, d_trace_geodesic_stokes :2307-2459): at a point of cylindrical
// radius R in [r_in, r_out] and height z (world units),
//   flux  = x^3 (1 - sqrt x), x = r_in / R
//   colour: three bands of flux^(1/4) (> 0.6, > 0.3, else)
//   Doppler factor D = 1 + 0.3 sqrt(rs / 2R) cos(phi), emissivity j = flux D^3 exp(-z^2 / 2h^2)
//   absorption alpha = opacity * j; intensity j (1 - e^-tau) / alpha per segment,
//   attenuated by the transmittance in front of it;
//   Stokes: j_Q = -0.75 j_I cos 2b, j_U = -0.75 j_I sin 2b (j_I the colour's
//   mean emissivity), Faraday rate rho_V = ne_scale exp(-z^2 / 2h^2), V not
//   emitted.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define BHV_HD __host__ __device__ __forceinline__
#else
#define BHV_HD inline
#endif

namespace bhvol {

struct Stokes {
  float i, q, u, v;
};

// One segment ds of polarized transfer with emission (jI, jQ, jU, jV), total
// absorption A (every channel) and Faraday rotation R (Q -> U at rate R):
//   dI/ds = jI - A I,  dV/ds = jV - A V,
//   d(Q, U)/ds = (jQ, jU) - A (Q, U) + R (-U, Q),
// solved exactly over the segment. With E = exp(-A ds) and phi = R ds, the
// homogeneous part scales (Q, U) by E and rotates it by phi; the source part
// is rot(R t) (jQ, jU) e^(-A t) integrated over t in [0, ds], i.e.
//   Ic = int e^(-At) cos(Rt) dt = (A (1 - E cos phi) + R E sin phi) / (A^2 + R^2),
//   Is = int e^(-At) sin(Rt) dt = (R (1 - E cos phi) - A E sin phi) / (A^2 + R^2),
// replaced by their Taylor series in ds when (A^2 + R^2) ds^2 is small, where
// the closed forms cancel.
BHV_HD Stokes stokes_step(Stokes s, float jI, float jQ, float jU, float jV, float A, float R, float ds) {
  if (!(ds > 0.0f)) return s;
  A = A > 0.0f ? A : 0.0f;
  const float tau = A * ds, phi = R * ds;
  const float E = tau < 80.0f ? expf(-tau) : 0.0f;
  // (1 - E) / A, the scalar channels' source weight, without cancellation at small tau
  const float w = tau < 1e-3f ? ds * (1.0f - tau * (0.5f - tau * (1.0f / 6.0f))) : (1.0f - E) / A;
  Stokes o;
  o.i = s.i * E + jI * w;
  o.v = s.v * E + jV * w;
  const float c = cosf(phi), sn = sinf(phi);
  float Ic, Is;
  if (tau * tau + phi * phi < 1e-6f) {  // Re, Im of ds (1 + z/2 + z^2/6), z = -tau + i phi
    Ic = ds * (1.0f - 0.5f * tau + (tau * tau - phi * phi) * (1.0f / 6.0f));
    Is = ds * phi * (0.5f - tau * (1.0f / 3.0f));
  } else {
    const float D = A * A + R * R;
    Ic = (A * (1.0f - E * c) + R * E * sn) / D;
    Is = (R * (1.0f - E * c) - A * E * sn) / D;
  }
  o.q = E * (s.q * c - s.u * sn) + jQ * Ic - jU * Is;
  o.u = E * (s.q * sn + s.u * c) + jQ * Is + jU * Ic;
  return o;
}

// Emission of the slab at world point (x, y, z): returns j, its colour band
// and the density weight rho = exp(-z^2 / 2h^2); -1 outside the slab's radii
// (where the reference neither emits, absorbs nor rotates).
BHV_HD float slab_emission(float x, float y, float z, float rs, float r_in, float r_out, float h, float col[3],
                           float &rho) {
  const float zh = z / h;
  rho = expf(-0.5f * zh * zh);
  const float R2 = x * x + y * y;
  if (!(R2 >= r_in * r_in && R2 <= r_out * r_out)) return -1.0f;
  const float R = sqrtf(R2);
  const float xr = r_in / R;
  const float flux = fmaxf(0.0f, xr * xr * xr * (1.0f - sqrtf(xr)));
  const float t = sqrtf(sqrtf(flux));
  if (t > 0.6f) {
    col[0] = 1.0f; col[1] = 0.9f; col[2] = 0.8f;
  } else if (t > 0.3f) {
    col[0] = 1.0f; col[1] = 0.6f; col[2] = 0.2f;
  } else {
    col[0] = 0.8f; col[1] = 0.2f; col[2] = 0.1f;
  }
  const float vel = sqrtf(0.5f * rs / R);
  const float dop = 1.0f + 0.3f * vel * (x / R);  // cos(phi) = x / R
  return flux * (dop * dop * dop) * rho;
}

// The running state of one ray through the slab.
struct Accum {
  float rgb[3];
  float T;     // transmittance in front of the next segment
  Stokes s;    // I unused (the colour accumulator carries intensity)
};

BHV_HD void accum_init(Accum &a) {
  a.rgb[0] = a.rgb[1] = a.rgb[2] = 0.0f;
  a.T = 1.0f;
  a.s = Stokes{0.0f, 0.0f, 0.0f, 0.0f};
}

// One emitting segment of length ds: emissivity j with colour col, density
// weight rho (for the Faraday rate). Returns true once the ray is opaque
// (transmittance below 0.005, where the reference stops).
BHV_HD bool accum_segment(Accum &a, float j, const float col[3], float rho, float ds, float opacity, int mode,
                          float cos2b, float sin2b, float ne_scale) {
  const float alpha = opacity * fmaxf(j, 0.0f);
  const float tau = alpha * ds;
  const float E = tau < 80.0f ? expf(-tau) : 0.0f;
  const float w = alpha < 1e-30f ? ds : (tau < 1e-3f ? ds * (1.0f - tau * (0.5f - tau * (1.0f / 6.0f))) : (1.0f - E) / alpha);
  const float e = j * w * a.T;
  a.rgb[0] += col[0] * e;
  a.rgb[1] += col[1] * e;
  a.rgb[2] += col[2] * e;
  a.T *= E;
  if (mode == 2) {
    const float jI = j * (col[0] + col[1] + col[2]) * (1.0f / 3.0f);
    a.s = stokes_step(a.s, 0.0f, -0.75f * jI * cos2b, -0.75f * jI * sin2b, 0.0f, alpha, ne_scale * rho, ds);
  }
  return a.T < 0.005f;
}

// The display colour of a Stokes-mode pixel: the intensity tinted by the
// polarization angle chi = atan2(U, Q) / 2 and degree P = |(Q, U)| / I (red by
// cos 2 chi, green by sin 2 chi, 0.4 P each) and blue by V / I (0.2, V / I
// clamped to +-0.5), I the mean of the three colour channels.
BHV_HD void stokes_tint(float rgb[3], float q, float u, float v) {
  const float I = (rgb[0] + rgb[1] + rgb[2]) * (1.0f / 3.0f);
  float p = 0.0f, vf = 0.0f;
  if (I > 1e-10f) {
    p = fminf(sqrtf(q * q + u * u) / I, 1.0f);
    vf = fmaxf(-0.5f, fminf(0.5f, v / I));
  }
  const float two_chi = atan2f(u, q);
  rgb[0] = fmaxf(rgb[0] * (1.0f + 0.4f * p * cosf(two_chi)), 0.0f);
  rgb[1] = fmaxf(rgb[1] * (1.0f + 0.4f * p * sinf(two_chi)), 0.0f);
  rgb[2] = fmaxf(rgb[2] * (1.0f + 0.2f * vf), 0.0f);
}

}  // namespace bhvol
