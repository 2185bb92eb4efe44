/*
 * bh_rt.h -- along-ray radiative transfer through a volumetric emitter.
 *
 * Counterpart of the reference's volumetric path: the GRMHD texture sampler
 * d_sample_grmhd (src/cuda/device_physics.cuh:1789-1829), the front-to-back
 * formal solution of d_rte_step / d_trace_geodesic_rte (:1988-2173), and the
 * FP64 physics it restates, physics::rteStep, synchrotronThermalEmissivity,
 * synchrotronThermalAbsorption and grTransform* (src/physics/rte_integrator.h:
 * 138-187, 291-356, 465-513). The medium is a grid of (n_e, Theta_e, |B|) on
 * log-spaced r, theta and phi; thermal synchrotron emission comes from a 2-D
 * table over (log Theta_e, log nu/nu_s), absorption from Kirchhoff's law at
 * the emitted frequency. Rays are the image tracer's FP64 DP45 geodesics
 * (bh_kerr.h); along every accepted step the medium is sampled at most
 * ds_max apart in affine length (cubic Hermite positions inside the step).
 *
 * Conventions follow bh_kerr.h (0 / -1 + bh_last_error, device pointers,
 * NULL stream = legacy default stream). Geometric units M = 1 for positions;
 * CGS for the radiative quantities.
 */
#ifndef BH_RT_H
#define BH_RT_H

#include <stdint.h>

#include "bh_kerr.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Device grid of float4 (n_e [cm^-3], Theta_e, |B| [G], 0), index
 * (i_r * n_theta + i_theta) * n_phi + i_phi. Nodes: r_i = r_min (r_max /
 * r_min)^(i / (n_r - 1)); theta_j = (j + 1/2) pi / n_theta; phi_k = 2 pi k /
 * n_phi (periodic). Trilinear interpolation; no emission outside [r_min, r_max]. */
typedef struct BH_GrmhdGrid {
    const void *cells;
    int32_t n_r, n_theta, n_phi, reserved;
    double r_min, r_max;
} BH_GrmhdGrid;

/* Synthetic torus: n_e = n0 T(r, theta) exp(F), Theta_e = theta0 r_peak / r,
 * |B| = b0 sqrt(n_e / n0). T = exp(-((R - r_peak)^2 + z^2) / (2 w^2)) with
 * R = r sin(theta), z = r cos(theta), times exp(-((r_in - r) / 1 M)^2) inside
 * r_in. F: Gaussian random field of standard deviation sigma and Gaussian
 * correlation of length corr_len (M), sampled as 256 random Fourier modes
 * in Cartesian space (seeded). */
typedef struct BH_TorusParams {
    double r_in, r_peak, width;
    double n0, theta0, b0;
    double sigma, corr_len;
    uint64_t seed;
} BH_TorusParams;

void bh_torus_defaults(BH_TorusParams *torus);  /* r_in 6, r_peak 12, width 3, n0 1e5, theta0 20,
                                                   b0 30, sigma 0.5, corr_len 2, seed 1 */

/* Fill grid->cells (already allocated: n_r * n_theta * n_phi float4). */
int bh_grmhd_synthetic(const BH_GrmhdGrid *grid, const BH_TorusParams *torus, void *stream);

/* ---- ingestion of simulation output ---------------------------------------
 *
 * A dataset written by the reference's tools/nubhlight_pack.cpp: a JSON
 * metadata file ("format" "RGBA32F", "bin" or legacy "binary_file": the blob
 * next to it, "grid_dims" [n_r, n_theta, n_phi], optional
 * "checksum_fnv1a64", "channels", "min", "max", "r_min", "r_max") and a blob
 * of float4 samples, raw values of four fields (rho, u, v1, v2 by default),
 * index (i_r n_theta + i_theta) n_phi + i_phi. Its sample positions follow the
 * reference renderer's 3-D texture (src/cuda/device_physics.cuh:1789-1829):
 * r_i = r_min + (i + 1/2)(r_max - r_min) / n_r (clamped outside), theta_j =
 * (j + 1/2) pi / n_theta, phi_k = (k + 1/2) 2 pi / n_phi (periodic).
 * Replaces loadGrmhdPackedTexture (src/grmhd_packed_loader.h:70-71). */
typedef struct BH_PackedGrmhdInfo {
    int32_t n_r, n_theta, n_phi, reserved;
    float r_min, r_max;     /* radial extent [M] ("r_min", "r_max"; 1 and 50 when absent) */
    float min_value[4], max_value[4];  /* per-channel ranges from the metadata (0 when absent) */
    char channels[4][32];   /* field names */
} BH_PackedGrmhdInfo;

/* Parse and validate the metadata at json_path and read its blob: format
 * RGBA32F, four channels, blob size n_r n_theta n_phi 4 floats, FNV-1a 64
 * checksum when present. host_samples (n_r n_theta n_phi 4 floats, may be
 * NULL: metadata only) receives the samples. Host only; no device work. */
int bh_grmhd_packed_read(const char *json_path, BH_PackedGrmhdInfo *info, float *host_samples,
                         int64_t capacity_floats);

/* From the fields to the emitting medium (channel 0 rho, channel 1 u, the
 * internal energy density, both in code units):
 *   n_e = n_scale rho,  Theta_e = theta_scale u / rho,  |B| = b_scale sqrt(u)
 * (temperature from u / rho; magnetic pressure a fixed fraction of the gas
 * pressure). The scales are the caller's unit choice. */
typedef struct BH_PackedConversion {
    double n_scale;      /* cm^-3 per unit rho (1e5) */
    double theta_scale;  /* Theta_e per unit u / rho (10) */
    double b_scale;      /* gauss per unit sqrt(u) (30) */
} BH_PackedConversion;

void bh_packed_conversion_defaults(BH_PackedConversion *conv);

/* Fill grid->cells (device) by sampling packed frames (device float4 arrays
 * as read above) trilinearly at every grid node, blending frame_left and
 * frame_right as (1 - alpha) left + alpha right (frame_right may be NULL:
 * alpha ignored), then converting. The reference blends two texture frames
 * the same way (device_physics.cuh:1816-1828). */
int bh_grmhd_from_packed(const BH_GrmhdGrid *grid, const BH_PackedGrmhdInfo *info, const void *frame_left,
                         const void *frame_right, double alpha, const BH_PackedConversion *conv, void *stream);

/* Thermal synchrotron table: float [n_theta][n_x] of ln(j_nu / (n_e nu_B))
 * (CGS emissivity per unit electron density and gyrofrequency) at nodes of
 * log Theta_e and log x (x = nu / nu_s, nu_s = 3/2 nu_B Theta_e^2) evenly
 * spaced over the given ranges, interpolated bilinearly in the logarithm;
 * zero emission beyond x_max, clamped below x_min. */
typedef struct BH_SynchrotronLut {
    const void *table;
    int32_t n_theta, n_x;
    double log_theta_min, log_theta_max;
    double log_x_min, log_x_max;
} BH_SynchrotronLut;

/* Fill lut->table (device, n_theta * n_x floats) on the host and copy it. */
int bh_synchrotron_lut(const BH_SynchrotronLut *lut, void *stream);
/* The same table into host memory (n_theta * n_x floats); lut->table unused. */
int bh_synchrotron_lut_host(const BH_SynchrotronLut *lut, float *out_host);

typedef struct BH_RtParams {
    double nu_hz;           /* observed frequency (230e9) */
    double length_cm;       /* cm per M (G M / c^2; 1.4766e6 for 10 solar masses) */
    double ds_max;          /* largest affine distance between samples, M (0.25) */
    double min_transmit;    /* stop a ray once its transmittance falls below this (1e-6) */
} BH_RtParams;

void bh_rt_defaults(BH_RtParams *rt);

/* Trace every pixel of `scene` (DP45 integrator; the thin disk is ignored)
 * through the medium. scene->precision BH_PRECISION_FP64: FP64 geodesic and
 * samples; BH_PRECISION_MIXED: the mixed-precision geodesic (FP32 bulk) and
 * FP32 samples with the emission carried as logarithms, intensity and depth
 * summed in FP64 (its accepted steps, hence its sample points, differ from
 * the FP64 ones: results agree to the sampling's discretization error).
 * Outputs per pixel (device,
 * NULL = not wanted): I_nu at the observer (erg s^-1 cm^-2 Hz^-1 sr^-1),
 * optical depth along the ray, class (0 captured, 2 escaped, 3 steps
 * exhausted, 4 stopped opaque) and accepted steps. */
int bh_kerr_trace_rt(const BH_KerrScene *scene, const BH_GrmhdGrid *grid, const BH_SynchrotronLut *lut,
                     const BH_RtParams *rt, double *i_nu, double *tau, int32_t *cls, int32_t *steps, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* BH_RT_H */
