// launch.h - internal C ABI between the C++23 host layer (csrc/host) and the
// CUDA translation units (csrc/device). POD structs and plain functions only,
// so that g++ -std=c++23 and nvcc see the same layout.
#pragma once

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// Everything the image kernels need about one scene, precomputed on the host
// (including every libm-derived constant, so that the device never calls a
// transcendental function that could differ from the CPU oracle by an ulp).
typedef struct BhkImageParams {
  double a, a2;            // spin and spin^2
  double r_obs;
  double r_plus, r_minus;  // outer / inner horizon (azimuth conversion)
  double r_hor;            // horizon_factor * r_+
  double r_esc;            // escape_factor * r_obs
  double r_in, r_out;      // disk edges
  double sin_o, cos_o;     // observer inclination
  double alpha_min, dalpha, beta_min, dbeta;  // pixel-centre grid
  double step_coeff, step_rcap;
  double rtol, atol;
  double nt_isco;          // ISCO of NovikovThorneDisk (pow form)
  double nt_flux_peak;     // its flux at 1.5 r_isco
  int64_t n_pix;
  int32_t width;
  int32_t max_steps;
  int32_t max_cross;       // 1..3
  int32_t form;            // 0 reference, 1 Carter
  int32_t integrator;      // 0 RK4, 1 DP45
  int32_t precision;       // 0 FP64, 1 mixed
  const uint16_t *sky;     // FP16 cubemap [6][sky_size][sky_size] added to escaped rays' intensity, or NULL
  int32_t sky_size;
  int32_t sky_pad;
} BhkImageParams;

typedef struct BhkImageOut {
  int32_t *cls, *steps, *n_cross;
  double *r_hit, *phi_hit, *g;  // [max_cross][n]
  double *flux, *intensity, *theta_inf, *phi_inf;
  // mixed tracer only: unit direction of motion of escaped rays, [3][n]
  // Cartesian (x, y, z) with x toward the observer's azimuth (zero if not escaped)
  float *esc_dir;
  // mixed camera tracer only: the ray's closest approach to the hole, [3][n]:
  // r [M], cos(theta) and phi (from the camera's azimuth) there; the camera's
  // own position if the ray never came closer
  float *closest;
  // [n] Carter-constant residual removed by the projection (mixed tracer)
  double *carter_drift;
  // mixed camera tracer with a BhkVolume: [8][n] front-to-back emission of
  // the disk slab (r, g, b), transmittance, Stokes Q, U, V, and 1 where the
  // slab made the ray opaque (0 otherwise)
  float *vol;
} BhkImageOut;

typedef struct BhkLaunch {
  int32_t grid;      // CTAs
  int32_t block;     // threads per CTA
  int32_t refill;    // integration steps between two refills of finished lanes (>= 1)
  int32_t pad;
} BhkLaunch;

// One frame of a batch as the device sees it.
typedef struct BhkFrame {
  BhkImageParams p;
  BhkImageOut o;
} BhkFrame;

// A batch of frames traced by one persistent launch. All pointers are device
// pointers owned by the host-side batch object.
typedef struct BhkBatchDev {
  const BhkFrame *frames;          // [n_frames]
  const long long *prefix;         // [n_frames + 1] first pixel of each frame in the work order
  unsigned int *done;              // [n_frames] finished pixels of the current trace
  unsigned long long *end_ns;      // [n_frames] %globaltimer when the frame's last pixel finished
  unsigned long long *start_ns;    // [1] earliest %globaltimer at which a CTA started
  long long n_total;               // sum of the frames' pixels
  int32_t n_frames;
  int32_t drift;                   // some frame asks for carter_drift
} BhkBatchDev;

// Persistent batch tracers (all frames share integrator and precision).
int bhk_trace_batch_fp64(const BhkBatchDev *b, int integrator, unsigned long long *work_counter, BhkLaunch L,
                         void *stream);
int bhk_trace_batch_mixed(const BhkBatchDev *b, int integrator, unsigned long long *work_counter, BhkLaunch L,
                          void *stream);
int bhk_trace_batch_fp64_occupancy(int integrator, int block, int *blocks_per_sm);
int bhk_trace_batch_mixed_occupancy(int integrator, int block, int *blocks_per_sm);

// FP64 image tracer. work_counter: one zeroed-on-stream 64-bit device word.
int bhk_trace_image_fp64(const BhkImageParams *p, const BhkImageOut *o, unsigned long long *work_counter,
                         BhkLaunch launch, void *stream);
// Occupancy query: max resident CTAs per SM for the given block size.
int bhk_trace_image_fp64_occupancy(int integrator, int block, int *blocks_per_sm);

// Mixed-precision image tracer (trace_image_mixed.cu), same contract.
int bhk_trace_image_mixed(const BhkImageParams *p, const BhkImageOut *o, unsigned long long *work_counter,
                          BhkLaunch launch, void *stream);
int bhk_trace_image_mixed_occupancy(int integrator, int block, int *blocks_per_sm);
// Mixed-precision tracer over the pixels named by a device list of *count
// entries (count written by an earlier kernel on the same stream).
int bhk_trace_list_mixed(const BhkImageParams *p, const BhkImageOut *o, const int *list, const unsigned int *count,
                         unsigned long long *work_counter, BhkLaunch L, void *stream);

// Output fields of a set of pixels gathered into compact arrays (the host-
// buffer render's rejected pixels, written after their rows were copied):
// src: the 10 BH_KerrImageOut fields in their order (NULL: skip), size 4 or
// 8 bytes, planes 1 or max_cross; dst[f][c * cap + w] = src[f][c * n_pix + list[w]]
// and list_out[w] = list[w] for w < min(*count, cap); *count_out = *count.
// The destinations may be mapped host memory (the writes end with a
// system-scope fence).
typedef struct BhkGather {
  const void *src[10];
  void *dst[10];
  int32_t size[10], planes[10];
  int *list_out;
  unsigned int *count_out;
} BhkGather;
int bhk_gather_pixels(const BhkGather *g, const int *list, const unsigned int *count, long long n_pix, int cap,
                      void *stream);

// Surrogate renderer (surrogate_render.cu): per-pixel acceptance of the
// network's head outputs [n_pix][16] for pixels [p0, p1), exact refinement of
// accepted disk hits, and the list of pixels left to the integrator. stats[5] += pixels accepted,
// low confidence, critical band, solve failed, disagreement.
int bhk_surrogate_refine(const BhkImageParams *p, const BhkImageOut *o, const float *head, float min_conf,
                         double band, int verify, int refine_fp64, long long p0, long long p1, int *list,
                         unsigned int *count, unsigned int *stats, void *stream);

// Reference stepper kernels (src/physics/kerr.cpp semantics), FP64.
typedef struct BhkStateSoA { double *r, *theta, *phi, *t, *sr, *sth; } BhkStateSoA;
typedef struct BhkConstsSoA { const double *e, *lz, *q; } BhkConstsSoA;

int bhk_kerr_potentials(int64_t n, const double *r, const double *theta, double mass, double a,
                        BhkConstsSoA c, double *rp, double *drp, double *tp, double *dtp, void *stream);
int bhk_kerr_step_mino(int64_t n, BhkStateSoA s, double mass, double a, BhkConstsSoA c, const double *dlam,
                       double dlam_scalar, void *stream);
int bhk_kerr_trace_rays(int64_t n, BhkStateSoA init, BhkConstsSoA c, double mass, double a, double r_horizon,
                        double r_escape, double step, int32_t max_steps, int32_t *status, int32_t *steps,
                        double *dist, double *rf, double *thf, double *phf, double *redshift, void *stream);

// Host layer (capi.cpp): scene validation + kernel parameters + persistent
// grid shape, allocating nothing; and setting the thread's last error.
struct BH_KerrScene;
int bhh_prepare_image_launch(const struct BH_KerrScene *scene, BhkImageParams *p, BhkLaunch *L);
// Validates one scene and fills its kernel parameters (no device call).
int bhh_make_params(const struct BH_KerrScene *scene, BhkImageParams *p);
// Launches the image kernel of p->precision (work counter zeroed on stream).
// The analytic integrator also needs a list of n_pix ints for the pixels it
// leaves to the DP45 tracer: `list`, or the device's grow-only list when NULL
// (its count lives in counter[1]; counter must hold two words).
int bhh_launch_image(const BhkImageParams *p, const BhkImageOut *o, unsigned long long *counter, BhkLaunch L,
                     void *stream, int *list);
int bhh_fail(const char *msg);
// The current device's persistent-kernel work counter (allocated once).
int bhh_work_counter(unsigned long long **counter);

// Along-ray radiative transfer (rt.cuh, trace_image_fp64.cu).
typedef struct BhkRtParams {
  const float *cells;   // float4 (n_e, Theta_e, |B|, 0) [n_r][n_th][n_ph]
  int32_t n_r, n_th, n_ph, pad0;
  double r_min, r_max, inv_log_range;  // 1 / log(r_max / r_min)
  const float *lut;     // [n_lt][n_lx] ln(j_nu / (n_e nu_B))
  int32_t n_lt, n_lx;
  double lt0, lt1, lx0, lx1;           // log Theta_e and log x ranges
  double nu, length_cm, ds_max, min_transmit;
} BhkRtParams;

// The same on the mixed-precision tracer with FP32 samples (trace_image_mixed.cu).
int bhk_trace_rt_mixed(const BhkImageParams *p, const BhkRtParams *q, double *i_nu, double *tau, int32_t *cls,
                       int32_t *steps, unsigned long long *work_counter, void *stream);
int bhk_trace_rt_fp64(const BhkImageParams *p, const BhkRtParams *q, double *i_nu, double *tau, int32_t *cls,
                      int32_t *steps, unsigned long long *work_counter, int grid, int block, void *stream);

// Synthetic torus grid (grmhd.cu): modes [n_modes] of (kx, ky, kz, phase).
// Resample packed simulation frames into the medium grid (grmhd.cu).
int bhk_grmhd_from_packed(float *cells, int n_r, int n_th, int n_ph, double r_min, double r_max, const float *left,
                          const float *right, double alpha, int pnr, int pnt, int pnp, double pr_min, double pr_max,
                          double n_scale, double theta_scale, double b_scale, void *stream);
int bhk_grmhd_fill(float *cells, int n_r, int n_th, int n_ph, double r_min, double r_max, double r_in, double r_peak,
                   double width, double n0, double theta0, double b0, double amp, const double *modes, int n_modes,
                   void *stream);

// Sky cubemap (sky.cu): noise texels for every texel, then the star texels
// (index, FP32 value) from the host list.
int bhk_sky_fill(uint16_t *tex, int size, uint64_t seed, const long long *star_idx, const float *star_val,
                 int n_stars, void *stream);

// FMA-throughput probe (probe.cu).
// A camera at finite distance (the reference renderer's camera model, in M
// units): pixel (px, py) looks along d = normalize(-u right - v up + fwd),
// u = (2 (px + 1/2) / width - 1) fov aspect + shift_x, v likewise with
// height and shift_y; the ray is the past-directed null geodesic whose
// direction in the camera's locally non-rotating frame is d.
typedef struct BhkCamera {
  double right[3], up[3], fwd[3];
  double fov, aspect, shift_x, shift_y;
  double r0, u0;      // camera radius [M] and cos(theta)
  double cphi, sphi;  // camera azimuth: cos, sin (the outputs' azimuths are relative to it)
  int32_t width, height;
} BhkCamera;

// The volumetric disk of the render launch ABI's RTE and Stokes modes (the
// reference's d_trace_geodesic_rte / d_trace_geodesic_stokes): a slab of
// Gaussian height h about z = 0 between r_in and r_out (cylindrical radius,
// world units), composited front to back along each camera ray with the
// reference's emission, opacity and polarization model. Path elements are the
// reference's: its Mino time in world units, d lambda = d tau / m.
typedef struct BhkVolume {
  int32_t mode;          // 1: intensity only (RTE), 2: with Stokes Q, U, V
  int32_t emit;          // the disk emits (adisk_enabled)
  float m, rs;           // world units per M; rs (world)
  float r_in, r_out, h;  // slab: cylindrical radii and Gaussian height (world)
  float opacity;         // absorption per unit emissivity (rte_opacity_scale)
  float b_angle, ne_scale;  // Stokes: field angle (EVPA of emission), Faraday rate per unit density
  float cphi, sphi;      // camera azimuth: tracer frame -> world
} BhkVolume;

// Traces every pixel of a camera with the mixed tracer (p: spin, horizon,
// escape and disk radii, integrator, tolerances; p.r_obs = cam.r0, Carter
// potentials). With vol (non-NULL, mode 1 or 2) the rays also integrate the disk slab
// into o->vol, and a ray the slab makes opaque stops with class 1.
int bhk_trace_camera_mixed(const BhkImageParams *p, const BhkCamera *cam, const BhkImageOut *o,
                           unsigned long long *work_counter, BhkLaunch L, void *stream, const BhkVolume *vol);
int bhk_trace_camera_mixed_occupancy(int block, int *blocks_per_sm);

// Positions (x, y, z) [M] after every FP64 RK4 step of image-plane rays, up
// to max_points per ray (initial point included): xyz [n][max_points][3],
// counts [n].
int bhk_trace_paths_fp64(const BhkImageParams *p, float *xyz, int32_t *counts, int max_points, void *stream);

// Legacy RGBA shading (legacy.cu).
typedef struct BhkShade {
  int64_t n;
  int32_t width;
  int32_t redshift_enabled, background_enabled, use_luts;
  float adisk_lit, background_intensity;
  float t_peak;          // disk temperature at the flux peak [K]
  float lut_r_min, lut_r_max, spec_r_min, spec_r_max;  // table domains in r / rs = r [M] / 2
  float cphi, sphi;      // camera azimuth (rotates escape directions into the world frame)
  unsigned long long tex_emissivity, tex_spectral, tex_galaxy, tex_equirect;
} BhkShade;
// The reference renderer's own look (legacy_look.cu): lengths in the
// caller's world unit (m of them per M), textures as CUDA texture objects
// (0 = not registered).
typedef struct BhkLook {
  int64_t n;
  float m;                       // world units per M (rs / 2)
  float rs, isco, spin;          // world units; spin a / M as the caller gave it
  double r_esc;                  // escape radius [M]
  float cam_pos[3], cam_right[3];
  float cphi, sphi;              // camera azimuth: tracer frame -> world
  int32_t redshift_enabled, use_luts, background_enabled;
  int32_t vol_mode;              // 1, 2: the slab of the RTE / Stokes modes was traced into `vol`
  float adisk_lit, doppler_strength, bg_intensity, time_sec, glow_strength;
  float bg_yaw, bg_pitch, bg_filter;
  float bg_layers[12], bg_lod_bias[3];
  float lut_r_min, lut_r_max, z_r_min, z_r_max, spec_r_min, spec_r_max;  // [rs]
  float grmhd_r_min, grmhd_r_max, grmhd_alpha;
  unsigned long long tex_emissivity, tex_redshift, tex_spectral, tex_galaxy, tex_grmhd, tex_grmhd_right,
      tex_equirect;
} BhkLook;
int bhk_legacy_look(const BhkLook *L, const int32_t *cls, const double *r_hit, const double *phi_hit,
                    const double *theta_inf, const double *phi_inf, const float *closest, const float *vol, float *rgba,
                    void *stream);

// n exact Stokes transfer steps (vol.cuh), device arrays state [n][4], coef [n][7], out [n][4].
int bhk_stokes_steps(long long n, const float *state, const float *coef, float *out, void *stream);

int bhk_legacy_set_blackbody(const float *rgb_table, int n, float log2_t0, float log2_t1);
int bhk_legacy_shade(const BhkShade *s, const int32_t *cls, const double *r_hit, const double *g, const double *flux,
                     const float *esc_dir, float *rgba, void *stream);
int bhk_legacy_lensing(int64_t n, const int32_t *cls, const double *r_hit, const double *g, float *rgba,
                       void *stream);
int bhk_legacy_disk_texture(double a, double r_isco, double r_out, double nt_flux_peak, double incl, float t_peak,
                            int width, int height, float *rgba, void *stream);

// Bloom and tone mapping (postprocess.cu). Taps: the normalized Gaussians
// of half-width 4, 8, 16, 32 (sigma = r / 2), 2r + 1 each, concatenated.
typedef struct BhkPostTaps {
  float w[124];
} BhkPostTaps;
int64_t bhk_post_scratch_floats(int w, int h);
int bhk_post_process(float *fb, int w, int h, const BhkPostTaps *taps, float threshold, float strength,
                     float exposure, float *scratch, void *stream);

// Closed-form tracer (trace_image_analytic.cu): pixels it does not cover go to list[0..*count).
int bhk_trace_image_analytic(const BhkImageParams *p, const BhkImageOut *o, int *list, unsigned int *count,
                             BhkLaunch L, void *stream);
int bhk_trace_image_analytic_occupancy(int block, int *blocks_per_sm);
int bhk_trace_image_analytic_block(void);  // threads per CTA the closed form is compiled for
// The same over list[0..*count); pixels it does not cover go to list2[0..*count2).
int bhk_trace_list_analytic(const BhkImageParams *p, const BhkImageOut *o, const int *list, const unsigned int *count,
                            int *list2, unsigned int *count2, BhkLaunch L, void *stream);
int bhk_trace_list_fp64(const BhkImageParams *p, const BhkImageOut *o, const int *list, const unsigned int *count,
                        unsigned long long *counter, BhkLaunch L, void *stream);


// Last CUDA error string of the device layer (thread-local).
const char *bhk_last_error(void);

#ifdef __cplusplus
}
#endif
