/*
 * bh_legacy.h -- the reference renderer's launch ABI, served by the B200 tracer.
 *
 * Drop-ins for the entry points that the reference's desktop application and
 * Blender bridge call to render an RGBA image with its CUDA kernels:
 *
 *   kernel launch   src/cuda/kernel_launch.h:28-190  (BH_LaunchParams, BH_KernelVariant,
 *                   bh_launch_geodesic_kernel, bh_select_kernel_variant,
 *                   bh_upload_lut_textures, bh_upload_bridge_background_texture)
 *   backend         src/cuda/cuda_backend.h:33-103   (bhCuda*)
 *   Blender bridge  src/blender_bridge/blender_bridge.h:348-405 and the snake_case
 *                   aliases of src/blender_bridge/blender_bridge.cpp:716-730 (bhbCuda*,
 *                   bhb_cuda_*)
 *
 * BH_LaunchParams keeps the reference's field order and types, so a caller
 * compiled against the reference header passes the same bytes. What happens
 * behind the calls is this library's: every pixel's ray is a Kerr null
 * geodesic traced by the mixed-precision DP45 tracer of bh_kerr.h (FP32 bulk,
 * FP64 set-up). Two ways to colour it (bh_legacy_set_shading):
 *   BH_SHADING_REFERENCE (the default): the reference shader's own look
 *     (src/cuda/device_physics.cuh, d_shade_hit and what it calls) -- colour
 *     ramp, tints, Doppler beaming, sector shaping, static-observer redshift,
 *     procedural stars or the caller's textures, escaped-sky shaping and
 *     photon-ring glow -- evaluated on this tracer's hit points, closest
 *     approaches and escape positions, so existing callers get the picture
 *     they were tuned for;
 *   BH_SHADING_PHYSICAL: the observed blackbody of a Novikov-Thorne disk
 *     (exact Keplerian redshift g) and the caller's texture in the ray's
 *     escape direction.
 * Still accepted and ignored in both: wiregrid, debug exports, Stokes and
 * volumetric (RTE) modes. The calls that need an OpenGL texture return -1 (no
 * graphics stack).
 *
 * Conventions: 0 on success, -1 on error with the message in bh_last_error()
 * (bh_kerr.h). World coordinates are those of the reference renderer: lengths
 * in units of rs (the Schwarzschild radius, 2M), spin axis along +z, the disk
 * in the z = 0 plane between isco and 30 rs, camera basis column-major with
 * columns right, up, forward.
 */
#ifndef BH_LEGACY_H
#define BH_LEGACY_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- kernel launch (src/cuda/kernel_launch.h) ------------------------------- */

struct BH_LaunchParams {
    /* black hole */
    float rs;        /* Schwarzschild radius: the world's unit of length */
    float spin;      /* a / M */
    float isco;      /* inner disk edge [rs] */
    float step_size; /* accepted and ignored: the tracer's steps are adaptive */
    float fov_scale; /* tangent of the half field of view */
    float max_dist;  /* escape radius [rs] */

    /* camera */
    float cam_pos[3];     /* world position [rs] */
    float cam_basis[9];   /* column-major: right, up, forward */
    float frame_shift_x;  /* image-plane offsets added to the pixel's (u, v) */
    float frame_shift_y;

    /* integration */
    int max_steps; /* accepted-step budget per ray */
    int width;
    int height;

    /* feature flags */
    int adisk_enabled;    /* 0: the disk is transparent */
    int redshift_enabled; /* 0: shade the disk at g = 1 */
    int kerr_enabled;     /* 0: spin taken as 0 */
    int use_luts;         /* 1: sample the registered emissivity / spectral tables */

    /* table domains (radius in rs mapped to the texture's [0, 1]) */
    float lut_radius_min;
    float lut_radius_max;
    float redshift_radius_min;
    float redshift_radius_max;
    float spectral_radius_min;
    float spectral_radius_max;

    float time_sec;
    float doppler_strength;     /* reference look: strength of its Doppler approximation */
    float background_intensity; /* background texture multiplier */
    int background_enabled;
    float photon_glow_strength;
    int debug_pre_redshift_background;
    int debug_pre_shaping_background;
    int debug_post_shaping_background;
    int debug_shaper_inputs;
    int debug_closest_approach_state;
    int debug_closest_approach_timeline;
    int debug_closest_approach_direction;
    int debug_escaped_direction;
    float background_yaw_rad;
    float background_pitch_rad;
    float background_filter_radius;
    float background_layer_params[12];
    float background_layer_lod_bias[3];

    int wiregrid_enabled;
    float wiregrid_show_ergo;
    float wiregrid_grid_scale;
    float wiregrid_motion_scale;
    float wiregrid_infall_scale;
    float wiregrid_strength;
    float wiregrid_scene_preserve;
    float wiregrid_color[4];

    float grmhd_r_min;
    float grmhd_r_max;
    int rte_enabled;
    float rte_opacity_scale;
    float grmhd_alpha;
    int stokes_enabled;
    float stokes_b_field_angle;
    float stokes_ne_scale;

    float adisk_lit; /* disk brightness multiplier */
};

enum BH_KernelVariant {
    BH_KERNEL_FP32_BASELINE = 0,
    BH_KERNEL_FP32_COARSENED = 1,
    BH_KERNEL_FP16_STORAGE = 2,
    BH_KERNEL_FP16_H2_ILP = 3,
    BH_KERNEL_COUNT = 4
};

/* Render params->width x params->height float4 RGBA pixels (linear, row 0 at
 * the top, alpha 1) into the device framebuffer, asynchronously on `stream`.
 * variant: any BH_KernelVariant value or negative for automatic; all of them
 * run the same mixed-precision tracer. The first call on a device allocates
 * the per-pixel scratch (grow-only, kept until bhbCudaResetDevice or exit).
 * Replaces bh_launch_geodesic_kernel, src/cuda/kernel_launch.h:143-146. */
int bh_launch_geodesic_kernel(void *framebuffer, const struct BH_LaunchParams *params, int variant, void *stream);

/* Shading of the render calls (no counterpart in the reference, whose look is
 * fixed): BH_SHADING_REFERENCE (0, default) or BH_SHADING_PHYSICAL (1); the
 * default can also be set by BLACKHOLE_SHADING=physical in the environment,
 * read on the first render. Process-wide; returns -1 on an unknown mode. */
enum BH_Shading { BH_SHADING_REFERENCE = 0, BH_SHADING_PHYSICAL = 1 };
int bh_legacy_set_shading(int mode);
int bh_legacy_get_shading(void);

/* The polarized transfer step of the render calls' Stokes mode
 * (stokes_enabled; replaces d_stokes_step, src/cuda/device_physics.cuh:
 * 2216-2284), on n independent states at once, on the GPU. Device arrays:
 * state [n][4] (I, Q, U, V), coef [n][7] (jI, jQ, jU, jV, alpha_I, rho_V, ds),
 * out [n][4]. The step is the exact solution over ds of
 *   dI/ds = jI - alpha_I I,  dV/ds = jV - alpha_I V,
 *   d(Q, U)/ds = (jQ, jU) - alpha_I (Q, U) + rho_V (-U, Q)
 * (absorption alpha_I on every channel, Faraday rotation rho_V of Q into U),
 * in FP32; ds <= 0 leaves the state unchanged, alpha_I < 0 counts as 0.
 * Asynchronous on `stream`; -1 on NULL arrays or n < 0. */
int bh_stokes_steps(long long n, const float *state, const float *coef, float *out, void *stream);

/* BH_KERNEL_FP32_BASELINE (kernel_launch.h:156). */
int bh_select_kernel_variant(void);

/* CUDA texture objects the next launches sample (0 = none); the values are
 * copied into each launch. Slot meanings as the reference (kernel_launch.h:
 * 158-180): emissivity (2D, float, sampled at (u, 0.5)), redshift (unused:
 * g is exact), spectral (2D, float), grb, galaxy (cube map, float4), grmhd,
 * synch_g, grmhd_right (unused here). */
void bh_upload_lut_textures(unsigned long long emissivity, unsigned long long redshift,
                            unsigned long long spectral, unsigned long long grb, unsigned long long galaxy,
                            unsigned long long grmhd, unsigned long long synch_g,
                            unsigned long long grmhd_right);

/* An equirectangular float4 background (2D texture object, normalized
 * coordinates; u = azimuth / 2 pi + 1/2, v = polar angle / pi), used when no
 * galaxy cube map is set (kernel_launch.h:182-189). */
void bh_upload_bridge_background_texture(unsigned long long background_equirect);

/* ---- backend (src/cuda/cuda_backend.h) ------------------------------------ */

typedef struct BhCudaBackend BH_CudaBackend;

/* A headless backend owning a width x height float4 device framebuffer on the
 * current device. gl_texture is accepted and ignored: there is no OpenGL
 * interop here, the image stays in device memory (bhCudaFramebuffer). */
BH_CudaBackend *bhCudaInit(unsigned int gl_texture, int width, int height);
/* Render one frame (params->width/height must match) and wait for it. */
int bhCudaRenderFrame(BH_CudaBackend *backend, const struct BH_LaunchParams *params);
int bhCudaResize(BH_CudaBackend *backend, unsigned int gl_texture, int width, int height);
/* OpenGL textures cannot be registered here: both return -1; pass CUDA
 * texture objects to bh_upload_lut_textures instead. */
int bhCudaRegisterLut(BH_CudaBackend *backend, int slot, unsigned int gl_texture, unsigned int target);
int bhCudaRegisterBackgroundTexture(BH_CudaBackend *backend, unsigned int gl_texture, unsigned int target);
/* Returns the variant in use (negative = automatic), -1 for an invalid one. */
int bhCudaSetVariant(BH_CudaBackend *backend, int variant);
int bhCudaGetVariant(BH_CudaBackend *backend);
void bhCudaShutdown(BH_CudaBackend *backend); /* NULL-safe */
/* The backend's device framebuffer (float4 [height][width]); not in the
 * reference, which hands the image to OpenGL instead. */
void *bhCudaFramebuffer(BH_CudaBackend *backend);

/* ---- Blender bridge (src/blender_bridge/blender_bridge.h) ------------------- */

struct BhbDiskParams {
    double aStar;
    double massMsun;
    double mdotEdd;
    double rOutRg;
    double inclinationRad;
};

int bhbHasCuda(void);
/* Releases this layer's device buffers. The reference resets the device; the
 * primary context is shared here with the rest of the library (and torch), so
 * it is left alone. */
int bhbCudaResetDevice(void);

/* Camera on the (y, z) circle of radius observerR [rs] at inclination from
 * +z, looking at the hole, field of view fovScale (1.0 for the plain call);
 * the frame is post-processed by bhb_cuda_postprocess (bloom threshold 1,
 * strength 0, exposure 12) into outRgba (host, width * height * 4 floats).
 * BLACKHOLE_BRIDGE_* environment variables override the render settings as in
 * src/blender_bridge/cuda_renderer.cu:425-552, 665-673 (STEP_SIZE, MAX_DIST,
 * MAX_STEPS, FRAME_SHIFT_X/Y, ADISK_ENABLED, REDSHIFT_ENABLED,
 * DOPPLER_STRENGTH, BACKGROUND_*, PHOTON_GLOW_STRENGTH, ADISK_LIT,
 * BLOOM_THRESHOLD, BLOOM_STRENGTH, EXPOSURE). */
int bhbCudaRenderRaytraced(float spin, float observerR, float inclinationRad, int width, int height,
                           float *outRgba);
int bhbCudaRenderRaytracedCamera(float spin, float observerR, float inclinationRad, float fovScale, int width,
                                 int height, float *outRgba);
/* Camera from a world position [rs] and column-major basis (right, up, forward). */
int bhbCudaRenderRaytracedView(float spin, const float *camPos, const float *camBasis, float fovScale, int width,
                               int height, float *outRgba);

/* Distant observer at observerRRg [M], image plane alpha = 30 (ix / width - 1/2),
 * beta = 30 (1/2 - iy / height) [M]; per pixel R = sqrt(1 - 2 / r) at the disk
 * hit (1 for escaped rays, 0 for captured ones), G = the disk redshift g
 * (1 off the disk), B = 1 on a disk hit (isco <= r <= 100 M), A = 1. */
int bhbCudaRenderLensingMap(double aStar, double observerRRg, double inclinationRad, int width, int height,
                            float *outRgba);

/* Disk emission texture: row iy at r = isco + (rOutRg - isco) iy / height,
 * column ix at azimuth 2 pi ix / width; RGB = blackbody colour of the observed
 * temperature g T(r) (T from the Novikov-Thorne flux, g of a Keplerian
 * emitter seen from a distant observer at the inclination) times g^4 F / F_max,
 * A = T / T_max. */
int bhbCudaRenderDiskTexture(const struct BhbDiskParams *params, int width, int height, float *outRgba);

/* Paths of an image plane of Kerr rays from a distant observer at observerRRg
 * [M]: alpha_i = alphaMin + (alphaMax - alphaMin) i / (nAlpha - 1), beta
 * likewise. Each ray (index j * nAlpha + i) writes the Cartesian position
 * (x, y, z) = r (sin th cos ph, sin th sin ph, cos th) [M] after every step of
 * the FP64 RK4 tracer with affine step stepSize min(1, r / 20), up to
 * maxSteps points, into outXyz (host, nAlpha * nBeta * maxSteps * 3 floats);
 * outCounts receives the points written. Rays stop at the horizon or at
 * 1.01 observerRRg; the disk is transparent. The reference returns -1 here
 * (src/blender_bridge/blender_bridge.cpp:706-714). */
int bhbCudaTraceGeodesics(double aStar, double observerRRg, double inclinationRad, double alphaMin, double alphaMax,
                          int nAlpha, double betaMin, double betaMax, int nBeta, int maxSteps, double stepSize,
                          float *outXyz, int *outCounts);

/* Post-processing of a device float4 framebuffer (width * height RGBA), in
 * place (src/blender_bridge/cuda_postprocess.cu:237-275): bloom = the sum over
 * half-widths 4, 8, 16, 32 of the Gaussian blur (sigma = half-width / 2,
 * clamped edges) of the bright-pass (colour scaled by max(0, L - threshold) / L,
 * L the Rec. 709 luminance, 0 where L <= 0.001), added times bloom_strength
 * (skipped when it is 0); then per pixel: x exposure_gain, x the vignette
 * sqrt(max(0, 1 - d^2 / 2)) (d the distance from the centre in uv), the ACES
 * fit of Narkowicz (2015) clamped to [0, 1], gamma 1 / 2.2, alpha 1. Red and
 * blue are read at (int(u w), int(v h)) of the float uv, as the reference's
 * chromatic-aberration lookup at strength 0 does. time_sec is accepted and
 * unused (the reference's film grain is absent from its kernel too). Returns
 * 0 after the work has finished, -1 on a NULL framebuffer, a non-positive
 * size or a CUDA error. */
int bhb_cuda_postprocess(float *d_framebuffer, int width, int height, float bloom_threshold, float bloom_strength,
                         float exposure_gain, float time_sec);

/* snake_case aliases used by the add-on's ctypes binding (float arguments). */
int bhb_cuda_render_raytraced(float spin, float observer_r, float inclination_rad, int width, int height,
                              float *out_rgba);
int bhb_cuda_render_raytraced_camera(float spin, float observer_r, float inclination_rad, float fov_scale,
                                     int width, int height, float *out_rgba);
int bhb_cuda_render_raytraced_view(float spin, const float *cam_pos, const float *cam_basis, float fov_scale,
                                   int width, int height, float *out_rgba);
int bhb_cuda_render_lensing_map(float a_star, float obs_r, float inc_rad, int width, int height, float *out_rgba);
int bhb_cuda_render_disk_texture(float a_star, float r_out_rg, float inc_rad, int width, int height,
                                 float *out_rgba);

#ifdef __cplusplus
}
#endif

#endif /* BH_LEGACY_H */
