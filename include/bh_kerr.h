/*
 * bh_kerr.h - C ABI of the B200 Kerr null-geodesic tracer.
 *
 * Plain C (C99) header: no C++ types, no CUDA types, no torch types. Every
 * pointer is either a device pointer (functions without a _host suffix) or a
 * host pointer (functions with a _host suffix). All functions return 0 on
 * success and -1 on error; the message of the last error on the calling
 * thread is available from bh_last_error().
 *
 * Two families of entry points live here:
 *
 *  1. Batched drop-ins for the reference's src/physics Kerr API (CGS units,
 *     mass in grams, spin parameter a in cm, exactly as the reference):
 *       bh_kerr_potentials      <- physics::kerrPotentials   (src/physics/kerr.cpp:69-97)
 *       bh_kerr_step_mino       <- physics::kerrStepMino     (src/physics/kerr.cpp:99-134)
 *       bh_kerr_trace_rays      <- physics::KerrRaytracer::trace (src/physics/raytracer.h:324-378)
 *     These reproduce the reference's first-order, sign-flip Mino-time scheme
 *     operation for operation (FP64, no FMA contraction).
 *
 *  2. The image-plane tracer (geometric units, M = 1):
 *       bh_kerr_trace_image / bh_kerr_trace_image_host
 *     Per-pixel backward null geodesics from a distant observer, classified as
 *     captured / disk / escaped, with disk-hit radius, azimuth, redshift g,
 *     Novikov-Thorne flux and intensity. Integrates the reference's Mino-time
 *     potentials (kerr.cpp:69-97) in second-order form.
 */
#ifndef BH_KERR_H
#define BH_KERR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BH_KERR_ABI_VERSION 1

/* ---------------------------------------------------------------------------
 * Common
 * ------------------------------------------------------------------------- */

/** Message of the last failed call on this thread ("" if none). Never NULL. */
const char *bh_last_error(void);

/** ABI version of the loaded library (BH_KERR_ABI_VERSION it was built with). */
int bh_abi_version(void);

/* ---------------------------------------------------------------------------
 * 1. Reference src/physics API, batched on the GPU (CGS units)
 * ------------------------------------------------------------------------- */

/** Status codes of physics::RayStatus (src/physics/raytracer.h:46-52). */
enum BH_RayStatus {
    BH_STATUS_PROPAGATING = 0,
    BH_STATUS_ESCAPED = 1,
    BH_STATUS_CAPTURED = 2,
    BH_STATUS_HIT_DISK = 3,
    BH_STATUS_MAX_STEPS = 4
};

/**
 * Structure-of-arrays view of n Kerr geodesic states
 * (physics::KerrGeodesicState, src/physics/kerr.h:381-388). Device pointers,
 * each of length n. sign_r / sign_theta hold +1.0 or -1.0.
 */
typedef struct BH_KerrStateSoA {
    double *r;
    double *theta;
    double *phi;
    double *t;
    double *sign_r;
    double *sign_theta;
} BH_KerrStateSoA;

/**
 * Structure-of-arrays view of n constants of motion
 * (physics::KerrGeodesicConsts, src/physics/kerr.h:362-366). Device pointers.
 */
typedef struct BH_KerrConstsSoA {
    const double *e;
    const double *lz;
    const double *q;
} BH_KerrConstsSoA;

/**
 * Batched physics::kerrPotentials (src/physics/kerr.cpp:69-97).
 * out_* are device arrays of length n; any of them may be NULL.
 */
int bh_kerr_potentials(int64_t n, const double *r, const double *theta,
                       double mass, double a, BH_KerrConstsSoA consts,
                       double *out_r_pot, double *out_dr_pot,
                       double *out_theta_pot, double *out_dtheta_pot,
                       void *stream);

/**
 * Batched physics::kerrStepMino (src/physics/kerr.cpp:99-134): one Mino-time
 * RK4 step of each state, in place. dlam is a device array of length n, or
 * NULL to use dlam_scalar for every state.
 */
int bh_kerr_step_mino(int64_t n, BH_KerrStateSoA state, double mass, double a,
                      BH_KerrConstsSoA consts, const double *dlam,
                      double dlam_scalar, void *stream);

/**
 * Parameters of physics::KerrRaytracer (src/physics/raytracer.h:309-399).
 * bh_kerr_raytracer_defaults() fills them exactly as the reference's
 * constructor does: horizon = outer horizon (or r_s if not finite/positive),
 * escape radius = 1000 r_s, step = 0.02 r_s, 10000 steps.
 */
typedef struct BH_KerrRaytracerParams {
    double mass;          /**< black-hole mass [g] */
    double a;             /**< spin parameter [cm], already clamped like physics::Kerr */
    double r_horizon;     /**< capture when r <= 1.001 * r_horizon */
    double r_escape;      /**< escape when r >= r_escape */
    double step_size;     /**< Mino-time step dlam */
    int32_t max_steps;
    int32_t reserved;
} BH_KerrRaytracerParams;

/** Fill params as physics::KerrRaytracer(mass, spinParam) does. */
int bh_kerr_raytracer_defaults(double mass, double spin_param,
                               BH_KerrRaytracerParams *out_params);

/**
 * Batched physics::KerrRaytracer::trace (src/physics/raytracer.h:324-378).
 * initial: n start states (not modified). Outputs (device, length n, any may
 * be NULL): status (BH_RayStatus), steps taken, total distance, final
 * (r, theta, phi) and the redshift 1 + kerrRedshift(r_final, theta_final).
 */
int bh_kerr_trace_rays(int64_t n, BH_KerrStateSoA initial, BH_KerrConstsSoA consts,
                       const BH_KerrRaytracerParams *params,
                       int32_t *out_status, int32_t *out_steps,
                       double *out_total_distance, double *out_r,
                       double *out_theta, double *out_phi, double *out_redshift,
                       void *stream);

/**
 * The same three calls with HOST arrays (every pointer above in host memory,
 * outputs NULL = not wanted): the library stages them through device buffers
 * of the calling thread and returns when the results are back. These serve
 * callers of the reference's scalar C++ API (include/bh_physics_compat.hpp)
 * that hold their states in host memory.
 */
int bh_kerr_potentials_host(int64_t n, const double *r, const double *theta,
                            double mass, double a, BH_KerrConstsSoA consts,
                            double *out_r_pot, double *out_dr_pot,
                            double *out_theta_pot, double *out_dtheta_pot);
int bh_kerr_step_mino_host(int64_t n, BH_KerrStateSoA state, double mass, double a,
                           BH_KerrConstsSoA consts, const double *dlam,
                           double dlam_scalar);
int bh_kerr_trace_rays_host(int64_t n, BH_KerrStateSoA initial, BH_KerrConstsSoA consts,
                            const BH_KerrRaytracerParams *params,
                            int32_t *out_status, int32_t *out_steps,
                            double *out_total_distance, double *out_r,
                            double *out_theta, double *out_phi, double *out_redshift);

/* ---------------------------------------------------------------------------
 * 2. Image-plane tracer (geometric units G = c = M = 1)
 * ------------------------------------------------------------------------- */

/** Per-pixel termination class. */
enum BH_PixelClass {
    BH_CLASS_CAPTURED = 0,  /**< r <= horizon_factor * r_+ */
    BH_CLASS_DISK = 1,      /**< stopped by the thin disk (opaque, or last allowed crossing) */
    BH_CLASS_ESCAPED = 2,   /**< r >= escape_factor * r_obs */
    BH_CLASS_MAX_STEPS = 3  /**< step budget exhausted */
};

enum BH_Integrator {
    BH_INTEGRATOR_RK4 = 0,  /**< fixed affine step h = step_coeff * min(r, step_rcap), dsigma = h / Sigma */
    BH_INTEGRATOR_DP45 = 1, /**< Dormand-Prince 5(4), rtol/atol on (r, cos theta, phi, p_r, p_u) */
    /** No stepping: each ray in closed form (Jacobi elliptic functions of Mino time for r, the polar
     *  angle and the azimuth; elliptic integrals in Carlson's form), FP64 whatever the precision,
     *  the same cost per crossing in the photon-ring band as elsewhere. Single-frame calls only
     *  (bh_kerr_trace_image*, bh_kerr_trace_image_sky). Rays it does not cover (a turning point
     *  between r+ and the horizon cut, q_R < 0 rays that reach the equator or escape, four complex
     *  roots with equator crossings) are traced by DP45 at the scene's precision with its rtol/atol.
     *  steps = 0 on analytic pixels; escaped rays report theta_inf, phi_inf and the sky radiance
     *  at exactly escape_factor * r_obs (the steppers report them after their last step's
     *  overshoot past it). The analytic counterpart of src/physics/analytic_kerr_geodesic.h
     *  (rAnalytic for bound orbits) and src/cuda/device_analytic_kerr.cuh, for image rays. */
    BH_INTEGRATOR_ANALYTIC = 2
};

enum BH_Precision {
    BH_PRECISION_FP64 = 0,  /**< every operation in FP64 */
    BH_PRECISION_MIXED = 1  /**< FP32 right-hand sides with compensated FP32 state; FP64 set-up,
                                 horizon-approach and disk-crossing steps */
};

/**
 * Meaning of the Carter constant inside the potentials.
 * REFERENCE: R(r) and Theta(theta) both take the reference's single q
 *   (kerr.cpp:81-89, Theta = q + a^2 cos^2 - Lz^2 / sin^2); the image-plane
 *   set-up uses q = eta + lambda^2 so that Theta matches the camera ray, the
 *   convention of the reference's GPU set-up (src/cuda/device_physics.cuh:381-390).
 * CARTER: the textbook Carter potentials (R with eta, Theta with eta + lambda^2).
 */
enum BH_PotentialForm {
    BH_POTENTIAL_REFERENCE = 0,
    BH_POTENTIAL_CARTER = 1
};

#define BH_MAX_CROSSINGS 3

/** One image-plane scene. Pixel (i, j) looks at the centre of its cell:
 *  alpha = alpha_min + (i + 0.5) (alpha_max - alpha_min) / width, same for beta/height. */
typedef struct BH_KerrScene {
    double spin;            /**< a/M, |spin| < 1 */
    double r_obs;           /**< observer radius [M] */
    double theta_obs;       /**< observer inclination [rad], in (0, pi) */
    double alpha_min, alpha_max;
    double beta_min, beta_max;
    int32_t width, height;
    int32_t integrator;     /**< BH_Integrator */
    int32_t precision;      /**< BH_Precision */
    int32_t potential_form; /**< BH_PotentialForm */
    int32_t max_crossings;  /**< 1 = opaque disk; 2..3 = transparent disk, stop at that crossing */
    int32_t max_steps;      /**< accepted-step budget per ray */
    int32_t reserved0;
    double step_coeff;      /**< RK4: affine h = step_coeff * min(r, step_rcap); DP45: first trial step */
    double step_rcap;
    double rtol, atol;      /**< DP45 tolerances */
    double horizon_factor;  /**< capture radius = horizon_factor * r_+ (1.001) */
    double escape_factor;   /**< escape radius = escape_factor * r_obs (1.01) */
    double disk_r_in;       /**< <= 0 selects the prograde ISCO (physics::kerrIscoRadius) */
    double disk_r_out;      /**< outer disk edge [M] (30) */
} BH_KerrScene;

/** Fill a scene with the defaults of the 256x256 a=0.9 disk scene
 *  (r_obs = 1000, theta_obs = 60 deg, alpha, beta in [-12, 12], RK4,
 *  h = 0.02 min(r, 20), 20000 steps, opaque disk r_isco..30). */
void bh_kerr_scene_defaults(BH_KerrScene *scene);

/**
 * Per-pixel outputs, structure of arrays, n = width * height, row-major
 * (pixel = j * width + i). Crossing-indexed arrays hold max_crossings planes
 * of n values (plane k at offset k * n). Any pointer may be NULL.
 * Values of crossings that did not happen are 0.
 */
typedef struct BH_KerrImageOut {
    int32_t *cls;        /**< [n] BH_PixelClass */
    int32_t *steps;      /**< [n] accepted integration steps */
    int32_t *n_cross;    /**< [n] disk crossings recorded */
    double *r_hit;       /**< [max_crossings * n] crossing radius [M] */
    double *phi_hit;     /**< [max_crossings * n] crossing azimuth [rad], observer at phi = 0 */
    double *g;           /**< [max_crossings * n] redshift g = E_obs / E_emit (Keplerian emitter) */
    double *flux;        /**< [n] Novikov-Thorne normalised flux at the first crossing */
    double *intensity;   /**< [n] sum_k g_k^4 (r_in / r_k)^3 */
    double *theta_inf;   /**< [n] polar angle at escape [rad] */
    double *phi_inf;     /**< [n] azimuth at escape [rad] */
    /** [n] Carter-constant check of the mixed-precision tracer: the largest,
     *  over the ray's accepted steps, of |eta(state) - eta| / (|q_Th| + a^2),
     *  eta(state) = (p_u^2 + lambda^2 u^2) / (1 - u^2) - a^2 u^2 from the FP32
     *  step before its momenta are projected back onto the first integrals
     *  (evaluated in FP64, away from polar turning points; the reference's
     *  ConservationMonitor drift of Q, src/physics/conservation_monitor.h:64-105).
     *  Written by the mixed tracer only (0 for pixels the surrogate or the
     *  closed form answer); not returned by the host-buffer entry points. */
    double *carter_drift;
} BH_KerrImageOut;

/** Check a scene; returns 0 if valid, else -1 with bh_last_error() set. */
int bh_kerr_scene_validate(const BH_KerrScene *scene);

/**
 * Trace every pixel of the scene on the current CUDA device.
 * out holds DEVICE pointers. stream is a cudaStream_t (NULL = legacy default).
 * Asynchronous with respect to the host.
 */
int bh_kerr_trace_image(const BH_KerrScene *scene, const BH_KerrImageOut *out, void *stream);

/**
 * Same as bh_kerr_trace_image with HOST output pointers: device buffers are
 * allocated, the trace runs, the results are copied back, and the call
 * returns after the copies have completed.
 */
int bh_kerr_trace_image_host(const BH_KerrScene *scene, const BH_KerrImageOut *out_host);

/**
 * Size of the fixed device scratch of bh_kerr_trace_image_host_noalloc:
 * 32 MiB, resident on every GPU that loads the library until process exit.
 */
#define BH_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)

/**
 * Same as bh_kerr_trace_image_host, but allocates nothing. (It has no
 * counterpart in the reference.)
 *
 * For callers that cannot allocate device memory: a plug-in running inside a
 * host application that owns the GPU's memory (it reserves the device pool
 * up front, or forbids cudaMalloc/cudaFree on its render thread because they
 * can synchronise the whole device and stall its frame), or a real-time loop
 * that must not block on an allocation. The caller passes the scene and HOST
 * output buffers exactly as for bh_kerr_trace_image_host; the work counter
 * and the device copies of the outputs live in one fixed device array of
 * BH_NOALLOC_SCRATCH_BYTES. A call whose requested outputs (each rounded up
 * to 256 bytes) plus 256 bytes exceed that size is rejected with -1 and a
 * message; with BH_INTEGRATOR_ANALYTIC the list of pixels the closed form
 * leaves to DP45 takes 4 more bytes per pixel (rounded up to 256). With
 * every field and one disk crossing that allows about 490,000 pixels
 * (700 x 700), 465,000 (680 x 680) with the closed form.
 *
 * stream: cudaStream_t to run on (NULL = legacy default stream); the call
 * returns after that stream has finished the copies. It creates no stream
 * and calls no cudaMalloc, cudaFree or allocating library routine.
 * Every call looks up the array's device address on the current device
 * (cudaGetSymbolAddress; it allocates nothing). The first call on a device
 * also loads the library's device code there: make that first call before
 * any stream capture. Every call shares the array
 * and overwrites the previous call's contents: calls whose GPU work overlaps
 * race and must be serialised by the caller.
 */
int bh_kerr_trace_image_host_noalloc(const BH_KerrScene *scene, const BH_KerrImageOut *out_host, void *stream);

/** Launch configuration of the image tracer (0 = automatic; the closed-form
 * integrator keeps the CTA size it is compiled for). */
int bh_kerr_set_launch(int32_t block_threads, int32_t ctas_per_sm);

/* ---------------------------------------------------------------------------
 * 3. Batches: many frames of uneven size in one persistent launch
 * ------------------------------------------------------------------------- */

/** Opaque batch of frames (device frame table, work counter, per-frame timers). */
typedef struct BH_KerrBatch BH_KerrBatch;

/** Persistent-grid shape of a batch (0 = automatic for block / ctas_per_sm). */
typedef struct BH_KerrLaunchConfig {
    int32_t block_threads;  /**< 32..128, multiple of 32 */
    int32_t ctas_per_sm;    /**< resident CTAs per SM (<= occupancy limit) */
    int32_t refill_steps;   /**< integration steps between refills of finished lanes (>= 1) */
    int32_t reserved;
} BH_KerrLaunchConfig;

/**
 * Create a batch of n_frames frames on the current device. scenes[i] and
 * outs[i] (DEVICE output pointers, as for bh_kerr_trace_image) describe frame
 * i; all frames must share integrator and precision, everything else (size,
 * spin, inclination, observer radius, window, tolerances, disk) may differ.
 * The frame table is copied to the device now; returns NULL on error.
 */
BH_KerrBatch *bh_kerr_batch_create(const BH_KerrScene *scenes, const BH_KerrImageOut *outs, int32_t n_frames);

/** Trace every frame of the batch in one persistent launch (asynchronous). */
int bh_kerr_batch_trace(BH_KerrBatch *batch, void *stream);

/**
 * Same as bh_kerr_batch_trace through a CUDA graph: the first call captures
 * the launch (on stream, which must not be the legacy default stream), later
 * calls replay it. Changing the launch configuration drops the graph.
 */
int bh_kerr_batch_trace_graph(BH_KerrBatch *batch, void *stream);

/** Set / get the persistent-grid shape used by the next trace. */
int bh_kerr_batch_set_launch(BH_KerrBatch *batch, const BH_KerrLaunchConfig *cfg);
int bh_kerr_batch_get_launch(const BH_KerrBatch *batch, BH_KerrLaunchConfig *cfg);

/**
 * Autotune the grid shape: time the candidate configurations (block size,
 * resident CTAs per SM, refill interval) on the batch's first frames, up to
 * max_pixels pixels (0: 4 Mi), keep the fastest and return it in best.
 * Synchronous; overwrites those frames' outputs.
 */
int bh_kerr_batch_autotune(BH_KerrBatch *batch, int64_t max_pixels, void *stream, BH_KerrLaunchConfig *best);

/**
 * Completion time of each frame in the last trace, in milliseconds after the
 * launch's first CTA started (0 for frames without pixels). Synchronises with
 * the device. frame_ms: host array of n_frames floats.
 */
int bh_kerr_batch_frame_times(BH_KerrBatch *batch, float *frame_ms);

/** Number of frames and total pixels of the batch. */
int32_t bh_kerr_batch_frames(const BH_KerrBatch *batch);
int64_t bh_kerr_batch_pixels(const BH_KerrBatch *batch);

/** Free the batch (NULL is allowed). */
void bh_kerr_batch_destroy(BH_KerrBatch *batch);

/* ------------------------------------------------------------------------ */
/* Part 4: background sky of escaping rays                                   */
/* ------------------------------------------------------------------------ */

/**
 * A cubemap of FP16 texels on the device: [6][size][size], faces +X, -X, +Y,
 * -Y, +Z, -Z with the OpenGL cube-map addressing; an escaped ray samples the
 * nearest texel in its direction (theta_inf, phi_inf) at the escape radius.
 * The reference renders its sky from textures bound to its GL/CUDA kernels
 * (src/cuda/device_physics.cuh, background sampling of d_shade_hit); this is
 * its headless counterpart.
 */
typedef struct BH_SkyCubemap {
    const void *texels;
    int32_t size;
    int32_t reserved;
} BH_SkyCubemap;

/**
 * Fill `texels` (device, 6 * size^2 FP16) with the seeded sky: uniform noise
 * in [0, 1) plus n_stars point stars of brightness in [2, 20) added to single
 * texels (stars on the same texel add up). Deterministic in (size, n_stars,
 * seed); synchronises with the device when n_stars > 0.
 */
int bh_sky_generate(void *texels, int32_t size, int32_t n_stars, uint64_t seed, void *stream);

/** bh_kerr_trace_image plus the sky: escaped rays add the radiance of their
 *  texel to `intensity` (sky NULL: same as bh_kerr_trace_image). */
int bh_kerr_trace_image_sky(const BH_KerrScene *scene, const BH_KerrImageOut *out, const BH_SkyCubemap *sky,
                            void *stream);

/** Attach a sky to every frame of a batch (NULL detaches). */
int bh_kerr_batch_set_sky(BH_KerrBatch *batch, const BH_SkyCubemap *sky);

/* ---------------------------------------------------------------------------
 * 5. Diagnostics of device allocation (no counterpart in the reference, whose
 *    renderer reports a failed allocation only by returning -1 and asks its
 *    caller to re-initialise, src/cuda/cuda_render_manager.h:155-199)
 * ------------------------------------------------------------------------- */

/** Device allocations (cudaMalloc) the library has made in this process. */
int64_t bh_debug_device_allocations(void);

/**
 * Make the library's nth device allocation from now fail as if the device
 * were out of memory (nth = 1: the next one; 0: off). The entry point that
 * makes it returns -1 with a message naming the allocation and leaves its
 * cached buffers consistent, so the next call allocates afresh. For tests of
 * the error paths; a process uses it from one thread at a time.
 */
int bh_debug_fail_device_allocation(int64_t nth);

#ifdef __cplusplus
}
#endif

#endif /* BH_KERR_H */
