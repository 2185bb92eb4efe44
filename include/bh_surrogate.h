/*
 * bh_surrogate.h -- learned transfer function for Kerr image-plane rays.
 *
 * No counterpart in the reference: the reference's renderer always
 * integrates every pixel (src/cuda/device_physics.cuh:912-1017,
 * src/physics/raytracer.h:324-378). This interface adds a small MLP that maps
 * (alpha, beta, spin, cos theta_obs) to the ray's termination class (captured,
 * disk, escaped), the radius and azimuth of its first two disk crossings, the
 * redshift g of the first, and its escape direction. The network is trained
 * on rays the integrator itself traces (bh_kerr_trace_image /
 * bh_kerr_batch_*) by BF16 tensor-core kernels (tcgen05, FP32 accumulation):
 * forward, backward and Adam all run on the GPU.
 *
 * Conventions follow bh_kerr.h: 0 = success, -1 = error with a message in
 * bh_last_error(); device pointers unless a name says host; a NULL stream is
 * the legacy default stream. Inputs are FP32 [n][4] rows (alpha, beta, spin,
 * cos theta_obs). Head outputs are FP32 [n][16] rows:
 *   0..2  class logits (captured, disk, escaped)
 *   3     ln r1 - 2     4, 5  cos phi1, sin phi1
 *   6     ln r2 - 2     7, 8  cos phi2, sin phi2
 *   9     g1 - 1        10    cos theta_inf     11, 12  cos phi_inf, sin phi_inf
 *   13..15 unused
 * Training targets are FP32 [n][16] rows (bh_surrogate_make_targets):
 *   0 opaque-disk class (0, 1, 2; -1 = not used), 1 disk crossings (0..2),
 *   2..11 the regression targets of head outputs 3..12, 12..15 zero.
 */
#ifndef BH_SURROGATE_H
#define BH_SURROGATE_H

#include <stdint.h>

#include "bh_kerr.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct BH_Surrogate BH_Surrogate;

typedef struct BH_AdamConfig {
    float lr;
    float beta1;
    float beta2;
    float eps;
} BH_AdamConfig;

/* Number of FP32 parameters: per layer l = 0..4, W_l [N_l][K_l] then b_l [N_l];
 * K = 192, 256, 256, 256, 256 and N = 256, 256, 256, 256, 16. */
int64_t bh_surrogate_param_count(void);

/* A network with seeded random weights on the current device, with training
 * buffers for batches of up to max_batch rows (a multiple of 128). */
BH_Surrogate* bh_surrogate_create(int64_t max_batch, uint64_t seed);
void bh_surrogate_destroy(BH_Surrogate* s); /* NULL-safe */

int bh_surrogate_get_params(const BH_Surrogate* s, float* host_params, int64_t n);
int bh_surrogate_set_params(BH_Surrogate* s, const float* host_params, int64_t n);

/* Adam state (first and second moments, bh_surrogate_param_count() values
 * each, and the step count) for checkpoints; set_params resets it, so
 * restore it after the parameters. */
int bh_surrogate_get_state(const BH_Surrogate* s, float* adam_m, float* adam_v, int64_t n, int64_t* step);
int bh_surrogate_set_state(BH_Surrogate* s, const float* adam_m, const float* adam_v, int64_t n, int64_t step);

/* Input features (BF16 [n][192]) of n rows; diagnostic. */
int bh_surrogate_features(const float* inputs, int64_t n, void* features_bf16, void* stream);

/* Head outputs [n][16] for n rows (inference, any n). */
int bh_surrogate_forward(BH_Surrogate* s, const float* inputs, int64_t n, float* head, void* stream);

/* Loss gradient w.r.t. every parameter (FP32, bh_surrogate_param_count()
 * values) for one batch; loss4 (4 floats, may be NULL) receives the sums of
 * cross entropy, squared regression error, correctly classified rows and
 * classified rows. Parameters are not changed. */
int bh_surrogate_gradients(BH_Surrogate* s, const float* inputs, const float* targets, int64_t batch,
                           float* grad, float* loss4, void* stream);

/* One Adam step on one batch (forward, backward, update). */
int bh_surrogate_train_step(BH_Surrogate* s, const float* inputs, const float* targets, int64_t batch,
                            const BH_AdamConfig* adam, float* loss4, void* stream);

/* Synchronise the device and return the first kernel error code recorded by
 * a bounded wait since the last call (0 = none), then clear it. */
int bh_surrogate_device_error(BH_Surrogate* s);

/* Limit of each wait of the network's tensor-core kernels on another warp's
 * progress (an mbarrier phase), in ns; 0 restores the default of 2 s. A wait
 * that runs out records an error code (bh_surrogate_device_error), lets the
 * work its own thread started finish, frees its tensor memory and returns,
 * so the context stays usable. The reference has no counterpart; its
 * renderer's contract on a failure is an error return after which the caller
 * re-initialises (src/cuda/cuda_render_manager.h:155-199). */
int bh_surrogate_set_wait_limit(BH_Surrogate* s, int64_t ns);

/* Training targets from integrator outputs (device planes as written by
 * bh_kerr_trace_image with the given max_crossings). */
int bh_surrogate_make_targets(const BH_KerrImageOut* outs, int64_t n, int max_crossings, float* targets,
                              void* stream);

/* Inputs [width * height][4] of a scene's pixel centres. */
int bh_surrogate_grid_inputs(const BH_KerrScene* scene, float* inputs, void* stream);

/* Which pixels the surrogate renderer leaves to the integrator. */
typedef struct BH_SurrogatePolicy {
    float min_confidence;  /* softmax class probability below this -> integrator (0.99) */
    int32_t verify;        /* 1: check the radial kind of captured/escaped predictions;
                              2: run the exact crossing search on every pixel, and send a
                                 pixel whose solved class contradicts the network's to the
                                 integrator;
                              3: as 2, but the solved class stands (the network only seeds
                                 the Newton iteration of the solve) */
    double critical_band;  /* first-order image-plane distance to the critical curve, M,
                              below which a pixel goes to the integrator (0.05) */
    int32_t refine_fp64;   /* 0: Mino-time quadrature in FP32 (r_hit to ~4e-6, up to ~5e-5 for rays
                              just outside the critical band); 1: all FP64 (~1e-8) */
    int32_t chunks;        /* pixel chunks whose refinement (second stream) overlaps the next
                              chunk's inference; 0 = default (1..8) */
} BH_SurrogatePolicy;

typedef struct BH_SurrogateStats {
    int64_t pixels;
    int64_t accepted;        /* answered without the integrator */
    int64_t low_confidence;
    int64_t critical_band;
    int64_t solve_failed;    /* radial potential not handled or no convergence */
    int64_t disagreement;    /* exact solve contradicts the network's class */
} BH_SurrogateStats;

void bh_surrogate_policy_defaults(BH_SurrogatePolicy* policy);

/* Render a scene through the surrogate: network inference on every pixel,
 * exact Mino-time refinement of accepted disk hits (r_hit, g, flux,
 * intensity, phi_hit) and of escaped pixels' theta_inf and phi_inf, and the
 * closed-form tracer (DP45 at the scene's precision on the rays it does not
 * cover) on every pixel the policy rejects. Outputs as bh_kerr_trace_image;
 * for accepted pixels steps = 0. No output field is the network's own
 * answer: it decides the class (checked per `verify`) and seeds the solve.
 * The azimuths are solved only when out->phi_hit or out->phi_inf is given.
 * Asynchronous on `stream`; no host sync. */
int bh_surrogate_trace_image(BH_Surrogate* s, const BH_KerrScene* scene, const BH_KerrImageOut* out,
                             const BH_SurrogatePolicy* policy, void* stream);

/* The same with HOST output buffers (BH_KerrImageOut of host pointers, NULL =
 * not wanted): grow-only device buffers owned by the network; returns when
 * the copies are done. With page-locked buffers (cudaMallocHost,
 * cudaHostRegister) the frame is rendered in policy->chunks chunks (0: 8)
 * and each chunk's rows are copied while the next one is inferred; the
 * pixels the policy rejected follow, gathered on the device into compact
 * arrays and scattered on the host (past max(4096, pixels / 25) of them the
 * frame is copied again; the gathered pixels go through a mapped page-locked
 * buffer the network keeps). Pageable buffers, or a failed allocation of that
 * buffer, get one copy per field after the render. The outputs are the same
 * either way.
 * Returns -1 with a message when an allocation fails or when a bounded wait
 * of the network's kernels ran out (the outputs are then not valid); the
 * next call starts afresh. */
int bh_surrogate_trace_image_host(BH_Surrogate* s, const BH_KerrScene* scene, const BH_KerrImageOut* out_host,
                                  const BH_SurrogatePolicy* policy);

/* Counts of the last bh_surrogate_trace_image (synchronises the device). */
int bh_surrogate_last_stats(BH_Surrogate* s, BH_SurrogateStats* stats);

/* C = A * B^T in FP32 for BF16 A [M][K], B [N][K] (K a multiple of 8;
 * N = 16, 192 or a multiple of 256): the tensor-core GEMM the network uses. */
int bh_bf16_gemm(const void* A, const void* B, int64_t M, int N, int K, float* C, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BH_SURROGATE_H */
