// Shapes, parameter layout and internal launchers of the learned transfer
// function: an MLP from image-plane position, spin and inclination to the
// ray's termination class, disk crossings, redshift and escape direction.
//
//   input   (alpha, beta, spin, cos theta_obs) -> 192 features (BF16):
//           16 Fourier frequencies x 4 inputs x (sin, cos) in columns 0..127,
//           the 4 scaled inputs and lambda, eta (the ray's constants of
//           motion) in 128..133, zero padding
//   hidden  4 layers x 256, SiLU, BF16 weights, FP32 accumulation
//   head    16 outputs (FP32): 3 class logits (captured, disk, escaped),
//           ln r1 - 2, cos phi1, sin phi1, ln r2 - 2, cos phi2, sin phi2,
//           g1 - 1, cos theta_inf, cos phi_inf, sin phi_inf, 3 unused
//
// Parameters (FP32 master copy, flat): for each layer l = 0..4 the weights
// W_l [N_l][K_l] (row-major, output-major) followed by the bias b_l [N_l].
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#define BHS_FEATURES 192
#define BHS_FEATURES_USED 134
#define BHS_HIDDEN 256
#define BHS_LAYERS 5
#define BHS_HEAD 16
#define BHS_HEAD_PAD 64
#define BHS_TARGETS 16
#define BHS_FOURIER 16

#ifdef __cplusplus
extern "C" {
#endif

// K_l (input width) and N_l (output width) of layer l.
static inline int bhs_layer_k(int l) { return l == 0 ? BHS_FEATURES : BHS_HIDDEN; }
static inline int bhs_layer_n(int l) { return l == BHS_LAYERS - 1 ? BHS_HEAD : BHS_HIDDEN; }
static inline int64_t bhs_weight_offset(int l) {
  int64_t off = 0;
  for (int j = 0; j < l; ++j) off += (int64_t)bhs_layer_n(j) * bhs_layer_k(j) + bhs_layer_n(j);
  return off;
}
static inline int64_t bhs_bias_offset(int l) {
  return bhs_weight_offset(l) + (int64_t)bhs_layer_n(l) * bhs_layer_k(l);
}
static inline int64_t bhs_param_count(void) { return bhs_weight_offset(BHS_LAYERS); }

// Epilogues of the BF16 GEMM C = A * B^T (A [M][K], B [N][K], both K-major).
enum BhsEpilogue {
  BHS_EPI_F32 = 0,     // C (FP32) [split][M][N] -- split-K partial sums
  BHS_EPI_HIDDEN = 1,  // H = SiLU(C + b) -> BF16 [M][N]; optional H^T [N][ld_t], pre-activation Y (FP32)
  BHS_EPI_HEAD = 2,    // out = C + b -> FP32 [M][16]
  BHS_EPI_BACKWARD = 3 // dY = C * SiLU'(Y) -> BF16 [M][N] and dY^T [N][ld_t]
};

typedef struct BhsGemm {
  const void* A;  // BF16 [M][lda]
  const void* B;  // BF16 [N][ldb]
  int64_t M;
  int N, K;
  int lda, ldb;
  int kchunks_per_split;  // 64-wide K chunks per split (0 = all)
  int epilogue;
  const float* bias;      // HIDDEN, HEAD
  const float* Y;         // BACKWARD: pre-activation [M][N]
  void* out;              // F32 partials, BF16 H / dY, or FP32 head
  void* out_t;            // BF16 transposed copy [N][ld_t] (optional)
  float* y_out;           // HIDDEN: pre-activation (optional)
  int64_t ld_t;
  uint64_t wait_ns;       // limit of each wait on another warp (>= 1)
} BhsGemm;

int bhs_launch_gemm(const BhsGemm* g, int* d_err, cudaStream_t stream);

// Fused inference of n rows (features, 4 hidden layers, head) in one
// persistent launch: head [n][16] = network(inputs [n][4]), FP16 weights wh
// (bhs_launch_refresh_f16) and activations, FP32 accumulation. host_bias:
// the 4 x 256 hidden biases then the 16 head biases (host memory, copied
// into the launch's parameters).
int bhs_launch_infer(const __half* const* wh, const float* host_bias, const float* inputs, int64_t n,
                     float* head, int* d_err, uint64_t wait_ns, cudaStream_t stream);

// FP16 inference weights W_l [N][K] from the master parameters.
int bhs_launch_refresh_f16(const float* params, __half* const* wh, cudaStream_t stream);

// Features of n rays from inputs [n][4] = (alpha, beta, spin, cos theta_obs).
int bhs_launch_features(const float* inputs, int64_t n, __nv_bfloat16* F, __nv_bfloat16* FT, int64_t ld_t,
            cudaStream_t stream);

// Loss and its gradient w.r.t. the head outputs. out [B][16], targets [B][16].
// dout [B][64] (columns >= 16 left untouched), dout_t [16][B]. loss[0..3] +=
// (cross entropy, regression, correct class count, counted rows).
int bhs_launch_loss(const float* out, const float* targets, int64_t B, __nv_bfloat16* dout,
          __nv_bfloat16* dout_t, float* loss, cudaStream_t stream);

// grad[bias of layer l][n] = sum_b dY_l^T[n][b] for all layers at once.
int bhs_launch_bias_grads(const __nv_bfloat16* const* dyt, int64_t B, float* grad, cudaStream_t stream);

// grad[W_l] = sum over splits of the partials (layer 4 stored transposed).
int bhs_launch_collect_dw(const float* const* partials, const int* splits, float* grad, cudaStream_t stream);

// Adam on the master parameters; refreshes the BF16 weights W_l [N][K] and
// their transposes W_l^T [K][N] (layer 4: [256][64], zero beyond 16).
int bhs_launch_adam(float* params, const float* grad, float* m, float* v, int64_t n, float lr_t, float beta1,
          float beta2, float eps, __nv_bfloat16* const* wb, __nv_bfloat16* const* wt,
          cudaStream_t stream);

// BF16 weights (and transposes) from the master parameters.
int bhs_launch_refresh_bf16(const float* params, __nv_bfloat16* const* wb, __nv_bfloat16* const* wt,
              cudaStream_t stream);

// Training targets from tracer outputs (planes [max_crossings][n]).
int bhs_launch_make_targets(const int* cls, const int* n_cross, const double* r_hit, const double* phi_hit,
              const double* g, const double* theta_inf, const double* phi_inf, int64_t n,
              int max_crossings, float* targets, cudaStream_t stream);

// Inputs [n][4] of every pixel of an image-plane grid.
int bhs_launch_grid_inputs(double spin, double cos_theta, double alpha_min, double dalpha, double beta_min,
              double dbeta, int width, int64_t n, float* inputs, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
