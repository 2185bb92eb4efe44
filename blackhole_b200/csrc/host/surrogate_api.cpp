// surrogate_api.cpp - C++23 host side of include/bh_surrogate.h.
//
// Owns the network's FP32 master parameters, Adam moments, BF16 weight
// copies (W_l and W_l^T) and the training activations, and sequences the
// GEMM and element-wise kernels of csrc/device/surrogate.cu for inference,
// gradients and training steps. Nothing here computes on the host except
// the seeded weight initialisation.
#include <cuda_bf16.h>
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <vector>

#include "../../../include/bh_surrogate.h"
#include "../device/launch.h"
#include "../device/surrogate_net.h"
#include "dalloc.hpp"

using bf16 = __nv_bfloat16;

constexpr int kRenderChunks = 8;   // most chunks a render splits into
constexpr int kDefaultChunks = 2;
constexpr uint64_t kDefaultWaitNs = 2000000000ull;  // 2 s per bounded device wait

struct BH_Surrogate {
  int device = -1;
  int64_t max_batch = 0;
  int64_t n_params = 0;
  int64_t step = 0;
  std::vector<void *> allocs;
  float *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
  bf16 *wb[BHS_LAYERS] = {}, *wt[BHS_LAYERS] = {};
  __half *wh[BHS_LAYERS] = {};  // FP16 inference copies, refreshed with the host biases
  // training activations, batch-major [B][.] and transposed [.][B]
  bf16 *F = nullptr, *FT = nullptr;
  bf16 *h[4] = {}, *ht[4] = {};
  float *y[4] = {};
  float *out = nullptr;
  bf16 *dout = nullptr, *dout_t = nullptr;
  bf16 *dy[4] = {}, *dyt[4] = {};
  float *part[BHS_LAYERS] = {};
  float *loss = nullptr;
  int *err = nullptr;
  // renderer buffers (grow-only)
  int64_t ren_pixels = 0;
  float *r_inputs = nullptr, *r_head = nullptr;
  int *r_list = nullptr;
  int *r_list2 = nullptr;            // rejected pixels the closed form leaves to DP45
  unsigned int *r_counts = nullptr;  // [0] list length, [1..5] stats, [6] list2 length
  unsigned long long *r_counter = nullptr;
  int64_t last_pixels = 0;
  // renderer concurrency: refine of chunk k on `side` while chunk k+1 is inferred
  cudaStream_t side = nullptr;
  cudaEvent_t ev[kRenderChunks + 2] = {};
  // device outputs and stream of the host-buffer entry point (grow-only)
  char *host_out = nullptr;
  size_t host_out_bytes = 0;
  cudaStream_t host_stream = nullptr;
  // its copies: each chunk's rows go to the host as soon as they are refined
  // (copy_stream), and the rejected pixels, which the fallback writes later,
  // follow in compact form
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_ev[kRenderChunks] = {};    // chunk k refined (recorded on side)
  cudaEvent_t copy_done[kRenderChunks] = {};  // chunk k's rows on the host (copy_stream)
  cudaEvent_t gathered = nullptr;             // compact arrays written (host_stream)
  char *gather_host = nullptr;  // mapped, page-locked: written by the gather kernel over the bus
  char *gather_dev = nullptr;   // its device address
  size_t gather_bytes = 0;
  // host copy of the biases for the fused inference launch
  std::vector<float> host_bias;
  bool bias_stale = true;
  // limit of each bounded device wait on another warp's progress
  uint64_t wait_ns = kDefaultWaitNs;
};

namespace {

constexpr int kDwChunks = 8;  // 64-row K chunks per split of the batch reduction

int fail_msg(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
int fail_msg(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return bhh_fail(buf);
}

int cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return 0;
  return fail_msg("%s: %s", what, cudaGetErrorString(e));
}

template <class T>
int alloc(BH_Surrogate *s, T **p, size_t count, const char *what) {
  void *q = nullptr;
  if (int rc = cuda_check(bhh_malloc(&q, std::max<size_t>(count, 1) * sizeof(T)), what)) return rc;
  s->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return 0;
}

int64_t dw_splits(int64_t batch) {
  const int64_t chunks = (batch + 63) / 64;
  return (chunks + kDwChunks - 1) / kDwChunks;
}

uint64_t splitmix(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Uniform weights of variance 1/fan_in (fan_in = the used input width),
// zero for the padded feature columns, smaller for the head, zero biases.
std::vector<float> init_params(uint64_t seed) {
  std::vector<float> p(static_cast<size_t>(bhs_param_count()), 0.0f);
  uint64_t st = seed ^ 0x5DEECE66Dull;
  for (int l = 0; l < BHS_LAYERS; ++l) {
    const int K = bhs_layer_k(l), N = bhs_layer_n(l);
    const int used = l == 0 ? BHS_FEATURES_USED : K;
    const double scale = std::sqrt(3.0 / used) * (l == BHS_LAYERS - 1 ? 0.5 : 1.0);
    float *W = p.data() + bhs_weight_offset(l);
    for (int n = 0; n < N; ++n)
      for (int k = 0; k < used; ++k) {
        const double u = static_cast<double>(splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
        W[static_cast<size_t>(n) * K + k] = static_cast<float>((2.0 * u - 1.0) * scale);
      }
  }
  return p;
}

int refresh(BH_Surrogate *s, cudaStream_t st) {
  if (bhs_launch_refresh_bf16(s->w, s->wb, s->wt, st) != 0) return fail_msg("surrogate: weight refresh launch failed");
  return 0;
}

int gemm(BH_Surrogate *s, const BhsGemm &g0, cudaStream_t st, const char *what) {
  BhsGemm g = g0;
  g.wait_ns = s->wait_ns;
  if (bhs_launch_gemm(&g, s->err, st) != 0)
    return fail_msg("surrogate: GEMM launch failed (%s: M=%lld N=%d K=%d)", what, static_cast<long long>(g.M), g.N,
                    g.K);
  return 0;
}

BhsGemm make_gemm(const void *A, int lda, const void *B, int ldb, int64_t M, int N, int K, int epi) {
  BhsGemm g{};
  g.A = A;
  g.B = B;
  g.M = M;
  g.N = N;
  g.K = K;
  g.lda = lda;
  g.ldb = ldb;
  g.epilogue = epi;
  return g;
}

// Forward (saving what backward needs), loss, backward, gradient collection.
int forward_backward(BH_Surrogate *s, const float *inputs, const float *targets, int64_t B, float *loss4,
                     cudaStream_t st) {
  if (B <= 0 || B > s->max_batch || B % 128 != 0)
    return fail_msg("surrogate: batch %lld must be a positive multiple of 128 up to %lld", static_cast<long long>(B),
                    static_cast<long long>(s->max_batch));
  if (int rc = cuda_check(cudaMemsetAsync(s->loss, 0, 4 * sizeof(float), st), "cudaMemsetAsync(loss)")) return rc;
  if (bhs_launch_features(inputs, B, s->F, s->FT, B, st) != 0) return fail_msg("surrogate: feature launch failed");
  for (int l = 0; l < 4; ++l) {
    const bf16 *X = l == 0 ? s->F : s->h[l - 1];
    const int K = bhs_layer_k(l);
    BhsGemm g = make_gemm(X, K, s->wb[l], K, B, BHS_HIDDEN, K, BHS_EPI_HIDDEN);
    g.bias = s->w + bhs_bias_offset(l);
    g.out = s->h[l];
    g.out_t = s->ht[l];
    g.y_out = s->y[l];
    g.ld_t = B;
    if (int rc = gemm(s, g, st, "forward")) return rc;
  }
  {
    BhsGemm g = make_gemm(s->h[3], BHS_HIDDEN, s->wb[4], BHS_HIDDEN, B, BHS_HEAD, BHS_HIDDEN, BHS_EPI_HEAD);
    g.bias = s->w + bhs_bias_offset(4);
    g.out = s->out;
    if (int rc = gemm(s, g, st, "head")) return rc;
  }
  if (bhs_launch_loss(s->out, targets, B, s->dout, s->dout_t, s->loss, st) != 0)
    return fail_msg("surrogate: loss launch failed");
  {  // head: dW4^T = H4^T dout, dY4 = (dout W4) * SiLU'(Y4)
    BhsGemm g = make_gemm(s->ht[3], static_cast<int>(B), s->dout_t, static_cast<int>(B), BHS_HIDDEN, BHS_HEAD,
                          static_cast<int>(B), BHS_EPI_F32);
    g.kchunks_per_split = kDwChunks;
    g.out = s->part[4];
    if (int rc = gemm(s, g, st, "dW4")) return rc;
    BhsGemm d = make_gemm(s->dout, BHS_HEAD_PAD, s->wt[4], BHS_HEAD_PAD, B, BHS_HIDDEN, BHS_HEAD_PAD,
                          BHS_EPI_BACKWARD);
    d.Y = s->y[3];
    d.out = s->dy[3];
    d.out_t = s->dyt[3];
    d.ld_t = B;
    if (int rc = gemm(s, d, st, "dH4")) return rc;
  }
  for (int l = 3; l >= 0; --l) {
    const int K = bhs_layer_k(l);
    const bf16 *XT = l == 0 ? s->FT : s->ht[l - 1];
    BhsGemm g = make_gemm(s->dyt[l], static_cast<int>(B), XT, static_cast<int>(B), BHS_HIDDEN, K,
                          static_cast<int>(B), BHS_EPI_F32);
    g.kchunks_per_split = kDwChunks;
    g.out = s->part[l];
    if (int rc = gemm(s, g, st, "dW")) return rc;
    if (l == 0) break;
    BhsGemm d = make_gemm(s->dy[l], BHS_HIDDEN, s->wt[l], BHS_HIDDEN, B, BHS_HIDDEN, BHS_HIDDEN, BHS_EPI_BACKWARD);
    d.Y = s->y[l - 1];
    d.out = s->dy[l - 1];
    d.out_t = s->dyt[l - 1];
    d.ld_t = B;
    if (int rc = gemm(s, d, st, "dH")) return rc;
  }
  const bf16 *dyt[BHS_LAYERS] = {s->dyt[0], s->dyt[1], s->dyt[2], s->dyt[3], s->dout_t};
  if (bhs_launch_bias_grads(dyt, B, s->grad, st) != 0) return fail_msg("surrogate: bias-gradient launch failed");
  const float *parts[BHS_LAYERS] = {s->part[0], s->part[1], s->part[2], s->part[3], s->part[4]};
  const int sp = static_cast<int>(dw_splits(B));
  const int splits[BHS_LAYERS] = {sp, sp, sp, sp, sp};
  if (bhs_launch_collect_dw(parts, splits, s->grad, st) != 0) return fail_msg("surrogate: dW collection failed");
  if (loss4)
    if (int rc = cuda_check(cudaMemcpyAsync(loss4, s->loss, 4 * sizeof(float), cudaMemcpyDeviceToDevice, st),
                            "cudaMemcpyAsync(loss)"))
      return rc;
  return 0;
}

}  // namespace

extern "C" {

int64_t bh_surrogate_param_count(void) { return bhs_param_count(); }

void bh_surrogate_destroy(BH_Surrogate *s) {
  if (!s) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (s->device >= 0) cudaSetDevice(s->device);
  for (void *p : s->allocs) cudaFree(p);
  for (cudaEvent_t e : s->ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : s->copy_ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : s->copy_done)
    if (e) cudaEventDestroy(e);
  if (s->gathered) cudaEventDestroy(s->gathered);
  if (s->side) cudaStreamDestroy(s->side);
  if (s->host_stream) cudaStreamDestroy(s->host_stream);
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  if (s->gather_host) cudaFreeHost(s->gather_host);
  if (cur >= 0) cudaSetDevice(cur);
  delete s;
}

BH_Surrogate *bh_surrogate_create(int64_t max_batch, uint64_t seed) {
  if (max_batch < 128 || max_batch % 128 != 0) {
    fail_msg("surrogate: max_batch must be a positive multiple of 128, got %lld", static_cast<long long>(max_batch));
    return nullptr;
  }
  auto *s = new BH_Surrogate();
  s->max_batch = max_batch;
  s->n_params = bhs_param_count();
  const size_t B = static_cast<size_t>(max_batch);
  const size_t P = static_cast<size_t>(s->n_params);
  auto bad = [&]() {
    bh_surrogate_destroy(s);
    return static_cast<BH_Surrogate *>(nullptr);
  };
  if (cuda_check(cudaGetDevice(&s->device), "cudaGetDevice")) return bad();
  if (alloc(s, &s->w, P, "cudaMalloc(params)") || alloc(s, &s->m, P, "cudaMalloc(adam m)") ||
      alloc(s, &s->v, P, "cudaMalloc(adam v)") || alloc(s, &s->grad, P, "cudaMalloc(grad)"))
    return bad();
  for (int l = 0; l < BHS_LAYERS; ++l) {
    const size_t nk = static_cast<size_t>(bhs_layer_n(l)) * bhs_layer_k(l);
    if (alloc(s, &s->wb[l], nk, "cudaMalloc(bf16 weights)") || alloc(s, &s->wh[l], nk, "cudaMalloc(f16 weights)"))
      return bad();
    const size_t tsz = l == BHS_LAYERS - 1 ? static_cast<size_t>(BHS_HIDDEN) * BHS_HEAD_PAD : nk;
    if (alloc(s, &s->wt[l], tsz, "cudaMalloc(bf16 weights^T)")) return bad();
  }
  if (alloc(s, &s->F, B * BHS_FEATURES, "cudaMalloc(features)") ||
      alloc(s, &s->FT, B * BHS_FEATURES, "cudaMalloc(features^T)"))
    return bad();
  for (int i = 0; i < 4; ++i) {
    if (alloc(s, &s->h[i], B * BHS_HIDDEN, "cudaMalloc(H)") || alloc(s, &s->ht[i], B * BHS_HIDDEN, "cudaMalloc(H^T)") ||
        alloc(s, &s->y[i], B * BHS_HIDDEN, "cudaMalloc(Y)") || alloc(s, &s->dy[i], B * BHS_HIDDEN, "cudaMalloc(dY)") ||
        alloc(s, &s->dyt[i], B * BHS_HIDDEN, "cudaMalloc(dY^T)"))
      return bad();
  }
  if (alloc(s, &s->out, B * BHS_HEAD, "cudaMalloc(head)") ||
      alloc(s, &s->dout, B * BHS_HEAD_PAD, "cudaMalloc(dout)") ||
      alloc(s, &s->dout_t, B * BHS_HEAD, "cudaMalloc(dout^T)"))
    return bad();
  const size_t sp = static_cast<size_t>(dw_splits(max_batch));
  for (int l = 0; l < BHS_LAYERS; ++l) {
    const size_t per = l == BHS_LAYERS - 1 ? static_cast<size_t>(BHS_HIDDEN) * BHS_HEAD
                                           : static_cast<size_t>(BHS_HIDDEN) * bhs_layer_k(l);
    if (alloc(s, &s->part[l], sp * per, "cudaMalloc(dW partials)")) return bad();
  }
  if (alloc(s, &s->loss, 4, "cudaMalloc(loss)") || alloc(s, &s->err, 1, "cudaMalloc(error flag)")) return bad();
  // Zero what is only partly written: padded dout columns, W4^T padding, moments, flags.
  if (cuda_check(cudaMemset(s->dout, 0, B * BHS_HEAD_PAD * sizeof(bf16)), "cudaMemset") ||
      cuda_check(cudaMemset(s->wt[BHS_LAYERS - 1], 0, static_cast<size_t>(BHS_HIDDEN) * BHS_HEAD_PAD * sizeof(bf16)),
                 "cudaMemset") ||
      cuda_check(cudaMemset(s->m, 0, P * sizeof(float)), "cudaMemset") ||
      cuda_check(cudaMemset(s->v, 0, P * sizeof(float)), "cudaMemset") ||
      cuda_check(cudaMemset(s->err, 0, sizeof(int)), "cudaMemset"))
    return bad();
  const std::vector<float> init = init_params(seed);
  if (bh_surrogate_set_params(s, init.data(), s->n_params) != 0) return bad();
  return s;
}

int bh_surrogate_get_params(const BH_Surrogate *s, float *host, int64_t n) {
  if (!s || !host || n != s->n_params) return fail_msg("surrogate: get_params needs %lld values", s ? static_cast<long long>(s->n_params) : 0LL);
  return cuda_check(cudaMemcpy(host, s->w, static_cast<size_t>(n) * sizeof(float), cudaMemcpyDeviceToHost),
                    "cudaMemcpy(params)");
}

int bh_surrogate_set_params(BH_Surrogate *s, const float *host, int64_t n) {
  if (!s || !host || n != s->n_params) return fail_msg("surrogate: set_params needs %lld values", s ? static_cast<long long>(s->n_params) : 0LL);
  if (int rc = cuda_check(cudaMemcpy(s->w, host, static_cast<size_t>(n) * sizeof(float), cudaMemcpyHostToDevice),
                          "cudaMemcpy(params)"))
    return rc;
  if (int rc = refresh(s, nullptr)) return rc;
  s->bias_stale = true;
  s->step = 0;
  if (int rc = cuda_check(cudaMemset(s->m, 0, static_cast<size_t>(n) * sizeof(float)), "cudaMemset")) return rc;
  if (int rc = cuda_check(cudaMemset(s->v, 0, static_cast<size_t>(n) * sizeof(float)), "cudaMemset")) return rc;
  return cuda_check(cudaDeviceSynchronize(), "set_params");
}

int bh_surrogate_get_state(const BH_Surrogate *s, float *m, float *v, int64_t n, int64_t *step) {
  if (!s || !m || !v || !step || n != s->n_params)
    return fail_msg("surrogate: get_state needs two arrays of %lld values and a step pointer",
                    s ? static_cast<long long>(s->n_params) : 0LL);
  const size_t b = static_cast<size_t>(n) * sizeof(float);
  if (int rc = cuda_check(cudaMemcpy(m, s->m, b, cudaMemcpyDeviceToHost), "cudaMemcpy(adam m)")) return rc;
  if (int rc = cuda_check(cudaMemcpy(v, s->v, b, cudaMemcpyDeviceToHost), "cudaMemcpy(adam v)")) return rc;
  *step = s->step;
  return 0;
}

int bh_surrogate_set_state(BH_Surrogate *s, const float *m, const float *v, int64_t n, int64_t step) {
  if (!s || !m || !v || n != s->n_params || step < 0)
    return fail_msg("surrogate: set_state needs two arrays of %lld values and step >= 0",
                    s ? static_cast<long long>(s->n_params) : 0LL);
  const size_t b = static_cast<size_t>(n) * sizeof(float);
  if (int rc = cuda_check(cudaMemcpy(s->m, m, b, cudaMemcpyHostToDevice), "cudaMemcpy(adam m)")) return rc;
  if (int rc = cuda_check(cudaMemcpy(s->v, v, b, cudaMemcpyHostToDevice), "cudaMemcpy(adam v)")) return rc;
  s->step = step;
  return 0;
}

int bh_surrogate_features(const float *inputs, int64_t n, void *features, void *stream) {
  if (n < 0 || (n > 0 && (!inputs || !features))) return fail_msg("surrogate: bad feature arguments");
  if (bhs_launch_features(inputs, n, static_cast<bf16 *>(features), nullptr, 0, static_cast<cudaStream_t>(stream)))
    return fail_msg("surrogate: feature launch failed");
  return 0;
}

int bh_surrogate_forward(BH_Surrogate *s, const float *inputs, int64_t n, float *head, void *stream) {
  if (!s || n < 0 || (n > 0 && (!inputs || !head))) return fail_msg("surrogate: bad forward arguments");
  if (n == 0) return 0;
  if (s->bias_stale) {  // after training steps: fetch the biases once (synchronous), refresh the FP16 weights
    if (bhs_launch_refresh_f16(s->w, s->wh, static_cast<cudaStream_t>(stream)) != 0)
      return fail_msg("surrogate: FP16 weight refresh launch failed");
    s->host_bias.resize(4 * BHS_HIDDEN + BHS_HEAD);
    for (int l = 0; l < BHS_LAYERS; ++l)
      if (int rc = cuda_check(cudaMemcpy(s->host_bias.data() + l * BHS_HIDDEN, s->w + bhs_bias_offset(l),
                                         static_cast<size_t>(bhs_layer_n(l)) * sizeof(float), cudaMemcpyDeviceToHost),
                              "cudaMemcpy(biases)"))
        return rc;
    s->bias_stale = false;
  }
  if (bhs_launch_infer(s->wh, s->host_bias.data(), inputs, n, head, s->err, s->wait_ns,
                       static_cast<cudaStream_t>(stream)) != 0)
    return fail_msg("surrogate: fused inference launch failed");
  return 0;
}

int bh_surrogate_gradients(BH_Surrogate *s, const float *inputs, const float *targets, int64_t batch, float *grad,
                           float *loss4, void *stream) {
  if (!s || !inputs || !targets || !grad) return fail_msg("surrogate: bad gradient arguments");
  auto st = static_cast<cudaStream_t>(stream);
  if (int rc = forward_backward(s, inputs, targets, batch, loss4, st)) return rc;
  return cuda_check(cudaMemcpyAsync(grad, s->grad, static_cast<size_t>(s->n_params) * sizeof(float),
                                    cudaMemcpyDeviceToDevice, st),
                    "cudaMemcpyAsync(grad)");
}

int bh_surrogate_train_step(BH_Surrogate *s, const float *inputs, const float *targets, int64_t batch,
                            const BH_AdamConfig *adam, float *loss4, void *stream) {
  if (!s || !inputs || !targets || !adam) return fail_msg("surrogate: bad train-step arguments");
  if (!(adam->lr > 0.0f) || !(adam->beta1 >= 0.0f && adam->beta1 < 1.0f) || !(adam->beta2 >= 0.0f && adam->beta2 < 1.0f) ||
      !(adam->eps > 0.0f))
    return fail_msg("surrogate: Adam needs lr > 0, betas in [0, 1), eps > 0");
  auto st = static_cast<cudaStream_t>(stream);
  if (int rc = forward_backward(s, inputs, targets, batch, loss4, st)) return rc;
  s->step += 1;
  const double t = static_cast<double>(s->step);
  const float lr_t = static_cast<float>(adam->lr * std::sqrt(1.0 - std::pow(adam->beta2, t)) /
                                        (1.0 - std::pow(adam->beta1, t)));
  if (bhs_launch_adam(s->w, s->grad, s->m, s->v, s->n_params, lr_t, adam->beta1, adam->beta2, adam->eps, s->wb, s->wt,
                      st) != 0)
    return fail_msg("surrogate: Adam launch failed");
  s->bias_stale = true;
  return 0;
}

int bh_surrogate_set_wait_limit(BH_Surrogate *s, int64_t ns) {
  if (!s || ns < 0) return fail_msg("surrogate: set_wait_limit needs a handle and ns >= 0");
  s->wait_ns = ns == 0 ? kDefaultWaitNs : static_cast<uint64_t>(ns);
  return 0;
}

int bh_surrogate_device_error(BH_Surrogate *s) {
  if (!s) return fail_msg("surrogate: NULL handle");
  if (int rc = cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize")) return rc;
  int code = 0;
  if (int rc = cuda_check(cudaMemcpy(&code, s->err, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy(error flag)"))
    return rc;
  if (code) cudaMemset(s->err, 0, sizeof(int));
  return code;
}

int bh_surrogate_make_targets(const BH_KerrImageOut *o, int64_t n, int max_crossings, float *targets, void *stream) {
  if (!o || !targets || n < 0 || max_crossings < 1 || max_crossings > BH_MAX_CROSSINGS)
    return fail_msg("surrogate: bad make_targets arguments");
  if (!o->cls || !o->n_cross || !o->r_hit || !o->phi_hit || !o->g || !o->theta_inf || !o->phi_inf)
    return fail_msg("surrogate: make_targets needs cls, n_cross, r_hit, phi_hit, g, theta_inf and phi_inf");
  if (bhs_launch_make_targets(static_cast<const int *>(o->cls), static_cast<const int *>(o->n_cross),
                              static_cast<const double *>(o->r_hit), static_cast<const double *>(o->phi_hit),
                              static_cast<const double *>(o->g), static_cast<const double *>(o->theta_inf),
                              static_cast<const double *>(o->phi_inf), n, max_crossings, targets,
                              static_cast<cudaStream_t>(stream)))
    return fail_msg("surrogate: target launch failed");
  return 0;
}

int bh_surrogate_grid_inputs(const BH_KerrScene *sc, float *inputs, void *stream) {
  if (!sc || !inputs) return fail_msg("surrogate: bad grid_inputs arguments");
  if (bh_kerr_scene_validate(sc) != 0) return -1;
  const int64_t n = static_cast<int64_t>(sc->width) * sc->height;
  const double da = (sc->alpha_max - sc->alpha_min) / sc->width;
  const double db = (sc->beta_max - sc->beta_min) / sc->height;
  if (bhs_launch_grid_inputs(sc->spin, std::cos(sc->theta_obs), sc->alpha_min, da, sc->beta_min, db, sc->width, n,
                             inputs, static_cast<cudaStream_t>(stream)))
    return fail_msg("surrogate: grid-input launch failed");
  return 0;
}

void bh_surrogate_policy_defaults(BH_SurrogatePolicy *p) {
  if (!p) return;
  p->min_confidence = 0.99f;
  p->verify = 1;
  p->critical_band = 0.05;
  p->refine_fp64 = 0;
  p->chunks = 0;
}

}  // extern "C"

namespace {

// The render of bh_surrogate_trace_image; after the refinement of each chunk
// of pixels [p0, p1) is enqueued on s->side, chunk_done(k, p0, p1) is called
// (when given), and `chunks` (1..kRenderChunks) overrides the policy's.
int render(BH_Surrogate *s, const BH_KerrScene *scene, const BH_KerrImageOut *out, const BH_SurrogatePolicy *policy,
           void *stream, int chunks, const std::function<int(int, int64_t, int64_t)> &chunk_done) {
  if (!s || !scene || !out) return fail_msg("surrogate render: NULL argument");
  BH_SurrogatePolicy pol;
  bh_surrogate_policy_defaults(&pol);
  if (policy) pol = *policy;
  if (!(pol.min_confidence >= 0.0f && pol.min_confidence <= 1.0f) || pol.verify < 1 || pol.verify > 3 ||
      !(pol.critical_band >= 0.0) || pol.chunks < 0 || pol.chunks > kRenderChunks)
    return fail_msg("surrogate render: policy needs min_confidence in [0, 1], verify 1, 2 or 3, critical_band >= 0, "
                    "chunks in [0, %d]", kRenderChunks);
  const int n_chunks = chunks > 0 ? chunks : (pol.chunks > 0 ? pol.chunks : kDefaultChunks);
  BH_KerrScene sc = *scene;
  sc.precision = BH_PRECISION_MIXED;  // the fallback integrator
  if (sc.integrator == BH_INTEGRATOR_ANALYTIC) sc.integrator = BH_INTEGRATOR_DP45;
  BhkImageParams p;
  BhkLaunch L;
  if (bhh_prepare_image_launch(&sc, &p, &L) != 0) return -1;
  const int64_t n = p.n_pix;
  s->last_pixels = n;
  if (n == 0) return 0;
  if (n > s->ren_pixels) {
    for (void *q : {static_cast<void *>(s->r_inputs), static_cast<void *>(s->r_head), static_cast<void *>(s->r_list),
                    static_cast<void *>(s->r_list2)}) {
      if (!q) continue;
      auto it = std::find(s->allocs.begin(), s->allocs.end(), q);
      if (it != s->allocs.end()) s->allocs.erase(it);
      cudaFree(q);
    }
    s->r_inputs = s->r_head = nullptr;
    s->r_list = s->r_list2 = nullptr;
    s->ren_pixels = 0;
    if (int rc = alloc(s, &s->r_inputs, static_cast<size_t>(n) * 4, "cudaMalloc(render inputs)")) return rc;
    if (int rc = alloc(s, &s->r_head, static_cast<size_t>(n) * BHS_HEAD, "cudaMalloc(render head)")) return rc;
    if (int rc = alloc(s, &s->r_list, static_cast<size_t>(n), "cudaMalloc(fallback list)")) return rc;
    if (int rc = alloc(s, &s->r_list2, static_cast<size_t>(n), "cudaMalloc(second fallback list)")) return rc;
    s->ren_pixels = n;
  }
  if (!s->r_counts && alloc(s, &s->r_counts, 8, "cudaMalloc(render counters)")) return -1;
  if (!s->r_counter && alloc(s, &s->r_counter, 1, "cudaMalloc(work counter)")) return -1;
  auto st = static_cast<cudaStream_t>(stream);
  const double da = (sc.alpha_max - sc.alpha_min) / sc.width, db = (sc.beta_max - sc.beta_min) / sc.height;
  if (bhs_launch_grid_inputs(sc.spin, std::cos(sc.theta_obs), sc.alpha_min, da, sc.beta_min, db, sc.width, n,
                             s->r_inputs, st))
    return fail_msg("surrogate render: input launch failed");
  if (int rc = cuda_check(cudaMemsetAsync(s->r_counts, 0, 8 * sizeof(unsigned int), st), "cudaMemsetAsync"))
    return rc;
  const BhkImageOut o{out->cls,   out->steps,     out->n_cross,   out->r_hit,     out->phi_hit,
                      out->g,     out->flux,      out->intensity, out->theta_inf, out->phi_inf, nullptr, nullptr, out->carter_drift, nullptr};
  if (!s->side) {
    // The refinement and fallback go first when SMs free up: a chunk's rows
    // are then final (and, in the host-buffer render, copied) while later
    // chunks are still being inferred. The total work is the same.
    int least = 0, greatest = 0;
    if (int rc = cuda_check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "cudaDeviceGetStreamPriorityRange"))
      return rc;
    if (int rc = cuda_check(cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, greatest),
                            "cudaStreamCreateWithPriority"))
      return rc;
    for (cudaEvent_t &e : s->ev)
      if (int rc = cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate")) return rc;
  }
  // Chunks of whole tile pairs (256 rows): the network infers chunk k on the
  // caller's stream while `side` refines chunk k - 1; then the integrator
  // traces the rejected pixels on `side`, which the caller's stream joins.
  const int64_t chunk = ((n + n_chunks - 1) / n_chunks + 255) / 256 * 256;
  if (int rc = cuda_check(cudaEventRecord(s->ev[kRenderChunks], st), "cudaEventRecord")) return rc;
  if (int rc = cuda_check(cudaStreamWaitEvent(s->side, s->ev[kRenderChunks], 0), "cudaStreamWaitEvent")) return rc;
  for (int k = 0; k < n_chunks; ++k) {
    const int64_t p0 = k * chunk, p1 = std::min<int64_t>(n, p0 + chunk);
    if (p1 <= p0) break;
    if (int rc = bh_surrogate_forward(s, s->r_inputs + 4 * p0, p1 - p0, s->r_head + BHS_HEAD * p0, stream)) return rc;
    if (int rc = cuda_check(cudaEventRecord(s->ev[k], st), "cudaEventRecord")) return rc;
    if (int rc = cuda_check(cudaStreamWaitEvent(s->side, s->ev[k], 0), "cudaStreamWaitEvent")) return rc;
    if (bhk_surrogate_refine(&p, &o, s->r_head, pol.min_confidence, pol.critical_band, pol.verify, pol.refine_fp64,
                             p0, p1, s->r_list, s->r_counts, s->r_counts + 1, s->side))
      return fail_msg("surrogate render: refine launch failed");
    if (chunk_done)
      if (int rc = chunk_done(k, p0, p1)) return rc;
  }
  // Rejected pixels: the closed-form tracer (O(1) per crossing, so the
  // near-critical band costs no more than the rest), then mixed DP45 on what
  // it does not cover.
  int per_sm = 0;
  const int a_block = bhk_trace_image_analytic_block();
  if (bhk_trace_image_analytic_occupancy(a_block, &per_sm) != 0 || per_sm < 1)
    return fail_msg("surrogate render: occupancy query failed");
  int dev = 0, sms = 0;
  if (int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
  if (int rc = cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count")) return rc;
  const BhkLaunch La{sms * per_sm, a_block, 1, 0};
  if (bhk_trace_list_analytic(&p, &o, s->r_list, s->r_counts, s->r_list2, s->r_counts + 6, La, s->side))
    return fail_msg("surrogate render: closed-form fallback launch failed");
  if (bhk_trace_list_mixed(&p, &o, s->r_list2, s->r_counts + 6, s->r_counter, L, s->side))
    return fail_msg("surrogate render: fallback tracer launch failed");
  if (int rc = cuda_check(cudaEventRecord(s->ev[kRenderChunks + 1], s->side), "cudaEventRecord")) return rc;
  return cuda_check(cudaStreamWaitEvent(st, s->ev[kRenderChunks + 1], 0), "cudaStreamWaitEvent");
}

// A bounded wait of the network's kernels that ran out leaves its pixels
// undefined: report it (and clear the flag) after a synchronized render.
int check_wait_flag(BH_Surrogate *s) {
  int code = 0;
  if (int rc = cuda_check(cudaMemcpy(&code, s->err, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy(error flag)"))
    return rc;
  if (code) {
    cudaMemset(s->err, 0, sizeof(int));
    return fail_msg("bh_surrogate_trace_image_host: a bounded device wait of the network ran out (code %d); "
                    "the outputs are not valid", code);
  }
  return 0;
}

}  // namespace

extern "C" {

int bh_surrogate_trace_image(BH_Surrogate *s, const BH_KerrScene *scene, const BH_KerrImageOut *out,
                             const BH_SurrogatePolicy *policy, void *stream) {
  return render(s, scene, out, policy, stream, 0, nullptr);
}

int bh_surrogate_trace_image_host(BH_Surrogate *s, const BH_KerrScene *scene, const BH_KerrImageOut *h,
                                  const BH_SurrogatePolicy *policy) {
  if (!s || !scene || !h) return fail_msg("surrogate render: NULL argument");
  if (bh_kerr_scene_validate(scene) != 0) return -1;
  const size_t n = size_t(scene->width) * size_t(scene->height);
  if (n == 0) return 0;
  const size_t mc = size_t(scene->max_crossings);
  void *const host[10] = {h->cls, h->steps, h->n_cross, h->r_hit, h->phi_hit,
                          h->g,   h->flux,  h->intensity, h->theta_inf, h->phi_inf};
  const size_t bytes[10] = {4 * n, 4 * n, 4 * n, 8 * n * mc, 8 * n * mc, 8 * n * mc, 8 * n, 8 * n, 8 * n, 8 * n};
  size_t total = 0, off[10];
  for (int i = 0; i < 10; ++i) {
    off[i] = total;
    if (host[i]) total += (bytes[i] + 255) & ~size_t(255);
  }
  if (total == 0) return 0;
  if (total > s->host_out_bytes) {
    if (s->host_out) {
      auto it = std::find(s->allocs.begin(), s->allocs.end(), s->host_out);
      if (it != s->allocs.end()) s->allocs.erase(it);
      cudaFree(s->host_out);
      s->host_out = nullptr;
      s->host_out_bytes = 0;
    }
    if (int rc = alloc(s, &s->host_out, total, "cudaMalloc(render outputs)")) return rc;
    s->host_out_bytes = total;
  }
  if (!s->host_stream) {
    if (int rc = cuda_check(cudaStreamCreateWithFlags(&s->host_stream, cudaStreamNonBlocking), "cudaStreamCreate"))
      return rc;
    if (int rc = cuda_check(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate"))
      return rc;
    for (cudaEvent_t &e : s->copy_ev)
      if (int rc = cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate")) return rc;
    for (cudaEvent_t &e : s->copy_done)
      if (int rc = cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate")) return rc;
    if (int rc = cuda_check(cudaEventCreateWithFlags(&s->gathered, cudaEventDisableTiming), "cudaEventCreate"))
      return rc;
  }
  void *d[10];
  for (int i = 0; i < 10; ++i) d[i] = host[i] ? s->host_out + off[i] : nullptr;
  const BH_KerrImageOut dev{static_cast<int32_t *>(d[0]), static_cast<int32_t *>(d[1]), static_cast<int32_t *>(d[2]),
                            static_cast<double *>(d[3]),  static_cast<double *>(d[4]),  static_cast<double *>(d[5]),
                            static_cast<double *>(d[6]),  static_cast<double *>(d[7]),  static_cast<double *>(d[8]),
                            static_cast<double *>(d[9]), nullptr};  // the drift diagnostic is not staged
  const int planes[10] = {1, 1, 1, int(mc), int(mc), int(mc), 1, 1, 1, 1};
  const int esize[10] = {4, 4, 4, 8, 8, 8, 8, 8, 8, 8};
  // Copies into pageable memory return only when done, which would hold back
  // the next chunk's launch: those buffers get the whole frame at the end.
  bool pinned = true;
  for (int i = 0; i < 10; ++i) {
    if (!host[i]) continue;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, host[i]) != cudaSuccess || at.type != cudaMemoryTypeHost) {
      cudaGetLastError();
      pinned = false;
    }
  }
  // compact buffers: the count, the list, then each field's planes of `cap`
  // entries, in mapped page-locked memory; where that cannot be had, the
  // frame takes the path of pageable buffers
  const int64_t cap = std::min<int64_t>(int64_t(n), std::max<int64_t>(4096, int64_t(n) / 25));
  size_t gbytes = 256 + ((size_t(cap) * 4 + 255) & ~size_t(255)), goff[10];
  for (int i = 0; i < 10; ++i) {
    goff[i] = gbytes;
    if (host[i]) gbytes += (size_t(cap) * planes[i] * esize[i] + 255) & ~size_t(255);
  }
  if (pinned && gbytes > s->gather_bytes) {
    if (s->gather_host) cudaFreeHost(s->gather_host);
    s->gather_host = s->gather_dev = nullptr;
    s->gather_bytes = 0;
    if (cudaHostAlloc(&s->gather_host, gbytes, cudaHostAllocMapped) != cudaSuccess) {
      cudaGetLastError();
      s->gather_host = nullptr;
      pinned = false;
    } else if (cudaHostGetDevicePointer(&s->gather_dev, s->gather_host, 0) != cudaSuccess) {
      cudaGetLastError();
      cudaFreeHost(s->gather_host);
      s->gather_host = s->gather_dev = nullptr;
      pinned = false;
    } else {
      s->gather_bytes = gbytes;
    }
  }
  if (!pinned) {
    if (int rc = render(s, scene, &dev, policy, s->host_stream, 0, nullptr)) return rc;
    for (int i = 0; i < 10; ++i)
      if (host[i])
        if (int rc = cuda_check(cudaMemcpyAsync(host[i], d[i], bytes[i], cudaMemcpyDeviceToHost, s->host_stream),
                                "cudaMemcpyAsync(D2H)"))
          return rc;
    if (int rc = cuda_check(cudaStreamSynchronize(s->host_stream), "bh_surrogate_trace_image_host")) return rc;
    return check_wait_flag(s);
  }
  // Rows go to the host chunk by chunk while the next chunk is inferred: the
  // accepted pixels of [p0, p1) are final once its refinement has run. The
  // rejected ones are written later by the fallback tracers; the gather
  // kernel writes them in compact form straight into mapped host memory (a
  // copy would queue behind the rows on the copy engine), and each chunk's
  // share is scattered here as soon as that chunk's rows have landed. Past
  // `cap` rejected pixels the whole frame is copied again.
  int64_t cp0[kRenderChunks] = {}, cp1[kRenderChunks] = {};
  int n_done = 0;
  auto copy_rows = [&](int k, int64_t p0, int64_t p1) -> int {
    if (int rc = cuda_check(cudaEventRecord(s->copy_ev[k], s->side), "cudaEventRecord")) return rc;
    if (int rc = cuda_check(cudaStreamWaitEvent(s->copy_stream, s->copy_ev[k], 0), "cudaStreamWaitEvent")) return rc;
    for (int i = 0; i < 10; ++i) {
      if (!host[i]) continue;
      for (int c = 0; c < planes[i]; ++c) {
        const size_t at = (size_t(c) * n + size_t(p0)) * esize[i];
        if (int rc = cuda_check(cudaMemcpyAsync(static_cast<char *>(host[i]) + at, static_cast<char *>(d[i]) + at,
                                                size_t(p1 - p0) * esize[i], cudaMemcpyDeviceToHost, s->copy_stream),
                                "cudaMemcpyAsync(D2H rows)"))
          return rc;
      }
    }
    cp0[k] = p0;
    cp1[k] = p1;
    n_done = k + 1;
    return cuda_check(cudaEventRecord(s->copy_done[k], s->copy_stream), "cudaEventRecord");
  };
  // on a failure after rows were enqueued: no copy may still be writing into
  // the caller's buffers when the call returns
  auto drained = [&](int rc) {
    cudaStreamSynchronize(s->copy_stream);
    cudaStreamSynchronize(s->host_stream);
    return rc;
  };
  const int chunks = policy && policy->chunks > 0 ? policy->chunks : kRenderChunks;
  if (int rc = render(s, scene, &dev, policy, s->host_stream, chunks, copy_rows)) return drained(rc);
  BhkGather g{};
  for (int i = 0; i < 10; ++i) {
    g.src[i] = d[i];
    g.dst[i] = host[i] ? s->gather_dev + goff[i] : nullptr;
    g.size[i] = esize[i];
    g.planes[i] = planes[i];
  }
  g.count_out = reinterpret_cast<unsigned int *>(s->gather_dev);
  g.list_out = reinterpret_cast<int *>(s->gather_dev + 256);
  if (bhk_gather_pixels(&g, s->r_list, s->r_counts, int64_t(n), int(cap), s->host_stream))
    return drained(fail_msg("bh_surrogate_trace_image_host: gather launch failed"));
  if (int rc = cuda_check(cudaEventRecord(s->gathered, s->host_stream), "cudaEventRecord")) return drained(rc);
  if (int rc = cuda_check(cudaEventSynchronize(s->gathered), "bh_surrogate_trace_image_host")) return drained(rc);
  const int64_t m = *reinterpret_cast<volatile const unsigned int *>(s->gather_host);
  if (m <= cap) {
    // bucket the compact entries by chunk, then scatter each bucket once its rows are on the host
    const int *list = reinterpret_cast<const int *>(s->gather_host + 256);
    const int64_t csize = n_done > 0 ? cp1[0] - cp0[0] : 1;
    std::vector<int64_t> start(static_cast<size_t>(n_done) + 1, 0);
    std::vector<int32_t> order(static_cast<size_t>(m));
    for (int64_t w = 0; w < m; ++w) ++start[size_t(std::min<int64_t>(list[w] / csize, n_done - 1)) + 1];
    for (int k = 0; k < n_done; ++k) start[size_t(k) + 1] += start[size_t(k)];
    {
      std::vector<int64_t> fill(start.begin(), start.end() - 1);
      for (int64_t w = 0; w < m; ++w)
        order[size_t(fill[size_t(std::min<int64_t>(list[w] / csize, n_done - 1))]++)] = int32_t(w);
    }
    for (int k = 0; k < n_done; ++k) {
      if (int rc = cuda_check(cudaEventSynchronize(s->copy_done[k]), "bh_surrogate_trace_image_host"))
        return drained(rc);
      for (int i = 0; i < 10; ++i) {
        if (!host[i]) continue;
        for (int c = 0; c < planes[i]; ++c) {
          const char *from = s->gather_host + goff[i] + size_t(c) * cap * esize[i];
          char *to = static_cast<char *>(host[i]) + size_t(c) * n * esize[i];
          for (int64_t e = start[size_t(k)]; e < start[size_t(k) + 1]; ++e) {
            const int32_t w = order[size_t(e)];
            if (esize[i] == 4)
              reinterpret_cast<int32_t *>(to)[list[w]] = reinterpret_cast<const int32_t *>(from)[w];
            else
              reinterpret_cast<double *>(to)[list[w]] = reinterpret_cast<const double *>(from)[w];
          }
        }
      }
    }
    if (int rc = cuda_check(cudaStreamSynchronize(s->copy_stream), "bh_surrogate_trace_image_host")) return rc;
  } else {
    // more rejected pixels than the compact buffers hold: the whole frame again
    if (int rc = cuda_check(cudaStreamSynchronize(s->copy_stream), "bh_surrogate_trace_image_host")) return rc;
    for (int i = 0; i < 10; ++i)
      if (host[i])
        if (int rc = cuda_check(cudaMemcpyAsync(host[i], d[i], bytes[i], cudaMemcpyDeviceToHost, s->host_stream),
                                "cudaMemcpyAsync(D2H)"))
          return rc;
    if (int rc = cuda_check(cudaStreamSynchronize(s->host_stream), "bh_surrogate_trace_image_host")) return rc;
  }
  return check_wait_flag(s);
}

int bh_surrogate_last_stats(BH_Surrogate *s, BH_SurrogateStats *out) {
  if (!s || !out) return fail_msg("surrogate stats: NULL argument");
  unsigned int c[8] = {};
  if (s->r_counts) {
    if (int rc = cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize")) return rc;
    if (int rc = cuda_check(cudaMemcpy(c, s->r_counts, sizeof(c), cudaMemcpyDeviceToHost), "cudaMemcpy(stats)"))
      return rc;
  }
  out->pixels = s->last_pixels;
  out->accepted = c[1];
  out->low_confidence = c[2];
  out->critical_band = c[3];
  out->solve_failed = c[4];
  out->disagreement = c[5];
  return 0;
}

int bh_bf16_gemm(const void *A, const void *B, int64_t M, int N, int K, float *C, void *stream) {
  if (!A || !B || !C || M < 0 || K <= 0 || K % 8 != 0) return fail_msg("bf16 gemm: bad arguments");
  if (!(N == 16 || N == 192 || (N > 0 && N % 256 == 0))) return fail_msg("bf16 gemm: N must be 16, 192 or k*256");
  static int *err = nullptr;
  if (!err) {
    if (int rc = cuda_check(bhh_malloc(&err, sizeof(int)), "cudaMalloc(error flag)")) return rc;
    cudaMemset(err, 0, sizeof(int));
  }
  BhsGemm g = make_gemm(A, K, B, K, M, N, K, BHS_EPI_F32);
  g.out = C;
  g.wait_ns = kDefaultWaitNs;
  if (bhs_launch_gemm(&g, err, static_cast<cudaStream_t>(stream)) != 0) return fail_msg("bf16 gemm: launch failed");
  return 0;
}

}  // extern "C"
