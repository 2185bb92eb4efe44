// batch.cpp - C++23 host side of BH_KerrBatch (include/bh_kerr.h, part 3).
//
// A batch owns one device allocation holding the frame table (kernel
// parameters and output pointers of every frame), the prefix sums of the
// frames' pixel counts, per-frame completion counters and timestamps, and the
// persistent kernel's work counter. A trace is three memsets and one launch,
// so it can be captured once into a CUDA graph and replayed.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/bh_kerr.h"
#include "../device/launch.h"
#include "dalloc.hpp"

struct BH_KerrBatch {
  int device = -1;
  int32_t n_frames = 0;
  int64_t n_total = 0;
  int32_t integrator = 0;
  int32_t precision = 0;
  int sms = 0;
  int max_per_sm = 0;  // occupancy limit at the current block size
  BH_KerrLaunchConfig cfg{};
  void *dev = nullptr;  // one allocation for everything below
  BhkBatchDev d{};
  unsigned long long *counter = nullptr;
  std::vector<BhkFrame> frames;        // host copy of the table
  std::vector<long long> prefix;       // host copy of the prefix sums
  cudaStream_t own_stream = nullptr;   // for graph capture when the caller passes NULL
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t graph_stream = nullptr;
};

namespace {

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

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

int occupancy(const BH_KerrBatch *b, int block, int *per_sm) {
  const int rc = (b->precision == BH_PRECISION_MIXED)
                     ? bhk_trace_batch_mixed_occupancy(b->integrator, block, per_sm)
                     : bhk_trace_batch_fp64_occupancy(b->integrator, block, per_sm);
  if (rc != 0) return cuda_check(cudaGetLastError(), "batch occupancy query");
  return 0;
}

void drop_graph(BH_KerrBatch *b) {
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->graph_exec = nullptr;
  b->graph = nullptr;
  b->graph_stream = nullptr;
}

BhkLaunch launch_of(const BH_KerrBatch *b) {
  const int per_sm = std::min(b->cfg.ctas_per_sm, b->max_per_sm);
  const int64_t full = int64_t(b->sms) * std::max(1, per_sm);
  const int64_t need = (b->n_total + b->cfg.block_threads - 1) / b->cfg.block_threads;
  return BhkLaunch{int32_t(std::max<int64_t>(1, std::min(full, need))), b->cfg.block_threads,
                   std::max(1, b->cfg.refill_steps), 0};
}

int enqueue_trace(BH_KerrBatch *b, cudaStream_t s) {
  if (b->n_total == 0) return 0;
  if (cuda_check(cudaMemsetAsync(b->d.done, 0, sizeof(unsigned int) * b->n_frames, s), "batch memset") ||
      cuda_check(cudaMemsetAsync(b->d.end_ns, 0, sizeof(unsigned long long) * b->n_frames, s), "batch memset") ||
      cuda_check(cudaMemsetAsync(b->d.start_ns, 0xff, sizeof(unsigned long long), s), "batch memset"))
    return -1;
  const BhkLaunch L = launch_of(b);
  const int rc = (b->precision == BH_PRECISION_MIXED) ? bhk_trace_batch_mixed(&b->d, b->integrator, b->counter, L, s)
                                                     : bhk_trace_batch_fp64(&b->d, b->integrator, b->counter, L, s);
  if (rc != 0) return cuda_check(cudaGetLastError(), "batch kernel launch");
  return 0;
}

}  // namespace

extern "C" {

BH_KerrBatch *bh_kerr_batch_create(const BH_KerrScene *scenes, const BH_KerrImageOut *outs, int32_t n_frames) {
  if (!scenes || !outs || n_frames <= 0) {
    fail_msg("bh_kerr_batch_create: need scenes, outs and n_frames > 0 (got %d)", n_frames);
    return nullptr;
  }
  auto b = std::make_unique<BH_KerrBatch>();
  b->n_frames = n_frames;
  b->frames.resize(size_t(n_frames));
  b->prefix.resize(size_t(n_frames) + 1);
  b->prefix[0] = 0;
  for (int32_t i = 0; i < n_frames; ++i) {
    if (bhh_make_params(&scenes[i], &b->frames[i].p) != 0) {
      char msg[600];
      std::snprintf(msg, sizeof(msg), "frame %d: %s", i, bh_last_error());
      bhh_fail(msg);
      return nullptr;
    }
    const BH_KerrImageOut &o = outs[i];
    b->frames[i].o = BhkImageOut{o.cls, o.steps, o.n_cross, o.r_hit, o.phi_hit, o.g, o.flux, o.intensity,
                                 o.theta_inf, o.phi_inf, nullptr, nullptr, o.carter_drift, nullptr};
    if (i > 0 && (scenes[i].integrator != scenes[0].integrator || scenes[i].precision != scenes[0].precision)) {
      fail_msg("frame %d: all frames of a batch must share integrator and precision", i);
      return nullptr;
    }
    b->prefix[i + 1] = b->prefix[i] + b->frames[i].p.n_pix;
  }
  b->n_total = b->prefix[n_frames];
  if (scenes[0].integrator == BH_INTEGRATOR_ANALYTIC) {
    fail_msg("the analytic integrator traces single frames (bh_kerr_trace_image); batches step RK4 or DP45");
    return nullptr;
  }
  b->integrator = scenes[0].integrator;
  b->precision = scenes[0].precision;
  if (cuda_check(cudaGetDevice(&b->device), "cudaGetDevice") ||
      cuda_check(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device), "SM count"))
    return nullptr;
  b->cfg = BH_KerrLaunchConfig{128, 0, 1, 0};
  if (occupancy(b.get(), 128, &b->max_per_sm) != 0) return nullptr;
  b->cfg.ctas_per_sm = b->max_per_sm;

  const size_t n = size_t(n_frames);
  const size_t o_frames = 0;
  const size_t o_prefix = o_frames + align256(sizeof(BhkFrame) * n);
  const size_t o_done = o_prefix + align256(sizeof(long long) * (n + 1));
  const size_t o_end = o_done + align256(sizeof(unsigned int) * n);
  const size_t o_start = o_end + align256(sizeof(unsigned long long) * n);
  const size_t o_counter = o_start + 256;
  const size_t total = o_counter + 256;
  if (cuda_check(bhh_malloc(&b->dev, total), "cudaMalloc(batch)")) return nullptr;
  char *base = static_cast<char *>(b->dev);
  b->d.frames = reinterpret_cast<const BhkFrame *>(base + o_frames);
  b->d.prefix = reinterpret_cast<const long long *>(base + o_prefix);
  b->d.done = reinterpret_cast<unsigned int *>(base + o_done);
  b->d.end_ns = reinterpret_cast<unsigned long long *>(base + o_end);
  b->d.start_ns = reinterpret_cast<unsigned long long *>(base + o_start);
  b->d.n_total = b->n_total;
  b->d.n_frames = n_frames;
  b->d.drift = 0;
  for (int i = 0; i < n_frames; ++i) b->d.drift |= outs[i].carter_drift != nullptr ? 1 : 0;
  b->counter = reinterpret_cast<unsigned long long *>(base + o_counter);
  if (cuda_check(cudaMemcpy(base + o_frames, b->frames.data(), sizeof(BhkFrame) * n, cudaMemcpyHostToDevice),
                 "frame table upload") ||
      cuda_check(cudaMemcpy(base + o_prefix, b->prefix.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice),
                 "prefix upload")) {
    cudaFree(b->dev);
    return nullptr;
  }
  return b.release();
}

void bh_kerr_batch_destroy(BH_KerrBatch *b) {
  if (!b) return;
  drop_graph(b);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  if (b->dev) cudaFree(b->dev);
  delete b;
}

int32_t bh_kerr_batch_frames(const BH_KerrBatch *b) { return b ? b->n_frames : 0; }
int64_t bh_kerr_batch_pixels(const BH_KerrBatch *b) { return b ? b->n_total : 0; }

int bh_kerr_batch_trace(BH_KerrBatch *b, void *stream) {
  if (!b) return bhh_fail("batch is NULL");
  return enqueue_trace(b, static_cast<cudaStream_t>(stream));
}

int bh_kerr_batch_trace_graph(BH_KerrBatch *b, void *stream) {
  if (!b) return bhh_fail("batch is NULL");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!s) {
    if (!b->own_stream && cuda_check(cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking), "stream"))
      return -1;
    s = b->own_stream;
  }
  if (b->graph_exec && b->graph_stream != s) drop_graph(b);
  if (!b->graph_exec) {
    if (cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture")) return -1;
    const int rc = enqueue_trace(b, s);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc != 0) {
      if (g) cudaGraphDestroy(g);
      return -1;
    }
    if (cuda_check(e, "cudaStreamEndCapture")) return -1;
    b->graph = g;
    if (cuda_check(cudaGraphInstantiate(&b->graph_exec, g, 0), "cudaGraphInstantiate")) {
      drop_graph(b);
      return -1;
    }
    b->graph_stream = s;
  }
  if (cuda_check(cudaGraphLaunch(b->graph_exec, s), "cudaGraphLaunch")) return -1;
  if (!stream) return cuda_check(cudaStreamSynchronize(s), "batch graph replay");
  return 0;
}

int bh_kerr_batch_set_launch(BH_KerrBatch *b, const BH_KerrLaunchConfig *cfg) {
  if (!b || !cfg) return bhh_fail("batch or config is NULL");
  const int block = cfg->block_threads ? cfg->block_threads : 128;
  if (block < 32 || block > 128 || block % 32 != 0)
    return fail_msg("block_threads must be 32, 64, 96 or 128, got %d", block);
  if (cfg->refill_steps < 0 || cfg->refill_steps > 64) return fail_msg("refill_steps must be in [0, 64]");
  int per_sm_max = 0;
  if (occupancy(b, block, &per_sm_max) != 0) return -1;
  if (per_sm_max < 1) return fail_msg("the batch kernel does not fit at %d threads per CTA", block);
  const int per_sm = cfg->ctas_per_sm ? std::min(cfg->ctas_per_sm, per_sm_max) : per_sm_max;
  if (per_sm < 1) return fail_msg("ctas_per_sm must be >= 0");
  b->max_per_sm = per_sm_max;
  b->cfg = BH_KerrLaunchConfig{block, per_sm, std::max(1, cfg->refill_steps), 0};
  drop_graph(b);
  return 0;
}

int bh_kerr_batch_set_sky(BH_KerrBatch *b, const BH_SkyCubemap *sky) {
  if (!b) return bhh_fail("batch is NULL");
  if (sky && (!sky->texels || sky->size < 1)) return bhh_fail("sky cubemap needs texels and size >= 1");
  for (BhkFrame &f : b->frames) {
    f.p.sky = sky ? static_cast<const uint16_t *>(sky->texels) : nullptr;
    f.p.sky_size = sky ? sky->size : 0;
  }
  // The kernel reads the frame table at run time: a captured graph stays valid.
  return cuda_check(cudaMemcpy(const_cast<BhkFrame *>(b->d.frames), b->frames.data(), sizeof(BhkFrame) * b->frames.size(),
                               cudaMemcpyHostToDevice),
                    "frame table");
}

int bh_kerr_batch_get_launch(const BH_KerrBatch *b, BH_KerrLaunchConfig *cfg) {
  if (!b || !cfg) return bhh_fail("batch or config is NULL");
  *cfg = b->cfg;
  return 0;
}

int bh_kerr_batch_frame_times(BH_KerrBatch *b, float *frame_ms) {
  if (!b || !frame_ms) return bhh_fail("batch or output is NULL");
  std::vector<unsigned long long> end(size_t(b->n_frames));
  unsigned long long start = 0;
  if (cuda_check(cudaDeviceSynchronize(), "bh_kerr_batch_frame_times") ||
      cuda_check(cudaMemcpy(end.data(), b->d.end_ns, sizeof(unsigned long long) * end.size(), cudaMemcpyDeviceToHost),
                 "frame times") ||
      cuda_check(cudaMemcpy(&start, b->d.start_ns, sizeof(start), cudaMemcpyDeviceToHost), "start time"))
    return -1;
  for (int32_t i = 0; i < b->n_frames; ++i)
    frame_ms[i] = (end[i] == 0 || end[i] < start) ? 0.0f : float(double(end[i] - start) * 1e-6);
  return 0;
}

int bh_kerr_batch_autotune(BH_KerrBatch *b, int64_t max_pixels, void *stream, BH_KerrLaunchConfig *best) {
  if (!b) return bhh_fail("batch is NULL");
  if (max_pixels <= 0) max_pixels = int64_t(4) << 20;
  // Sub-batch: the leading frames up to max_pixels pixels (at least one frame).
  int32_t nf = 1;
  while (nf < b->n_frames && b->prefix[nf + 1] <= max_pixels) ++nf;
  BH_KerrBatch sub = *b;  // shares the device table; only the totals differ
  sub.n_frames = nf;
  sub.n_total = b->prefix[nf];
  sub.d.n_frames = nf;
  sub.d.n_total = sub.n_total;
  sub.graph = nullptr;
  sub.graph_exec = nullptr;
  sub.own_stream = nullptr;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaEvent_t e0, e1;
  if (cuda_check(cudaEventCreate(&e0), "event") || cuda_check(cudaEventCreate(&e1), "event")) return -1;
  float best_ms = 1e30f;
  BH_KerrLaunchConfig best_cfg = b->cfg;
  int rc = 0;
  for (int block : {64, 128}) {
    int per_sm_max = 0;
    if ((rc = occupancy(b, block, &per_sm_max)) != 0) break;
    for (int per_sm = per_sm_max; per_sm >= std::max(1, per_sm_max - 1); --per_sm) {
      for (int refill : {1, 2, 4}) {
        sub.cfg = BH_KerrLaunchConfig{block, per_sm, refill, 0};
        sub.max_per_sm = per_sm_max;
        if ((rc = enqueue_trace(&sub, s)) != 0) break;  // warm-up
        cudaEventRecord(e0, s);
        if ((rc = enqueue_trace(&sub, s)) != 0) break;
        cudaEventRecord(e1, s);
        if ((rc = cuda_check(cudaEventSynchronize(e1), "autotune")) != 0) break;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
          best_ms = ms;
          best_cfg = sub.cfg;
        }
      }
      if (rc) break;
    }
    if (rc) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return -1;
  if (bh_kerr_batch_set_launch(b, &best_cfg) != 0) return -1;
  if (best) *best = b->cfg;
  return 0;
}

}  // extern "C"
