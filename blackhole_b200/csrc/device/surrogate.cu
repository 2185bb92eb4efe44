// Learned transfer function: BF16 tensor-core (tcgen05) GEMM with fused
// epilogues, input features, loss, gradient collection and Adam.
//
// One GEMM kernel serves every matrix product of training and inference:
// C = A * B^T with A [M][K] and B [N][K] both K-major BF16 in HBM, tiles of
// 128 x BN (BN = 16, 192 or 256), K in chunks of 64 streamed by TMA into a
// 4-stage shared-memory ring (128-byte swizzle), FP32 accumulation in TMEM,
// one thread issuing tcgen05.mma, four warps in the epilogue (one TMEM lane
// quarter each). Backward products that reduce over the batch read
// transposed activations (written by the forward epilogue), so every operand
// is K-major and no transpose pass exists.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "surrogate_net.h"
#include "umma.cuh"

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;
constexpr int kStages = 4;
// Waits on other warps' progress run out after the caller's limit (default
// 2 s; bh_surrogate_set_wait_limit) and record an error code. Work this
// thread itself started (TMA loads, MMAs) is then drained with a fixed limit
// before TMEM is freed and the CTA exits: it completes on its own.
constexpr uint64_t kDrainNs = 1000000000ull;

enum : int { kErrProducer = 11, kErrMma = 12, kErrDone = 13 };

template <int BN>
struct GemmCfg {
  static constexpr int kABytes = kBM * kBK * 2;
  static constexpr int kBBytes = BN * kBK * 2;
  static constexpr int kStage = kABytes + kBBytes;
  static constexpr int kSmem = kStages * kStage + 1024 + 256;
  static constexpr uint32_t kTmemCols = BN <= 32 ? 32u : (BN <= 64 ? 64u : (BN <= 128 ? 128u : 256u));
  static_assert(kStage % 1024 == 0, "stage buffers must stay 1024-byte aligned");
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N for M = 128");
};

__device__ __forceinline__ float tanh_approx(float x) {
  float r;
  asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// SiLU(y) = y sigmoid(y) with sigmoid(y) = (1 + tanh(y/2)) / 2: one MUFU
// operation per element (training and inference use the same form).
__device__ __forceinline__ float silu(float y) {
  const float h = 0.5f * y;
  return fmaf(h, tanh_approx(h), h);
}

__device__ __forceinline__ float silu_grad(float y) {
  const float s = fmaf(0.5f, tanh_approx(0.5f * y), 0.5f);
  return s * (1.0f + y * (1.0f - s));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ uint32_t pack_f16(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

// SiLU of two pre-activations given as halves hy = y / 2 (FP32), returned as
// packed FP16: hy (1 + tanh hy) = y sigmoid(y), with one tanh.approx.f16x2
// (one MUFU operation for both) and one f16x2 FMA. The activation is the next
// layer's FP16 operand, so nothing is unpacked; FP16 keeps 11 significant
// bits, as many as the MUFU tanh delivers.
__device__ __forceinline__ uint32_t silu_f16x2(float hy_lo, float hy_hi) {
  const uint32_t h = pack_f16(hy_lo, hy_hi);
  uint32_t t, r;
  asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(h));
  asm("fma.rn.f16x2 %0, %1, %2, %2;" : "=r"(r) : "r"(t), "r"(h));
  return r;
}

__device__ __forceinline__ void store_bf16x16(__nv_bfloat16* dst, const float (&h)[16]) {
  uint4* p = reinterpret_cast<uint4*>(dst);
  p[0] = make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]), pack_bf16(h[6], h[7]));
  p[1] = make_uint4(pack_bf16(h[8], h[9]), pack_bf16(h[10], h[11]), pack_bf16(h[12], h[13]),
           pack_bf16(h[14], h[15]));
}

__device__ __forceinline__ void store_f32x16(float* dst, const float (&h)[16]) {
  float4* p = reinterpret_cast<float4*>(dst);
#pragma unroll
  for (int q = 0; q < 4; ++q) p[q] = make_float4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]);
}

// ---- epilogues: (row, first column, 16 accumulator values, split index) ---

struct EpiF32 {
  float* C;
  int64_t M;
  int N;
  __device__ void operator()(int64_t row, int col, const float (&v)[16], int split) const {
    if (row >= M) return;
    store_f32x16(C + ((int64_t)split * M + row) * N + col, v);
  }
};

struct EpiHidden {
  const float* bias;
  __nv_bfloat16* H;
  __nv_bfloat16* HT;
  float* Y;
  int64_t M;
  int N;
  int64_t ldt;
  __device__ void operator()(int64_t row, int col, const float (&v)[16], int) const {
    if (row >= M) return;
    float y[16], h[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      y[i] = v[i] + __ldg(bias + col + i);
      h[i] = silu(y[i]);
    }
    if (Y) store_f32x16(Y + row * N + col, y);
    store_bf16x16(H + row * N + col, h);
    if (HT) {
#pragma unroll
      for (int i = 0; i < 16; ++i) HT[(int64_t)(col + i) * ldt + row] = __float2bfloat16_rn(h[i]);
    }
  }
};

struct EpiHead {
  const float* bias;
  float* out;
  int64_t M;
  __device__ void operator()(int64_t row, int col, const float (&v)[16], int) const {
    if (row >= M) return;
    float o[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) o[i] = v[i] + __ldg(bias + col + i);
    store_f32x16(out + row * BHS_HEAD + col, o);
  }
};

struct EpiBackward {
  const float* Y;
  __nv_bfloat16* dY;
  __nv_bfloat16* dYT;
  int64_t M;
  int N;
  int64_t ldt;
  __device__ void operator()(int64_t row, int col, const float (&v)[16], int) const {
    if (row >= M) return;
    const float4* yp = reinterpret_cast<const float4*>(Y + row * N + col);
    float d[16];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 y = yp[q];
      d[4 * q + 0] = v[4 * q + 0] * silu_grad(y.x);
      d[4 * q + 1] = v[4 * q + 1] * silu_grad(y.y);
      d[4 * q + 2] = v[4 * q + 2] * silu_grad(y.z);
      d[4 * q + 3] = v[4 * q + 3] * silu_grad(y.w);
    }
    store_bf16x16(dY + row * N + col, d);
#pragma unroll
    for (int i = 0; i < 16; ++i) dYT[(int64_t)(col + i) * ldt + row] = __float2bfloat16_rn(d[i]);
  }
};

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
     "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
     "=r"(r[15])
    : "r"(taddr)
    : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// One 128 x BN output tile per CTA; blockIdx = (M tile, N tile, K split).
template <int BN, class Epi>
__global__ void __launch_bounds__(128, 1)
  k_gemm_bf16(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, int K,
        int kchunks_per_split, Epi epi, int* err, uint64_t wait_ns) {
  using Cfg = GemmCfg<BN>;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = umma::smem_u32(smem_raw);
  const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  uint8_t* smem = smem_raw + pad;
  const uint32_t sbase = raw + pad;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * Cfg::kStage);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 1);
  const uint32_t bar0 = umma::smem_u32(bars);
  auto full = [&](int s) { return bar0 + 8u * s; };
  auto empty = [&](int s) { return bar0 + 8u * (kStages + s); };
  const uint32_t done = bar0 + 8u * (2 * kStages);
  auto sA = [&](int s) { return sbase + (uint32_t)(s * Cfg::kStage); };
  auto sB = [&](int s) { return sbase + (uint32_t)(s * Cfg::kStage + Cfg::kABytes); };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  const int total = (K + kBK - 1) / kBK;
  const int c0 = blockIdx.z * kchunks_per_split;
  const int nch = max(0, min(total, c0 + kchunks_per_split) - c0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      umma::mbar_init(full(s), 1);
      umma::mbar_init(empty(s), 1);
    }
    umma::mbar_init(done, 1);
    umma::fence_mbar_init();
    umma::tma_prefetch_desc(&ta);
    umma::tma_prefetch_desc(&tb);
  }
  if (warp == 0) {
    umma::tmem_alloc(umma::smem_u32(tmem_slot), Cfg::kTmemCols);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    int issued = 0;
    for (int i = 0; i < nch; ++i) {
      const int s = i % kStages;
      if (i >= kStages && !umma::mbar_wait(empty(s), ((i / kStages) - 1) & 1, wait_ns)) {
        atomicExch(err, kErrProducer);
        break;
      }
      umma::mbar_arrive_expect_tx(full(s), Cfg::kStage);
      const int kx = (c0 + i) * kBK;
      umma::tma_load_2d(sA(s), &ta, full(s), kx, m0);
      umma::tma_load_2d(sB(s), &tb, full(s), kx, n0);
      issued = i + 1;
    }
    // the last load issued on each stage has landed before the CTA may exit
    for (int i = max(0, issued - kStages); i < issued; ++i)
      umma::mbar_wait(full(i % kStages), (i / kStages) & 1, kDrainNs);
  } else if (warp == 1 && lane == 0) {
    constexpr uint32_t idesc = umma::idesc_bf16_f32(kBM, BN);
    for (int i = 0; i < nch; ++i) {
      const int s = i % kStages;
      if (!umma::mbar_wait(full(s), (i / kStages) & 1, wait_ns)) {
        atomicExch(err, kErrMma);
        break;
      }
      umma::tc_fence_after();
      const uint64_t ad = umma::sw128_desc(sA(s));
      const uint64_t bd = umma::sw128_desc(sB(s));
#pragma unroll
      for (int k = 0; k < kBK / 16; ++k)
        umma::mma_bf16(tmem, ad + 2u * k, bd + 2u * k, idesc, (i > 0 || k > 0) ? 1u : 0u);
      umma::mma_commit(empty(s));
    }
    umma::mma_commit(done);
  }
  __syncwarp();

  bool ok = umma::mbar_wait(done, 0, wait_ns);
  if (!ok) {
    atomicExch(err, kErrDone);
    umma::mbar_wait(done, 0, kDrainNs);  // let tensor-core work in flight drain before TMEM is freed
  }
  umma::tc_fence_after();
  const int64_t row = (int64_t)m0 + warp * 32 + lane;
  const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
  for (int j = 0; j < BN / 16; ++j) {
    float v[16];
    tmem_ld16(taddr + 16u * j, v);
    if (!ok || nch == 0) {
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = 0.0f;
    }
    epi(row, n0 + 16 * j, v, (int)blockIdx.z);
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, Cfg::kTmemCols);
}

// ---- features ----------------------------------------------------------------

// 2^(k/3), k = 0..15: Fourier frequencies in units of pi.
__constant__ float c_freq[BHS_FOURIER] = {1.0f,
                     1.2599210498948732f,
                     1.5874010519681994f,
                     2.0f,
                     2.5198420997897464f,
                     3.1748021039363987f,
                     4.0f,
                     5.0396841995794928f,
                     6.3496042078727974f,
                     8.0f,
                     10.079368399158986f,
                     12.699208415745595f,
                     16.0f,
                     20.158736798317971f,
                     25.398416831491190f,
                     32.0f};

// Fourier features of one input x: (sin, cos)(pi 2^(k/3) x), k = 0..15,
// interleaved. Frequencies k = 0, 1, 2 come from sincospif; every further
// one doubles the angle of the one three below (sin 2t = 2 s c,
// cos 2t = (c - s)(c + s)), which keeps the absolute error near 1e-6.
__device__ __forceinline__ void fourier_pairs(float x, float (&v)[2 * BHS_FOURIER]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) sincospif(c_freq[k] * x, &v[2 * k], &v[2 * k + 1]);
#pragma unroll
  for (int k = 3; k < BHS_FOURIER; ++k) {
    const float sn = v[2 * (k - 3)], cs = v[2 * (k - 3) + 1];
    v[2 * k] = 2.0f * sn * cs;
    v[2 * k + 1] = (cs - sn) * (cs + sn);
  }
}

// The network's scaled inputs: x = (alpha/15, beta/15, 2a - 1, 2 cos theta - 1)
// and the constants of motion lambda/15, eta/225.
__device__ __forceinline__ void scaled_inputs(float4 q, float (&x)[4], float& lam, float& eta) {
  x[0] = q.x * (1.0f / 15.0f);
  x[1] = q.y * (1.0f / 15.0f);
  x[2] = 2.0f * q.z - 1.0f;
  x[3] = 2.0f * q.w - 1.0f;
  const float st = sqrtf(fmaxf(0.0f, 1.0f - q.w * q.w));
  lam = -q.x * st * (1.0f / 15.0f);
  eta = (q.y * q.y + (q.x * q.x - q.z * q.z) * q.w * q.w) * (1.0f / 225.0f);
}

// The network's input features of one ray: columns 32 d + 2k, 32 d + 2k + 1
// = Fourier pair k of input d (d = 0..3), columns 128..133 = the scaled
// inputs and constants of motion, 134..191 zero.
__device__ __forceinline__ void ray_features(float4 q, float (&f)[BHS_FEATURES_USED]) {
  float x[4], lam, eta;
  scaled_inputs(q, x, lam, eta);
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    float v[2 * BHS_FOURIER];
    fourier_pairs(x[d], v);
#pragma unroll
    for (int j = 0; j < 2 * BHS_FOURIER; ++j) f[2 * BHS_FOURIER * d + j] = v[j];
  }
  f[128] = x[0];
  f[129] = x[1];
  f[130] = x[2];
  f[131] = x[3];
  f[132] = lam;
  f[133] = eta;
}

__global__ void k_features(const float* __restrict__ in, int64_t n, __nv_bfloat16* __restrict__ F,
                           __nv_bfloat16* __restrict__ FT, int64_t ldt) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  float f[BHS_FEATURES_USED];
  ray_features(reinterpret_cast<const float4*>(in)[r], f);
  uint4* row = reinterpret_cast<uint4*>(F + r * BHS_FEATURES);
#pragma unroll
  for (int u = 0; u < BHS_FEATURES / 8; ++u) {
    float h[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int j = u * 8 + e;
      h[e] = j < BHS_FEATURES_USED ? f[j] : 0.0f;
    }
    row[u] = make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]),
              pack_bf16(h[6], h[7]));
  }
  if (FT) {
#pragma unroll
    for (int j = 0; j < BHS_FEATURES; ++j)
      FT[(int64_t)j * ldt + r] = __float2bfloat16_rn(j < BHS_FEATURES_USED ? f[j] : 0.0f);
  }
}

// ---- loss ------------------------------------------------------------------

// Regression output j (head column 3 + j, target column 2 + j) counts when:
// j = 0..2, 6: a first disk hit; j = 3..5: a second hit; j = 7..9: escaped.
__device__ __forceinline__ bool reg_mask(int j, int cls, int nc) {
  if (j <= 2 || j == 6) return nc >= 1;
  if (j <= 5) return nc >= 2;
  return cls == 2;
}

__global__ void k_loss(const float* __restrict__ out, const float* __restrict__ tg, int64_t B,
            __nv_bfloat16* __restrict__ dout, __nv_bfloat16* __restrict__ dout_t,
            float* __restrict__ loss) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  if (r < B) {
    const float* o = out + r * BHS_HEAD;
    const float* t = tg + r * BHS_TARGETS;
    const int cls = (int)t[0];
    const int nc = (int)t[1];
    const float invB = 1.0f / (float)B;
    float d[BHS_HEAD];
#pragma unroll
    for (int i = 0; i < BHS_HEAD; ++i) d[i] = 0.0f;
    if (cls >= 0) {
      const float m = fmaxf(o[0], fmaxf(o[1], o[2]));
      const float e0 = expf(o[0] - m), e1 = expf(o[1] - m), e2 = expf(o[2] - m);
      const float Z = e0 + e1 + e2;
      acc[0] = -(o[cls] - m - logf(Z));
      d[0] = (e0 / Z - (cls == 0 ? 1.f : 0.f)) * invB;
      d[1] = (e1 / Z - (cls == 1 ? 1.f : 0.f)) * invB;
      d[2] = (e2 / Z - (cls == 2 ? 1.f : 0.f)) * invB;
      const int am = (o[1] > o[0] && o[1] >= o[2]) ? 1 : ((o[2] > o[0] && o[2] > o[1]) ? 2 : 0);
      acc[2] = am == cls ? 1.f : 0.f;
      acc[3] = 1.f;
    }
#pragma unroll
    for (int j = 0; j < 10; ++j) {
      if (reg_mask(j, cls, nc)) {
        const float e = o[3 + j] - t[2 + j];
        acc[1] += e * e;
        d[3 + j] = 2.0f * e * invB;
      }
    }
    uint4* row = reinterpret_cast<uint4*>(dout + r * BHS_HEAD_PAD);
    row[0] = make_uint4(pack_bf16(d[0], d[1]), pack_bf16(d[2], d[3]), pack_bf16(d[4], d[5]),
              pack_bf16(d[6], d[7]));
    row[1] = make_uint4(pack_bf16(d[8], d[9]), pack_bf16(d[10], d[11]), pack_bf16(d[12], d[13]),
              pack_bf16(d[14], d[15]));
#pragma unroll
    for (int i = 0; i < BHS_HEAD; ++i) dout_t[(int64_t)i * B + r] = __float2bfloat16_rn(d[i]);
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    float v = acc[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0f) atomicAdd(loss + c, v);
  }
}

// ---- fused inference -----------------------------------------------------------
//
// One persistent CTA per SM runs the whole network on pairs of 128-row tiles,
// in FP16 (weights and activations; FP32 accumulation): the network is
// trained in BF16, and FP16's 11 significant bits evaluate it more closely,
// while letting SiLU run as tanh.approx.f16x2 -- one MUFU operation per two
// activations, which halves the epilogue's bound (at one tanh per element
// the MUFU pipe alone took as long as the layer's MMAs).
// Warp 0 streams weight K-chunks by TMA through a 3-stage ring (each chunk
// is loaded once per tile), warp 1 issues the tcgen05 MMAs, warps 2-9 and
// 10-17 are the epilogues of tile slots 0 and 1 (two warps per TMEM lane
// quarter, 128 columns each). The activations of a slot
// stay in shared memory, in the 128-byte-swizzled K-major layout the MMA
// reads; its FP32 accumulator is one half of the CTA's 512 TMEM columns.
// While one slot's epilogue (bias, SiLU, BF16, store to shared) runs, the
// tensor core works on the other slot.

#ifndef BHS_EPI_PIPE
#define BHS_EPI_PIPE 1
#endif

// K steps (16 columns each) of layer 0's last 64-column chunk that can hold a
// nonzero term: features 128..133 lie in the first.
constexpr int kFeatTailSteps = (BHS_FEATURES_USED - 128 + 15) / 16;
static_assert(BHS_FEATURES_USED > 128 && BHS_FEATURES_USED <= 144, "feature tail within one K step");

constexpr int kInfThreads = 576;  // 2 control warps + 2 slots x 8 epilogue warps
constexpr int kEpiThreads = 256;  // epilogue threads per slot
constexpr int kInfRing = 3;
constexpr int kActChunk = kBM * kBK * 2;       // 16 KB: one 64-column chunk of a tile
constexpr int kActBytes = 4 * kActChunk;        // 64 KB: 256 columns
constexpr int kWChunk = BHS_HIDDEN * kBK * 2;   // 32 KB: [256 x 64] weights
constexpr int kInfSmem = 2 * kActBytes + kInfRing * kWChunk + 1024 + 256;

// Biases travel in kernel parameter space: every lane of a warp reads the
// same column, so the loads are constant-bank broadcasts, not global loads.
constexpr int kBiasCount = 4 * BHS_HIDDEN + BHS_HEAD;

struct InferArgs {
  const float* in;
  float* out;
  int64_t n;
  int64_t pairs;
  int* err;
  uint64_t wait_ns;  // limit of each wait on another warp's progress
  float bias[kBiasCount];  // layers 0..3 (256 each, halved: b / 2), then the head (16, as is)
};

__device__ __forceinline__ int layer_chunks(int l) { return (l == 0 ? BHS_FEATURES : BHS_HIDDEN) / kBK; }

// One 16-byte unit (8 BF16, unit j of 8 in a 64-column chunk) of row r of a
// K-major 128-byte-swizzled tile chunk at shared address cb.
__device__ __forceinline__ void st_unit(uint32_t cb, int r, int j, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  const uint32_t addr = cb + (uint32_t)r * 128u + ((uint32_t)(j ^ (r & 7)) << 4);
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

__global__ void __launch_bounds__(kInfThreads, 1)
    k_mlp_infer(const __grid_constant__ CUtensorMap w0, const __grid_constant__ CUtensorMap w1,
                const __grid_constant__ CUtensorMap w2, const __grid_constant__ CUtensorMap w3,
                const __grid_constant__ CUtensorMap w4, InferArgs A) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = umma::smem_u32(smem_raw);
  const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  const uint32_t act0 = raw + pad;
  const uint32_t ring0 = act0 + 2u * kActBytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + pad + 2 * kActBytes + kInfRing * kWChunk);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kInfRing + 5);
  const uint32_t b0 = umma::smem_u32(bars);
  auto full = [&](int i) { return b0 + 8u * i; };
  auto empty = [&](int i) { return b0 + 8u * (kInfRing + i); };
  auto act_ready = [&](int s) { return b0 + 8u * (2 * kInfRing + s); };
  auto acc_full = [&](int s) { return b0 + 8u * (2 * kInfRing + 2 + s); };
  const uint32_t drained = b0 + 8u * (2 * kInfRing + 4);  // every MMA issued has completed
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kInfRing; ++i) {
      umma::mbar_init(full(i), 1);
      umma::mbar_init(empty(i), 1);
    }
    for (int s = 0; s < 2; ++s) {
      umma::mbar_init(act_ready(s), kEpiThreads);
      umma::mbar_init(acc_full(s), 1);
    }
    umma::mbar_init(drained, 1);
    umma::fence_mbar_init();
    umma::tma_prefetch_desc(&w0);
    umma::tma_prefetch_desc(&w1);
    umma::tma_prefetch_desc(&w2);
    umma::tma_prefetch_desc(&w3);
    umma::tma_prefetch_desc(&w4);
  }
  if (warp == 0) {
    umma::tmem_alloc(umma::smem_u32(tmem_slot), 512);
    umma::tmem_relinquish();
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // weight producer
      const CUtensorMap* maps[BHS_LAYERS] = {&w0, &w1, &w2, &w3, &w4};
      uint32_t it = 0;
      bool ok = true;
      for (int64_t p = blockIdx.x; ok && p < A.pairs; p += gridDim.x)
        for (int l = 0; ok && l < BHS_LAYERS; ++l) {
          const uint32_t bytes = (uint32_t)((l == BHS_LAYERS - 1 ? BHS_HEAD : BHS_HIDDEN) * kBK * 2);
          for (int s = 0; ok && s < 2; ++s)
            for (int c = 0; c < layer_chunks(l); ++c, ++it) {
              const int st = (int)(it % kInfRing);
              if (it >= (uint32_t)kInfRing && !umma::mbar_wait(empty(st), ((it / kInfRing) - 1) & 1, A.wait_ns)) {
                atomicExch(A.err, kErrProducer);
                ok = false;
                break;
              }
              umma::mbar_arrive_expect_tx(full(st), bytes);
              umma::tma_load_2d(ring0 + (uint32_t)st * kWChunk, maps[l], full(st), c * kBK, 0);
            }
        }
      // the last load issued on each ring stage has landed before the CTA may exit
      for (uint32_t i = it > (uint32_t)kInfRing ? it - kInfRing : 0u; i < it; ++i)
        umma::mbar_wait(full((int)(i % kInfRing)), (i / kInfRing) & 1, kDrainNs);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      uint32_t it = 0, ph[2] = {0u, 0u};
      bool ok = true;
      for (int64_t p = blockIdx.x; ok && p < A.pairs; p += gridDim.x)
        for (int l = 0; ok && l < BHS_LAYERS; ++l)
          for (int s = 0; ok && s < 2; ++s) {
            if (!umma::mbar_wait(act_ready(s), ph[s], A.wait_ns)) {
              atomicExch(A.err, kErrMma);
              ok = false;
              break;
            }
            ph[s] ^= 1u;
            umma::tc_fence_after();
            const uint32_t idesc = umma::idesc_f16_f32(kBM, l == BHS_LAYERS - 1 ? BHS_HEAD : BHS_HIDDEN);
            const uint32_t d = tmem + (uint32_t)s * 256u;
            for (int c = 0; c < layer_chunks(l); ++c, ++it) {
              const int st = (int)(it % kInfRing);
              if (!umma::mbar_wait(full(st), (it / kInfRing) & 1, A.wait_ns)) {
                atomicExch(A.err, kErrMma);
                ok = false;
                break;
              }
              umma::tc_fence_after();
              const uint64_t ad = umma::sw128_desc(act0 + (uint32_t)s * kActBytes + (uint32_t)c * kActChunk);
              const uint64_t bd = umma::sw128_desc(ring0 + (uint32_t)st * kWChunk);
              // layer 0's last chunk holds features 128..133 and zero padding
              // (zero weights too): its first K step covers every nonzero term
              const int ksteps = (l == 0 && c == layer_chunks(0) - 1) ? kFeatTailSteps : kBK / 16;
#pragma unroll
              for (int k = 0; k < kBK / 16; ++k)
                if (k < ksteps) umma::mma_bf16(d, ad + 2u * k, bd + 2u * k, idesc, (c > 0 || k > 0) ? 1u : 0u);
              umma::mma_commit(empty(st));
            }
            umma::mma_commit(acc_full(s));
          }
      // every MMA issued has completed (and stopped writing TMEM) before TMEM is freed
      umma::mma_commit(drained);
      umma::mbar_wait(drained, 0, kDrainNs);
    }
  } else {  // epilogue of slot s: TMEM lane quarter q (warp % 4), column half hf
    const int e = warp - 2;
    const int s = e >> 3;
    const int hf = (e & 7) >> 2;
    const int q = warp & 3;
    const int r = q * 32 + lane;
    const uint32_t act = act0 + (uint32_t)s * kActBytes;
    const uint32_t tacc = tmem + (uint32_t)s * 256u + ((uint32_t)(q * 32) << 16);
    uint32_t ph = 0;
    for (int64_t p = blockIdx.x; p < A.pairs; p += gridDim.x) {
      const int64_t row = (2 * p + s) * kBM + r;
      const bool valid = row < A.n;
      {  // features: half 0 writes inputs 0, 1 (units 0..7), half 1 inputs 2, 3 and the rest (units 8..23)
        const float4 in = valid ? reinterpret_cast<const float4*>(A.in)[row] : make_float4(0.f, 0.f, 0.f, 0.5f);
        float x[4], lam, eta;
        scaled_inputs(in, x, lam, eta);
        const float z = valid ? 1.0f : 0.0f;
#pragma unroll 1
        for (int d = 2 * hf; d < 2 * hf + 2; ++d) {  // columns 32 d .. 32 d + 31: units 4 d .. 4 d + 3
          float v[2 * BHS_FOURIER];
          fourier_pairs(x[d], v);
#pragma unroll
          for (int uu = 0; uu < 4; ++uu) {
            const int u = 4 * d + uu;
            st_unit(act + (uint32_t)(u >> 3) * kActChunk, r, u & 7, pack_f16(z * v[8 * uu], z * v[8 * uu + 1]),
                    pack_f16(z * v[8 * uu + 2], z * v[8 * uu + 3]), pack_f16(z * v[8 * uu + 4], z * v[8 * uu + 5]),
                    pack_f16(z * v[8 * uu + 6], z * v[8 * uu + 7]));
          }
        }
        if (hf == 1) {
          // unit 16: columns 128..135 (scaled inputs, lambda, eta, two zeros); unit 17: zero
          st_unit(act + 2u * kActChunk, r, 0, pack_f16(z * x[0], z * x[1]), pack_f16(z * x[2], z * x[3]),
                  pack_f16(z * lam, z * eta), 0u);
          st_unit(act + 2u * kActChunk, r, 1, 0u, 0u, 0u, 0u);  // unit 17; units 18..23 are never read
        }
      }
      umma::fence_async_smem();
      umma::mbar_arrive(act_ready(s));
      bool ok = true;
      for (int l = 0; l < BHS_LAYERS - 1; ++l) {
        ok = __all_sync(0xffffffffu, umma::mbar_wait(acc_full(s), ph, A.wait_ns));
        ph ^= 1u;
        if (!ok) break;
        umma::tc_fence_after();
        const float* b = A.bias + l * BHS_HIDDEN;
#if BHS_EPI_PIPE
        // 32 columns at a time, the next chunk's TMEM load in flight while
        // this one is activated and stored (two register buffers).
        float va[32], vb[32];
        umma::tmem_ld32_nowait(tacc + 32u * (4 * hf), va);
        umma::tmem_wait_ld();
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int j = 4 * hf + h;
          if (h < 3) umma::tmem_ld32_nowait(tacc + 32u * (j + 1), (h & 1) ? va : vb);
          const float* v = (h & 1) ? vb : va;
          uint32_t pk[16];
#pragma unroll
          for (int i = 0; i < 16; ++i)  // b: halved biases, so hy = acc / 2 + b / 2
            pk[i] = silu_f16x2(fmaf(v[2 * i], 0.5f, b[32 * j + 2 * i]), fmaf(v[2 * i + 1], 0.5f, b[32 * j + 2 * i + 1]));
          const uint32_t cb = act + (uint32_t)(j >> 1) * kActChunk;
#pragma unroll
          for (int uu = 0; uu < 4; ++uu)
            st_unit(cb, r, (j & 1) * 4 + uu, pk[4 * uu], pk[4 * uu + 1], pk[4 * uu + 2], pk[4 * uu + 3]);
          if (h < 3) umma::tmem_wait_ld();
        }
#else
#pragma unroll 1
        for (int jj = 0; jj < 2; ++jj) {  // 64 columns per TMEM wait: two loads in flight
          const int j0 = 4 * hf + 2 * jj;
          float v[64];
          umma::tmem_ld32_nowait(tacc + 32u * j0, v);
          umma::tmem_ld32_nowait(tacc + 32u * (j0 + 1), v + 32);
          umma::tmem_wait_ld();
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int j = j0 + h;
            uint32_t pk[16];
#pragma unroll
            for (int i = 0; i < 16; ++i)  // b: halved biases, so hy = acc / 2 + b / 2
              pk[i] = silu_f16x2(fmaf(v[32 * h + 2 * i], 0.5f, b[32 * j + 2 * i]),
                                 fmaf(v[32 * h + 2 * i + 1], 0.5f, b[32 * j + 2 * i + 1]));
            const uint32_t cb = act + (uint32_t)(j >> 1) * kActChunk;
#pragma unroll
            for (int uu = 0; uu < 4; ++uu)
              st_unit(cb, r, (j & 1) * 4 + uu, pk[4 * uu], pk[4 * uu + 1], pk[4 * uu + 2], pk[4 * uu + 3]);
          }
        }
#endif
        umma::fence_async_smem();
        umma::tc_fence_before();
        umma::mbar_arrive(act_ready(s));
      }
      if (ok) ok = __all_sync(0xffffffffu, umma::mbar_wait(acc_full(s), ph, A.wait_ns));
      ph ^= 1u;
      if (!ok) {
        if (lane == 0) atomicExch(A.err, kErrDone);
        break;
      }
      umma::tc_fence_after();
      if (hf == 0) {
        float v[16];
        tmem_ld16(tacc, v);
        if (valid) {
          const float* b = A.bias + 4 * BHS_HIDDEN;
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] += b[i];
          store_f32x16(A.out + row * BHS_HEAD, v);
        }
      }
      umma::tc_fence_before();
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 512);
}

// ---- gradients and optimiser -------------------------------------------------

struct Ptr5 {
  const void* p[BHS_LAYERS];
};
struct MutPtr5 {
  void* p[BHS_LAYERS];
};
struct LayerTable {
  int k[BHS_LAYERS], n[BHS_LAYERS];
  int64_t w_off[BHS_LAYERS], b_off[BHS_LAYERS];
  int splits[BHS_LAYERS];
};

LayerTable make_table() {
  LayerTable t{};
  for (int l = 0; l < BHS_LAYERS; ++l) {
    t.k[l] = bhs_layer_k(l);
    t.n[l] = bhs_layer_n(l);
    t.w_off[l] = bhs_weight_offset(l);
    t.b_off[l] = bhs_bias_offset(l);
  }
  return t;
}

// One block per (layer, output unit): grad[b_l][n] = sum_b dY^T[n][b].
__global__ void k_bias_grads(Ptr5 dyt, LayerTable t, int64_t B, float* __restrict__ grad) {
  int u = blockIdx.x, l = 0;
  while (l < BHS_LAYERS - 1 && u >= t.n[l]) u -= t.n[l++];
  const __nv_bfloat16* row = static_cast<const __nv_bfloat16*>(dyt.p[l]) + (int64_t)u * B;
  float s = 0.0f;
  for (int64_t b = threadIdx.x; b < B; b += blockDim.x) s += __bfloat162float(row[b]);
  __shared__ float red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) grad[t.b_off[l] + u] = s;
  }
}

// grad[W_l][n][k] = sum_s P_l[s][n][k]; layer 4's partials are [s][k][n].
__global__ void k_collect_dw(Ptr5 parts, LayerTable t, float* __restrict__ grad) {
  const int64_t total = t.b_off[BHS_LAYERS - 1];
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < total;
     p += (int64_t)gridDim.x * blockDim.x) {
    int l = BHS_LAYERS - 1;
    while (l > 0 && p < t.w_off[l]) --l;
    const int64_t q = p - t.w_off[l];
    if (q >= (int64_t)t.n[l] * t.k[l]) continue;  // a bias slot
    const int n = (int)(q / t.k[l]), k = (int)(q % t.k[l]);
    const float* P = static_cast<const float*>(parts.p[l]);
    float s = 0.0f;
    if (l == BHS_LAYERS - 1) {
      const int64_t stride = (int64_t)t.k[l] * t.n[l];
      for (int sp = 0; sp < t.splits[l]; ++sp) s += P[sp * stride + (int64_t)k * t.n[l] + n];
    } else {
      const int64_t stride = (int64_t)t.n[l] * t.k[l];
      for (int sp = 0; sp < t.splits[l]; ++sp) s += P[sp * stride + q];
    }
    grad[p] = s;
  }
}

__device__ __forceinline__ void write_bf16_weight(const LayerTable& t, const MutPtr5& wb, const MutPtr5& wt,
                         int64_t p, float w) {
  int l = BHS_LAYERS - 1;
  while (l > 0 && p < t.w_off[l]) --l;
  const int64_t q = p - t.w_off[l];
  if (q >= (int64_t)t.n[l] * t.k[l]) return;  // bias
  const int n = (int)(q / t.k[l]), k = (int)(q % t.k[l]);
  const __nv_bfloat16 h = __float2bfloat16_rn(w);
  static_cast<__nv_bfloat16*>(wb.p[l])[q] = h;
  if (l == BHS_LAYERS - 1)
    static_cast<__nv_bfloat16*>(wt.p[l])[(int64_t)k * BHS_HEAD_PAD + n] = h;
  else if (l > 0)
    static_cast<__nv_bfloat16*>(wt.p[l])[(int64_t)k * t.n[l] + n] = h;
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
            float* __restrict__ v, int64_t n, float lr_t, float b1, float b2, float eps, LayerTable t,
            MutPtr5 wb, MutPtr5 wt) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const float gp = g[p];
    const float mp = b1 * m[p] + (1.0f - b1) * gp;
    const float vp = b2 * v[p] + (1.0f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    const float wp = w[p] - lr_t * mp / (sqrtf(vp) + eps);
    w[p] = wp;
    write_bf16_weight(t, wb, wt, p, wp);
  }
}

// FP16 copies of the weights for inference, K-major [N][K] like the BF16 ones.
__global__ void k_refresh_f16(const float* __restrict__ w, int64_t n, LayerTable t, MutPtr5 wh) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    int l = BHS_LAYERS - 1;
    while (l > 0 && p < t.w_off[l]) --l;
    const int64_t q = p - t.w_off[l];
    if (q < (int64_t)t.n[l] * t.k[l]) static_cast<__half*>(wh.p[l])[q] = __float2half_rn(w[p]);
  }
}

__global__ void k_refresh_bf16(const float* __restrict__ w, int64_t n, LayerTable t, MutPtr5 wb, MutPtr5 wt) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
    write_bf16_weight(t, wb, wt, p, w[p]);
}

// ---- data --------------------------------------------------------------------

__global__ void k_make_targets(const int* __restrict__ cls, const int* __restrict__ ncr,
                const double* __restrict__ r_hit, const double* __restrict__ phi_hit,
                const double* __restrict__ g, const double* __restrict__ th_inf,
                const double* __restrict__ ph_inf, int64_t n, int mc, float* __restrict__ tg) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float t[BHS_TARGETS];
#pragma unroll
  for (int j = 0; j < BHS_TARGETS; ++j) t[j] = 0.0f;
  const int nc = min(ncr[i], 2);
  const int c = cls[i];
  const int oc = nc >= 1 ? 1 : (c == 0 ? 0 : (c == 2 ? 2 : -1));
  t[0] = (float)oc;
  t[1] = (float)nc;
  if (nc >= 1) {
    t[2] = (float)(log(r_hit[i]) - 2.0);
    t[3] = (float)cos(phi_hit[i]);
    t[4] = (float)sin(phi_hit[i]);
    t[8] = (float)(g[i] - 1.0);
  }
  if (nc >= 2 && mc >= 2) {
    t[5] = (float)(log(r_hit[n + i]) - 2.0);
    t[6] = (float)cos(phi_hit[n + i]);
    t[7] = (float)sin(phi_hit[n + i]);
  }
  if (oc == 2) {
    t[9] = (float)cos(th_inf[i]);
    t[10] = (float)cos(ph_inf[i]);
    t[11] = (float)sin(ph_inf[i]);
  }
  float4* dst = reinterpret_cast<float4*>(tg + i * BHS_TARGETS);
#pragma unroll
  for (int q = 0; q < 4; ++q) dst[q] = make_float4(t[4 * q], t[4 * q + 1], t[4 * q + 2], t[4 * q + 3]);
}

__global__ void k_grid_inputs(double spin, double ct, double a0, double da, double b0, double db, int width,
               int64_t n, float* __restrict__ in) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int64_t i = p % width, j = p / width;
  const double al = a0 + ((double)i + 0.5) * da;
  const double be = b0 + ((double)j + 0.5) * db;
  reinterpret_cast<float4*>(in)[p] = make_float4((float)al, (float)be, (float)spin, (float)ct);
}

// ---- host side: tensor maps and launchers -----------------------------------

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
        cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// K-major 16-bit matrix [rows][ld] (K valid columns), box {64, box_rows}, 128-byte swizzle.
bool make_map(CUtensorMap* m, const void* base, int64_t rows, int K, int ld, int box_rows,
              CUtensorMapDataType type = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0 || (ld * 2) % 16 != 0) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  return fn(m, type, 2, const_cast<void*>(base), dims, strides, box, es,
       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, class Epi>
int launch_tile(const BhsGemm* g, const Epi& epi, int* err, cudaStream_t st) {
  using Cfg = GemmCfg<BN>;
  CUtensorMap ta, tb;
  if (!make_map(&ta, g->A, g->M, g->K, g->lda, kBM) || !make_map(&tb, g->B, g->N, g->K, g->ldb, BN)) {
    std::fprintf(stderr, "blackhole_b200: tensor map encoding failed\n");
    return -1;
  }
  static bool attr_set = false;  // per template instance
  if (!attr_set) {
    if (cudaFuncSetAttribute(k_gemm_bf16<BN, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::kSmem) !=
      cudaSuccess)
      return -1;
    attr_set = true;
  }
  const int total = (g->K + kBK - 1) / kBK;
  const int kcps = g->kchunks_per_split > 0 ? g->kchunks_per_split : total;
  const int splits = (total + kcps - 1) / kcps;
  const dim3 grid((unsigned)((g->M + kBM - 1) / kBM), (unsigned)(g->N / BN), (unsigned)splits);
  k_gemm_bf16<BN, Epi><<<grid, 128, Cfg::kSmem, st>>>(ta, tb, g->K, kcps, epi, err, g->wait_ns);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <int BN>
int launch_bn(const BhsGemm* g, int* err, cudaStream_t st) {
  switch (g->epilogue) {
    case BHS_EPI_F32:
      return launch_tile<BN>(g, EpiF32{static_cast<float*>(g->out), g->M, g->N}, err, st);
    case BHS_EPI_HIDDEN:
      return launch_tile<BN>(g,
                  EpiHidden{g->bias, static_cast<__nv_bfloat16*>(g->out),
                       static_cast<__nv_bfloat16*>(g->out_t), g->y_out, g->M, g->N, g->ld_t},
                  err, st);
    case BHS_EPI_HEAD:
      return launch_tile<BN>(g, EpiHead{g->bias, static_cast<float*>(g->out), g->M}, err, st);
    case BHS_EPI_BACKWARD:
      return launch_tile<BN>(g,
                  EpiBackward{g->Y, static_cast<__nv_bfloat16*>(g->out),
                        static_cast<__nv_bfloat16*>(g->out_t), g->M, g->N, g->ld_t},
                  err, st);
    default:
      return -1;
  }
}

int blocks_for(int64_t n, int threads) { return (int)((n + threads - 1) / threads); }

}  // namespace

extern "C" int bhs_launch_infer(const __half* const* wh, const float* host_bias, const float* inputs,
                                int64_t n, float* head, int* d_err, uint64_t wait_ns, cudaStream_t stream) {
  if (n <= 0) return 0;
  CUtensorMap m[BHS_LAYERS];
  for (int l = 0; l < BHS_LAYERS; ++l)
    if (!make_map(&m[l], wh[l], bhs_layer_n(l), bhs_layer_k(l), bhs_layer_k(l), bhs_layer_n(l),
                  CU_TENSOR_MAP_DATA_TYPE_FLOAT16)) {
      std::fprintf(stderr, "blackhole_b200: tensor map encoding failed\n");
      return -1;
    }
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return -1;
    if (cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kInfSmem) != cudaSuccess)
      return -1;
  }
  InferArgs a{};
  a.in = inputs;
  a.out = head;
  a.n = n;
  const int64_t tiles = (n + kBM - 1) / kBM;
  a.pairs = (tiles + 1) / 2;
  for (int i = 0; i < kBiasCount; ++i) a.bias[i] = i < 4 * BHS_HIDDEN ? 0.5f * host_bias[i] : host_bias[i];
  a.err = d_err;
  a.wait_ns = wait_ns;
  const int grid = (int)std::min<int64_t>(sms, a.pairs);
  k_mlp_infer<<<grid, kInfThreads, kInfSmem, stream>>>(m[0], m[1], m[2], m[3], m[4], a);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhs_launch_gemm(const BhsGemm* g, int* d_err, cudaStream_t stream) {
  if (g->M <= 0) return 0;
  if (g->K <= 0 || g->lda % 8 || g->ldb % 8) return -1;
  if (g->epilogue == BHS_EPI_HEAD && g->N != BHS_HEAD) return -1;
  if (g->N == 256) return launch_bn<256>(g, d_err, stream);
  if (g->N == 192) return launch_bn<192>(g, d_err, stream);
  if (g->N == 16) return launch_bn<16>(g, d_err, stream);
  if (g->N % 256 == 0) return launch_bn<256>(g, d_err, stream);
  return -1;
}

extern "C" int bhs_launch_features(const float* inputs, int64_t n, __nv_bfloat16* F, __nv_bfloat16* FT,
                  int64_t ld_t, cudaStream_t stream) {
  if (n <= 0) return 0;
  k_features<<<blocks_for(n, 128), 128, 0, stream>>>(inputs, n, F, FT, ld_t);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhs_launch_loss(const float* out, const float* targets, int64_t B, __nv_bfloat16* dout,
                __nv_bfloat16* dout_t, float* loss, cudaStream_t stream) {
  if (B <= 0) return 0;
  k_loss<<<blocks_for(B, 256), 256, 0, stream>>>(out, targets, B, dout, dout_t, loss);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhs_launch_bias_grads(const __nv_bfloat16* const* dyt, int64_t B, float* grad, cudaStream_t stream) {
  Ptr5 p{};
  for (int l = 0; l < BHS_LAYERS; ++l) p.p[l] = dyt[l];
  int blocks = 0;
  for (int l = 0; l < BHS_LAYERS; ++l) blocks += bhs_layer_n(l);
  k_bias_grads<<<blocks, 256, 0, stream>>>(p, make_table(), B, grad);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhs_launch_collect_dw(const float* const* partials, const int* splits, float* grad,
                   cudaStream_t stream) {
  Ptr5 p{};
  LayerTable t = make_table();
  for (int l = 0; l < BHS_LAYERS; ++l) {
    p.p[l] = partials[l];
    t.splits[l] = splits[l];
  }
  k_collect_dw<<<592, 256, 0, stream>>>(p, t, grad);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhs_launch_adam(float* params, const float* grad, float* m, float* v, int64_t n, float lr_t,
                float beta1, float beta2, float eps, __nv_bfloat16* const* wb,
                __nv_bfloat16* const* wt, cudaStream_t stream) {
  MutPtr5 b{}, t{};
  for (int l = 0; l < BHS_LAYERS; ++l) {
    b.p[l] = wb[l];
    t.p[l] = wt[l];
  }
  k_adam<<<592, 256, 0, stream>>>(params, grad, m, v, n, lr_t, beta1, beta2, eps, make_table(), b, t);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhs_launch_refresh_bf16(const float* params, __nv_bfloat16* const* wb, __nv_bfloat16* const* wt,
                    cudaStream_t stream) {
  MutPtr5 b{}, t{};
  for (int l = 0; l < BHS_LAYERS; ++l) {
    b.p[l] = wb[l];
    t.p[l] = wt[l];
  }
  k_refresh_bf16<<<592, 256, 0, stream>>>(params, bhs_param_count(), make_table(), b, t);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhs_launch_refresh_f16(const float* params, __half* const* wh, cudaStream_t stream) {
  MutPtr5 h{};
  for (int l = 0; l < BHS_LAYERS; ++l) h.p[l] = wh[l];
  k_refresh_f16<<<592, 256, 0, stream>>>(params, bhs_param_count(), make_table(), h);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhs_launch_make_targets(const int* cls, const int* n_cross, const double* r_hit,
                    const double* phi_hit, const double* g, const double* theta_inf,
                    const double* phi_inf, int64_t n, int max_crossings, float* targets,
                    cudaStream_t stream) {
  if (n <= 0) return 0;
  k_make_targets<<<blocks_for(n, 256), 256, 0, stream>>>(cls, n_cross, r_hit, phi_hit, g, theta_inf, phi_inf,
                              n, max_crossings, targets);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bhs_launch_grid_inputs(double spin, double cos_theta, double alpha_min, double dalpha,
                   double beta_min, double dbeta, int width, int64_t n, float* inputs,
                   cudaStream_t stream) {
  if (n <= 0) return 0;
  k_grid_inputs<<<blocks_for(n, 256), 256, 0, stream>>>(spin, cos_theta, alpha_min, dalpha, beta_min, dbeta,
                              width, n, inputs);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
