// postprocess.cu - bloom and tone mapping of an RGBA float4 framebuffer, the
// bridge's post-processing (src/blender_bridge/cuda_postprocess.cu:237-275).
//
// The reference's pipeline, per frame:
//   bright = bright_pass(fb)            luminance excess over the threshold
//   accum  = sum over r in {4, 8, 16, 32} of V_r(H_r(bright))
//   fb    += strength * accum
//   fb     = tone(fb)                   exposure, vignette, ACES, gamma 1/2.2
// with H_r / V_r the normalized Gaussian of half-width r (sigma = r / 2),
// clamped at the image edges. Each scale blurs the bright-pass itself (the
// reference re-extracts it between scales).
//
// Here that is three launches instead of nineteen:
//   k_post_rows : bright-pass fused into the four horizontal blurs. A tile of
//                 32 rows x 128 columns (+ 32-column halos) in shared memory,
//                 one lane per row, 8 consecutive outputs per thread, so each
//                 loaded tap feeds up to 8 FMAs (pitch 193 = 1 mod 32: the
//                 lanes' rows fall in distinct banks); each output plane is
//                 staged in shared memory and stored row-coalesced.
//   k_post_cols : the four vertical blurs, summed in the reference's order
//                 (r = 4, 8, 16, 32), and the composite; one lane per
//                 column, 8 rows per thread; the next scale's planes arrive
//                 by cp.async while this one is blurred.
//   k_post_tone : the tone map into the caller's framebuffer.
// The horizontal results travel through 12 float planes (4 scales x RGB,
// structure of arrays); the composite goes to a separate buffer because the
// tone map reads a neighbour's colour (below), which an in-place pass would
// race on. Bytes per pixel: rows 16 in + 48 out, cols 48 + 16 in + 16 out,
// tone 16 in + 16 out.
//
// The tone map's red and blue come from pixel (rx, ry) = (int(u w), int(v h))
// with u = px / w, v = py / h rounded to float (cuda_postprocess.cu:165-176,
// chromatic aberration at strength 0): for most widths a few columns take
// them from the pixel to their left (fl(fl(px / w) w) < px). That index is
// kept bit for bit; the colour read there is the composite before tone
// mapping.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "launch.h"

namespace {

constexpr int kHalo = 32;  // the largest blur half-width
constexpr int kRun = 8;    // outputs per thread along the blur direction

// Rows pass tile.
constexpr int kRowsY = 32;
constexpr int kRowsX = 128;
constexpr int kRowsW = kRowsX + 2 * kHalo;
constexpr int kRowsPitch = kRowsW + 1;
constexpr int kRowsThreads = kRowsY * (kRowsX / kRun);  // 512
constexpr int kOutPitch = kRowsX + 1;
constexpr size_t kRowsSmem = sizeof(float) * (3 * kRowsY * kRowsPitch + kRowsY * kOutPitch);

// Columns pass tile.
constexpr int kColsX = 32;
constexpr int kColsY = 64;
constexpr int kColsH = kColsY + 2 * kHalo;
constexpr int kColsThreads = kColsX * (kColsY / kRun);  // 256
constexpr size_t kColsSmem = sizeof(float) * 2 * 3 * kColsH * kColsX;  // double-buffered scales

// Scale index and offset of the normalized taps (2r + 1 each) of half-width R.
__host__ __device__ constexpr int scale_of(int R) { return R == 4 ? 0 : R == 8 ? 1 : R == 16 ? 2 : 3; }
__host__ __device__ constexpr int tap_off(int R) { return R == 4 ? 0 : R == 8 ? 9 : R == 16 ? 26 : 59; }

__device__ __forceinline__ float bright_scale(float4 c, float threshold) {
  const float lum = 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
  const float excess = fmaxf(0.0f, lum - threshold);
  return lum > 0.001f ? excess / lum : 0.0f;
}

// acc[j] += sum_t w[t] src[(j + t) * stride], t = 0..2R: the blur of R taps
// either side of output j, src pointing at output 0's first tap. Unrolled,
// so w[] is read with constant indices from the kernel's parameter bank.
template <int R>
__device__ __forceinline__ void blur_run(const float *src, int stride, const float *w, float (&acc)[kRun]) {
#pragma unroll
  for (int k = 0; k < kRun + 2 * R; ++k) {
    const float v = src[k * stride];
#pragma unroll
    for (int j = 0; j < kRun; ++j) {
      const int t = k - j;
      if (t >= 0 && t <= 2 * R) acc[j] = fmaf(w[t], v, acc[j]);
    }
  }
}

__global__ void __launch_bounds__(kRowsThreads, 2) k_post_rows(const __grid_constant__ BhkPostTaps taps,
                                                             const float4 *__restrict__ fb, int w, int h,
                                                             float threshold, float *__restrict__ planes) {
  extern __shared__ float sm[];  // [3][kRowsY][kRowsPitch] bright-pass, then [kRowsY][kOutPitch] one output plane
  float *stage = sm + 3 * kRowsY * kRowsPitch;
  const int x0 = blockIdx.x * kRowsX, y0 = blockIdx.y * kRowsY;
  static_assert(kRowsY * kRowsW % kRowsThreads == 0, "whole load rounds");
  constexpr int kLoads = kRowsY * kRowsW / kRowsThreads;  // 12, all in flight at once
  float4 v[kLoads];
#pragma unroll
  for (int k = 0; k < kLoads; ++k) {
    const int e = threadIdx.x + k * kRowsThreads, row = e / kRowsW, col = e - row * kRowsW;
    const int y = y0 + row;
    v[k] = y < h ? fb[(int64_t)y * w + min(max(x0 - kHalo + col, 0), w - 1)] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
#pragma unroll
  for (int k = 0; k < kLoads; ++k) {
    const int e = threadIdx.x + k * kRowsThreads, row = e / kRowsW, col = e - row * kRowsW;
    const float s = bright_scale(v[k], threshold);
    sm[(0 * kRowsY + row) * kRowsPitch + col] = v[k].x * s;
    sm[(1 * kRowsY + row) * kRowsPitch + col] = v[k].y * s;
    sm[(2 * kRowsY + row) * kRowsPitch + col] = v[k].z * s;
  }
  const int lane = threadIdx.x & 31, run = threadIdx.x >> 5;
  const int64_t n = (int64_t)w * h;
  // Results leave through the stage, so that a warp stores 32 consecutive
  // floats of one row (the compute layout has a lane per row).
  auto scale = [&](auto rtag) {
    constexpr int R = decltype(rtag)::value, si = scale_of(R);
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      __syncthreads();  // bright-pass written / the previous plane copied out
      float acc[kRun] = {};
      blur_run<R>(sm + (c * kRowsY + lane) * kRowsPitch + kHalo + run * kRun - R, 1, taps.w + tap_off(R), acc);
#pragma unroll
      for (int j = 0; j < kRun; ++j) stage[lane * kOutPitch + run * kRun + j] = acc[j];
      __syncthreads();
      float *out = planes + (int64_t)(si * 3 + c) * n;
      for (int e = threadIdx.x; e < kRowsY * kRowsX; e += kRowsThreads) {
        const int row = e / kRowsX, col = e - row * kRowsX;
        if (y0 + row < h && x0 + col < w) out[(int64_t)(y0 + row) * w + x0 + col] = stage[row * kOutPitch + col];
      }
    }
  };
  scale(std::integral_constant<int, 4>{});
  scale(std::integral_constant<int, 8>{});
  scale(std::integral_constant<int, 16>{});
  scale(std::integral_constant<int, 32>{});
}

// One scale's three planes (rows y0 - 32 .. y0 + 95 clamped, columns x0 ..
// x0 + 31; zeros past the right edge) into a shared buffer, by cp.async.
__device__ __forceinline__ void cols_fetch(float *buf, const float *__restrict__ planes, int si, int64_t n, int x0,
                                           int y0, int w, int h) {
  const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
  const int x = x0 + lane;
#pragma unroll 4
  for (int k = 0; k < 3 * kColsH / (kColsThreads / kColsX); ++k) {  // 48 rounds of 8 rows
    const int cr = grp + k * (kColsThreads / kColsX);                 // channel * kColsH + row
    const int c = cr / kColsH, row = cr - c * kColsH;
    const int y = min(max(y0 - kHalo + row, 0), h - 1);
    float *dst = buf + cr * kColsX + lane;
    if (x < w) {
      const float *src = planes + (int64_t)(si * 3 + c) * n + (int64_t)y * w + x;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                   "l"(src)
                   : "memory");
    } else {
      *dst = 0.0f;
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__global__ void __launch_bounds__(kColsThreads) k_post_cols(const __grid_constant__ BhkPostTaps taps,
                                                             const float *__restrict__ planes,
                                                             const float4 *__restrict__ fb, int w, int h,
                                                             float strength, float4 *__restrict__ out) {
  extern __shared__ float sm[];  // two buffers of [3][kColsH][kColsX]: scale s in buffer s % 2
  constexpr int kBuf = 3 * kColsH * kColsX;
  const int x0 = blockIdx.x * kColsX, y0 = blockIdx.y * kColsY;
  const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
  const int64_t n = (int64_t)w * h;
  float tot[3][kRun] = {};
  cols_fetch(sm, planes, 0, n, x0, y0, w, h);
  cols_fetch(sm + kBuf, planes, 1, n, x0, y0, w, h);
  auto scale = [&](auto rtag) {
    constexpr int R = decltype(rtag)::value, si = scale_of(R);
    if constexpr (si < 3)
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // scale si landed, si + 1 may be in flight
    else
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    const float *buf = sm + (si & 1) * kBuf;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float acc[kRun] = {};
      blur_run<R>(buf + (c * kColsH + kHalo + grp * kRun - R) * kColsX + lane, kColsX, taps.w + tap_off(R), acc);
#pragma unroll
      for (int j = 0; j < kRun; ++j) tot[c][j] += acc[j];
    }
    if constexpr (si + 2 < 4) {
      __syncthreads();  // every warp is done with this buffer
      cols_fetch(sm + (si & 1) * kBuf, planes, si + 2, n, x0, y0, w, h);
    }
  };
  scale(std::integral_constant<int, 4>{});
  scale(std::integral_constant<int, 8>{});
  scale(std::integral_constant<int, 16>{});
  scale(std::integral_constant<int, 32>{});
  const int x = x0 + lane;
  if (x >= w) return;
#pragma unroll
  for (int j = 0; j < kRun; ++j) {
    const int y = y0 + grp * kRun + j;
    if (y >= h) break;
    const int64_t i = (int64_t)y * w + x;
    const float4 b = fb[i];
    out[i] = make_float4(b.x + tot[0][j] * strength, b.y + tot[1][j] * strength, b.z + tot[2][j] * strength, 1.0f);
  }
}

// ACES filmic curve, the fit of K. Narkowicz (2015), clamped to [0, 1].
__device__ __forceinline__ float aces(float x) {
  const float y = (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
  return fminf(fmaxf(y, 0.0f), 1.0f);
}

// Exposure, vignette, ACES, gamma 1/2.2, in the reference's order.
__device__ __forceinline__ float tone_channel(float x, float exposure, float vignette) {
  return powf(fmaxf(aces((x * exposure) * vignette), 0.0f), 1.0f / 2.2f);
}

__global__ void __launch_bounds__(256) k_post_tone(const float4 *__restrict__ src, int w, int h, float exposure,
                                                   float4 *__restrict__ fb) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)w * h) return;
  const int py = (int)(i / w), px = (int)(i - (int64_t)py * w);
  const float u = __fdiv_rn((float)px, (float)w), v = __fdiv_rn((float)py, (float)h);
  const int rx = min(max((int)__fmul_rn(u, (float)w), 0), w - 1);
  const int ry = min(max((int)__fmul_rn(v, (float)h), 0), h - 1);
  const float4 rb = src[(int64_t)ry * w + rx];
  const float gch = src[i].y;
  const float du = u - 0.5f, dv = v - 0.5f;
  const float dist = sqrtf(du * du + dv * dv);
  const float vig = sqrtf(fmaxf(1.0f - dist * dist * 0.5f, 0.0f));
  fb[i] = make_float4(tone_channel(rb.x, exposure, vig), tone_channel(gch, exposure, vig),
                      tone_channel(rb.z, exposure, vig), 1.0f);
}

}  // namespace

extern "C" int64_t bhk_post_scratch_floats(int w, int h) { return (int64_t)16 * w * h; }

extern "C" int bhk_post_process(float *fb, int w, int h, const BhkPostTaps *taps, float threshold, float strength,
                                float exposure, float *scratch, void *stream) {
  if (w <= 0 || h <= 0) return 0;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = (int64_t)w * h;
  float *planes = scratch;                                  // 12 n floats
  float4 *comp = reinterpret_cast<float4 *>(scratch + 12 * n);  // n float4
  float4 *f4 = reinterpret_cast<float4 *>(fb);
  if (strength != 0.0f) {
    if (cudaFuncSetAttribute(k_post_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRowsSmem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_post_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kColsSmem) !=
            cudaSuccess)
      return -1;
    const dim3 gr((w + kRowsX - 1) / kRowsX, (h + kRowsY - 1) / kRowsY);
    k_post_rows<<<gr, kRowsThreads, kRowsSmem, st>>>(*taps, f4, w, h, threshold, planes);
    const dim3 gc((w + kColsX - 1) / kColsX, (h + kColsY - 1) / kColsY);
    k_post_cols<<<gc, kColsThreads, kColsSmem, st>>>(*taps, planes, f4, w, h, strength, comp);
  } else if (cudaMemcpyAsync(comp, fb, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
    return -1;
  }
  k_post_tone<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(comp, w, h, exposure, f4);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
