// sky_api.cpp - C++23 host side of the background sky (include/bh_kerr.h, part 4):
// the seeded star list (deterministic, collisions merged in star order) and
// the cubemap attached to image traces and batches.
#include <cuda_runtime_api.h>

#include <cstdio>
#include <map>
#include <vector>

#include "../../../include/bh_kerr.h"
#include "../device/launch.h"
#include "../device/sky.cuh"
#include "dalloc.hpp"

namespace {

int fail_msg(const char* msg) { return bhh_fail(msg); }

}  // namespace

extern "C" {

int bh_sky_generate(void* texels, int32_t size, int32_t n_stars, uint64_t seed, void* stream) {
  if (!texels) return fail_msg("bh_sky_generate: texels is NULL");
  if (size < 1 || size > 8192) return fail_msg("bh_sky_generate: size must be in [1, 8192]");
  if (n_stars < 0) return fail_msg("bh_sky_generate: negative star count");
  const long long n = 6LL * size * size;
  // Star s: texel splitmix64((seed ^ "STARS") + 2s) mod n, brightness
  // 2 + 18 u with u the top 24 bits of splitmix64((seed ^ "STARS") + 2s + 1).
  std::map<long long, float> stars;
  const uint64_t base = seed ^ 0x5354415253ull;
  for (int32_t s = 0; s < n_stars; ++s) {
    const uint64_t h1 = bhsky::splitmix64(base + 2ull * (uint64_t)s);
    const uint64_t h2 = bhsky::splitmix64(base + 2ull * (uint64_t)s + 1ull);
    const long long k = (long long)(h1 % (uint64_t)n);
    const float b = 2.0f + 18.0f * ((float)(h2 >> 40) * (1.0f / 16777216.0f));
    auto it = stars.find(k);
    if (it == stars.end())
      stars.emplace(k, bhsky::noise(seed, (uint64_t)k) + b);
    else
      it->second += b;
  }
  std::vector<long long> idx;
  std::vector<float> val;
  idx.reserve(stars.size());
  val.reserve(stars.size());
  for (const auto& [k, v] : stars) {
    idx.push_back(k);
    val.push_back(v);
  }
  long long* d_idx = nullptr;
  float* d_val = nullptr;
  const int m = (int)idx.size();
  if (m > 0) {
    if (bhh_malloc((&d_idx), m * sizeof(long long)) != cudaSuccess ||
        bhh_malloc((&d_val), m * sizeof(float)) != cudaSuccess) {
      cudaFree(d_idx);
      return fail_msg("bh_sky_generate: cudaMalloc failed");
    }
    cudaMemcpy(d_idx, idx.data(), m * sizeof(long long), cudaMemcpyHostToDevice);
    cudaMemcpy(d_val, val.data(), m * sizeof(float), cudaMemcpyHostToDevice);
  }
  const int rc = bhk_sky_fill(static_cast<uint16_t*>(texels), size, seed, d_idx, d_val, m, stream);
  if (m > 0) {
    cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    cudaFree(d_idx);
    cudaFree(d_val);
  }
  if (rc != 0) return fail_msg("bh_sky_generate: launch failed");
  return 0;
}

int bh_kerr_trace_image_sky(const BH_KerrScene* scene, const BH_KerrImageOut* out, const BH_SkyCubemap* sky,
                            void* stream) {
  if (!out) return fail_msg("output descriptor is NULL");
  if (sky && (!sky->texels || sky->size < 1)) return fail_msg("sky cubemap needs texels and size >= 1");
  BhkImageParams p;
  BhkLaunch L;
  if (bhh_prepare_image_launch(scene, &p, &L) != 0) return -1;
  if (p.n_pix == 0) return 0;
  p.sky = sky ? static_cast<const uint16_t*>(sky->texels) : nullptr;
  p.sky_size = sky ? sky->size : 0;
  unsigned long long* counter = nullptr;
  if (bhh_work_counter(&counter) != 0) return -1;
  const BhkImageOut o{out->cls,   out->steps,     out->n_cross,   out->r_hit,     out->phi_hit,
                      out->g,     out->flux,      out->intensity, out->theta_inf, out->phi_inf, nullptr, nullptr, out->carter_drift, nullptr};
  return bhh_launch_image(&p, &o, counter, L, stream, nullptr);
}

}  // extern "C"
