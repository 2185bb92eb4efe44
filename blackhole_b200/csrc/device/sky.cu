// sky.cu - fills the background cubemap of escaping rays (see sky.cuh).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "launch.h"
#include "sky.cuh"

namespace {

__global__ void k_sky_noise(uint16_t* __restrict__ tex, long long n, uint64_t seed) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  tex[k] = __half_as_ushort(__float2half_rn(bhsky::noise(seed, (uint64_t)k)));
}

__global__ void k_sky_stars(uint16_t* __restrict__ tex, const long long* __restrict__ idx,
                            const float* __restrict__ val, int n) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  tex[idx[s]] = __half_as_ushort(__float2half_rn(val[s]));
}

}  // namespace

extern "C" int bhk_sky_fill(uint16_t* tex, int size, uint64_t seed, const long long* star_idx, const float* star_val,
                            int n_stars, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long n = 6LL * size * size;
  k_sky_noise<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(tex, n, seed);
  if (n_stars > 0) k_sky_stars<<<(n_stars + 255) / 256, 256, 0, s>>>(tex, star_idx, star_val, n_stars);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
