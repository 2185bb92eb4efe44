// fma_probe.cu - FMA-throughput probe giving the measured FP64 / FP32 pipe
// peak that bench.py divides the tracer kernels' FLOP rates by. A measuring
// tool of the bench, built into its own library (lib/libbh_bench_probe.so),
// not part of the tracer library.
//
// Each thread runs 8 independent FMA chains for `iters` iterations; the grid
// covers every SM at full occupancy. FLOPs = 2 * 8 * iters * threads.
#include <cuda_runtime.h>

namespace {

template <class T>
__global__ void __launch_bounds__(256) k_fma_probe(T *out, int iters, T x, T y) {
  T a0 = x + (T)threadIdx.x, a1 = a0 + (T)1, a2 = a0 + (T)2, a3 = a0 + (T)3;
  T a4 = a0 + (T)4, a5 = a0 + (T)5, a6 = a0 + (T)6, a7 = a0 + (T)7;
  for (int i = 0; i < iters; ++i) {
    a0 = fma(a0, y, x);
    a1 = fma(a1, y, x);
    a2 = fma(a2, y, x);
    a3 = fma(a3, y, x);
    a4 = fma(a4, y, x);
    a5 = fma(a5, y, x);
    a6 = fma(a6, y, x);
    a7 = fma(a7, y, x);
  }
  const T s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (s == (T)-12345.678) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace

// Best of `repeats` launches (after one warm-up), in TFLOP/s (FMA = 2 FLOPs).
extern "C" int bh_bench_fma_peak(int fp64, int repeats, double *tflops) {
  const int iters = 1 << 14;
  if (!tflops) return -1;
  if (repeats < 1) repeats = 1;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int per_sm = 0;
  if (fp64)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_probe<double>, 256, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_probe<float>, 256, 0);
  const int grid = sms * (per_sm > 0 ? per_sm : 1);
  void *buf = nullptr;
  if (cudaMalloc(&buf, grid * sizeof(double)) != cudaSuccess) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int r = 0; r < repeats + 1; ++r) {
    cudaEventRecord(e0);
    if (fp64)
      k_fma_probe<double><<<grid, 256>>>((double *)buf, iters, 1.0000001, 0.9999999);
    else
      k_fma_probe<float><<<grid, 256>>>((float *)buf, iters, 1.0000001f, 0.9999999f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms < best) best = ms;  // first launch is warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return -1;
  const double flops = 2.0 * 8.0 * double(iters) * double(grid) * 256.0;
  *tflops = flops / (double(best) * 1e-3) / 1e12;
  return 0;
}
