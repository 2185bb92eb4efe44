// noalloc.cu - bh_kerr_trace_image_host_noalloc: the host-buffer image trace
// for callers that cannot allocate device memory.
//
// bh_kerr_trace_image_host stages the outputs in device buffers it allocates
// (and bh_kerr_trace_image allocates the persistent kernel's work counter on
// first use). This variant allocates nothing: the work counter and the
// output staging live in the fixed array below, which is part of the
// library's device image and so exists on every GPU that loads the library
// until the process exits.
//
// Layout of the array for one call: bytes [0, 256) hold the work counter
// (zeroed on the stream before every launch); each requested output field
// follows at a 256-byte boundary. Every call reuses the same bytes, so calls
// whose GPU work overlaps (several host threads, or calls on streams that run
// concurrently) race and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../../include/bh_kerr.h"
#include "launch.h"

static __device__ __align__(256) unsigned char g_noalloc_scratch[BH_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of g_noalloc_scratch on the current device, looked up on
// every call with that device current (cudaGetSymbolAddress allocates
// nothing; once the module is loaded it is a table lookup). An address kept
// from an earlier call would dangle after cudaDeviceReset, which reloads the
// module elsewhere. In host code the array's name is only a host-side
// stand-in and must never be handed to a kernel.
int scratch_address(void **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    char msg[256];
    std::snprintf(msg, sizeof(msg), "cudaGetSymbolAddress(no-allocation scratch): %s", cudaGetErrorString(e));
    return bhh_fail(msg);
  }
  *out = p;
  return 0;
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" int bh_kerr_trace_image_host_noalloc(const BH_KerrScene *scene, const BH_KerrImageOut *h,
                                                 void *stream) {
  if (!h) return bhh_fail("output descriptor is NULL");
  BhkImageParams p;
  BhkLaunch L;
  if (bhh_prepare_image_launch(scene, &p, &L) != 0) return -1;
  if (p.n_pix == 0) return 0;

  const size_t n = size_t(p.n_pix), mc = size_t(p.max_cross);
  void *host[10] = {h->cls, h->steps, h->n_cross, h->r_hit, h->phi_hit, h->g, h->flux, h->intensity, h->theta_inf,
                    h->phi_inf};
  const size_t bytes[10] = {4 * n, 4 * n, 4 * n, 8 * n * mc, 8 * n * mc, 8 * n * mc, 8 * n, 8 * n, 8 * n, 8 * n};
  size_t off[10];
  size_t used = 256;  // work counter (and the analytic integrator's list count)
  for (int i = 0; i < 10; ++i) {
    off[i] = used;
    if (host[i]) used += round256(bytes[i]);
  }
  const size_t list_off = used;  // the analytic integrator's fallback list
  if (p.integrator == BH_INTEGRATOR_ANALYTIC) used += round256(4 * n);
  if (used > size_t(BH_NOALLOC_SCRATCH_BYTES)) {
    char msg[320];
    std::snprintf(msg, sizeof(msg),
                  "bh_kerr_trace_image_host_noalloc: the requested outputs of %lld pixels need %zu bytes of "
                  "device staging, more than its fixed %u-byte scratch; trace the image in tiles or use "
                  "bh_kerr_trace_image_host",
                  (long long)p.n_pix, used, (unsigned)BH_NOALLOC_SCRATCH_BYTES);
    return bhh_fail(msg);
  }

  void *base = nullptr;
  if (scratch_address(&base) != 0) return -1;
  char *b = static_cast<char *>(base);
  void *d[10];
  for (int i = 0; i < 10; ++i) d[i] = host[i] ? b + off[i] : nullptr;
  const BhkImageOut o{static_cast<int32_t *>(d[0]), static_cast<int32_t *>(d[1]), static_cast<int32_t *>(d[2]),
                      static_cast<double *>(d[3]),  static_cast<double *>(d[4]),  static_cast<double *>(d[5]),
                      static_cast<double *>(d[6]),  static_cast<double *>(d[7]),  static_cast<double *>(d[8]),
                      static_cast<double *>(d[9])};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // bhh_launch_image zeroes the work counter on s before the launch.
  if (bhh_launch_image(&p, &o, reinterpret_cast<unsigned long long *>(b), L, stream,
                       reinterpret_cast<int *>(b + list_off)) != 0)
    return -1;
  for (int i = 0; i < 10; ++i) {
    if (!host[i]) continue;
    const cudaError_t e = cudaMemcpyAsync(host[i], d[i], bytes[i], cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return bhh_fail(cudaGetErrorString(e));
  }
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return bhh_fail(cudaGetErrorString(e));
  return 0;
}
