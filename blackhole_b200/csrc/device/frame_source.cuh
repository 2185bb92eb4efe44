// frame_source.cuh - where a persistent tracer's work items come from.
//
// The tracing loop hands out global work indices w = 0, 1, ... from one
// counter. SingleSrc maps them to the pixels of one frame whose parameters
// live in kernel parameter space; BatchSrc maps them through a device frame
// table (prefix sums of the frames' pixel counts) so that one launch traces
// frames of uneven size, spin, inclination and observer radius back to back,
// and records when each frame's last pixel finished.
#pragma once

#include "launch.h"

namespace bhsrc {

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct SingleSrc {
  const BhkImageParams &p;
  const BhkImageOut &o;
  __device__ __forceinline__ long long total() const { return p.n_pix; }
  __device__ __forceinline__ int frame_of(long long w, long long &pix) const {
    pix = w;
    return 0;
  }
  __device__ __forceinline__ const BhkImageParams &params(int) const { return p; }
  __device__ __forceinline__ const BhkImageOut &out(int) const { return o; }
  __device__ __forceinline__ void pixel_done(int) const {}
};

// The pixels of one frame named by a device list whose length a previous
// kernel wrote (the surrogate renderer's integrator fallback).
struct ListSrc {
  const BhkImageParams &p;
  const BhkImageOut &o;
  const int *list;
  const unsigned int *count;
  __device__ __forceinline__ long long total() const { return (long long)*count; }
  __device__ __forceinline__ int frame_of(long long w, long long &pix) const {
    pix = list[w];
    return 0;
  }
  __device__ __forceinline__ const BhkImageParams &params(int) const { return p; }
  __device__ __forceinline__ const BhkImageOut &out(int) const { return o; }
  __device__ __forceinline__ void pixel_done(int) const {}
};

struct BatchSrc {
  const BhkBatchDev &b;
  __device__ __forceinline__ long long total() const { return b.n_total; }
  // Largest f with prefix[f] <= w (binary search; prefix[0] = 0).
  __device__ __forceinline__ int frame_of(long long w, long long &pix) const {
    int lo = 0, hi = b.n_frames - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (b.prefix[mid] <= w)
        lo = mid;
      else
        hi = mid - 1;
    }
    pix = w - b.prefix[lo];
    return lo;
  }
  __device__ __forceinline__ const BhkImageParams &params(int f) const { return b.frames[f].p; }
  __device__ __forceinline__ const BhkImageOut &out(int f) const { return b.frames[f].o; }
  // The lane that finishes a frame's last pixel stamps the frame's end time.
  __device__ __forceinline__ void pixel_done(int f) const {
    const unsigned int n = (unsigned int)b.frames[f].p.n_pix;
    if (atomicAdd(&b.done[f], 1u) + 1u == n) b.end_ns[f] = globaltimer_ns();
  }
};

}  // namespace bhsrc
