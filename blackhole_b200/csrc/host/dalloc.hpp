// dalloc.hpp - the one door through which the library allocates device memory.
//
// Every cudaMalloc of the host layer goes through bhh_malloc, which counts
// the allocations that succeeded (bh_debug_device_allocations) and can be told
// to fail the n-th one from now as if the device were out of memory
// (bh_debug_fail_device_allocation), so that the error paths of the entry
// points can be exercised without exhausting a GPU.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

cudaError_t bhh_malloc(void **p, size_t bytes);

template <class T>
cudaError_t bhh_malloc(T **p, size_t bytes) {
  return bhh_malloc(reinterpret_cast<void **>(p), bytes);
}
