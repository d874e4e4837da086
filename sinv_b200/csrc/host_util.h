// Host-side helpers shared by the entry points of libsinvb.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "../../include/sinvb.h"

namespace sinvb {

#define SINVB_CUDA(call)                            \
  do {                                              \
    cudaError_t sinvb_err_ = (call);                \
    if (sinvb_err_ != cudaSuccess) {                \
      sinvb::set_last_cuda_error(sinvb_err_);       \
      return SINVB_ECUDA;                           \
    }                                               \
  } while (0)

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Records the last CUDA error seen by an entry point (per thread).
void set_last_cuda_error(cudaError_t e);

// SM count of the current device (cached per device).
int device_sm_count();

// SINVB_OK on an sm_100 device, SINVB_EUNSUPPORTED otherwise (cached per device).
int check_device();

}  // namespace sinvb
