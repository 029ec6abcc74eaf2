// Host-side RAII: makes a CUDA device current for the calling thread for the duration of one
// C-ABI call and restores the caller's current device afterwards, so that no entry point
// leaves the thread on another GPU than the one its caller had selected.
#pragma once

#include <cuda_runtime.h>

namespace frb {

struct DeviceGuard {
  int prev = -1;
  cudaError_t err = cudaSuccess;  // of making `device` current
  explicit DeviceGuard(int device)
  {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    if (prev != device) err = cudaSetDevice(device);
  }
  ~DeviceGuard()
  {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;
};

}// namespace frb
