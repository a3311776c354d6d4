// Shared helpers of the C ABI layer: thread-local error text and a current-device guard.
#ifndef EBG_CAPI_COMMON_H
#define EBG_CAPI_COMMON_H

#include <string>

#include <cuda_runtime.h>

#include "ebgeometry_b200.h"

namespace ebg {

// Records msg as the calling thread's last error and returns code.
ebg_status setError(ebg_status code, const std::string& msg);

// Restores the caller's current CUDA device on scope exit (entry points switch to the handle's).
struct DeviceGuard
{
  int prev = -1;
  DeviceGuard() { cudaGetDevice(&prev); }
  ~DeviceGuard()
  {
    if (prev >= 0) {
      cudaSetDevice(prev);
    }
  }
};

} // namespace ebg

#endif
