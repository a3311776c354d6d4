// Shared helpers of the C ABI layer: thread-local error text and a current-device guard.
#ifndef EBG_CAPI_COMMON_H
#define EBG_CAPI_COMMON_H

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "ebgeometry_b200.h"

namespace ebg {

// Records msg as the calling thread's last error and returns code.
ebg_status setError(ebg_status code, const std::string& msg);

// Keeps freed stream-ordered allocations in the current device's default memory pool.  Query calls
// take their workspace from that pool; with the driver's default release threshold (0) the pool
// returns its memory at every synchronisation and the next call maps it again, which costs
// milliseconds per call and varies from call to call.  Called by every create entry point.
void keepPoolMemory();

// True when every one of the n floats is finite (checked on all host threads).
bool allFinite(const float* x, int64_t n);

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
