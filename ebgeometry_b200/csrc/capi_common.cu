// Library-wide C ABI entry points (errors, version, devices).
#include <cmath>
#include <string>

#include <cuda_runtime.h>

#include "capi_common.h"
#include "ebgeometry_b200.h"

namespace ebg {

namespace {
thread_local std::string g_lastError;
}

ebg_status setError(ebg_status code, const std::string& msg)
{
  g_lastError = msg;
  return code;
}

bool allFinite(const float* x, int64_t n)
{
  int64_t bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
  for (int64_t i = 0; i < n; i++) {
    bad += std::isfinite(x[i]) ? 0 : 1;
  }
  return bad == 0;
}

void keepPoolMemory()
{
  int           device = 0;
  cudaMemPool_t pool;
  if (cudaGetDevice(&device) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
}

} // namespace ebg

extern "C" {

const char* ebg_last_error(void) { return ebg::g_lastError.c_str(); }

const char* ebg_version(void) { return "ebgeometry_b200 0.1.0 (sm_100a)"; }

int ebg_device_count(void)
{
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

} // extern "C"
