// Measurement probe used by bench.py (not part of the library's C ABI): the read bandwidth of a
// kernel streaming a device buffer, which with a buffer well under the L2 size (126 MB on B200)
// gives the L2 read roof the traversal kernels are compared with.  Built into its own library,
// libebgprobe.so.  Returns 0 on success, 1 bad arguments, 2 CUDA failure, 3 no memory.
#include <cstdint>

#include <cuda_runtime.h>

namespace {

// Streams float4 loads over a buffer (grid-stride, 4 independent loads in flight per thread) and
// folds them into one word per block, so the loads cannot be removed.
__global__ void kReadBandwidth(const float4* __restrict__ buf, int64_t n4, int reps, float* __restrict__ sink)
{
  float         acc  = 0.f;
  const int64_t step = int64_t(gridDim.x) * blockDim.x;
  for (int r = 0; r < reps; r++) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    for (; i + 3 * step < n4; i += 4 * step) {
      const float4 a = __ldcg(buf + i), b = __ldcg(buf + i + step), c = __ldcg(buf + i + 2 * step),
                   d = __ldcg(buf + i + 3 * step);
      acc += (a.x + b.y) + (c.z + d.w);
    }
    for (; i < n4; i += step) {
      const float4 a = __ldcg(buf + i);
      acc += a.x;
    }
  }
  if (acc == 12345.678f) {
    sink[blockIdx.x] = acc;
  }
}

} // namespace

extern "C" {

int ebgprobe_read_bandwidth(int64_t bytes, int32_t iters, double* gbs)
{
  if (bytes < (1 << 20) || iters < 1 || gbs == nullptr) {
    return 1;
  }
  const int64_t n4  = bytes / 16;
  float4*       buf = nullptr;
  float*        sink = nullptr;
  int           dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8;
  if (cudaMalloc(&buf, size_t(n4) * 16) != cudaSuccess || cudaMalloc(&sink, blocks * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(buf);
    return 3;
  }
  cudaMemset(buf, 0, size_t(n4) * 16);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // each launch streams the buffer `reps` times so launch overhead is negligible
  const int reps = 32;
  for (int w = 0; w < 3; w++) {
    kReadBandwidth<<<blocks, 256>>>(buf, n4, reps, sink);
  }
  cudaEventRecord(e0);
  for (int it = 0; it < iters; it++) {
    kReadBandwidth<<<blocks, 256>>>(buf, n4, reps, sink);
  }
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  cudaFree(sink);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) {
    return 2;
  }
  *gbs = double(n4) * 16.0 * iters * reps / (double(ms) * 1e-3) / 1e9;
  return 0;
}

} // extern "C"
