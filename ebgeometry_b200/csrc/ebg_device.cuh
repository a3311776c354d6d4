// Device helpers shared by the mesh kernels.
#ifndef EBG_DEVICE_CUH
#define EBG_DEVICE_CUH

#include <cstdint>
#include <cuda_runtime.h>

#include "ebg_layout.h"

namespace ebg {

constexpr unsigned FULL = 0xffffffffu;

// Device-side status word values (host reads them after the call).
constexpr int ST_STACK = 1;  // traversal stack would overflow (never for trees the builder accepts)
constexpr int ST_ITERS = 2;  // iteration cap reached
constexpr int ST_INPUT = 4;  // a query coordinate was NaN or infinite (its result is meaningless)
constexpr int ST_COPY  = 8;  // an asynchronous copy did not signal completion within its wait limit

// Iteration cap per packet traversal: far above any real traversal (a packet visits at most
// every node and leaf once per pass), so hitting it means corrupt input; the kernel then stops,
// records ST_ITERS and returns instead of spinning.
constexpr uint32_t MAX_ITERS = 1u << 26;

// Squared distance from p to an axis-aligned box, the reference's AABBT::getDistance2
// (BoundingVolumesImplem.hpp:480-496): sum over axes of max(0, lo - p, p - hi)^2.
__device__ __forceinline__ float boxDist2(float lx, float ly, float lz, float hx, float hy, float hz, float px,
                                          float py, float pz)
{
  const float dx = fmaxf(0.f, fmaxf(lx - px, px - hx));
  const float dy = fmaxf(0.f, fmaxf(ly - py, py - hy));
  const float dz = fmaxf(0.f, fmaxf(lz - pz, pz - hz));
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

// Squared distance between two axis-aligned boxes, every step rounded down (a lower bound of the
// true distance).
__device__ __forceinline__ float boxBoxDist2(float alx, float aly, float alz, float ahx, float ahy, float ahz, float blx,
                                             float bly, float blz, float bhx, float bhy, float bhz)
{
  const float dx = fmaxf(0.f, fmaxf(__fsub_rd(blx, ahx), __fsub_rd(alx, bhx)));
  const float dy = fmaxf(0.f, fmaxf(__fsub_rd(bly, ahy), __fsub_rd(aly, bhy)));
  const float dz = fmaxf(0.f, fmaxf(__fsub_rd(blz, ahz), __fsub_rd(alz, bhz)));
  return __fadd_rd(__fadd_rd(__fmul_rd(dx, dx), __fmul_rd(dy, dy)), __fmul_rd(dz, dz));
}

__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }

// Quotients by a leaf's primitive count c (1..32) without integer division: 32 / c, and
// ceil(4096 / c), with which (a * ceil(4096 / c)) >> 12 == a / c for every 0 <= a < 64.
static __constant__ uint16_t c_lanesPer[33] = {0, 32, 16, 10, 8, 6, 5, 4, 4, 3, 3, 2, 2, 2, 2, 2, 2,
                                               1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
static __constant__ uint16_t c_recip12[33] = {0,   4096, 2048, 1366, 1024, 820, 683, 586, 512, 456, 410,
                                              373, 342,  316,  293,  274,  256, 241, 228, 216, 205, 196,
                                              187, 179,  171,  164,  158,  152, 147, 142, 137, 133, 128};
__device__ __forceinline__ int divSmall(int a, int c) { return (a * int(c_recip12[c])) >> 12; }

// 10 bits per axis -> 30-bit Morton code.
__device__ __forceinline__ uint32_t spread10(uint32_t x)
{
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__device__ __forceinline__ float warpSum(float v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(FULL, v, o);
  }
  return v;
}

} // namespace ebg

#endif
