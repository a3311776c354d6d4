// FP64 near-surface re-evaluation (sm_100a).  Compiled with -fmad=false: the point-triangle
// arithmetic below keeps the reference's separate multiplies and adds in the reference's order.
//
// Queries whose FP32 distance fell inside the band |d| <= band (default 1e-4 x the mesh's bounding
// box diagonal, where the sign is ill-conditioned) are re-evaluated here with the reference's own
// FP64 triangle test -- a lane-by-lane restatement of the AVX W=4 double path of
// TriangleSoAT::signedDistance (TriangleSoAImplem.hpp:1029-1180) -- over every triangle whose FP32
// (outward-rounded) box lies within |d32| + delta of the point, keeping the value of smallest
// magnitude with strict < (MeshDistanceFunctionsImplem.hpp:492-502).  delta covers the FP32
// distance error, so the FP64 winner is never pruned; leaves and nodes are also pruned by their
// oriented boxes, which bound the exact distance to every triangle inside from below.  Packets of 32 band queries share one
// traversal stack exactly as in the FP32 kernel.
#include <cfloat>

#include <math_constants.h>

#include "band64.cuh"
#include "ebg_device.cuh"
#include "mesh_kernels.h"
#include "mesh_traverse.cuh"

namespace ebg {

namespace {

// Eight 128-thread blocks per SM (at most 64 registers, a few spills): the FP64 test is latency
// bound, and the extra warps outweigh the spills (12 % faster than 90 registers and five blocks).
// EVAL 0: the reference's Triangle/TriangleSoA test (TriMeshSDF); 1: the DCEL face (MeshSDF).
template <int EVAL>
__global__ void __launch_bounds__(128, 8) kMeshBand64(const MeshQueryArgs a, float delta)
{
  __shared__ float4  smem[4 * 2 * EBG_STACK_DEPTH];
  const int          lane  = threadIdx.x & 31;
  float4*            stk   = smem + (threadIdx.x >> 5) * (2 * EBG_STACK_DEPTH);
  const EbgMeshView& m     = a.mesh;
  const uint32_t     count = *a.band_count;
  const uint32_t     numPk = (count + 31) / 32;
  const uint32_t     warpId = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t     nWarps = (gridDim.x * blockDim.x) >> 5;

  for (uint32_t pk = warpId; pk < numPk; pk += nWarps) {
    const uint32_t j     = pk * 32 + lane;
    const bool     valid = j < count;
    const uint32_t jj    = valid ? j : count - 1;
    const uint32_t pos   = a.band_list[jj];
    const uint32_t id    = a.order ? a.order[pos] : pos;
    // the FP64 point: the caller's own when it passed FP64, else its FP32 point
    const D3       P     = a.points64 ? D3{a.points64[3 * size_t(id)], a.points64[3 * size_t(id) + 1],
                                          a.points64[3 * size_t(id) + 2]}
                                      : D3{double(a.points[3 * size_t(id)]), double(a.points[3 * size_t(id) + 1]),
                                           double(a.points[3 * size_t(id) + 2])};
    const float    px = a.points[3 * size_t(id)], py = a.points[3 * size_t(id) + 1], pz = a.points[3 * size_t(id) + 2];
    const float    d32 = a.band_d32 ? a.band_d32[jj] : a.out_d[id]; // the FP32 pass's distance
    // Boxes are tested at the FP32 point, `shift` from the FP64 point.  The mesh is within
    // |d32| + delta of the FP32 point (delta covers the FP32 distance error near the surface, the
    // relative term far from it), so the FP64 winner is within |d32| + delta + shift of the FP64
    // point and within |d32| + delta + 2 shift of the FP32 point.
    const double   ex = P.x - double(px), ey = P.y - double(py), ez = P.z - double(pz);
    const float    shift = float(sqrt(ex * ex + ey * ey + ez * ez)) * 1.0001f;
    float          r   = (fabsf(d32) * 1.00001f + delta + 2.f * shift) * 1.000001f;
    float          bound = r * r;
    double         best  = DBL_MAX;
    int            bt    = -1;
    uint32_t       iters = 0;
    int            err   = 0;

    band64Mesh<EVAL>(m, P, px, py, pz, shift, bound, best, bt, stk, iters, err);
    if (err && lane == 0) {
      atomicOr(a.status, err);
    }
    if (valid && a.out_d64 != nullptr) {
      a.out_d64[id] = bt >= 0 ? best : double(d32);
    }
    if (valid && bt >= 0) {
      a.out_d[id] = float(best);
      if (a.out_tri) {
        a.out_tri[id] = m.tri_id[bt];
      }
    }
  }
}

// FlatMeshSDF (MeshT::DirectSignedDistance2, DCEL_MeshImplem.hpp:574-595): every face, the first
// in soup order with the smallest unsigned distance^2 wins, and its signed distance is the value.
// One query per thread; the block walks the triangles (leaf order) through shared-memory tiles of
// their vertices and DCEL normals and keeps the lexicographic minimum of (d^2, soup index).
constexpr int FLAT_TILE = 64;

__global__ void __launch_bounds__(128) kMeshFlat64(const EbgMeshView m, int64_t numTris, const double* __restrict__ pts,
                                                   int64_t n, double* __restrict__ out, int32_t* __restrict__ outTri,
                                                   int* __restrict__ status)
{
  __shared__ double  sv[FLAT_TILE][12];
  __shared__ int32_t sid[FLAT_TILE];
  for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < n; base += int64_t(gridDim.x) * blockDim.x) {
    const int64_t q     = base + threadIdx.x;
    const bool    valid = q < n;
    const D3      P     = valid ? D3{pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]} : D3{0.0, 0.0, 0.0};
    const bool    finite = isfinite(P.x) && isfinite(P.y) && isfinite(P.z);
    if (valid && !finite) {
      atomicOr(status, ST_INPUT);
    }
    double        best  = CUDART_INF;
    int32_t       bsoup = INT32_MAX;
    int64_t       bpos  = -1;
    for (int64_t t0 = 0; t0 < numTris; t0 += FLAT_TILE) {
      __syncthreads();
      for (int k = threadIdx.x; k < FLAT_TILE * 12; k += blockDim.x) {
        const int64_t tt = t0 + k / 12;
        const int     c  = k % 12;
        sv[k / 12][c]    = tt < numTris ? (c < 9 ? m.tri64[30 * tt + c] : m.dcel_n[3 * tt + (c - 9)]) : 0.0;
      }
      for (int k = threadIdx.x; k < FLAT_TILE; k += blockDim.x) {
        sid[k] = t0 + k < numTris ? m.tri_id[t0 + k] : INT32_MAX;
      }
      __syncthreads();
      const int cnt = int(numTris - t0 < FLAT_TILE ? numTris - t0 : FLAT_TILE);
      for (int k = 0; k < cnt; k++) {
        const double d2 = dcelFaceUd2(sv[k], sv[k] + 9, P);
        if (d2 < best || (d2 == best && sid[k] < bsoup)) {
          best  = d2;
          bsoup = sid[k];
          bpos  = t0 + k;
        }
      }
    }
    if (valid) {
      // a non-finite point (reported through the status word) gets NaN
      out[q] = (finite && bpos >= 0) ? dcelFaceSd(m.tri64 + 30 * bpos, m.dcel_n + 3 * bpos, P) : CUDART_NAN;
      if (outTri) {
        outTri[q] = (finite && bpos >= 0) ? bsoup : -1;
      }
    }
  }
}

} // namespace

cudaError_t launchMeshFlat64(const EbgMeshView& m, int64_t numTris, const double* pts, int64_t n, double* out,
                             int32_t* outTri, int* status, int numSms, cudaStream_t s)
{
  int64_t blocks = (n + 127) / 128;
  blocks         = blocks < int64_t(numSms) * 16 ? blocks : int64_t(numSms) * 16;
  kMeshFlat64<<<unsigned(blocks < 1 ? 1 : blocks), 128, 0, s>>>(m, numTris, pts, n, out, outTri, status);
  return cudaGetLastError();
}

namespace {
__global__ void kDoubleToFloat(const double* __restrict__ in, float* __restrict__ out, int64_t count)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x) {
    out[i] = float(in[i]);
  }
}
} // namespace

void launchDoubleToFloat(const double* in, float* out, int64_t count, cudaStream_t s)
{
  int64_t blocks = (count + 255) / 256;
  blocks         = blocks < 4096 ? blocks : 4096;
  kDoubleToFloat<<<unsigned(blocks < 1 ? 1 : blocks), 256, 0, s>>>(in, out, count);
}

cudaError_t launchMeshBand64(const MeshQueryArgs& a, float delta, int numSms, cudaStream_t s)
{
  if (a.eval == 1) {
    kMeshBand64<1><<<unsigned(numSms * 8), 128, 0, s>>>(a, delta);
  }
  else {
    kMeshBand64<0><<<unsigned(numSms * 8), 128, 0, s>>>(a, delta);
  }
  return cudaGetLastError();
}

} // namespace ebg
