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
#include "cells_kernels.h"
#include "ebg_device.cuh"
#include "mesh_kernels.h"
#include "mesh_traverse.cuh"

namespace ebg {

namespace {

// A band packet's start from its cell's cut (queries that pass an attached model).  The packet's
// box over its valid lanes must fit its cell grown by the margin, exactly as the FP32 kernel tests
// it, and every lane's bound must lie below R_C by the FP32 kernel's margin: every triangle within a
// lane's bound of its point is then under the cut.  The cut comes onto the stack and the entries
// farther from the packet's box than the largest bound are dropped.  Returns the entries kept (0:
// start at the root).
__device__ int bandCutStart(const SeedCellsView& cv, bool valid, float px, float py, float pz, float bound,
                            float4* stk)
{
  const int   lane = threadIdx.x & 31;
  const float inf  = __int_as_float(0x7f800000);
  float       mnx = valid ? px : inf, mny = valid ? py : inf, mnz = valid ? pz : inf;
  float       mxx = valid ? px : -inf, mxy = valid ? py : -inf, mxz = valid ? pz : -inf;
  float       bmax = bound;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mnx  = fminf(mnx, __shfl_xor_sync(FULL, mnx, o));
    mny  = fminf(mny, __shfl_xor_sync(FULL, mny, o));
    mnz  = fminf(mnz, __shfl_xor_sync(FULL, mnz, o));
    mxx  = fmaxf(mxx, __shfl_xor_sync(FULL, mxx, o));
    mxy  = fmaxf(mxy, __shfl_xor_sync(FULL, mxy, o));
    mxz  = fmaxf(mxz, __shfl_xor_sync(FULL, mxz, o));
    bmax = fmaxf(bmax, __shfl_xor_sync(FULL, bmax, o));
  }
  const float fx = (0.5f * (mnx + mxx) - cv.lo[0]) * cv.inv[0];
  const float fy = (0.5f * (mny + mxy) - cv.lo[1]) * cv.inv[1];
  const float fz = (0.5f * (mnz + mxz) - cv.lo[2]) * cv.inv[2];
  const float g  = float(cv.g);
  if (!(fx >= 0.f && fx < g && fy >= 0.f && fy < g && fz >= 0.f && fz < g)) {
    return 0;
  }
  const int  ix = min(int(fx), cv.g - 1), iy = min(int(fy), cv.g - 1), iz = min(int(fz), cv.g - 1);
  const bool inside =
    mnx >= __fsub_rd(__fadd_rd(cv.lo[0], float(ix) * cv.size[0]), cv.margin[0]) &&
    mny >= __fsub_rd(__fadd_rd(cv.lo[1], float(iy) * cv.size[1]), cv.margin[1]) &&
    mnz >= __fsub_rd(__fadd_rd(cv.lo[2], float(iz) * cv.size[2]), cv.margin[2]) &&
    mxx <= __fadd_ru(__fadd_ru(cv.lo[0], float(ix + 1) * cv.size[0]), cv.margin[0]) &&
    mxy <= __fadd_ru(__fadd_ru(cv.lo[1], float(iy + 1) * cv.size[1]), cv.margin[1]) &&
    mxz <= __fadd_ru(__fadd_ru(cv.lo[2], float(iz + 1) * cv.size[2]), cv.margin[2]);
  if (!inside) {
    return 0;
  }
  const int64_t cell = (int64_t(iz) * cv.g + iy) * cv.g + ix;
  const int     ne   = int(__ldg(cv.count + cell));
  const float   R    = __ldg(cv.radius + cell);
  if (ne == 0 || !(isfinite(R) && bmax <= __fmul_rd(__fmul_rd(R, R), 0.99998f))) {
    return 0;
  }
  const float4* src = cv.entries + size_t(cell) * size_t(cv.lmax) * 2;
  __syncwarp(); // the stack's previous reads are done
  for (int i = lane; i < 2 * ne; i += 32) {
    stk[i] = __ldg(src + i);
  }
  __syncwarp();
  int kept = 0;
#pragma unroll 1
  for (int base = 0; base < ne; base += 32) {
    const int i    = base + lane;
    float4    eA   = make_float4(0.f, 0.f, 0.f, 0.f), eB = eA;
    bool      keep = false;
    if (i < ne) {
      eA   = stk[2 * i];
      eB   = stk[2 * i + 1];
      keep = boxBoxDist2(eA.x, eA.y, eA.z, eB.x, eB.y, eB.z, mnx, mny, mnz, mxx, mxy, mxz) <= bmax;
    }
    const unsigned km = __ballot_sync(FULL, keep);
    __syncwarp(); // every entry of this step is read before any is overwritten
    if (keep) {
      const int r    = kept + __popc(km & ((1u << lane) - 1u));
      stk[2 * r]     = eA;
      stk[2 * r + 1] = eB;
    }
    kept += __popc(km);
    __syncwarp();
  }
  return kept;
}

// Eight 128-thread blocks per SM (at most 64 registers, a few spills): the FP64 test is latency
// bound, and the extra warps outweigh the spills (12 % faster than 90 registers and five blocks).
// EVAL 0: the reference's Triangle/TriangleSoA test (TriMeshSDF); 1: the DCEL face (MeshSDF).
// CUT: the queries passed an attached model, and packets start from their cells' cuts where they
// can (bandCutStart).
template <int EVAL, bool CUT>
__global__ void __launch_bounds__(128, 8) kMeshBand64(const MeshQueryArgs a, float delta)
{
  constexpr int      STACK = CUT ? CUT_STACK_DEPTH : EBG_STACK_DEPTH;
  __shared__ float4  smem[4 * 2 * STACK];
  const int          lane  = threadIdx.x & 31;
  float4*            stk   = smem + (threadIdx.x >> 5) * (2 * STACK);
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

    const int sp0 = CUT ? bandCutStart(a.cells, valid, px, py, pz, bound, stk) : 0;
    band64Mesh<EVAL, STACK>(m, P, px, py, pz, shift, bound, best, bt, stk, iters, err, sp0);
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
  const bool cut = a.cells.count != nullptr;
  if (a.eval == 1) {
    if (cut) {
      kMeshBand64<1, true><<<unsigned(numSms * 8), 128, 0, s>>>(a, delta);
    }
    else {
      kMeshBand64<1, false><<<unsigned(numSms * 8), 128, 0, s>>>(a, delta);
    }
  }
  else if (cut) {
    kMeshBand64<0, true><<<unsigned(numSms * 8), 128, 0, s>>>(a, delta);
  }
  else {
    kMeshBand64<0, false><<<unsigned(numSms * 8), 128, 0, s>>>(a, delta);
  }
  return cudaGetLastError();
}

} // namespace ebg
