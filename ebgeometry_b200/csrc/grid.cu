// PointCloudHashGrid on the device (sm_100a): a dense uniform grid over a point cloud and its
// expanding-shell k-nearest-neighbour search (PointCloudHashGridImplem.hpp).  The same queries as
// the BVH cloud (PointCloudBVH's interface) with the same results: the k nearest by the reference's
// float squared distance, in (d2, index) order -- ties to the lowest index.
//
// Build: the cloud's box; the cell size h = cbrt(box volume / n * target) (a characteristic length
// for a flat box), coarsened until the grid holds at most 64 + 8 n cells, as the reference sizes
// it; cell coordinates floor((p - lo) / h) in FP64, clamped; a radix sort of (cell, index) makes
// every cell a contiguous range of points (float4: xyz and the index bits).
// Query: one thread per query (queries in Morton order), k best in registers; shells of cells at
// Chebyshev distance r = 0, 1, ... around the query's cell.  After shell r, every point not yet seen
// lies outside the box of cells [c - r, c + r]; its distance is at least the distance from the query
// to the nearest open side of that box (FP64, minus a relative 1e-9 of h).  The search stops once
// the k-th best squared distance is strictly below that bound squared, so no point that could
// enter the result (even on a tie) is skipped.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include "capi_common.h"
#include "ebg_device.cuh"
#include "ebgeometry_b200.h"
#include "mesh_kernels.h"

namespace ebg {
namespace {

struct GridView
{
  const float4*   points;    // sorted by cell: xyz + index bits
  const uint32_t* cellStart; // numCells + 1
  double          lo[3];
  double          h, invH;
  int             n[3];
  int64_t         numPoints;
};

__device__ __forceinline__ int cellCoord(double x, double lo, double invH, int n)
{
  const double c = floor((x - lo) * invH);
  return c < 0.0 ? 0 : (c > double(n - 1) ? n - 1 : int(c));
}

// the reference's squared distance: (p - q) . (p - q) in float, each operation rounded
__device__ __forceinline__ float gridD2(float px, float py, float pz, float qx, float qy, float qz)
{
  const float dx = __fsub_rn(px, qx), dy = __fsub_rn(py, qy), dz = __fsub_rn(pz, qz);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

__device__ __forceinline__ bool lexLessG(float da, uint32_t ia, float db, uint32_t ib)
{
  return da < db || (da == db && ia < ib);
}

__global__ void kGridBounds(const float* __restrict__ pts, int64_t n, unsigned int* __restrict__ box)
{
  // box: [0..2] min keys, [3..5] max keys (order-preserving uint32 of the float)
  unsigned int k[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    for (int a = 0; a < 3; a++) {
      const unsigned int b   = __float_as_uint(pts[3 * i + a]);
      const unsigned int key = (b >> 31) ? ~b : (b | 0x80000000u);
      k[a]                   = min(k[a], key);
      k[3 + a]               = max(k[3 + a], key);
    }
  }
  for (int j = 0; j < 6; j++) {
    for (int off = 16; off > 0; off >>= 1) {
      const unsigned int o = __shfl_xor_sync(FULL, k[j], off);
      k[j]                 = j < 3 ? min(k[j], o) : max(k[j], o);
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int j = 0; j < 3; j++) {
      atomicMin(box + j, k[j]);
      atomicMax(box + 3 + j, k[3 + j]);
    }
  }
}

__global__ void kGridCells(const float* __restrict__ pts, int64_t n, const GridView g, uint32_t* __restrict__ cell,
                           uint32_t* __restrict__ ids, uint32_t* __restrict__ counts)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int cx = cellCoord(double(pts[3 * i]), g.lo[0], g.invH, g.n[0]);
    const int cy = cellCoord(double(pts[3 * i + 1]), g.lo[1], g.invH, g.n[1]);
    const int cz = cellCoord(double(pts[3 * i + 2]), g.lo[2], g.invH, g.n[2]);
    const uint32_t c = (uint32_t(cz) * uint32_t(g.n[1]) + uint32_t(cy)) * uint32_t(g.n[0]) + uint32_t(cx);
    cell[i]          = c;
    ids[i]           = uint32_t(i);
    atomicAdd(counts + c, 1u);
  }
}

__global__ void kGridGather(const float* __restrict__ pts, const uint32_t* __restrict__ ids, int64_t n,
                            float4* __restrict__ out, uint32_t* __restrict__ inv)
{
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t i = ids[j];
    out[j]           = make_float4(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], __uint_as_float(i));
    inv[i]           = uint32_t(j);
  }
}

struct GridQueryArgs
{
  GridView        g;
  const float*    queries;  // caller's xyz (nullptr: self queries)
  const uint32_t* order;    // sorted position -> caller index (external queries)
  const int64_t*  pointIds; // self queries of these cloud indices (nullptr: every point, in cell order)
  const uint32_t* inv;      // cloud index -> sorted position
  int64_t         n;
  int             k;
  int32_t*        outIdx;
  float*          outD2;
  int*            status;
};

// The distance from q to the nearest open side of the searched cells [c - r, c + r] along one axis
// (a side is open if cells lie beyond it), less the rounding of this FP64 arithmetic (relative to
// the magnitudes involved) and of the cell assignment (floor((x - lo) / h) with a rounded 1 / h).
__device__ __forceinline__ void sideBound(double q, int c, int r, int n, double lo, double h, double& lb, bool& open)
{
  const double err = 1e-15 * (fabs(q) + fabs(lo) + double(n + 1) * h) + 1e-9 * h;
  if (c - r > 0) {
    open = true;
    lb   = fmin(lb, q - (lo + double(c - r) * h) - err);
  }
  if (c + r < n - 1) {
    open = true;
    lb   = fmin(lb, (lo + double(c + r + 1) * h) - q - err);
  }
}

// 12 blocks per SM for k <= 2 and 8 for k <= 8 (at most 42 and 64 registers): the walk waits on
// the latency of its cell-bound and point loads, and the extra warps hide more of it (2-10 % faster
// than the compiler's own 56 and 71 registers).
template <int K>
__global__ void __launch_bounds__(128, (K <= 2 ? 12 : (K <= 8 ? 8 : 1))) kGridKnn(const GridQueryArgs a)
{
  const GridView& g = a.g;
  for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < a.n; t += int64_t(gridDim.x) * blockDim.x) {
    float    qx, qy, qz;
    uint32_t self = 0xffffffffu, row;
    if (a.queries == nullptr && a.pointIds == nullptr) {
      const float4 q = g.points[t];
      qx             = q.x;
      qy             = q.y;
      qz             = q.z;
      self           = __float_as_uint(q.w);
      row            = self;
    }
    else if (a.queries == nullptr) {
      row              = uint32_t(t);
      const int64_t id = a.pointIds[t];
      if (id < 0 || id >= g.numPoints) {
        atomicOr(a.status, ST_INPUT);
        for (int j = 0; j < a.k; j++) {
          a.outIdx[size_t(row) * a.k + j] = -1;
          a.outD2[size_t(row) * a.k + j]  = __int_as_float(0x7f800000);
        }
        continue;
      }
      const float4 q = g.points[a.inv[id]];
      qx             = q.x;
      qy             = q.y;
      qz             = q.z;
      self           = uint32_t(id);
    }
    else {
      row = a.order ? a.order[t] : uint32_t(t);
      qx  = a.queries[3 * size_t(row)];
      qy  = a.queries[3 * size_t(row) + 1];
      qz  = a.queries[3 * size_t(row) + 2];
    }
    if (!(isfinite(qx) && isfinite(qy) && isfinite(qz))) {
      atomicOr(a.status, ST_INPUT);
      qx = qy = qz = 0.f;
    }
    float    kd[K];
    uint32_t ki[K];
    // The k best sit in the LAST k slots, in (d2, index) order, so that slot K - 1 is the k-th
    // best; the first K - k slots hold d2 = -1, below any distance, and never move.
    const int pad = K - a.k;
#pragma unroll
    for (int j = 0; j < K; j++) {
      kd[j] = j < pad ? -1.f : __int_as_float(0x7f800000);
      ki[j] = j < pad ? 0u : 0xffffffffu;
    }
    const double Qx = double(qx), Qy = double(qy), Qz = double(qz);
    const int    cx = cellCoord(Qx, g.lo[0], g.invH, g.n[0]);
    const int    cy = cellCoord(Qy, g.lo[1], g.invH, g.n[1]);
    const int    cz = cellCoord(Qz, g.lo[2], g.invH, g.n[2]);
    const int    rMax = max(max(max(cx, g.n[0] - 1 - cx), max(cy, g.n[1] - 1 - cy)), max(cz, g.n[2] - 1 - cz));
    // one point into the sorted k-best list (lowest index on equal distances)
    auto scan = [&](uint32_t b, uint32_t e) {
#pragma unroll 1
      for (uint32_t s = b; s < e; s++) {
        const float4   p  = __ldg(g.points + s);
        const uint32_t ii = __float_as_uint(p.w);
        const float    dd = gridD2(p.x, p.y, p.z, qx, qy, qz);
        if (ii != self && lexLessG(dd, ii, kd[K - 1], ki[K - 1])) {
          kd[K - 1] = dd;
          ki[K - 1] = ii;
#pragma unroll
          for (int j = K - 1; j > 0; j--) {
            if (lexLessG(kd[j], ki[j], kd[j - 1], ki[j - 1])) {
              const float    td = kd[j];
              const uint32_t ti = ki[j];
              kd[j]             = kd[j - 1];
              ki[j]             = ki[j - 1];
              kd[j - 1]         = td;
              ki[j - 1]         = ti;
            }
          }
        }
      }
    };
    // After shell r: stop once the k-th best is below every distance a later shell can hold (a point
    // in a cell outside [c - r, c + r] on some axis lies beyond that side's plane, at least lb away;
    // the comparison leaves room for the rounding of the float squared distances, a relative 1e-6
    // against their 3e-7), or when no side is open.
    auto done = [&](int r) {
      if (ki[K - 1] == 0xffffffffu) {
        return false;
      }
      double lb   = DBL_MAX;
      bool   open = false;
      sideBound(Qx, cx, r, g.n[0], g.lo[0], g.h, lb, open);
      sideBound(Qy, cy, r, g.n[1], g.lo[1], g.h, lb, open);
      sideBound(Qz, cz, r, g.n[2], g.lo[2], g.h, lb, open);
      if (!open) {
        return true;
      }
      lb = fmax(0.0, lb);
      return double(kd[K - 1]) < lb * lb * (1.0 - 1e-6);
    };
    // Shells 0 and 1: the query's cell, then the rest of the 3 x 3 rows around it, x from cx - 1 to
    // cx + 1 (each row a contiguous range of sorted points).  The bounds of all nine rows and of the
    // query's cell are loaded before any point, so those reads overlap instead of following one
    // another; the check after shell 0 keeps dense cells from scanning their neighbours.
    bool stop;
    {
      const int      xlo = max(0, cx - 1), xhi = min(g.n[0] - 1, cx + 1);
      uint32_t       rb[9], re[9];
      const uint32_t rowc = (uint32_t(cz) * uint32_t(g.n[1]) + uint32_t(cy)) * uint32_t(g.n[0]);
      const uint32_t cb = __ldg(g.cellStart + rowc + cx), ce = __ldg(g.cellStart + rowc + cx + 1);
#pragma unroll
      for (int j = 0; j < 9; j++) {
        const int iz = cz - 1 + j / 3, iy = cy - 1 + j % 3;
        rb[j] = re[j] = 0;
        if (iz >= 0 && iz < g.n[2] && iy >= 0 && iy < g.n[1]) {
          const uint32_t row0 = (uint32_t(iz) * uint32_t(g.n[1]) + uint32_t(iy)) * uint32_t(g.n[0]);
          rb[j]               = __ldg(g.cellStart + row0 + xlo);
          re[j]               = __ldg(g.cellStart + row0 + xhi + 1);
        }
      }
      scan(cb, ce);
      stop = done(0);
      if (!stop) {
#pragma unroll
        for (int j = 0; j < 9; j++) {
          if (j == 4) {
            scan(rb[4], cb); // the query's row without its cell
            scan(ce, re[4]);
          }
          else {
            scan(rb[j], re[j]);
          }
        }
        stop = done(1);
      }
    }
#pragma unroll 1
    for (int r = 2; !stop && r <= rMax; r++) {
      // the shell at Chebyshev radius r: on its two z faces and two y faces a whole x row of cells
      // (contiguous in the sorted points), elsewhere the two cells at x = cx -/+ r
      const int xlo = max(0, cx - r), xhi = min(g.n[0] - 1, cx + r);
      const int ylo = max(0, cy - r), yhi = min(g.n[1] - 1, cy + r);
      const int zlo = max(0, cz - r), zhi = min(g.n[2] - 1, cz + r);
#pragma unroll 1
      for (int iz = zlo; iz <= zhi; iz++) {
        const bool zEdge = (iz == cz - r) || (iz == cz + r);
#pragma unroll 1
        for (int iy = ylo; iy <= yhi; iy++) {
          const bool     yEdge = (iy == cy - r) || (iy == cy + r);
          const uint32_t row0  = (uint32_t(iz) * uint32_t(g.n[1]) + uint32_t(iy)) * uint32_t(g.n[0]);
          if (zEdge || yEdge) {
            scan(g.cellStart[row0 + xlo], g.cellStart[row0 + xhi + 1]);
          }
          else {
            if (cx - r >= 0) {
              scan(g.cellStart[row0 + cx - r], g.cellStart[row0 + cx - r + 1]);
            }
            if (cx + r < g.n[0]) {
              scan(g.cellStart[row0 + cx + r], g.cellStart[row0 + cx + r + 1]);
            }
          }
        }
      }
      stop = done(r);
    }
#pragma unroll
    for (int j = 0; j < K; j++) {
      if (j >= pad) {
        const bool   found = ki[j] != 0xffffffffu;
        const size_t o     = size_t(row) * a.k + (j - pad);
        a.outIdx[o]        = found ? int32_t(ki[j]) : -1;
        a.outD2[o]         = found ? kd[j] : __int_as_float(0x7f800000);
      }
    }
  }
}

template <int K>
cudaError_t launchGridK(const GridQueryArgs& a, int numSms, cudaStream_t s)
{
  int64_t blocks = (a.n + 127) / 128;
  blocks         = std::min<int64_t>(blocks, int64_t(numSms) * 32);
  kGridKnn<K><<<unsigned(std::max<int64_t>(blocks, 1)), 128, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launchGridKnn(const GridQueryArgs& a, int kt, int numSms, cudaStream_t s)
{
  switch (kt) {
  case 1:
    return launchGridK<1>(a, numSms, s);
  case 2:
    return launchGridK<2>(a, numSms, s);
  case 4:
    return launchGridK<4>(a, numSms, s);
  case 8:
    return launchGridK<8>(a, numSms, s);
  case 16:
    return launchGridK<16>(a, numSms, s);
  default:
    return launchGridK<32>(a, numSms, s);
  }
}

unsigned gridBlocks(int64_t n) { return unsigned(std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 1 << 20)); }

double hostKeyToFloat(unsigned int k)
{
  const unsigned int b = (k >> 31) ? (k & 0x7fffffffu) : ~k;
  float              f;
  std::memcpy(&f, &b, 4);
  return double(f);
}

} // namespace
} // namespace ebg

struct ebg_grid
{
  int            device = 0;
  int            numSms = 148;
  ebg::GridView  view{};
  float4*        dPoints = nullptr;
  uint32_t*      dStart  = nullptr;
  uint32_t*      dInv    = nullptr;
  int*           dStatus = nullptr;
  double         target  = 1.0;
};

using namespace ebg;

extern "C" {

ebg_status ebg_grid_create(const float* points_host, int64_t n, double target_per_cell, int32_t device, ebg_grid** out)
{
  if (out == nullptr || n < 0 || (n > 0 && points_host == nullptr)) {
    return setError(EBG_ERR_INVALID, "null output or point array");
  }
  *out = nullptr;
  if (n > int64_t(INT32_MAX) - 1) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-2 points");
  }
  if (!allFinite(points_host, 3 * n)) {
    return setError(EBG_ERR_INVALID, "non-finite point coordinate");
  }
  DeviceGuard guard;
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess) {
    return setError(EBG_ERR_NOT_FOUND, "cannot select CUDA device " + std::to_string(device));
  }
  keepPoolMemory();
  auto* G   = new ebg_grid;
  G->target = target_per_cell > 0 ? target_per_cell : 1.0;
  cudaGetDevice(&G->device);
  cudaDeviceGetAttribute(&G->numSms, cudaDevAttrMultiProcessorCount, G->device);
  if (n == 0) {
    // an empty cloud: one empty cell; every query reports nothing found
    const uint32_t zero[2] = {0u, 0u};
    if (cudaMalloc((void**)&G->dPoints, 16) != cudaSuccess || cudaMalloc((void**)&G->dStart, 8) != cudaSuccess ||
        cudaMalloc((void**)&G->dStatus, sizeof(int)) != cudaSuccess ||
        cudaMemcpy(G->dStart, zero, 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(G->dStatus, 0, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      ebg_grid_destroy(G);
      return setError(EBG_ERR_NO_MEMORY, "grid allocation");
    }
    GridView& g = G->view;
    g.h         = 1.0;
    g.invH      = 1.0;
    g.n[0] = g.n[1] = g.n[2] = 1;
    g.points                 = G->dPoints;
    g.cellStart              = G->dStart;
    *out                     = G;
    return EBG_OK;
  }
  cudaStream_t s = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  std::vector<void*> tmp;
  auto alloc = [&](void** p, size_t bytes) {
    if (cudaMallocAsync(p, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
      return false;
    }
    tmp.push_back(*p);
    return true;
  };
  auto fail = [&](ebg_status code, const std::string& msg) {
    for (void* p : tmp) {
      cudaFreeAsync(p, s);
    }
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    ebg_grid_destroy(G);
    return setError(code, msg);
  };
  float*        dPts = nullptr;
  unsigned int* dBox = nullptr;
  if (!alloc((void**)&dPts, 12 * size_t(n)) || !alloc((void**)&dBox, 24)) {
    return fail(EBG_ERR_NO_MEMORY, "grid build workspace");
  }
  cudaMemcpyAsync(dPts, points_host, 12 * size_t(n), cudaMemcpyHostToDevice, s);
  const unsigned int init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  cudaMemcpyAsync(dBox, init, sizeof(init), cudaMemcpyHostToDevice, s);
  kGridBounds<<<std::min(gridBlocks(n), 4096u), 256, 0, s>>>(dPts, n, dBox);
  unsigned int hb[6];
  cudaMemcpyAsync(hb, dBox, sizeof(hb), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return fail(EBG_ERR_CUDA, std::string("grid bounds: ") + cudaGetErrorString(cudaGetLastError()));
  }
  // cell size as the reference sizes it (PointCloudHashGridImplem.hpp:63-125, the cell size and its cap)
  GridView& g = G->view;
  double    lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    lo[a] = hostKeyToFloat(hb[a]);
    hi[a] = hostKeyToFloat(hb[3 + a]);
  }
  const double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const double vol    = ext[0] * ext[1] * ext[2];
  double       h      = vol > 0 ? std::cbrt(vol / double(n) * G->target)
                                : (std::max({ext[0], ext[1], ext[2]}) > 0 ? std::max({ext[0], ext[1], ext[2]}) / std::cbrt(double(n))
                                                                          : 1.0);
  if (!(h > 0)) {
    h = 1.0;
  }
  const double maxCells = std::min(64.0 + 8.0 * double(n), double(INT32_MAX - 1));
  auto         cellsFor = [&](double hh) {
    return (std::floor(ext[0] / hh) + 1) * (std::floor(ext[1] / hh) + 1) * (std::floor(ext[2] / hh) + 1);
  };
  for (int guard2 = 0; guard2 < 100 && cellsFor(h) > maxCells; guard2++) {
    h *= std::cbrt(cellsFor(h) / maxCells);
  }
  if (!(cellsFor(h) <= maxCells)) {
    return fail(EBG_ERR_INVALID, "grid cell size did not converge");
  }
  for (int a = 0; a < 3; a++) {
    g.lo[a] = lo[a];
    g.n[a]  = int(std::floor(ext[a] / h)) + 1;
  }
  g.h               = h;
  g.invH            = 1.0 / h;
  g.numPoints       = n;
  const int64_t nc  = int64_t(g.n[0]) * g.n[1] * g.n[2];
  uint32_t *cell = nullptr, *cellOut = nullptr, *ids = nullptr, *idsOut = nullptr, *counts = nullptr;
  if (!alloc((void**)&cell, 4 * size_t(n)) || !alloc((void**)&cellOut, 4 * size_t(n)) ||
      !alloc((void**)&ids, 4 * size_t(n)) || !alloc((void**)&idsOut, 4 * size_t(n)) ||
      !alloc((void**)&counts, 4 * size_t(nc + 1)) ||
      cudaMalloc((void**)&G->dPoints, 16 * size_t(n)) != cudaSuccess ||
      cudaMalloc((void**)&G->dStart, 4 * size_t(nc + 1)) != cudaSuccess ||
      cudaMalloc((void**)&G->dInv, 4 * size_t(n)) != cudaSuccess ||
      cudaMalloc((void**)&G->dStatus, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return fail(EBG_ERR_NO_MEMORY, "grid allocation");
  }
  cudaMemsetAsync(counts, 0, 4 * size_t(nc + 1), s);
  cudaMemsetAsync(G->dStatus, 0, sizeof(int), s);
  kGridCells<<<gridBlocks(n), 256, 0, s>>>(dPts, n, g, cell, ids, counts);
  size_t sortBytes = 0, scanBytes = 0;
  int cellBits = 1;
  while (cellBits < 32 && (int64_t(1) << cellBits) < nc) {
    cellBits++;
  }
  cub::DeviceRadixSort::SortPairs(nullptr, sortBytes, cell, cellOut, ids, idsOut, int(n), 0, cellBits, s);
  cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, counts, G->dStart, int(nc + 1), s);
  void* work = nullptr;
  if (!alloc(&work, std::max(sortBytes, scanBytes))) {
    return fail(EBG_ERR_NO_MEMORY, "grid sort workspace");
  }
  cub::DeviceRadixSort::SortPairs(work, sortBytes, cell, cellOut, ids, idsOut, int(n), 0, cellBits, s);
  cub::DeviceScan::ExclusiveSum(work, scanBytes, counts, G->dStart, int(nc + 1), s);
  kGridGather<<<gridBlocks(n), 256, 0, s>>>(dPts, idsOut, n, G->dPoints, G->dInv);
  for (void* p : tmp) {
    cudaFreeAsync(p, s);
  }
  tmp.clear();
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return fail(EBG_ERR_CUDA, std::string("grid build: ") + cudaGetErrorString(cudaGetLastError()));
  }
  cudaStreamDestroy(s);
  g.points    = G->dPoints;
  g.cellStart = G->dStart;
  *out        = G;
  return EBG_OK;
}

ebg_status ebg_grid_destroy(ebg_grid* G)
{
  if (G == nullptr) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(G->device);
  cudaFree(G->dPoints);
  cudaFree(G->dStart);
  cudaFree(G->dInv);
  cudaFree(G->dStatus);
  delete G;
  return EBG_OK;
}

ebg_status ebg_grid_info(const ebg_grid* G, int32_t* cells_xyz, double* cell_size)
{
  if (G == nullptr) {
    return setError(EBG_ERR_INVALID, "null grid");
  }
  if (cells_xyz) {
    for (int a = 0; a < 3; a++) {
      cells_xyz[a] = G->view.n[a];
    }
  }
  if (cell_size) {
    *cell_size = G->view.h;
  }
  return EBG_OK;
}

// The three query forms: external points (queries), self queries of listed cloud indices (ids) and
// self queries of every point (neither).  Asynchronous on s.
static ebg_status gridQuery(const ebg_grid* G, const float* queries_dev, const int64_t* ids_dev, int64_t nq, int32_t k,
                            int32_t* idx_dev, float* d2_dev, cudaStream_t s)
{
  int kt = 1;
  while (kt < k) {
    kt *= 2;
  }
  std::vector<void*> ws;
  auto get = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMallocAsync(&p, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    ws.push_back(p);
    return p;
  };
  auto release = [&]() {
    for (void* p : ws) {
      cudaFreeAsync(p, s);
    }
  };
  uint32_t* order = nullptr;
  if (queries_dev) {
    // Morton order of the queries over the grid's box, so that a warp's queries visit nearby cells
    auto* kin  = static_cast<uint32_t*>(get(4 * size_t(nq)));
    auto* kout = static_cast<uint32_t*>(get(4 * size_t(nq)));
    auto* iin  = static_cast<uint32_t*>(get(4 * size_t(nq)));
    order      = static_cast<uint32_t*>(get(4 * size_t(nq)));
    size_t tb  = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, iin, order, int(nq), 0, 30, s);
    void* tmpb = get(tb);
    if (!kin || !kout || !iin || !order || !tmpb) {
      release();
      return setError(EBG_ERR_NO_MEMORY, "grid query workspace");
    }
    float lo[3], scale[3];
    for (int a = 0; a < 3; a++) {
      const double ext = std::max(double(G->view.n[a]) * G->view.h, 1e-30);
      lo[a]            = float(G->view.lo[a]);
      scale[a]         = float(1024.0 / ext);
    }
    launchQueryKeys(queries_dev, nq, lo, scale, kin, iin, s);
    cub::DeviceRadixSort::SortPairs(tmpb, tb, kin, kout, iin, order, int(nq), 0, 30, s);
  }
  GridQueryArgs a{};
  a.g        = G->view;
  a.queries  = queries_dev;
  a.order    = order;
  a.pointIds = ids_dev;
  a.inv      = G->dInv;
  a.n        = nq;
  a.k        = k;
  a.outIdx   = idx_dev;
  a.outD2    = d2_dev;
  a.status   = G->dStatus;
  const cudaError_t e = launchGridKnn(a, kt, G->numSms, s);
  release();
  if (e != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("grid k-NN launch failed: ") + cudaGetErrorString(e));
  }
  return EBG_OK;
}

static ebg_status gridCheck(const ebg_grid* G, cudaStream_t s)
{
  int st = 0;
  if (cudaMemcpyAsync(&st, G->dStatus, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  if (st != 0) {
    cudaMemsetAsync(G->dStatus, 0, sizeof(int), s);
    cudaStreamSynchronize(s);
    return setError(EBG_ERR_INVALID, "non-finite query coordinate or cloud index out of range");
  }
  return EBG_OK;
}

// host arrays in and out around one of the device forms; synchronous
static ebg_status gridHost(const ebg_grid* G, const float* queries_host, const int64_t* ids_host, int64_t nq,
                           int32_t k, int32_t* idx_host, float* d2_host, cudaStream_t s)
{
  if (nq == 0) {
    return EBG_OK;
  }
  void *q = nullptr, *ids = nullptr, *idx = nullptr, *d2 = nullptr;
  const size_t outN = size_t(nq) * size_t(k);
  bool         ok   = cudaMallocAsync(&idx, 4 * outN, s) == cudaSuccess && cudaMallocAsync(&d2, 4 * outN, s) == cudaSuccess;
  if (ok && queries_host) {
    ok = cudaMallocAsync(&q, 12 * size_t(nq), s) == cudaSuccess &&
         cudaMemcpyAsync(q, queries_host, 12 * size_t(nq), cudaMemcpyHostToDevice, s) == cudaSuccess;
  }
  if (ok && ids_host) {
    ok = cudaMallocAsync(&ids, 8 * size_t(nq), s) == cudaSuccess &&
         cudaMemcpyAsync(ids, ids_host, 8 * size_t(nq), cudaMemcpyHostToDevice, s) == cudaSuccess;
  }
  ebg_status st = ok ? EBG_OK : setError(EBG_ERR_NO_MEMORY, "grid host-call buffers");
  if (st == EBG_OK) {
    st = gridQuery(G, static_cast<const float*>(q), static_cast<const int64_t*>(ids), nq, k, static_cast<int32_t*>(idx),
                   static_cast<float*>(d2), s);
  }
  if (st == EBG_OK) {
    cudaMemcpyAsync(idx_host, idx, 4 * outN, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(d2_host, d2, 4 * outN, cudaMemcpyDeviceToHost, s);
  }
  for (void* p : {q, ids, idx, d2}) {
    if (p) {
      cudaFreeAsync(p, s);
    }
  }
  cudaGetLastError();
  const ebg_status cs = gridCheck(G, s);
  return st != EBG_OK ? st : cs;
}

static bool kOk(int32_t k) { return k >= 1 && k <= 32; }

ebg_status ebg_grid_knn(const ebg_grid* G, const float* queries_dev, int64_t nq, int32_t k, int32_t* idx_dev,
                        float* d2_dev, void* stream)
{
  if (G == nullptr || nq < 0 || !kOk(k) || (nq > 0 && (!queries_dev || !idx_dev || !d2_dev))) {
    return setError(EBG_ERR_INVALID, "bad grid k-NN arguments (k must be in [1, 32])");
  }
  if (nq > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 queries per call");
  }
  if (nq == 0) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(G->device);
  return gridQuery(G, queries_dev, nullptr, nq, k, idx_dev, d2_dev, static_cast<cudaStream_t>(stream));
}

ebg_status ebg_grid_knn_host(const ebg_grid* G, const float* queries_host, int64_t nq, int32_t k, int32_t* idx_host,
                             float* d2_host, void* stream)
{
  if (G == nullptr || nq < 0 || !kOk(k) || (nq > 0 && (!queries_host || !idx_host || !d2_host))) {
    return setError(EBG_ERR_INVALID, "bad grid k-NN arguments (k must be in [1, 32])");
  }
  if (nq > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 queries per call");
  }
  DeviceGuard guard;
  cudaSetDevice(G->device);
  return gridHost(G, queries_host, nullptr, nq, k, idx_host, d2_host, static_cast<cudaStream_t>(stream));
}

ebg_status ebg_grid_self_knn(const ebg_grid* G, int32_t k, int32_t* idx_dev, float* d2_dev, void* stream)
{
  if (G == nullptr || !kOk(k) || (G->view.numPoints > 0 && (!idx_dev || !d2_dev))) {
    return setError(EBG_ERR_INVALID, "bad grid self k-NN arguments (k must be in [1, 32])");
  }
  if (G->view.numPoints == 0) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(G->device);
  return gridQuery(G, nullptr, nullptr, G->view.numPoints, k, idx_dev, d2_dev, static_cast<cudaStream_t>(stream));
}

ebg_status ebg_grid_self_knn_host(const ebg_grid* G, int32_t k, int32_t* idx_host, float* d2_host, void* stream)
{
  if (G == nullptr || !kOk(k) || (G->view.numPoints > 0 && (!idx_host || !d2_host))) {
    return setError(EBG_ERR_INVALID, "bad grid self k-NN arguments (k must be in [1, 32])");
  }
  DeviceGuard guard;
  cudaSetDevice(G->device);
  return gridHost(G, nullptr, nullptr, G->view.numPoints, k, idx_host, d2_host, static_cast<cudaStream_t>(stream));
}

ebg_status ebg_grid_self_knn_points(const ebg_grid* G, const int64_t* point_ids_dev, int64_t m, int32_t k,
                                    int32_t* idx_dev, float* d2_dev, void* stream)
{
  if (G == nullptr || m < 0 || !kOk(k) || (m > 0 && (!point_ids_dev || !idx_dev || !d2_dev))) {
    return setError(EBG_ERR_INVALID, "bad grid self k-NN arguments (k must be in [1, 32])");
  }
  if (m > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 queries per call");
  }
  if (m == 0) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(G->device);
  return gridQuery(G, nullptr, point_ids_dev, m, k, idx_dev, d2_dev, static_cast<cudaStream_t>(stream));
}

ebg_status ebg_grid_self_knn_points_host(const ebg_grid* G, const int64_t* point_ids_host, int64_t m, int32_t k,
                                         int32_t* idx_host, float* d2_host, void* stream)
{
  if (G == nullptr || m < 0 || !kOk(k) || (m > 0 && (!point_ids_host || !idx_host || !d2_host))) {
    return setError(EBG_ERR_INVALID, "bad grid self k-NN arguments (k must be in [1, 32])");
  }
  if (m > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 queries per call");
  }
  DeviceGuard guard;
  cudaSetDevice(G->device);
  return gridHost(G, nullptr, point_ids_host, m, k, idx_host, d2_host, static_cast<cudaStream_t>(stream));
}

int64_t ebg_grid_size(const ebg_grid* G) { return G ? G->view.numPoints : -1; }

ebg_status ebg_grid_check_status(const ebg_grid* G, void* stream)
{
  if (G == nullptr) {
    return setError(EBG_ERR_INVALID, "null grid");
  }
  DeviceGuard guard;
  cudaSetDevice(G->device);
  return gridCheck(G, static_cast<cudaStream_t>(stream));
}

} // extern "C"
