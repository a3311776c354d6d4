// Pseudonormals of a triangle soup on the device, bit-identical to the host restatement of the
// reference's DCEL (mesh_host.cpp: computePseudonormals): the same operations in the same order,
// compiled with -fmad=false so no multiply-add is fused.
//   face:   (x2 - x0) x (x2 - x1), normalised once (the Triangle's normal) and once more (the DCEL
//           face normal) -- division is a multiply by the reciprocal (Vec3T::operator/);
//   edge:   normalise(n_face + n_pair), the pair being the other triangle around the edge's first
//           vertex that holds its second vertex;
//   vertex: the sum over the vertex's triangles in facet order of alpha * n_face, alpha the angle
//           at the vertex, then normalised.
// The angles are acos(clamp(e1 . e2)) with the host C library's acos, as in the reference: the
// device computes the clamped cosines, the host takes their acos, the device does the rest.
#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include "capi_common.h"
#include "mesh_build_gpu.h"

namespace ebg {

namespace {

struct D3
{
  double x, y, z;
};
__device__ __forceinline__ D3 ld3(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ D3 sub3(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 cross3(D3 a, D3 b)
{
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double len3(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ D3 divs3(D3 a, double s)
{
  const double is = 1.0 / s;
  return {is * a.x, is * a.y, is * a.z};
}
__device__ __forceinline__ void st3(double* p, D3 a)
{
  p[0] = a.x;
  p[1] = a.y;
  p[2] = a.z;
}

// status bits
constexpr int NRM_DEGENERATE  = 1;
constexpr int NRM_NONMANIFOLD = 2;

__global__ void kFaceNormals(const double* __restrict__ V, const int32_t* __restrict__ F, int64_t nt,
                             double* __restrict__ triN, double* __restrict__ faceN, int* __restrict__ status)
{
  for (int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; f < nt; f += int64_t(gridDim.x) * blockDim.x) {
    const D3     x0 = ld3(V + 3 * int64_t(F[3 * f])), x1 = ld3(V + 3 * int64_t(F[3 * f + 1])),
             x2 = ld3(V + 3 * int64_t(F[3 * f + 2]));
    const D3     c = cross3(sub3(x2, x0), sub3(x2, x1));
    const double l = len3(c);
    if (!(l > 0.0)) {
      atomicOr(status, NRM_DEGENERATE);
      continue;
    }
    const D3 once = divs3(c, l);
    st3(triN + 3 * f, once);
    st3(faceN + 3 * f, divs3(once, len3(once)));
  }
}

// corner entry i = 3 f + k belongs to vertex F[i]
__global__ void kCornerKeys(const int32_t* __restrict__ F, int64_t n3, uint32_t* __restrict__ keys,
                            uint32_t* __restrict__ vals, uint32_t* __restrict__ counts)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n3; i += int64_t(gridDim.x) * blockDim.x) {
    keys[i] = uint32_t(F[i]);
    vals[i] = uint32_t(i);
    atomicAdd(counts + F[i], 1u);
  }
}

__global__ void kEdgeNormals(const int32_t* __restrict__ F, int64_t nt, const uint32_t* __restrict__ start,
                             const uint32_t* __restrict__ around, const double* __restrict__ faceN,
                             double* __restrict__ edgeN, int* __restrict__ status)
{
  for (int64_t h = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; h < 3 * nt; h += int64_t(gridDim.x) * blockDim.x) {
    const int64_t f = h / 3;
    const int     i = int(h - 3 * f);
    const int32_t a = F[3 * f + i], b = F[3 * f + (i + 1) % 3];
    int64_t       pair = -1, found = 0;
    for (uint32_t e = start[a]; e < start[a + 1]; e++) {
      const int64_t g = int64_t(around[e] / 3);
      if (g == f) {
        continue;
      }
      for (int k = 0; k < 3; k++) {
        if (F[3 * g + k] == b) {
          found++;
          pair = g;
        }
      }
    }
    if (found > 1) {
      atomicOr(status, NRM_NONMANIFOLD);
    }
    D3 n = ld3(faceN + 3 * f);
    if (pair >= 0) {
      n = {n.x + faceN[3 * pair], n.y + faceN[3 * pair + 1], n.z + faceN[3 * pair + 2]};
    }
    const double l = len3(n);
    st3(edgeN + 9 * f + 3 * i, (l > DBL_EPSILON) ? divs3(n, l) : D3{0.0, 0.0, 0.0});
  }
}

// the clamped cosine of the angle at each corner (neighbours in half-edge loop order: a:(b,c),
// b:(a,c), c:(b,a))
__global__ void kCornerCos(const double* __restrict__ V, const int32_t* __restrict__ F, int64_t nt,
                           double* __restrict__ cs)
{
  for (int64_t h = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; h < 3 * nt; h += int64_t(gridDim.x) * blockDim.x) {
    const int64_t f = h / 3;
    const int     k = int(h - 3 * f);
    const int32_t a = F[3 * f], b = F[3 * f + 1], c = F[3 * f + 2];
    const int32_t corner = k == 0 ? a : (k == 1 ? b : c);
    const int32_t n1     = k == 0 ? b : (k == 1 ? a : b);
    const int32_t n2     = k == 0 ? c : (k == 1 ? c : a);
    const D3      x0     = ld3(V + 3 * int64_t(corner));
    D3            e1     = sub3(ld3(V + 3 * int64_t(n1)), x0);
    D3            e2     = sub3(ld3(V + 3 * int64_t(n2)), x0);
    e1                   = divs3(e1, len3(e1));
    e2                   = divs3(e2, len3(e2));
    const double d       = dot3(e1, e2);
    cs[h]                = d < -1.0 ? -1.0 : (1.0 < d ? 1.0 : d);
  }
}

__global__ void kVertexNormals(int64_t nv, const uint32_t* __restrict__ start, const uint32_t* __restrict__ around,
                               const double* __restrict__ alpha, const double* __restrict__ faceN, double* __restrict__ vn)
{
  for (int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < nv; v += int64_t(gridDim.x) * blockDim.x) {
    double x = 0.0, y = 0.0, z = 0.0;
    for (uint32_t e = start[v]; e < start[v + 1]; e++) {
      const uint32_t i  = around[e];
      const double*  fn = faceN + 3 * size_t(i / 3);
      x += alpha[i] * fn[0];
      y += alpha[i] * fn[1];
      z += alpha[i] * fn[2];
    }
    const D3     n = {x, y, z};
    const double l = len3(n);
    st3(vn + 3 * v, (l > DBL_EPSILON) ? divs3(n, l) : n);
  }
}

__global__ void kCornerVN(const int32_t* __restrict__ F, int64_t nt, const double* __restrict__ vn,
                          double* __restrict__ cornerVN)
{
  for (int64_t h = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; h < 3 * nt; h += int64_t(gridDim.x) * blockDim.x) {
    const double* p = vn + 3 * int64_t(F[h]);
    cornerVN[3 * h]     = p[0];
    cornerVN[3 * h + 1] = p[1];
    cornerVN[3 * h + 2] = p[2];
  }
}

inline unsigned gridOf(int64_t n) { return unsigned(std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 1 << 20)); }

} // namespace

ebg_status pseudonormalsOnDevice(const double* dV, int64_t nv, const int32_t* dF, int64_t nt, double* dTriN,
                                 double* dCornerVN, double* dEdgeN, cudaStream_t s)
{
  const int64_t      n3 = 3 * nt;
  std::vector<void*> tmp;
  auto alloc = [&](void** p, size_t bytes) {
    if (cudaMallocAsync(p, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
      return false;
    }
    tmp.push_back(*p);
    return true;
  };
  struct Free
  {
    std::vector<void*>& t;
    cudaStream_t        s;
    ~Free()
    {
      for (void* p : t) {
        cudaFreeAsync(p, s);
      }
    }
  } freer{tmp, s};
  double *  faceN = nullptr, *cs = nullptr, *vn = nullptr;
  uint32_t *keys = nullptr, *keysOut = nullptr, *vals = nullptr, *around = nullptr, *counts = nullptr,
           *start = nullptr;
  int*      status = nullptr;
  if (!alloc((void**)&faceN, 24 * size_t(nt)) || !alloc((void**)&cs, 8 * size_t(n3)) ||
      !alloc((void**)&vn, 24 * size_t(nv)) || !alloc((void**)&keys, 4 * size_t(n3)) ||
      !alloc((void**)&keysOut, 4 * size_t(n3)) || !alloc((void**)&vals, 4 * size_t(n3)) ||
      !alloc((void**)&around, 4 * size_t(n3)) || !alloc((void**)&counts, 4 * size_t(nv + 1)) ||
      !alloc((void**)&start, 4 * size_t(nv + 1)) || !alloc((void**)&status, 4)) {
    return setError(EBG_ERR_NO_MEMORY, "device pseudonormal workspace");
  }
  cudaMemsetAsync(status, 0, 4, s);
  cudaMemsetAsync(counts, 0, 4 * size_t(nv + 1), s);
  kFaceNormals<<<gridOf(nt), 256, 0, s>>>(dV, dF, nt, dTriN, faceN, status);
  // triangles around each vertex in facet order: a stable sort of the corners by vertex
  kCornerKeys<<<gridOf(n3), 256, 0, s>>>(dF, n3, keys, vals, counts);
  size_t bytes = 0, scanBytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, keysOut, vals, around, int(n3), 0, 32, s);
  cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, counts, start, int(nv + 1), s);
  void* work = nullptr;
  if (!alloc(&work, std::max(bytes, scanBytes))) {
    return setError(EBG_ERR_NO_MEMORY, "device pseudonormal workspace");
  }
  cub::DeviceRadixSort::SortPairs(work, bytes, keys, keysOut, vals, around, int(n3), 0, 32, s);
  cub::DeviceScan::ExclusiveSum(work, scanBytes, counts, start, int(nv + 1), s);
  kEdgeNormals<<<gridOf(n3), 256, 0, s>>>(dF, nt, start, around, faceN, dEdgeN, status);
  kCornerCos<<<gridOf(n3), 256, 0, s>>>(dV, dF, nt, cs);
  // the angles: the host C library's acos of the device's cosines
  std::vector<double> h(static_cast<size_t>(n3));
  int                 st = 0;
  cudaMemcpyAsync(h.data(), cs, 8 * size_t(n3), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&st, status, 4, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("device pseudonormals: ") + cudaGetErrorString(cudaGetLastError()));
  }
  if (st & NRM_DEGENERATE) {
    return setError(EBG_ERR_INVALID, "degenerate (zero-area) triangle in the soup");
  }
  if (st & NRM_NONMANIFOLD) {
    return setError(EBG_ERR_INVALID, "non-manifold edge (shared by more than two triangles)");
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n3; i++) {
    h[size_t(i)] = std::acos(h[size_t(i)]);
  }
  cudaMemcpyAsync(cs, h.data(), 8 * size_t(n3), cudaMemcpyHostToDevice, s);
  kVertexNormals<<<gridOf(nv), 256, 0, s>>>(nv, start, around, cs, faceN, vn);
  kCornerVN<<<gridOf(n3), 256, 0, s>>>(dF, nt, vn, dCornerVN);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("device pseudonormals: ") + cudaGetErrorString(cudaGetLastError()));
  }
  return EBG_OK;
}

} // namespace ebg
