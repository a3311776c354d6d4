// C ABI of the point-cloud path: PointCloudBVH construction (on the device) and k-NN queries.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "capi_common.h"
#include "cloud_kernels.h"
#include "ebg_device.cuh"
#include "ebgeometry_b200.h"
#include "mesh_kernels.h"

using namespace ebg;

struct ebg_cloud
{
  int          device  = 0;
  int          numSms  = 148;
  int64_t      n       = 0;
  int          leaf    = 16;
  int          levels  = 0;     // node levels of the tree (0: the root is one leaf)
  int64_t      numNodes = 0;
  bool         radixTree = false; // false: the balanced fallback tree
  EbgCloudView view{};
  void*        dNodes  = nullptr;
  void*        dPoints = nullptr;
  uint32_t*    dInv    = nullptr; // cloud index -> leaf position (self queries of given points)
  int*         dStatus = nullptr;
};

namespace {

template <class T>
T* devAlloc(size_t count, cudaStream_t s, std::vector<void*>& list)
{
  void* p = nullptr;
  if (cudaMallocAsync(&p, std::max<size_t>(count * sizeof(T), 16), s) != cudaSuccess) {
    return nullptr;
  }
  list.push_back(p);
  return static_cast<T*>(p);
}

void freeAll(std::vector<void*>& list, cudaStream_t s)
{
  for (void* p : list) {
    cudaFreeAsync(p, s);
  }
  list.clear();
}

ebg_status createCloud(const float* pointsDev, int64_t n, const ebg_build_opts* opts, cudaStream_t s, ebg_cloud** out)
{
  const int L = (opts && opts->leaf_size > 0) ? opts->leaf_size : 8;
  if (L > EBG_MAX_LEAF) {
    return setError(EBG_ERR_INVALID, "leaf size must be in [1, 32]");
  }
  int device = 0;
  cudaGetDevice(&device);
  keepPoolMemory();
  auto* c   = new ebg_cloud;
  c->device = device;
  c->n      = n;
  c->leaf   = L;
  cudaDeviceGetAttribute(&c->numSms, cudaDevAttrMultiProcessorCount, device);

  if (cudaMalloc(&c->dPoints, size_t(n) * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&c->dInv), size_t(n) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&c->dStatus), sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    ebg_cloud_destroy(c);
    return setError(EBG_ERR_NO_MEMORY, "device allocation for the point cloud");
  }
  cudaMemsetAsync(c->dStatus, 0, sizeof(int), s);
  CloudTree   tree;
  const bool  balanced = opts && (opts->flags & EBG_CLOUD_BALANCED);
  cudaError_t e        = buildCloud(pointsDev, n, L, balanced, static_cast<float4*>(c->dPoints), tree, s);
  c->dNodes     = tree.nodes;
  if (e == cudaSuccess) {
    launchInvertOrder(static_cast<const float4*>(c->dPoints), n, c->dInv, s);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    e = cudaStreamSynchronize(s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    ebg_cloud_destroy(c);
    if (e == cudaErrorMemoryAllocation) {
      return setError(EBG_ERR_NO_MEMORY, "build workspace for the point cloud");
    }
    return setError(EBG_ERR_CUDA, std::string("point cloud build failed: ") + cudaGetErrorString(e));
  }
  c->levels      = tree.depth;
  c->numNodes    = tree.numNodes;
  c->radixTree   = tree.radix;
  const float* rootBox = tree.rootBox;
  EbgCloudView& v = c->view;
  v.nodes         = static_cast<const EbgNode4*>(c->dNodes);
  v.points        = static_cast<const float4*>(c->dPoints);
  for (int a = 0; a < 3; a++) {
    v.root_lo[a] = rootBox[a];
    v.root_hi[a] = rootBox[3 + a];
    const double lo = rootBox[a], hi = rootBox[3 + a];
    const double ext = std::max(hi - lo, 1e-30);
    v.morton_lo[a]    = float(lo);
    v.morton_scale[a] = float(1024.0 / ext);
  }
  if (c->levels == 0) {
    v.root_ref   = EBG_LEAF_BIT | 0u;
    v.root_count = uint32_t(n);
  }
  else {
    v.root_ref   = 0;
    v.root_count = 0;
  }
  *out = c;
  return EBG_OK;
}

// self = 1: the queries are the cloud's own points -- all of them in leaf order when selfIds is
// null (nq = n, rows = cloud indices), else the nq cloud indices in selfIds (rows = list order).
ebg_status runKnn(const ebg_cloud* c, const float* q, int64_t nq, int k, int32_t* idx, float* d2,
                  const ebg_query_opts* opts, cudaStream_t s, int self = 0, const int64_t* selfIds = nullptr)
{
  const bool sort = !self && !(opts && opts->no_sort);
  int        kt   = 1;
  while (kt < k) {
    kt *= 2;
  }
  std::vector<void*> ws;
  uint32_t*          order = nullptr;
  if (sort) {
    uint32_t* kin  = devAlloc<uint32_t>(nq, s, ws);
    uint32_t* kout = devAlloc<uint32_t>(nq, s, ws);
    uint32_t* iin  = devAlloc<uint32_t>(nq, s, ws);
    order          = devAlloc<uint32_t>(nq, s, ws);
    size_t tb      = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, iin, order, int(nq), 0, 30, s);
    void* tmp = devAlloc<char>(tb, s, ws);
    if (!kin || !kout || !iin || !order || !tmp) {
      freeAll(ws, s);
      return setError(EBG_ERR_NO_MEMORY, "k-NN query workspace");
    }
    launchQueryKeys(q, nq, c->view.morton_lo, c->view.morton_scale, kin, iin, s);
    cub::DeviceRadixSort::SortPairs(tmp, tb, kin, kout, iin, order, int(nq), 0, 30, s);
  }
  uint32_t* selfPos = nullptr;
  if (self && selfIds) {
    // leaf positions of the given points, sorted: leaf order is Morton order
    uint32_t* kin  = devAlloc<uint32_t>(nq, s, ws);
    uint32_t* rin  = devAlloc<uint32_t>(nq, s, ws);
    selfPos        = devAlloc<uint32_t>(nq, s, ws);
    order          = devAlloc<uint32_t>(nq, s, ws);
    size_t tb      = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, selfPos, rin, order, int(nq), 0, 32, s);
    void* tmp = devAlloc<char>(tb, s, ws);
    if (!kin || !rin || !selfPos || !order || !tmp) {
      freeAll(ws, s);
      return setError(EBG_ERR_NO_MEMORY, "k-NN query workspace");
    }
    launchSelfKeys(selfIds, nq, c->dInv, c->n, kin, rin, c->dStatus, s);
    cub::DeviceRadixSort::SortPairs(tmp, tb, kin, selfPos, rin, order, int(nq), 0, 32, s);
  }
  auto* work = devAlloc<unsigned long long>(1, s, ws);
  if (!work) {
    freeAll(ws, s);
    return setError(EBG_ERR_NO_MEMORY, "k-NN query workspace");
  }
  cudaMemsetAsync(work, 0, sizeof(unsigned long long), s);
  CloudQueryArgs a{};
  a.cloud   = c->view;
  a.queries = q;
  a.order    = order;
  a.self_pos = selfPos;
  a.n        = nq;
  a.k       = k;
  a.out_idx = idx;
  a.out_d2  = d2;
  a.work    = work;
  a.status  = c->dStatus;
  const cudaError_t e = launchCloudKnn(a, kt, c->numSms, s, self != 0);
  freeAll(ws, s);
  if (e != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("k-NN launch failed: ") + cudaGetErrorString(e));
  }
  return EBG_OK;
}

} // namespace

extern "C" {

ebg_status ebg_cloud_create(const float* points_host, int64_t n, const ebg_build_opts* opts, ebg_cloud** out)
{
  if (out == nullptr) {
    return setError(EBG_ERR_INVALID, "out handle pointer is null");
  }
  *out = nullptr;
  if (n <= 0 || points_host == nullptr) {
    return setError(EBG_ERR_INVALID, "point cloud needs at least one point");
  }
  if (n >= int64_t(EBG_LEAF_BIT)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 points");
  }
  if (!allFinite(points_host, 3 * n)) {
    return setError(EBG_ERR_INVALID, "non-finite point coordinate");
  }
  DeviceGuard guard;
  if (opts && opts->device >= 0 && cudaSetDevice(opts->device) != cudaSuccess) {
    return setError(EBG_ERR_NOT_FOUND, "cannot select CUDA device");
  }
  cudaStream_t s  = nullptr;
  float*       dp = nullptr;
  if (cudaMalloc(&dp, size_t(n) * 3 * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    return setError(EBG_ERR_NO_MEMORY, "device buffer for the points");
  }
  cudaMemcpy(dp, points_host, size_t(n) * 3 * sizeof(float), cudaMemcpyHostToDevice);
  const ebg_status rc = createCloud(dp, n, opts, s, out);
  cudaFree(dp);
  return rc;
}

ebg_status ebg_cloud_create_device(const float* points_dev, int64_t n, const ebg_build_opts* opts, ebg_cloud** out,
                                   void* stream)
{
  if (out == nullptr) {
    return setError(EBG_ERR_INVALID, "out handle pointer is null");
  }
  *out = nullptr;
  if (n <= 0 || points_dev == nullptr) {
    return setError(EBG_ERR_INVALID, "point cloud needs at least one point");
  }
  if (n >= int64_t(EBG_LEAF_BIT)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 points");
  }
  DeviceGuard guard;
  if (opts && opts->device >= 0 && cudaSetDevice(opts->device) != cudaSuccess) {
    return setError(EBG_ERR_NOT_FOUND, "cannot select CUDA device");
  }
  return createCloud(points_dev, n, opts, static_cast<cudaStream_t>(stream), out);
}

ebg_status ebg_cloud_destroy(ebg_cloud* c)
{
  if (c == nullptr) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(c->device);
  cudaFree(c->dNodes);
  cudaFree(c->dPoints);
  cudaFree(c->dInv);
  cudaFree(c->dStatus);
  delete c;
  return EBG_OK;
}

int64_t ebg_cloud_size(const ebg_cloud* c) { return c ? c->n : 0; }

ebg_status ebg_cloud_tree_info(const ebg_cloud* c, int64_t* num_nodes, int32_t* depth, int32_t* radix)
{
  if (c == nullptr) {
    return setError(EBG_ERR_INVALID, "null cloud");
  }
  if (num_nodes) {
    *num_nodes = c->numNodes;
  }
  if (depth) {
    *depth = c->levels;
  }
  if (radix) {
    *radix = c->radixTree ? 1 : 0;
  }
  return EBG_OK;
}

ebg_status ebg_cloud_knn(const ebg_cloud*      c,
                         const float*          queries_dev,
                         int64_t               nq,
                         int32_t               k,
                         int32_t*              idx_dev,
                         float*                d2_dev,
                         const ebg_query_opts* opts,
                         void*                 stream)
{
  if (c == nullptr || nq < 0 || k < 1 || k > 32 || (nq > 0 && (!queries_dev || !idx_dev || !d2_dev))) {
    return setError(EBG_ERR_INVALID, "bad k-NN arguments (k must be in [1, 32])");
  }
  if (nq > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 queries per call");
  }
  if (nq == 0) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(c->device);
  return runKnn(c, queries_dev, nq, k, idx_dev, d2_dev, opts, static_cast<cudaStream_t>(stream));
}

ebg_status ebg_cloud_knn_host(const ebg_cloud*      c,
                              const float*          queries_host,
                              int64_t               nq,
                              int32_t               k,
                              int32_t*              idx_host,
                              float*                d2_host,
                              const ebg_query_opts* opts,
                              void*                 stream)
{
  if (c == nullptr || nq < 0 || k < 1 || k > 32 || (nq > 0 && (!queries_host || !idx_host || !d2_host))) {
    return setError(EBG_ERR_INVALID, "bad k-NN arguments (k must be in [1, 32])");
  }
  if (nq == 0) {
    return EBG_OK;
  }
  if (!allFinite(queries_host, 3 * nq)) {
    return setError(EBG_ERR_INVALID, "non-finite query coordinate");
  }
  DeviceGuard        guard;
  cudaSetDevice(c->device);
  cudaStream_t       s = static_cast<cudaStream_t>(stream);
  std::vector<void*> ws;
  float*             dq = devAlloc<float>(3 * nq, s, ws);
  int32_t*           di = devAlloc<int32_t>(nq * k, s, ws);
  float*             dd = devAlloc<float>(nq * k, s, ws);
  if (!dq || !di || !dd) {
    freeAll(ws, s);
    return setError(EBG_ERR_NO_MEMORY, "device buffers for the host k-NN call");
  }
  cudaMemsetAsync(c->dStatus, 0, sizeof(int), s);
  cudaMemcpyAsync(dq, queries_host, size_t(nq) * 3 * sizeof(float), cudaMemcpyHostToDevice, s);
  ebg_status rc = runKnn(c, dq, nq, k, di, dd, opts, s);
  if (rc == EBG_OK) {
    cudaMemcpyAsync(idx_host, di, size_t(nq) * k * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(d2_host, dd, size_t(nq) * k * sizeof(float), cudaMemcpyDeviceToHost, s);
  }
  freeAll(ws, s);
  int st = 0;
  cudaMemcpyAsync(&st, c->dStatus, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  if (rc == EBG_OK && st != 0) {
    return setError(EBG_ERR_TRAVERSAL, "k-NN traversal stopped early (status " + std::to_string(st) + ")");
  }
  return rc;
}

ebg_status ebg_cloud_self_knn(const ebg_cloud* c, int32_t k, int32_t* idx_dev, float* d2_dev, void* stream)
{
  if (c == nullptr || k < 1 || k > 32 || idx_dev == nullptr || d2_dev == nullptr) {
    return setError(EBG_ERR_INVALID, "bad self k-NN arguments (k must be in [1, 32])");
  }
  if (c->n > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 points");
  }
  DeviceGuard guard;
  cudaSetDevice(c->device);
  return runKnn(c, nullptr, c->n, k, idx_dev, d2_dev, nullptr, static_cast<cudaStream_t>(stream), 1);
}

ebg_status ebg_cloud_self_knn_points(const ebg_cloud* c,
                                     const int64_t*   point_ids_dev,
                                     int64_t          m,
                                     int32_t          k,
                                     int32_t*         idx_dev,
                                     float*           d2_dev,
                                     void*            stream)
{
  if (c == nullptr || m < 0 || k < 1 || k > 32 || (m > 0 && (!point_ids_dev || !idx_dev || !d2_dev))) {
    return setError(EBG_ERR_INVALID, "bad self k-NN arguments (k must be in [1, 32])");
  }
  if (m > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 points per call");
  }
  if (m == 0) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(c->device);
  return runKnn(c, nullptr, m, k, idx_dev, d2_dev, nullptr, static_cast<cudaStream_t>(stream), 1, point_ids_dev);
}

ebg_status ebg_cloud_self_knn_host(const ebg_cloud* c, int32_t k, int32_t* idx_host, float* d2_host, void* stream)
{
  if (c == nullptr || k < 1 || k > 32 || idx_host == nullptr || d2_host == nullptr) {
    return setError(EBG_ERR_INVALID, "bad self k-NN arguments (k must be in [1, 32])");
  }
  DeviceGuard        guard;
  cudaSetDevice(c->device);
  cudaStream_t       s = static_cast<cudaStream_t>(stream);
  std::vector<void*> ws;
  int32_t*           di = devAlloc<int32_t>(c->n * k, s, ws);
  float*             dd = devAlloc<float>(c->n * k, s, ws);
  if (!di || !dd) {
    freeAll(ws, s);
    return setError(EBG_ERR_NO_MEMORY, "device buffers for the host self k-NN call");
  }
  cudaMemsetAsync(c->dStatus, 0, sizeof(int), s);
  ebg_status rc = ebg_cloud_self_knn(c, k, di, dd, stream);
  if (rc == EBG_OK) {
    cudaMemcpyAsync(idx_host, di, size_t(c->n) * k * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(d2_host, dd, size_t(c->n) * k * sizeof(float), cudaMemcpyDeviceToHost, s);
  }
  freeAll(ws, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  return rc == EBG_OK ? ebg_cloud_check_status(c, stream) : rc;
}

ebg_status ebg_cloud_self_knn_points_host(const ebg_cloud* c,
                                          const int64_t*   point_ids_host,
                                          int64_t          m,
                                          int32_t          k,
                                          int32_t*         idx_host,
                                          float*           d2_host,
                                          void*            stream)
{
  if (c == nullptr || m < 0 || k < 1 || k > 32 || (m > 0 && (!point_ids_host || !idx_host || !d2_host))) {
    return setError(EBG_ERR_INVALID, "bad self k-NN arguments (k must be in [1, 32])");
  }
  if (m == 0) {
    return EBG_OK;
  }
  DeviceGuard        guard;
  cudaSetDevice(c->device);
  cudaStream_t       s = static_cast<cudaStream_t>(stream);
  std::vector<void*> ws;
  int64_t*           dp = devAlloc<int64_t>(m, s, ws);
  int32_t*           di = devAlloc<int32_t>(m * k, s, ws);
  float*             dd = devAlloc<float>(m * k, s, ws);
  if (!dp || !di || !dd) {
    freeAll(ws, s);
    return setError(EBG_ERR_NO_MEMORY, "device buffers for the host self k-NN call");
  }
  cudaMemcpyAsync(dp, point_ids_host, size_t(m) * sizeof(int64_t), cudaMemcpyHostToDevice, s);
  ebg_status rc = ebg_cloud_self_knn_points(c, dp, m, k, di, dd, stream);
  if (rc == EBG_OK) {
    cudaMemcpyAsync(idx_host, di, size_t(m) * k * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(d2_host, dd, size_t(m) * k * sizeof(float), cudaMemcpyDeviceToHost, s);
  }
  freeAll(ws, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  return rc == EBG_OK ? ebg_cloud_check_status(c, stream) : rc;
}

ebg_status ebg_cloud_check_status(const ebg_cloud* c, void* stream)
{
  if (c == nullptr) {
    return setError(EBG_ERR_INVALID, "null cloud");
  }
  DeviceGuard  guard;
  cudaSetDevice(c->device);
  cudaStream_t s  = static_cast<cudaStream_t>(stream);
  int          st = 0;
  if (cudaMemcpyAsync(&st, c->dStatus, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  if (st != 0) {
    cudaMemsetAsync(c->dStatus, 0, sizeof(int), s);
    if (st & ST_INPUT) {
      return setError(EBG_ERR_INVALID, "point index out of range in a self k-NN query");
    }
    return setError(EBG_ERR_TRAVERSAL, "k-NN traversal stopped early (status " + std::to_string(st) + ")");
  }
  return EBG_OK;
}

} // extern "C"
