// C ABI of the CSG union: BVHUnion over spheres and posed mesh instances, batched queries.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <cuda_runtime.h>
#include <thrust/iterator/counting_iterator.h>

#include "capi_common.h"
#include "capi_internal.h"
#include "mesh_host.h"
#include "mesh_kernels.h"
#include "scene_kernels.h"

using namespace ebg;

struct ebg_scene
{
  int       device  = 0;
  int       numSms  = 148;
  SceneView view{};
  void*     dNodes   = nullptr;
  void*     dObjects = nullptr;
  void*     dObjects64 = nullptr;
  void*     dMeshes  = nullptr;
  int*      dStatus  = nullptr;
  int64_t   numObjects = 0;
  int       depth      = 0;
  double    diagonal   = 0.0; // of the scene's box
  double    errScale   = 0.0; // what the FP32 union value's rounding errors scale with (see below)
  int       tunedChunk = 0;   // work-queue chunk chosen by ebg_scene_autotune (0 = one packet)
};

namespace {

// RotateIF's point map as a matrix (TransformImplem.hpp:163-225): angle in degrees about one axis,
// local = R p.
void rotationMatrix(double angleDeg, int axis, double R[9])
{
  const double th = angleDeg * 3.14159265358979323846 / 180.0;
  const double c = std::cos(th), s = std::sin(th);
  const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  std::memcpy(R, I, sizeof(I));
  if (axis == 0) {
    R[4] = c;
    R[5] = s;
    R[7] = -s;
    R[8] = c;
  }
  else if (axis == 1) {
    R[0] = c;
    R[2] = -s;
    R[6] = s;
    R[8] = c;
  }
  else {
    R[0] = c;
    R[1] = s;
    R[3] = -s;
    R[4] = c;
  }
}

// The union query of one batch (points/out) or of several (batches), asynchronous on the stream:
// ordering, the FP32 pass, the band compaction and the FP64 pass.
ebg_status sceneQuery(const ebg_scene*      s,
                      const float*          points,
                      float*                out,
                      const SceneBatch*     batches,
                      int32_t               nb,
                      int64_t               n,
                      const ebg_query_opts* opts,
                      void*                 stream)
{
  if (n > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 points per call");
  }
  if (n == 0) {
    return EBG_OK;
  }
  DeviceGuard  guard;
  cudaSetDevice(s->device);
  cudaStream_t st     = static_cast<cudaStream_t>(stream);
  const bool   sort   = !(opts && opts->no_sort);
  const bool   band64 = !(opts && opts->no_fp64_band);
  std::vector<void*> ws;
  bool ok  = true;
  auto get = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (!ok || cudaMallocAsync(&p, std::max<size_t>(bytes, 16), st) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    ws.push_back(p);
    return p;
  };
  auto release = [&]() {
    for (void* p : ws) {
      cudaFreeAsync(p, st);
    }
  };
  SceneQueryArgs a{};
  a.scene       = s->view;
  a.points      = points;
  a.out         = out;
  a.batches     = batches;
  a.num_batches = nb;
  a.n           = n;
  a.status      = s->dStatus;
  a.band        = float((opts && opts->band > 0) ? opts->band : 1e-4 * s->errScale);
  auto* counters = static_cast<unsigned long long*>(get(2 * sizeof(unsigned long long))); // work, band count
  int64_t* starts = batches ? static_cast<int64_t*>(get(size_t(nb + 1) * sizeof(int64_t))) : nullptr;
  uint32_t* order = nullptr;
  if (sort) {
    order      = static_cast<uint32_t*>(get(n * 4));
    auto* iin  = static_cast<uint32_t*>(get(n * 4));
    size_t tb  = 0;
    if (batches) {
      auto* kin  = static_cast<uint32_t*>(get(n * 4));
      auto* kout = static_cast<uint32_t*>(get(n * 4));
      cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, iin, order, int(n), 0, 30, st);
      void* tmp = get(tb);
      if (!ok) {
        release();
        return setError(EBG_ERR_NO_MEMORY, "scene query workspace");
      }
      a.batch_start = starts;
      if (launchSceneBatchStarts(batches, nb, starts, s->dStatus, n, st) != cudaSuccess ||
          launchSceneBatchKeys(a, kin, iin, st) != cudaSuccess ||
          cub::DeviceRadixSort::SortPairs(tmp, tb, kin, kout, iin, order, int(n), 0, 30, st) != cudaSuccess) {
        release();
        return setError(EBG_ERR_CUDA, std::string("scene batch ordering: ") + cudaGetErrorString(cudaGetLastError()));
      }
    }
    else {
      auto* kin  = static_cast<uint32_t*>(get(n * 4));
      auto* kout = static_cast<uint32_t*>(get(n * 4));
      cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, iin, order, int(n), 0, 30, st);
      void* tmp = get(tb);
      if (!ok) {
        release();
        return setError(EBG_ERR_NO_MEMORY, "scene query workspace");
      }
      launchQueryKeys(points, n, s->view.morton_lo, s->view.morton_scale, kin, iin, st);
      if (cub::DeviceRadixSort::SortPairs(tmp, tb, kin, kout, iin, order, int(n), 0, 30, st) != cudaSuccess) {
        release();
        return setError(EBG_ERR_CUDA, "scene query sort failed");
      }
    }
  }
  else if (batches) {
    if (!ok) {
      release();
      return setError(EBG_ERR_NO_MEMORY, "scene query workspace");
    }
    a.batch_start = starts;
    if (launchSceneBatchStarts(batches, nb, starts, s->dStatus, n, st) != cudaSuccess) {
      release();
      return setError(EBG_ERR_CUDA, "scene batch starts launch failed");
    }
  }
  uint8_t*  flags    = band64 ? static_cast<uint8_t*>(get(size_t(n))) : nullptr;
  uint32_t* bandList = band64 ? static_cast<uint32_t*>(get(size_t(n) * 4)) : nullptr;
  size_t    selBytes = 0;
  void*     selTemp  = nullptr;
  auto*     bandCnt  = counters ? reinterpret_cast<uint32_t*>(counters + 1) : nullptr;
  if (band64 && ok) {
    cub::DeviceSelect::Flagged(nullptr, selBytes, thrust::counting_iterator<uint32_t>(0u), flags, bandList, bandCnt,
                               int(n), st);
    selTemp = get(selBytes);
  }
  if (!ok) {
    release();
    return setError(EBG_ERR_NO_MEMORY, "scene query workspace");
  }
  cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), st);
  a.order      = order;
  a.work       = counters;
  a.chunk      = (opts && opts->queue_chunk > 0) ? opts->queue_chunk : (s->tunedChunk > 0 ? s->tunedChunk : 1);
  a.band_flag  = flags;
  a.band_list  = bandList;
  a.band_count = bandCnt;
  cudaError_t e = launchSceneValue(a, s->numSms, st);
  if (e == cudaSuccess && band64) {
    if (cub::DeviceSelect::Flagged(selTemp, selBytes, thrust::counting_iterator<uint32_t>(0u), flags, bandList,
                                   bandCnt, int(n), st) != cudaSuccess) {
      e = cudaGetLastError();
      e = e == cudaSuccess ? cudaErrorUnknown : e;
    }
    else {
      // delta bounds the FP32 error of the union's value: the instance transform and the mesh distance
      e = launchSceneBand64(a, float(4e-6 * s->errScale) + 1e-30f, s->numSms, st);
    }
  }
  release();
  if (e != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("scene launch failed: ") + cudaGetErrorString(e));
  }
  return EBG_OK;
}

} // namespace

extern "C" {

ebg_status ebg_scene_create(int64_t                num_spheres,
                            const double*          spheres,
                            int64_t                num_meshes,
                            const ebg_mesh* const* meshes,
                            const double*          poses,
                            const ebg_build_opts*  opts,
                            ebg_scene**            out)
{
  if (out == nullptr) {
    return setError(EBG_ERR_INVALID, "out handle pointer is null");
  }
  *out = nullptr;
  if (num_spheres < 0 || num_meshes < 0 || num_spheres + num_meshes < 1 || (num_spheres > 0 && !spheres) ||
      (num_meshes > 0 && (!meshes || !poses))) {
    return setError(EBG_ERR_INVALID, "a scene needs at least one object and non-null arrays");
  }
  int device = -1;
  for (int64_t m = 0; m < num_meshes; m++) {
    if (meshes[m] == nullptr) {
      return setError(EBG_ERR_INVALID, "null mesh handle");
    }
    if (device >= 0 && meshes[m]->device != device) {
      return setError(EBG_ERR_INVALID, "all meshes of a scene must live on one device");
    }
    device = meshes[m]->device;
    const int axis = int(poses[5 * m + 1]);
    if (axis < 0 || axis > 2 || !std::isfinite(poses[5 * m])) {
      return setError(EBG_ERR_INVALID, "pose: rotation axis must be 0, 1 or 2 and the angle finite");
    }
  }
  for (int64_t i = 0; i < 4 * num_spheres; i++) {
    if (!std::isfinite(spheres[i])) {
      return setError(EBG_ERR_INVALID, "non-finite sphere parameter");
    }
  }
  DeviceGuard guard;
  if (device < 0) {
    device = (opts && opts->device >= 0) ? opts->device : -1;
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) {
      return setError(EBG_ERR_NOT_FOUND, "no CUDA device");
    }
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    return setError(EBG_ERR_NOT_FOUND, "cannot select CUDA device");
  }
  keepPoolMemory();
  const int64_t            no = num_spheres + num_meshes;
  std::vector<SceneObject> objs(no);
  std::vector<SceneObject64> objs64(no);
  std::vector<double>      lo(3 * no), hi(3 * no), cen(3 * no);
  for (int64_t i = 0; i < num_spheres; i++) {
    const double* s = spheres + 4 * i;
    SceneObject&  o = objs[i];
    std::memset(&o, 0, sizeof(o));
    o.kind   = 0;
    o.radius = float(s[3]);
    SceneObject64& o64 = objs64[i];
    std::memset(&o64, 0, sizeof(o64));
    o64.kind   = 0;
    o64.radius = s[3];
    for (int a = 0; a < 3; a++) {
      o64.t[a]          = s[a];
      o.t[a]            = float(s[a]);
      lo[3 * i + a]     = s[a] - std::fabs(s[3]);
      hi[3 * i + a]     = s[a] + std::fabs(s[3]);
      cen[3 * i + a]    = s[a];
    }
  }
  std::vector<EbgMeshView> views(std::max<int64_t>(num_meshes, 1));
  for (int64_t m = 0; m < num_meshes; m++) {
    const int64_t i = num_spheres + m;
    SceneObject&  o = objs[i];
    std::memset(&o, 0, sizeof(o));
    o.kind = 1;
    o.mesh = int32_t(m);
    double R[9];
    rotationMatrix(poses[5 * m], int(poses[5 * m + 1]), R);
    for (int k = 0; k < 9; k++) {
      o.R[k] = float(R[k]);
    }
    SceneObject64& o64 = objs64[i];
    std::memset(&o64, 0, sizeof(o64));
    o64.kind = 1;
    o64.axis = int32_t(poses[5 * m + 1]);
    // RotateIF's cosine and sine (TransformImplem.hpp:164-181): theta = angle * pi / 180
    const double theta = poses[5 * m] * 3.14159265358979323846 / 180.0;
    o64.c              = std::cos(theta);
    o64.s              = std::sin(theta);
    for (int a = 0; a < 3; a++) {
      o.t[a]   = float(poses[5 * m + 2 + a]);
      o64.t[a] = poses[5 * m + 2 + a];
    }
    views[m] = meshes[m]->view;
    // world box: the 8 corners of the local box mapped back (p = R^T local + t), grown by the
    // float rounding of the instance transform
    const ebg_mesh_info& inf = meshes[m]->info;
    double               wl[3] = {1e300, 1e300, 1e300}, wh[3] = {-1e300, -1e300, -1e300};
    for (int c = 0; c < 8; c++) {
      const double L[3] = {(c & 1) ? inf.hi[0] : inf.lo[0], (c & 2) ? inf.hi[1] : inf.lo[1],
                           (c & 4) ? inf.hi[2] : inf.lo[2]};
      for (int a = 0; a < 3; a++) {
        const double w = R[0 + a] * L[0] + R[3 + a] * L[1] + R[6 + a] * L[2] + poses[5 * m + 2 + a];
        wl[a]          = std::min(wl[a], w);
        wh[a]          = std::max(wh[a], w);
      }
    }
    for (int a = 0; a < 3; a++) {
      const double g   = 1e-5 * (std::fabs(wl[a]) + std::fabs(wh[a]) + inf.diagonal);
      lo[3 * i + a]    = wl[a] - g;
      hi[3 * i + a]    = wh[a] + g;
      cen[3 * i + a]   = 0.5 * (wl[a] + wh[a]);
    }
  }
  Bvh4        bvh;
  std::string msg;
  const int   leaf = (opts && opts->leaf_size > 0) ? opts->leaf_size : 3;
  if (!buildBvh4(lo, hi, cen, EBG_BUILD_SAH, leaf, bvh, msg)) {
    return setError(EBG_ERR_INVALID, msg);
  }
  if (3 * bvh.depth + 4 > sceneOuterDepth()) {
    return setError(EBG_ERR_TOO_LARGE, "object hierarchy too deep for the traversal stack");
  }
  std::vector<SceneObject> ordered(no);
  std::vector<SceneObject64> ordered64(no);
  for (int64_t i = 0; i < no; i++) {
    ordered[i]   = objs[bvh.order[i]];
    ordered64[i] = objs64[bvh.order[i]];
  }
  auto* s      = new ebg_scene;
  s->device    = device;
  s->numObjects = no;
  s->depth     = bvh.depth;
  cudaDeviceGetAttribute(&s->numSms, cudaDevAttrMultiProcessorCount, device);
  auto up = [](void** dst, const void* src, size_t bytes) {
    return cudaMalloc(dst, std::max<size_t>(bytes, 16)) == cudaSuccess &&
           (bytes == 0 || cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess);
  };
  if (!up(&s->dNodes, bvh.nodes.data(), bvh.nodes.size() * sizeof(EbgNode4)) ||
      !up(&s->dObjects, ordered.data(), no * sizeof(SceneObject)) ||
      !up(&s->dObjects64, ordered64.data(), no * sizeof(SceneObject64)) ||
      !up(&s->dMeshes, views.data(), views.size() * sizeof(EbgMeshView)) ||
      cudaMalloc(reinterpret_cast<void**>(&s->dStatus), sizeof(int)) != cudaSuccess ||
      cudaMemset(s->dStatus, 0, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    ebg_scene_destroy(s);
    return setError(EBG_ERR_NO_MEMORY, "scene upload");
  }
  SceneView& v = s->view;
  v.nodes      = static_cast<const EbgNode4*>(s->dNodes);
  v.objects    = static_cast<const SceneObject*>(s->dObjects);
  v.objects64  = static_cast<const SceneObject64*>(s->dObjects64);
  v.meshes     = static_cast<const EbgMeshView*>(s->dMeshes);
  v.root_ref   = bvh.rootRef;
  v.root_count = bvh.rootCount;
  s->diagonal = std::sqrt((bvh.hi[0] - bvh.lo[0]) * (bvh.hi[0] - bvh.lo[0]) +
                          (bvh.hi[1] - bvh.lo[1]) * (bvh.hi[1] - bvh.lo[1]) +
                          (bvh.hi[2] - bvh.lo[2]) * (bvh.hi[2] - bvh.lo[2]));
  // the scene's diagonal, or the magnitude of its world coordinates or of any mesh's local ones
  // when those are larger (FP32 rounds coordinates relative to their magnitude)
  s->errScale = s->diagonal;
  for (int a = 0; a < 3; a++) {
    s->errScale = std::max(s->errScale, std::max(std::fabs(bvh.lo[a]), std::fabs(bvh.hi[a])));
  }
  for (int64_t m = 0; m < num_meshes; m++) {
    s->errScale = std::max(s->errScale, fp32ErrorScale(meshes[m]));
  }
  for (int a = 0; a < 3; a++) {
    v.root_lo[a]      = roundDown(bvh.lo[a]);
    v.root_hi[a]      = roundUp(bvh.hi[a]);
    const double c    = 0.5 * (bvh.lo[a] + bvh.hi[a]);
    const double ext  = std::max(bvh.hi[a] - bvh.lo[a], 1e-30);
    v.morton_lo[a]    = float(c - ext);
    v.morton_scale[a] = float(1024.0 / (2.0 * ext));
  }
  *out = s;
  return EBG_OK;
}

ebg_status ebg_scene_destroy(ebg_scene* s)
{
  if (s == nullptr) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(s->device);
  cudaFree(s->dNodes);
  cudaFree(s->dObjects);
  cudaFree(s->dObjects64);
  cudaFree(s->dMeshes);
  cudaFree(s->dStatus);
  delete s;
  return EBG_OK;
}

ebg_status ebg_scene_value(const ebg_scene*      s,
                           const float*          points_dev,
                           int64_t               n,
                           float*                out_dev,
                           const ebg_query_opts* opts,
                           void*                 stream)
{
  if (s == nullptr || n < 0 || (n > 0 && (!points_dev || !out_dev))) {
    return setError(EBG_ERR_INVALID, "null scene/buffer or negative count");
  }
  return sceneQuery(s, points_dev, out_dev, nullptr, 0, n, opts, stream);
}

ebg_status ebg_scene_eval_batches(const ebg_scene*      s,
                                  const ebg_batch*      batches_dev,
                                  int32_t               num_batches,
                                  int64_t               total_points,
                                  const ebg_query_opts* opts,
                                  void*                 stream)
{
  if (s == nullptr || num_batches < 0 || total_points < 0 || (num_batches > 0 && batches_dev == nullptr)) {
    return setError(EBG_ERR_INVALID, "null scene/batches or negative count");
  }
  if (num_batches > (1 << 24)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^24 batches per call");
  }
  if (num_batches == 0 || total_points == 0) {
    return EBG_OK;
  }
  static_assert(sizeof(ebg_batch) == sizeof(SceneBatch), "ebg_batch and SceneBatch must match");
  return sceneQuery(s, nullptr, nullptr, reinterpret_cast<const SceneBatch*>(batches_dev), num_batches, total_points,
                    opts, stream);
}

ebg_status ebg_scene_value_host(const ebg_scene*      s,
                                const float*          points_host,
                                int64_t               n,
                                float*                out_host,
                                const ebg_query_opts* opts,
                                void*                 stream)
{
  if (s == nullptr || n < 0 || (n > 0 && (!points_host || !out_host))) {
    return setError(EBG_ERR_INVALID, "null scene/buffer or negative count");
  }
  if (n == 0) {
    return EBG_OK;
  }
  if (!allFinite(points_host, 3 * n)) {
    return setError(EBG_ERR_INVALID, "non-finite query coordinate");
  }
  DeviceGuard  guard;
  cudaSetDevice(s->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float*       dp = nullptr;
  float*       dd = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&dp), size_t(n) * 12, st) != cudaSuccess ||
      cudaMallocAsync(reinterpret_cast<void**>(&dd), size_t(n) * 4, st) != cudaSuccess) {
    cudaGetLastError();
    return setError(EBG_ERR_NO_MEMORY, "device buffers for the host scene call");
  }
  cudaMemsetAsync(s->dStatus, 0, sizeof(int), st);
  cudaMemcpyAsync(dp, points_host, size_t(n) * 12, cudaMemcpyHostToDevice, st);
  ebg_status rc = ebg_scene_value(s, dp, n, dd, opts, stream);
  if (rc == EBG_OK) {
    cudaMemcpyAsync(out_host, dd, size_t(n) * 4, cudaMemcpyDeviceToHost, st);
  }
  cudaFreeAsync(dp, st);
  cudaFreeAsync(dd, st);
  if (rc != EBG_OK) {
    return rc;
  }
  return ebg_scene_check_status(s, stream);
}

ebg_status ebg_scene_check_status(const ebg_scene* s, void* stream)
{
  if (s == nullptr) {
    return setError(EBG_ERR_INVALID, "null scene");
  }
  DeviceGuard  guard;
  cudaSetDevice(s->device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int          v  = 0;
  if (cudaMemcpyAsync(&v, s->dStatus, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  if (v != 0) {
    cudaMemsetAsync(s->dStatus, 0, sizeof(int), st);
    return setError(EBG_ERR_TRAVERSAL, "scene traversal stopped early (status " + std::to_string(v) + ")");
  }
  return EBG_OK;
}

int64_t ebg_scene_num_objects(const ebg_scene* s) { return s ? s->numObjects : 0; }

ebg_status ebg_scene_autotune(ebg_scene*   s,
                              const float* sample_points_dev,
                              int64_t      n,
                              int32_t*     best_queue_chunk,
                              float*       best_ms,
                              void*        stream)
{
  if (s == nullptr || sample_points_dev == nullptr || n < 32) {
    return setError(EBG_ERR_INVALID, "scene autotune needs a scene and at least 32 sample points");
  }
  DeviceGuard guard;
  cudaSetDevice(s->device);
  cudaStream_t st  = static_cast<cudaStream_t>(stream);
  float*       out = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&out), size_t(n) * sizeof(float), st) != cudaSuccess) {
    cudaGetLastError();
    return setError(EBG_ERR_NO_MEMORY, "scene autotune output buffer");
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float      bestMs = INFINITY;
  int        bestC  = 1;
  ebg_status rc     = EBG_OK;
  for (int c : {1, 2, 4, 8}) {
    ebg_query_opts q{};
    q.queue_chunk = c;
    float ms      = INFINITY;
    for (int rep = 0; rep < 3 && rc == EBG_OK; rep++) { // the first run warms caches and the pool
      cudaEventRecord(e0, st);
      rc = sceneQuery(s, sample_points_dev, out, nullptr, 0, n, &q, stream);
      cudaEventRecord(e1, st);
      if (rc == EBG_OK && cudaEventSynchronize(e1) != cudaSuccess) {
        rc = setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
      }
      float t = 0.f;
      if (rc == EBG_OK && rep > 0 && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess) {
        ms = std::min(ms, t);
      }
    }
    if (ms < bestMs) {
      bestMs = ms;
      bestC  = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(out, st);
  cudaStreamSynchronize(st);
  if (rc != EBG_OK) {
    return rc;
  }
  s->tunedChunk = bestC;
  if (best_queue_chunk) {
    *best_queue_chunk = bestC;
  }
  if (best_ms) {
    *best_ms = bestMs;
  }
  return EBG_OK;
}

} // extern "C"
