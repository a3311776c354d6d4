// C ABI of the CSG union: BVHUnion over spheres and posed mesh instances, batched queries.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

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
  void*     dMeshes  = nullptr;
  int*      dStatus  = nullptr;
  int64_t   numObjects = 0;
  int       depth      = 0;
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
  std::vector<double>      lo(3 * no), hi(3 * no), cen(3 * no);
  for (int64_t i = 0; i < num_spheres; i++) {
    const double* s = spheres + 4 * i;
    SceneObject&  o = objs[i];
    std::memset(&o, 0, sizeof(o));
    o.kind   = 0;
    o.radius = float(s[3]);
    for (int a = 0; a < 3; a++) {
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
    for (int a = 0; a < 3; a++) {
      o.t[a] = float(poses[5 * m + 2 + a]);
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
  for (int64_t i = 0; i < no; i++) {
    ordered[i] = objs[bvh.order[i]];
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
  v.meshes     = static_cast<const EbgMeshView*>(s->dMeshes);
  v.root_ref   = bvh.rootRef;
  v.root_count = bvh.rootCount;
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
  if (n > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 points per call");
  }
  if (n == 0) {
    return EBG_OK;
  }
  DeviceGuard  guard;
  cudaSetDevice(s->device);
  cudaStream_t st   = static_cast<cudaStream_t>(stream);
  const bool   sort = !(opts && opts->no_sort);
  std::vector<void*> ws;
  auto get = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMallocAsync(&p, std::max<size_t>(bytes, 16), st) != cudaSuccess) {
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
  uint32_t* order = nullptr;
  if (sort) {
    auto* kin  = static_cast<uint32_t*>(get(n * 4));
    auto* kout = static_cast<uint32_t*>(get(n * 4));
    auto* iin  = static_cast<uint32_t*>(get(n * 4));
    order      = static_cast<uint32_t*>(get(n * 4));
    size_t tb  = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, iin, order, int(n), 0, 30, st);
    void* tmp = get(tb);
    if (!kin || !kout || !iin || !order || !tmp) {
      release();
      return setError(EBG_ERR_NO_MEMORY, "scene query workspace");
    }
    launchQueryKeys(points_dev, n, s->view.morton_lo, s->view.morton_scale, kin, iin, st);
    cub::DeviceRadixSort::SortPairs(tmp, tb, kin, kout, iin, order, int(n), 0, 30, st);
  }
  auto* work = static_cast<unsigned long long*>(get(sizeof(unsigned long long)));
  if (!work) {
    release();
    return setError(EBG_ERR_NO_MEMORY, "scene query workspace");
  }
  cudaMemsetAsync(work, 0, sizeof(unsigned long long), st);
  SceneQueryArgs a{};
  a.scene  = s->view;
  a.points = points_dev;
  a.order  = order;
  a.n      = n;
  a.out    = out_dev;
  a.work   = work;
  a.status = s->dStatus;
  const cudaError_t e = launchSceneValue(a, s->numSms, st);
  release();
  if (e != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("scene launch failed: ") + cudaGetErrorString(e));
  }
  return EBG_OK;
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
  for (int64_t i = 0; i < 3 * n; i++) {
    if (!std::isfinite(points_host[i])) {
      return setError(EBG_ERR_INVALID, "non-finite query coordinate");
    }
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

} // extern "C"
