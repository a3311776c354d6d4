// CSG union scene: device view and launch wrapper.
#ifndef EBG_SCENE_KERNELS_H
#define EBG_SCENE_KERNELS_H

#include <cstdint>
#include <cuda_runtime.h>

#include "ebg_layout.h"

namespace ebg {

// One object of the union.  kind 0: sphere (centre t, radius); kind 1: mesh instance whose value
// at p is mesh(R (p - t)), R the row-major 3x3 rotation of RotateIF's point map.
struct alignas(16) SceneObject
{
  int32_t kind;
  int32_t mesh;
  float   radius;
  float   pad;
  float   t[3];
  float   R[9];
};

// The same object in FP64 for the near-surface pass, as the reference evaluates it:
// TranslateIF(RotateIF(mesh)).value(p) = mesh(rot(p - t)) with RotateIF's per-axis formulas and
// cos / sin of the angle in double (TransformImplem.hpp:152-225); a sphere is |p - t| - radius.
struct alignas(16) SceneObject64
{
  double  t[3];
  double  c, s;   // cos and sin of the rotation angle
  double  radius;
  int32_t kind;   // 0 sphere, 1 mesh instance
  int32_t axis;   // rotation axis 0, 1, 2
};

// One batch of a batched call: n points (xyz) and n results, device memory.
struct SceneBatch
{
  const float* points;
  int64_t      n;
  float*       out;
};

struct SceneView
{
  const EbgNode4*      nodes;     // object BVH (root at 0 unless root_ref is a leaf)
  const SceneObject*   objects;   // in BVH leaf order
  const SceneObject64* objects64; // the same objects in FP64
  const EbgMeshView*   meshes;
  float              root_lo[3], root_hi[3];
  uint32_t           root_ref, root_count;
  float              morton_lo[3], morton_scale[3];
};

struct SceneQueryArgs
{
  SceneView           scene;
  const float*        points;      // one batch: the caller's xyz (n x 3) ...
  float*              out;         // ... and results
  const SceneBatch*   batches;     // several batches (non-null): point g of the call is point
  const int64_t*      batch_start; // g - batch_start[b] of the last batch b with batch_start[b] <= g
  int32_t             num_batches;
  const uint32_t*     order;       // sorted position -> point of the call (nullptr = identity)
  int64_t             n;           // points of the call
  float               band;        // |value| <= band -> FP64 re-evaluation
  uint8_t*            band_flag;   // per sorted position (nullable = no band pass)
  const uint32_t*     band_list;   // sorted positions needing FP64 (compacted from band_flag)
  const uint32_t*     band_count;
  unsigned long long* work;
  int                 chunk;       // packets taken from the work counter at a time (0, 1: one)
  int*                status;
};

// Point g of a call (one batch or several) and where its result goes.
__device__ __forceinline__ const float* scenePoint(const SceneQueryArgs& a, uint32_t g, float** out)
{
  if (a.batches == nullptr) {
    *out = a.out + g;
    return a.points + 3 * size_t(g);
  }
  int lo = 0, hi = a.num_batches - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.batch_start[mid] <= int64_t(g)) {
      lo = mid;
    }
    else {
      hi = mid - 1;
    }
  }
  const int64_t i = int64_t(g) - a.batch_start[lo];
  *out            = a.batches[lo].out + i;
  return a.batches[lo].points + 3 * i;
}

int         sceneOuterDepth();
cudaError_t launchSceneValue(const SceneQueryArgs& a, int numSms, cudaStream_t s);
// FP64 re-evaluation of the band list (reads band_count on the device); delta bounds the FP32
// error of the union's value.
cudaError_t launchSceneBand64(const SceneQueryArgs& a, float delta, int numSms, cudaStream_t s);
// Sort keys of a batched call: the 30-bit Morton code of every point of every batch, and the
// identity.
cudaError_t launchSceneBatchKeys(const SceneQueryArgs& a, uint32_t* keys, uint32_t* ids, cudaStream_t s);
// batch_start[b] = sum of the first b batches' n, batch_start[nb] = the total (one small launch).
cudaError_t launchSceneBatchStarts(const SceneBatch* batches, int32_t nb, int64_t* start, int* status,
                                   int64_t expectTotal, cudaStream_t s);

} // namespace ebg

#endif
