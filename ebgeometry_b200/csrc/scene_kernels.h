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

struct SceneView
{
  const EbgNode4*    nodes;   // object BVH (root at 0 unless root_ref is a leaf)
  const SceneObject* objects; // in BVH leaf order
  const EbgMeshView* meshes;
  float              root_lo[3], root_hi[3];
  uint32_t           root_ref, root_count;
  float              morton_lo[3], morton_scale[3];
};

struct SceneQueryArgs
{
  SceneView           scene;
  const float*        points;
  const uint32_t*     order;
  int64_t             n;
  float*              out;
  unsigned long long* work;
  int*                status;
};

int         sceneOuterDepth();
cudaError_t launchSceneValue(const SceneQueryArgs& a, int numSms, cudaStream_t s);

} // namespace ebg

#endif
