// Device build of a mesh's Morton 4-wide BVH, leaf-ordered records and oriented boxes.
#ifndef EBG_MESH_BUILD_GPU_H
#define EBG_MESH_BUILD_GPU_H

#include <cstdint>

#include <cuda_runtime.h>

#include "capi_internal.h"

namespace ebg {

// Builds the tree and every device array of m (nodes, records, oriented boxes, DCEL normals) from
// the soup (V, F on the host) and m's pseudonormals (m->triN, cornerVN, edgeN, soup order; with
// normalsOnDevice they are computed here and copied into those vectors); fills
// m->areaCdf and m->info's num_nodes / num_leaves / depth, m->view's root reference, and the
// triangles' bounding box (outLo / outHi).  Synchronous on s.
ebg_status buildMeshOnDevice(ebg_mesh* m, const double* V, int64_t nv, const int32_t* F, int64_t nt, int leafSize,
                             double* outLo, double* outHi, cudaStream_t s, bool normalsOnDevice = false);

// The pseudonormals of the soup (device arrays dV, dF; outputs per triangle in soup order: the
// Triangle normal 3, corner vertex normals 9, edge normals 9), bit-identical to
// computePseudonormals (normals_gpu.cu).  Synchronous on s.
ebg_status pseudonormalsOnDevice(const double* dV, int64_t nv, const int32_t* dF, int64_t nt, double* dTriN,
                                 double* dCornerVN, double* dEdgeN, cudaStream_t s);

} // namespace ebg

#endif
