// Device build of a mesh's Morton 4-wide BVH, leaf-ordered records and oriented boxes.
#ifndef EBG_MESH_BUILD_GPU_H
#define EBG_MESH_BUILD_GPU_H

#include <cstdint>

#include <cuda_runtime.h>

#include "capi_internal.h"

namespace ebg {

// Builds the tree (build: EBG_BUILD_MORTON or EBG_BUILD_SAH, the host build's tree in either case)
// and every device array of m (nodes, records, oriented boxes, DCEL normals) from the soup (V, F on
// the host) and m's pseudonormals (m->triN, cornerVN, edgeN, soup order; with normalsOnDevice they
// are computed here instead, and the records are their only copy); fills m->areaCdf and m->info's
// num_nodes / num_leaves / depth, m->view's root reference, and the triangles' bounding box (outLo /
// outHi).  Synchronous on s.
ebg_status buildMeshOnDevice(ebg_mesh* m, const double* V, int64_t nv, const int32_t* F, int64_t nt, int build,
                             int leafSize, double* outLo, double* outHi, cudaStream_t s, bool normalsOnDevice = false);

// Refits m to moved vertices (same count, same triangles; V on the host, or on the device with
// vOnDevice): the pseudonormals, every triangle record, every leaf's and node's oriented box and
// every node's child boxes are recomputed on the device; the tree's topology and the triangles'
// leaf order stay.  Returns the moved triangles' bounding box.  Synchronous on s; on an error
// before the first device write (non-finite or degenerate geometry) m is unchanged.
ebg_status refitMeshOnDevice(ebg_mesh* m, const double* V, bool vOnDevice, int64_t nv, double* outLo, double* outHi,
                             cudaStream_t s);

// The normals held in m's FP64 records, in soup order: out = face normals (3n), corner vertex
// normals (9n), edge normals (9n).  Asynchronous on s.
void launchGatherNormals(const double* tri64, const int32_t* triId, int64_t n, double* out, cudaStream_t s);

// The pseudonormals of the soup (device arrays dV, dF; outputs per triangle in soup order: the
// Triangle normal 3, corner vertex normals 9, edge normals 9), bit-identical to
// computePseudonormals (normals_gpu.cu).  Synchronous on s.
ebg_status pseudonormalsOnDevice(const double* dV, int64_t nv, const int32_t* dF, int64_t nt, double* dTriN,
                                 double* dCornerVN, double* dEdgeN, cudaStream_t s);

} // namespace ebg

#endif
