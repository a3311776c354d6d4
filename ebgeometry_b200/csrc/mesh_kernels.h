// Launch wrappers of the mesh kernels (called from the C ABI layer).
#ifndef EBG_MESH_KERNELS_H
#define EBG_MESH_KERNELS_H

#include <cstdint>
#include <cuda_runtime.h>

#include "cells_kernels.h"
#include "ebg_layout.h"

namespace ebg {

struct MeshQueryArgs
{
  EbgMeshView        mesh;
  const float*       points;     // caller's xyz (n x 3)
  const double*      points64;   // the caller's FP64 xyz when it passed FP64 (nullable)
  const uint32_t*    order;      // sorted position -> caller index (nullptr = identity)
  const float*       hint;       // per query (caller order): radius upper bound (nullptr = none)
  int64_t            n;
  float*             out_d;      // caller order
  double*            out_d64;    // caller order, FP64 results of the band pass (nullable)
  int                eval;       // FP64 evaluator: 0 the Triangle test (TriMeshSDF), 1 the DCEL face (MeshSDF)
  int32_t*           out_tri;    // caller order (nullable)
  int                tri_leaf;   // 1: out_tri gets the leaf-order triangle (the device records' index)
  float              band;       // |d| <= band -> FP64 re-evaluation list
  uint32_t*          band_list;  // sorted positions needing FP64 (nullable = no band pass)
  uint32_t*          band_count;
  float*             band_d32;   // FP32 distance of each band entry (nullable: read out_d instead)
  uint8_t*           band_flag;  // per sorted position, 1 = needs FP64 (nullable: the traversal
                                 // appends to band_list itself, in completion order)
  unsigned long long* work;      // packet counter (zeroed before the launch)
  int                chunk;      // packets taken from the counter at a time (0, 1: one)
  int*               status;     // device status word (ST_* bits)
  unsigned long long* stats;     // 15 counters (nullable): 6 per query, 6 per packet, 2 of the cuts,
                                 // [14] triangle records of the leaves the warps opened
  SeedCellsView      cells;      // per-cell entry cuts (used when cells.count is non-null)
  uint32_t           top_nodes;  // nodes [0, top_nodes) and their oriented boxes are read from a copy
                                 // in each block's shared memory (0: none)
  int                node_width; // 8: mesh.nodes / mesh.node_obb are the 8-wide copy (EbgNode8; plain
                                 // and hinted queries, no top nodes); else the 4-wide tree
};

// Morton keys of the query points (30 bits) and the identity permutation.
void launchQueryKeys(const float* points, int64_t n, const float* lo, const float* scale, uint32_t* keys,
                     uint32_t* ids, cudaStream_t s);

// FP32 packet traversal.  warpsPerBlock in {1,2,4,8}; occupancy 0..3 (see ebg_query_opts).
cudaError_t launchMeshSdf32(const MeshQueryArgs& a, int warpsPerBlock, int numSms, cudaStream_t s, int occupancy = 0);

// FP64 re-evaluation of the band list (reads band_count on the device).
cudaError_t launchMeshBand64(const MeshQueryArgs& a, float delta, int numSms, cudaStream_t s);

// FlatMeshSDF over every triangle (FP64 points and results, DCEL face algorithm); outTri nullable;
// non-finite points set ST_INPUT in *status and get NaN.
cudaError_t launchMeshFlat64(const EbgMeshView& m, int64_t numTris, const double* pts, int64_t n, double* out,
                             int32_t* outTri, int* status, int numSms, cudaStream_t s);

// out[i] = float(in[i]) for i < count (round to nearest).
void launchDoubleToFloat(const double* in, float* out, int64_t count, cudaStream_t s);

} // namespace ebg

#endif
