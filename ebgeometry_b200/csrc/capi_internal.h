// Internal handle layouts shared by the C ABI translation units.
#ifndef EBG_CAPI_INTERNAL_H
#define EBG_CAPI_INTERNAL_H

#include <cmath>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "cells_kernels.h"
#include "ebg_layout.h"
#include "ebgeometry_b200.h"
#include "seed_kernels.h"

struct ebg_mesh
{
  int           device = 0;
  int           numSms = 148;
  EbgMeshView   view{};
  ebg_mesh_info info{};
  // device allocations
  void* dNodes  = nullptr;
  void* dHot    = nullptr;
  void* dSign   = nullptr;
  void* dTri64  = nullptr;
  void* dTriId  = nullptr;
  void* dObb    = nullptr;
  void* dNodeObb = nullptr;
  void* dDcelN   = nullptr;
  int*  dStatus = nullptr;
  // kept for refitting moved vertices: the soup's triangles, and each leaf's and each interior
  // node's range of leaf positions
  int32_t*  dF         = nullptr;
  uint32_t* dLeafFirst = nullptr;
  uint32_t* dLeafCount = nullptr;
  uint32_t* dNodeFirst = nullptr;
  uint32_t* dNodeEnd   = nullptr;
  // the pseudonormals (soup order) during a host build only -- afterwards they live in the FP64
  // records on the device -- and the cumulative triangle area (leaf order)
  std::vector<double> triN, cornerVN, edgeN;
  std::vector<double> areaCdf;
  // launch shape chosen by ebg_mesh_autotune (0 = library defaults)
  int tunedOccupancy = 0;
  int tunedWpb       = 0;
  int tunedChunk     = 0;
  int tunedWidth     = 0; // 8: plain queries take the 8-wide copy
  // the optional 8-wide copy of the tree (ebg_mesh_widen; plain FP32 queries): its nodes and their
  // oriented boxes, and the view the traversal reads them through (the 4-wide view with nodes,
  // node_obb and root replaced); a refit drops it
  bool        hasWide   = false;
  void*       dNodes8   = nullptr;
  void*       dNodeObb8 = nullptr;
  EbgMeshView view8{};
  int64_t     numNodes8 = 0;
  int32_t     depth8    = 0;
  // per-cell entry cuts built by ebg_seed_attach from `cellsSeed` (queries passing that model use
  // them); a refit drops them
  const ebg_seed*    cellsSeed    = nullptr;
  float4*            dCellEntries = nullptr;
  uint32_t*          dCellCount   = nullptr;
  float*             dCellRadius  = nullptr;
  int32_t*           dCellAnchor  = nullptr;
  ebg::SeedCellsView cellsView{};
  ebg_attach_report  cellsReport{};
};

struct ebg_seed
{
  int            device = 0;
  int            numSms = 148;
  ebg::SeedView  view{};
  int64_t        tableSize = 0; // L * T * 2 features
  float*         tableF32  = nullptr;
  __nv_bfloat16* tableBf16 = nullptr;
  float*         tableGrad = nullptr;
  float*         tableM    = nullptr;
  float*         tableV    = nullptr;
  float*         params    = nullptr;
  float*         paramGrad = nullptr;
  float*         paramM    = nullptr;
  float*         paramV    = nullptr;
  ebg_seed_report report{};
};

namespace ebg {

// Frees a mesh's entry cuts (if any) and forgets the model they came from.
void dropCells(ebg_mesh* m);

// Frees a mesh's 8-wide copy of the tree (if any); plain queries go back to the 4-wide tree.
void dropWide(ebg_mesh* m);

// The length that the FP32 pass's rounding errors scale with: the mesh's diagonal or, for a mesh
// far from the origin, the magnitude of its coordinates (FP32 rounds coordinates relative to it).
inline double fp32ErrorScale(const ebg_mesh* m)
{
  double s = m->info.diagonal;
  for (int a = 0; a < 3; a++) {
    s = s > std::fabs(m->info.lo[a]) ? s : std::fabs(m->info.lo[a]);
    s = s > std::fabs(m->info.hi[a]) ? s : std::fabs(m->info.hi[a]);
  }
  return s;
}

// Nodes of the tree's top levels that each block of the FP32 traversal copies into shared memory
// (ebg_query_opts.top_nodes, at most MAX_TOP_NODES and the tree's node count): plain queries
// descend through them from the root; a seeded query starts below them and copies none.
constexpr int64_t MAX_TOP_NODES = 512;
inline uint32_t   topNodesFor(const ebg_mesh* m, const ebg_query_opts* opts, bool seeded)
{
  if (seeded || opts == nullptr || opts->top_nodes <= 0) {
    return 0u;
  }
  int64_t t = opts->top_nodes < MAX_TOP_NODES ? opts->top_nodes : MAX_TOP_NODES;
  t         = t < m->info.num_nodes ? t : m->info.num_nodes;
  return uint32_t(t);
}

// The mesh query pipeline (ordering, optional seed inference, FP32 traversal, FP64 band pass) on
// device buffers, asynchronous on s.  With pts64/out64 (the caller's FP64 points, of which pts is
// the FP32 rounding, and an FP64 result array) every query is re-evaluated in FP64, with the
// Triangle test (evalKind 0, TriMeshSDF) or the DCEL face algorithm (1, MeshSDF).
ebg_status meshQuery(const ebg_mesh*       m,
                     const float*          pts,
                     int64_t               n,
                     float*                outD,
                     int32_t*              outTri,
                     const ebg_query_opts* opts,
                     unsigned long long*   statsDev,
                     cudaStream_t          s,
                     const double*         pts64    = nullptr,
                     double*               out64    = nullptr,
                     int                   evalKind = 0,
                     bool                  triLeafOrder = false);

} // namespace ebg

#endif
