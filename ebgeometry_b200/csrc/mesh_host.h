// Host-side (C++) preprocessing of the mesh path: pseudonormals and the 4-wide BVH build.
#ifndef EBG_MESH_HOST_H
#define EBG_MESH_HOST_H

#include <cstdint>
#include <string>
#include <vector>

#include "ebg_layout.h"

namespace ebg {

// Face, edge and angle-weighted vertex pseudonormals of a triangle soup, as the reference's DCEL
// computes them (see mesh_host.cpp).  Outputs per triangle: triN (3), cornerVN (9), edgeN (9).
// Returns false (with msg) on a non-manifold edge shared by more than two triangles or a
// degenerate triangle.
bool computePseudonormals(const double*        V,
                          int64_t              nv,
                          const int32_t*       F,
                          int64_t              nt,
                          std::vector<double>& triN,
                          std::vector<double>& cornerVN,
                          std::vector<double>& edgeN,
                          std::string&         msg);

struct Bvh4
{
  std::vector<EbgNode4> nodes;
  std::vector<uint32_t> order; // leaf position -> primitive index
  std::vector<uint32_t> leafFirst, leafCount; // per leaf id: first position and primitive count
  std::vector<uint32_t> nodeFirst, nodeEnd;   // per interior node: its subtree's positions [first, end)
  uint32_t              rootRef   = 0;
  uint32_t              rootCount = 0;
  int                   depth     = 0;
  int64_t               numLeaves = 0;
  double                lo[3], hi[3];
};

// The DCEL quantities of a polygon soup (faces: vertex lists idx[off[f] .. off[f+1]), each of at
// least three distinct vertices), as the reference's soupToDCEL + reconcile computes them: per face
// the DCEL normal (3) and centroid (3); per corner the vertex's pseudonormal (3) and the
// pseudonormal of the edge from that corner to the next (3).  Returns false (with msg) on a face
// whose vertices span no plane or an edge shared by more than two faces.
bool computePolygonNormals(const double*        V,
                           int64_t              nv,
                           const int64_t*       off,
                           const int32_t*       idx,
                           int64_t              nf,
                           std::vector<double>& faceN,
                           std::vector<double>& centroid,
                           std::vector<double>& cornerVN,
                           std::vector<double>& edgeN,
                           std::string&         msg);

// Builds a 4-wide BVH over primitives given by FP64 boxes (lo/hi, 3 per primitive) and
// centroids.  build: 0 = binned SAH, 1 = Morton.  leafSize: max primitives per leaf.
bool buildBvh4(const std::vector<double>& boxLo,
               const std::vector<double>& boxHi,
               const std::vector<double>& centroid,
               int                        build,
               int                        leafSize,
               Bvh4&                      out,
               std::string&               msg);

// The 8-wide copy of a 4-wide tree whose root is node 0 (mesh_wide.cpp): nodes in breadth-first
// order (the root first), each with the oriented box of the 4-wide node it was made from.  depth8
// counts the levels of the deepest path, the leaf level included.  Returns false (with msg) when a
// reference is out of range or the tree is too deep for the traversal stack.
bool widenBvh8(const std::vector<EbgNode4>& n4,
               const std::vector<EbgObb>&   obb4,
               int64_t                      numTris,
               int64_t                      numLeaves,
               std::vector<EbgNode8>&       n8,
               std::vector<EbgObb>&         obb8,
               int&                         depth8,
               std::string&                 msg);

// Outward rounding of FP64 box bounds to FP32.
float roundDown(double x);
float roundUp(double x);

} // namespace ebg

#endif
