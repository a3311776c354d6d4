// Device data layout shared by the host builder (C++) and the CUDA kernels.
//
// HBM layout of one triangle mesh (all arrays 16-byte aligned, leaf order = the order the BVH
// leaves reference triangles in):
//
//   Node4   nodes[num_nodes]      128 B each = one L2 line: the boxes of the node's four children
//                                 in structure-of-arrays form (lo.x[4] lo.y[4] lo.z[4] hi.x[4]
//                                 hi.y[4] hi.z[4], FP32, rounded outward from the FP64 boxes so
//                                 that pruning with them never drops a primitive the FP64 boxes
//                                 would keep), then child[4] and count[4].
//   TriHot  tri_hot[num_tris]     48 B: v0 and the two edge vectors ab, ac in FP32 with |ab|^2,
//                                 ab.ac, |ac|^2 in the .w slots -- everything the FP32
//                                 point-triangle distance test reads.
//   TriSign tri_sign[num_tris]    96 B: FP32 face normal, 3 vertex and 3 edge pseudonormals; read
//                                 once per query, for the winning triangle's sign.
//   double  tri64[num_tris][30]   240 B: FP64 vertices, face normal, vertex and edge
//                                 pseudonormals for the near-surface re-evaluation (the
//                                 reference's TriangleSoA lane data, TriangleSoAImplem.hpp:28-70).
//   int32   tri_id[num_tris]      leaf position -> triangle index in the caller's soup.
//
//   Obb     leaf_obb[num_leaves]  64 B: oriented box of each leaf's triangles.
//   Obb     node_obb[num_nodes]   64 B: oriented box of all triangles below each interior node.
//   double  dcel_n[num_tris][3]   24 B: the DCEL face normal (the Triangle normal normalised once
//                                 more), for the DCEL face distance of MeshSDF / FlatMeshSDF.
//
// child[k] of an interior slot is a node index and count[k] is 0, or EBG_NODE_HAS_OBB when the
// child's oriented box is tighter than its axis-aligned one (the traversal then tests it before
// reading the child); of a leaf slot, child[k] is the first triangle (leaf order) with
// EBG_LEAF_BIT set and count[k] its triangle count.  An empty slot has child 0, count 0 and an
// empty box (lo = +inf, hi = -inf), whose point distance is +inf.
#ifndef EBG_LAYOUT_H
#define EBG_LAYOUT_H

#include <stdint.h>

#define EBG_LEAF_BIT 0x80000000u
#define EBG_MAX_LEAF 32
// count[k] of a leaf slot packs the primitive count (low 6 bits) and the leaf's index (upper 26
// bits, mesh leaves only: it selects the leaf's oriented box).
#define EBG_COUNT_BITS 6u
#define EBG_COUNT_MASK 63u
#define EBG_MAX_LEAVES (1u << 26)
// count[k] of an interior slot: the child node has an oriented box worth testing.
#define EBG_NODE_HAS_OBB 0x80000000u

// Traversal stack depth (entries per warp).  The builder rejects trees whose depth would need
// more (a 4-wide node pushes at most 3 siblings per level besides the one it descends into).
#define EBG_STACK_DEPTH 96

struct alignas(128) EbgNode4
{
  float    lox[4], loy[4], loz[4];
  float    hix[4], hiy[4], hiz[4];
  uint32_t child[4];
  uint32_t count[4];
};

// The optional 8-wide copy of the tree (plain FP32 queries only; mesh_wide.cpp): two 128-byte
// lines per node, the boxes of eight children as structure-of-arrays (lo.x[8] ... hi.z[8]), then
// child[8] and count[8] with the 4-wide node's meanings.  Leaves and child boxes are the 4-wide
// tree's own, so results do not depend on the width.
struct alignas(128) EbgNode8
{
  float    lox[8], loy[8], loz[8];
  float    hix[8], hiy[8], hiz[8];
  uint32_t child[8];
  uint32_t count[8];
};

struct alignas(16) EbgTriHot
{
  float v0x, v0y, v0z, ab2;
  float abx, aby, abz, abac;
  float acx, acy, acz, ac2;
};

struct alignas(16) EbgTriSign
{
  float nx, ny, nz, pad0;
  float vn[9];
  float en[9];
  float pad1, pad2;
};

// Oriented box of the triangles of one mesh leaf or of one subtree, as three slabs: unit axes n
// (their area-weighted mean normal), u (in-plane principal axis) and v = n x u, each with the
// offset of the box centre along it (dn = n . c, ...), and the half-extents (hn, hu, hv), padded
// outward to cover FP32 evaluation.  A point's distance to the box follows from three plane
// distances (n . p - dn, ...).  A patch of a smooth surface is a thin slab, so its distance bounds
// the patch's triangles far more tightly than the axis-aligned box does.
struct alignas(16) EbgObb
{
  float nx, ny, nz, dn;
  float ux, uy, uz, du;
  float vx, vy, vz, dv;
  float hn, hu, hv, pad;
};

static_assert(sizeof(EbgNode4) == 128, "node must be one 128-byte line");
static_assert(sizeof(EbgNode8) == 256, "8-wide node must be two 128-byte lines");
static_assert(sizeof(EbgObb) == 64, "oriented box must be 64 bytes");
static_assert(sizeof(EbgTriHot) == 48, "hot triangle record must be 48 bytes");
static_assert(sizeof(EbgTriSign) == 96, "sign record must be 96 bytes");

// Device view of one mesh (passed by value to kernels).
struct EbgMeshView
{
  const EbgNode4*   nodes;
  const EbgTriHot*  hot;
  const EbgTriSign* sign;
  const double*     tri64;
  const int32_t*    tri_id;
  const EbgObb*     obb;                    // per leaf id
  const EbgObb*     node_obb;               // per interior node index
  const double*     dcel_n;                 // per triangle (leaf order): the DCEL face normal (3)
  float             root_lo[3], root_hi[3]; // root box (FP32, outward)
  uint32_t          root_ref;               // node index 0, or a leaf reference for tiny meshes
  uint32_t          root_count;             // leaf count when root_ref is a leaf
  float             morton_lo[3];           // Morton quantisation box for query ordering
  float             morton_scale[3];
};

#endif
