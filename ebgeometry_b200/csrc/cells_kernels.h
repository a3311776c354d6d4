// Per-cell entry cuts of a mesh BVH, built from a learned distance bound (sm_100a).
//
// A regular grid of G^3 cells covers the seed model's domain.  Each cell keeps a CUT of the mesh's
// BVH: a list of at most `lmax` subtrees (stack entries: child box, reference and count words, as
// the traversal pushes them) that together hold every triangle within the cell's radius R_C of the
// cell grown by `margin` on every side.  R_C bounds |d| over that grown cell: the model's
// calibrated radius at the cell centre plus the grown cell's half-diagonal (the SDF is 1-Lipschitz).
// The cut is refined best-first from the root (the subtree nearest to the cell centre is split
// first; a child farther than R_C from the grown cell is dropped) until `lmax` entries are reached
// or every entry is a leaf.  Entries are stored farthest first, so that copied onto a warp's stack
// the nearest is popped first.
//
// A packet of 32 sorted queries whose bounding box lies inside the grown cell of the cell holding
// the box's centre starts from that cut with its lanes' bound at R_C instead of descending from the
// root.  Whatever a lane finds within R_C is its exact nearest triangle (every triangle within R_C of
// a point of the grown cell is under the cut); a lane that finds nothing is traversed again from the
// root without a bound, so results never depend on the model.
#ifndef EBG_CELLS_KERNELS_H
#define EBG_CELLS_KERNELS_H

#include <cstdint>
#include <cuda_runtime.h>

#include "ebg_layout.h"

namespace ebg {

// Stack capacity (entries) of the traversal that starts from a cut: the cut's entries sit below
// what the traversal pushes (at most 3 per level of the tree below them).
constexpr int CUT_STACK_DEPTH = 160;
constexpr int CUT_MAX_ENTRIES = 112;

struct SeedCellsView
{
  const float4*   entries; // [cells][lmax][2] stack entries of each cell's cut, farthest first
  const uint32_t* count;   // [cells] entries in the cut (0: the cell's packets start at the root)
  const float*    radius;  // [cells] R_C, rounded up
  const int32_t*  anchor;  // [cells] leaf-order triangle nearest to the cell centre (-1: none; nullable)
  float           lo[3];   // domain corner
  float           inv[3];  // cells per unit length along each axis
  float           size[3]; // cell edge along each axis
  float           margin[3];
  int32_t         g;       // cells per axis
  int32_t         lmax;    // entry slots per cell
};

// Cell centres (x fastest), xyz per cell.
cudaError_t launchCellCentres(const SeedCellsView& v, float* out, cudaStream_t s);
// radius[c] from the value at cell c's centre: mode 0 learned ((1 + alpha) |value| + beta), 2 exact
// (|value| rounded up); plus the grown cell's half-diagonal.  Mode 1: +inf (cuts by distance order
// only, no radius).
cudaError_t launchCellRadius(const float* value, int64_t cells, int mode, float alpha, float beta, float halfDiag,
                             float* radius, cudaStream_t s);
// The cut of every cell (one warp per cell).
cudaError_t launchCellCuts(const EbgMeshView& m, const SeedCellsView& v, float4* entries, uint32_t* count,
                           cudaStream_t s);

} // namespace ebg

#endif
