// Point-cloud build and k-NN launch wrappers (called from the C ABI layer).
#ifndef EBG_CLOUD_KERNELS_H
#define EBG_CLOUD_KERNELS_H

#include <cstdint>
#include <cuda_runtime.h>

#include "ebg_layout.h"

namespace ebg {

// Device view of a point cloud: 4-wide nodes (root at 0) over leaves of consecutive float4
// (x, y, z, original index bits) points in Morton order.
struct EbgCloudView
{
  const EbgNode4* nodes;
  const float4*   points;
  float           root_lo[3], root_hi[3];
  uint32_t        root_ref, root_count;
  float           morton_lo[3], morton_scale[3];
};

struct CloudQueryArgs
{
  EbgCloudView        cloud;
  const float*        queries; // caller's xyz
  const uint32_t*     order;   // sorted position -> caller index (nullptr = identity; in self
                               // queries: the query point's own cloud index)
  const uint32_t*     self_pos; // self queries: sorted position -> the query's leaf position in
                                // cloud.points (nullptr = identity: every cloud point in leaf order)
  int64_t             n;
  int                 k;       // neighbours written per query (<= template K)
  int32_t*            out_idx; // n x k, caller order
  float*              out_d2;  // n x k
  unsigned long long* work;
  int*                status;
};

// A cloud's tree: 4-wide nodes (cudaMalloc'd by buildCloud, freed by the caller) and the root's box.
struct CloudTree
{
  EbgNode4* nodes    = nullptr;
  int64_t   numNodes = 0;
  int       depth    = 0;     // node levels; 0 when the root is a single leaf (n <= L)
  bool      radix    = false; // false: the balanced tree (fallback)
  float     rootBox[6]{};
};

// Builds the tree of n points on stream s and synchronises s: leafPts (n float4, the caller's)
// receives the points in Morton order, tree the nodes (the balanced tree when asked for, or when
// the radix tree would be too deep or too large).  Returns cudaErrorMemoryAllocation when
// device memory runs out, else the first failing call's error or cudaSuccess.
cudaError_t buildCloud(const float* points, int64_t n, int L, bool balanced, float4* leafPts, CloudTree& tree,
                       cudaStream_t s);
cudaError_t launchCloudKnn(const CloudQueryArgs& a, int kTemplate, int numSms, cudaStream_t s, bool self = false);

// inv[cloud index] = leaf position, from the leaf points' index words.
void launchInvertOrder(const float4* pts, int64_t n, uint32_t* inv, cudaStream_t s);

// Self queries of caller-given cloud indices: keys = their leaf positions (the sort key that makes
// packets coherent), rows = 0..m-1; out-of-range indices set ST_INPUT.
void launchSelfKeys(const int64_t* ids, int64_t m, const uint32_t* inv, int64_t n, uint32_t* keys, uint32_t* rows,
                    int* status, cudaStream_t s);

} // namespace ebg

#endif
