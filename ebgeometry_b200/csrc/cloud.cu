// Point-cloud nearest-neighbour search (sm_100a): GPU build + per-lane k-NN traversal.
//
// Reference: PointCloudBVH (PointCloudBVH.hpp:56-350, PointCloudBVHImplem.hpp:59-610): a K-wide
// packed BVH over SoA groups of W points, built by recursive longest-axis midpoint partitioning,
// queried by pruneTraverse with a {d2, index} state for k = 1 and an insertion-sorted Hit[k] for
// k > 1 (PointCloudBVHImplem.hpp:263-427).
//
// Build here (all on the device):
//   1. bounding box of the points; 2. 30-bit Morton key of each point in that box; 3. radix sort
//   of (key, index); 4. the points gathered into that order as float4 (x, y, z, original index);
//   5. a 4-wide tree built top-down, one launch per level: a node owns a range of sorted points,
//   divided at the highest bit in which the range's first and last keys differ (the middle when all
//   its keys are equal), and its largest part divided again, until it has four parts or none holds
//   more than L points; a part of at most L points is a leaf (a run of consecutive points);
//   6. node boxes bottom-up, one launch per level.  Cutting where the Morton curve jumps keeps
//   every box spatially compact.  (Fixed runs of L points grouped four at a time in Morton order --
//   the balanced tree kept as the fallback for clouds whose radix tree is too deep for the
//   traversal stack -- make long, thin boxes across those jumps that every nearby query opens.)
// Query: Morton-sorted queries, one per lane, each walking the tree with its own stack and keeping
// its k best (d2, index) pairs sorted in registers.  Order is lexicographic on
// (d2, index), so equal distances resolve to the lowest index, and d2 is the reference's float
// arithmetic (PointSoAImplem.hpp:214-230): dx = q - p, d2 = (dx*dx + dy*dy) + dz*dz, each operation
// rounded separately (no fused multiply-add).  Box distances use the same association, which makes
// the box distance of a leaf never exceed the computed d2 of any point inside it, so pruning with
// "box d2 > k-th best d2" never drops a point that belongs in the answer, ties included.
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "cloud_kernels.h"
#include "ebg_device.cuh"

namespace ebg {

namespace {

__device__ __forceinline__ float d2exact(float dx, float dy, float dz)
{
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

__device__ __forceinline__ float boxD2exact(float lx, float ly, float lz, float hx, float hy, float hz, float px,
                                            float py, float pz)
{
  const float gx = fmaxf(0.f, fmaxf(__fsub_rn(lx, px), __fsub_rn(px, hx)));
  const float gy = fmaxf(0.f, fmaxf(__fsub_rn(ly, py), __fsub_rn(py, hy)));
  const float gz = fmaxf(0.f, fmaxf(__fsub_rn(lz, pz), __fsub_rn(pz, hz)));
  return d2exact(gx, gy, gz);
}

// order-preserving float <-> uint mapping for atomic min/max of floats
__device__ __forceinline__ uint32_t fkey(float f)
{
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funkey(uint32_t k)
{
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void kBounds(const float* __restrict__ p, int64_t n, uint32_t* __restrict__ box)
{
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float v = p[3 * i + a];
      lo[a]         = fminf(lo[a], v);
      hi[a]         = fmaxf(hi[a], v);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = fminf(lo[a], __shfl_xor_sync(FULL, lo[a], o));
      hi[a] = fmaxf(hi[a], __shfl_xor_sync(FULL, hi[a], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; a++) {
      atomicMin(box + a, fkey(lo[a]));
      atomicMax(box + 3 + a, fkey(hi[a]));
    }
  }
}

__global__ void kCloudKeys(const float* __restrict__ p, int64_t n, const uint32_t* __restrict__ box,
                           uint32_t* __restrict__ keys, uint32_t* __restrict__ ids)
{
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  uint32_t q[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float lo = funkey(box[a]), hi = funkey(box[3 + a]);
    const float ext = hi - lo;
    const float s   = ext > 0.f ? 1023.f / ext : 0.f;
    q[a]            = uint32_t(fminf(fmaxf((p[3 * i + a] - lo) * s, 0.f), 1023.f));
  }
  keys[i] = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
  ids[i]  = uint32_t(i);
}

__global__ void kGatherLeaves(const float* __restrict__ p, const uint32_t* __restrict__ order, int64_t n,
                              float4* __restrict__ leafPts)
{
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  const uint32_t id = order[i];
  leafPts[i]        = make_float4(p[3 * size_t(id)], p[3 * size_t(id) + 1], p[3 * size_t(id) + 2], __uint_as_float(id));
}

// Box of each leaf (L consecutive points); boxes as 6 floats (lo xyz, hi xyz).
__global__ void kLeafBoxes(const float4* __restrict__ pts, int64_t n, int L, int64_t nLeaves, float* __restrict__ boxes)
{
  const int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (l >= nLeaves) {
    return;
  }
  float         lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  const int64_t b = l * L, e = (b + L < n) ? b + L : n;
  for (int64_t i = b; i < e; i++) {
    const float4 q = pts[i];
    lo[0] = fminf(lo[0], q.x);
    lo[1] = fminf(lo[1], q.y);
    lo[2] = fminf(lo[2], q.z);
    hi[0] = fmaxf(hi[0], q.x);
    hi[1] = fmaxf(hi[1], q.y);
    hi[2] = fmaxf(hi[2], q.z);
  }
  for (int a = 0; a < 3; a++) {
    boxes[6 * l + a]     = lo[a];
    boxes[6 * l + 3 + a] = hi[a];
  }
}

// One tree level: node j (0 <= j < nNodes) gets children 4j..4j+3 of the level below (nChild
// entries with boxes childBoxes).  childIsLeaf: children are point leaves (ref = LEAF | first point,
// count = points) else nodes at index childBase + c.  Writes the node record at nodes[nodeBase + j]
// and its own box into outBoxes[j].
__global__ void kTreeLevel(int64_t nNodes, int64_t nChild, const float* __restrict__ childBoxes, int childIsLeaf,
                           int64_t childBase, int L, int64_t nPoints, EbgNode4* __restrict__ nodes, int64_t nodeBase,
                           float* __restrict__ outBoxes)
{
  const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= nNodes) {
    return;
  }
  EbgNode4 nd;
  float    lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int64_t c = 4 * j + k;
    if (c < nChild) {
      const float* b = childBoxes + 6 * c;
      nd.lox[k] = b[0];
      nd.loy[k] = b[1];
      nd.loz[k] = b[2];
      nd.hix[k] = b[3];
      nd.hiy[k] = b[4];
      nd.hiz[k] = b[5];
      for (int a = 0; a < 3; a++) {
        lo[a] = fminf(lo[a], b[a]);
        hi[a] = fmaxf(hi[a], b[3 + a]);
      }
      if (childIsLeaf) {
        const int64_t first = c * L;
        const int64_t cnt   = (first + L < nPoints) ? L : nPoints - first;
        nd.child[k]         = EBG_LEAF_BIT | uint32_t(first);
        nd.count[k]         = uint32_t(cnt);
      }
      else {
        nd.child[k] = uint32_t(childBase + c);
        nd.count[k] = 0;
      }
    }
    else {
      nd.lox[k] = nd.loy[k] = nd.loz[k] = __int_as_float(0x7f800000);  // +inf
      nd.hix[k] = nd.hiy[k] = nd.hiz[k] = __int_as_float(0xff800000);  // -inf
      nd.child[k] = 0;
      nd.count[k] = 0;
    }
  }
  nodes[nodeBase + j] = nd;
  for (int a = 0; a < 3; a++) {
    outBoxes[6 * j + a]     = lo[a];
    outBoxes[6 * j + 3 + a] = hi[a];
  }
}

// ---- top-down radix build ----------------------------------------------------------------------

struct CloudTask
{
  uint32_t b, e, node; // sorted point range [b, e) of node `node`
};

// The first position of [b, e) (e - b >= 2) whose key differs from keys[b] in the highest bit where
// keys[b] and keys[e - 1] differ; the middle when the range's keys are all equal.
__device__ __forceinline__ uint32_t radixSplit(const uint32_t* __restrict__ keys, uint32_t b, uint32_t e)
{
  const uint32_t x = keys[b] ^ keys[e - 1];
  if (x == 0u) {
    return b + (e - b) / 2;
  }
  const int      bit = 31 - __clz(int(x));
  const uint32_t pre = keys[b] >> bit;
  uint32_t       lo = b + 1, hi = e - 1; // keys[e - 1] >> bit != pre: the answer lies in [b + 1, e - 1]
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if ((keys[mid] >> bit) == pre) {
      lo = mid + 1;
    }
    else {
      hi = mid;
    }
  }
  return lo;
}

// One level: each task's node gets 2-4 parts (the largest part of more than L points is divided
// until there are four, ties to the lowest slot); leaf parts get their boxes here, interior parts a
// node index (counters[0]), a task for the next level (counters[1]) and an empty box that the box
// pass fills.  A node index at or above maxNodes sets *overflow and leaves the slot empty.
__global__ void kCloudSplit(const CloudTask* __restrict__ tasks, uint32_t count, const uint32_t* __restrict__ keys,
                            const float4* __restrict__ pts, int L, EbgNode4* __restrict__ nodes,
                            CloudTask* __restrict__ next, uint32_t* __restrict__ counters,
                            uint32_t* __restrict__ parentSlot, uint32_t maxNodes, int* __restrict__ overflow)
{
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < count; w += gridDim.x * blockDim.x) {
    const CloudTask t = tasks[w];
    uint32_t        pb[4], pe[4];
    int             nc = 1;
    pb[0]              = t.b;
    pe[0]              = t.e;
    while (nc < 4) {
      int      pick = -1;
      uint32_t most = uint32_t(L);
      for (int i = 0; i < nc; i++) {
        if (pe[i] - pb[i] > most) {
          most = pe[i] - pb[i];
          pick = i;
        }
      }
      if (pick < 0) {
        break;
      }
      const uint32_t m = radixSplit(keys, pb[pick], pe[pick]);
      for (int i = nc; i > pick + 1; i--) {
        pb[i] = pb[i - 1];
        pe[i] = pe[i - 1];
      }
      pb[pick + 1] = m;
      pe[pick + 1] = pe[pick];
      pe[pick]     = m;
      nc++;
    }
    EbgNode4 nd;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float    lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      uint32_t child = 0, cnt = 0;
      bool     leafBox = false;
      if (k < nc) {
        const uint32_t c = pe[k] - pb[k];
        if (c <= uint32_t(L)) {
          for (uint32_t i = pb[k]; i < pe[k]; i++) {
            const float4 q = pts[i];
            lo[0]          = fminf(lo[0], q.x);
            lo[1]          = fminf(lo[1], q.y);
            lo[2]          = fminf(lo[2], q.z);
            hi[0]          = fmaxf(hi[0], q.x);
            hi[1]          = fmaxf(hi[1], q.y);
            hi[2]          = fmaxf(hi[2], q.z);
          }
          child   = EBG_LEAF_BIT | pb[k];
          cnt     = c;
          leafBox = true;
        }
        else {
          const uint32_t id = atomicAdd(counters, 1u);
          if (id >= maxNodes) {
            atomicOr(overflow, 1);
          }
          else {
            child            = id;
            parentSlot[id]   = t.node * 4u + uint32_t(k);
            const uint32_t q = atomicAdd(counters + 1, 1u);
            next[q]          = CloudTask{pb[k], pe[k], id};
          }
        }
      }
      nd.lox[k]   = leafBox ? lo[0] : __int_as_float(0x7f800000);
      nd.loy[k]   = leafBox ? lo[1] : __int_as_float(0x7f800000);
      nd.loz[k]   = leafBox ? lo[2] : __int_as_float(0x7f800000);
      nd.hix[k]   = leafBox ? hi[0] : __int_as_float(0xff800000);
      nd.hiy[k]   = leafBox ? hi[1] : __int_as_float(0xff800000);
      nd.hiz[k]   = leafBox ? hi[2] : __int_as_float(0xff800000);
      nd.child[k] = child;
      nd.count[k] = cnt;
    }
    nodes[t.node] = nd;
  }
}

// Boxes of one level's nodes [begin, end) (every deeper level done): the union of the node's
// occupied slots, written into its parent's slot (the root's into rootBox).
__global__ void kCloudBoxes(EbgNode4* __restrict__ nodes, uint32_t begin, uint32_t end,
                            const uint32_t* __restrict__ parentSlot, float* __restrict__ rootBox)
{
  for (uint32_t id = begin + blockIdx.x * blockDim.x + threadIdx.x; id < end; id += gridDim.x * blockDim.x) {
    const EbgNode4 nd    = nodes[id];
    float          lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if ((nd.child[k] | nd.count[k]) != 0u) {
        lo[0] = fminf(lo[0], nd.lox[k]);
        lo[1] = fminf(lo[1], nd.loy[k]);
        lo[2] = fminf(lo[2], nd.loz[k]);
        hi[0] = fmaxf(hi[0], nd.hix[k]);
        hi[1] = fmaxf(hi[1], nd.hiy[k]);
        hi[2] = fmaxf(hi[2], nd.hiz[k]);
      }
    }
    if (id == 0u) {
      for (int a = 0; a < 3; a++) {
        rootBox[a]     = lo[a];
        rootBox[3 + a] = hi[a];
      }
      continue;
    }
    const uint32_t ps = parentSlot[id];
    EbgNode4&      p  = nodes[ps >> 2];
    const int      k  = int(ps & 3u);
    p.lox[k]          = lo[0];
    p.loy[k]          = lo[1];
    p.loz[k]          = lo[2];
    p.hix[k]          = hi[0];
    p.hiy[k]          = hi[1];
    p.hiz[k]          = hi[2];
  }
}

// ---- query ---------------------------------------------------------------------------------------

__device__ __forceinline__ bool lexLess(float da, uint32_t ia, float db, uint32_t ib)
{
  return da < db || (da == db && ia < ib);
}

// One query per lane.  Each lane walks the tree on its own, nearest child first, with a private
// stack of (ref, count, box distance) entries (in local memory: at most 3 x depth + 1 of them); a
// popped entry whose distance exceeds the lane's k-th best is skipped.  Warps take packets of 32
// consecutive (Morton-ordered) queries from the work counter, so a warp's lanes walk nearby paths
// and mostly read the same node and point lines.  (A warp walking one shared stack for its 32
// queries opens every node any lane needs -- about four times what each lane needs on the k-NN
// workloads -- and costs more than the divergence of separate walks.)
// SELF: the queries are cloud points (self_pos), each excluded from its own neighbours
// (nearestNeighbors / allNearestNeighbors, PointCloudBVHImplem.hpp:455-507).
template <int K, bool SELF>
__global__ void __launch_bounds__(128, (K <= 2 ? 16 : (K <= 8 ? 10 : 1))) kCloudKnn(const CloudQueryArgs a)
{
  const int           lane       = threadIdx.x & 31;
  const EbgCloudView& c          = a.cloud;
  const uint64_t      numPackets = (uint64_t(a.n) + 31) / 32;
  while (true) {
    unsigned long long pk = 0;
    if (lane == 0) {
      pk = atomicAdd(a.work, 1ull);
    }
    pk = __shfl_sync(FULL, pk, 0);
    if (pk >= numPackets) {
      break;
    }
    const int64_t pos = int64_t(pk) * 32 + lane;
    if (pos >= a.n) {
      continue;
    }
    uint32_t id, self = 0xffffffffu;
    float    px, py, pz;
    if (SELF) {
      const uint32_t lp = a.self_pos ? __ldg(a.self_pos + pos) : uint32_t(pos);
      const float4   qp = __ldg(c.points + lp);
      px                = qp.x;
      py                = qp.y;
      pz                = qp.z;
      self              = __float_as_uint(qp.w);
      id                = a.order ? __ldg(a.order + pos) : self;
    }
    else {
      id = a.order ? __ldg(a.order + pos) : uint32_t(pos);
      px = __ldg(a.queries + 3 * size_t(id));
      py = __ldg(a.queries + 3 * size_t(id) + 1);
      pz = __ldg(a.queries + 3 * size_t(id) + 2);
    }
    const int pad = K - a.k;
    float     kd[K];
    uint32_t  ki[K];
#pragma unroll
    for (int j = 0; j < K; j++) {
      kd[j] = j < pad ? -1.f : __int_as_float(0x7f800000);
      ki[j] = j < pad ? 0u : 0xffffffffu;
    }
    uint4    stk[EBG_STACK_DEPTH];
    int      sp    = 1;
    uint32_t iters = 0;
    int      err   = 0;
    stk[0]         = make_uint4(c.root_ref, c.root_count,
                                __float_as_uint(boxD2exact(c.root_lo[0], c.root_lo[1], c.root_lo[2], c.root_hi[0],
                                                           c.root_hi[1], c.root_hi[2], px, py, pz)),
                                0u);
    while (sp > 0) {
      if (++iters > MAX_ITERS) {
        err |= ST_ITERS;
        break;
      }
      const uint4 e = stk[--sp];
      if (__uint_as_float(e.z) > kd[K - 1]) {
        continue;
      }
      if (e.x & EBG_LEAF_BIT) {
        const uint32_t p0 = e.x & ~EBG_LEAF_BIT, pe = p0 + e.y;
        for (uint32_t t = p0; t < pe; ++t) {
          const float4   q  = __ldg(c.points + t);
          const float    dd = d2exact(px - q.x, py - q.y, pz - q.z);
          const uint32_t ii = __float_as_uint(q.w);
          if ((!SELF || ii != self) && lexLess(dd, ii, kd[K - 1], ki[K - 1])) {
            kd[K - 1] = dd;
            ki[K - 1] = ii;
#pragma unroll
            for (int j = K - 1; j > 0; j--) {
              if (lexLess(kd[j], ki[j], kd[j - 1], ki[j - 1])) {
                const float    td = kd[j];
                const uint32_t ti = ki[j];
                kd[j]             = kd[j - 1];
                ki[j]             = ki[j - 1];
                kd[j - 1]         = td;
                ki[j - 1]         = ti;
              }
            }
          }
        }
        continue;
      }
      const float4* nd    = reinterpret_cast<const float4*>(c.nodes + e.x);
      const float4  lx    = __ldg(nd), ly = __ldg(nd + 1), lz = __ldg(nd + 2);
      const float4  hx    = __ldg(nd + 3), hy = __ldg(nd + 4), hz = __ldg(nd + 5);
      const uint4   ch    = __ldg(reinterpret_cast<const uint4*>(nd + 6));
      const uint4   cn    = __ldg(reinterpret_cast<const uint4*>(nd + 7));
      const float   bound = kd[K - 1];
      // (distance, ref, count) of each child; -1 marks an empty slot or a child beyond the bound
      float    d[4]  = {boxD2exact(lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, px, py, pz),
                        boxD2exact(lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, px, py, pz),
                        boxD2exact(lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, px, py, pz),
                        boxD2exact(lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, px, py, pz)};
      uint32_t r[4]  = {ch.x, ch.y, ch.z, ch.w};
      uint32_t n4[4] = {cn.x, cn.y, cn.z, cn.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (!(d[k] <= bound) || (r[k] | n4[k]) == 0u) {
          d[k] = -1.f;
        }
      }
      // farthest first onto the stack, so the nearest is popped next (ties by slot)
      auto cswap = [&](int i, int j) {
        if (d[i] < d[j]) {
          const float    td = d[i];
          const uint32_t tr = r[i], tn = n4[i];
          d[i]              = d[j];
          r[i]              = r[j];
          n4[i]             = n4[j];
          d[j]              = td;
          r[j]              = tr;
          n4[j]             = tn;
        }
      };
      cswap(0, 1);
      cswap(2, 3);
      cswap(0, 2);
      cswap(1, 3);
      cswap(1, 2);
      const int np = int(d[0] >= 0.f) + int(d[1] >= 0.f) + int(d[2] >= 0.f) + int(d[3] >= 0.f);
      if (sp + np > EBG_STACK_DEPTH) {
        err |= ST_STACK;
        break;
      }
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (d[k] >= 0.f) {
          stk[sp++] = make_uint4(r[k], n4[k], __float_as_uint(d[k]), 0u);
        }
      }
    }
    if (err) {
      atomicOr(a.status, err);
    }
#pragma unroll
    for (int j = 0; j < K; j++) {
      if (j >= pad) {
        const bool   found = ki[j] != 0xffffffffu;
        const size_t o     = size_t(id) * a.k + (j - pad);
        a.out_idx[o]       = found ? int32_t(ki[j]) : -1;
        a.out_d2[o]        = found ? kd[j] : __int_as_float(0x7f800000);
      }
    }
  }
}

template <int K, bool SELF>
cudaError_t launchKnnKS(const CloudQueryArgs& a, int numSms, cudaStream_t s)
{
  int perSm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kCloudKnn<K, SELF>, 128, 0);
  perSm              = perSm < 1 ? 1 : perSm;
  const int64_t need = ((int64_t(a.n) + 31) / 32 + 3) / 4;
  int64_t       grid = int64_t(numSms) * perSm;
  grid               = grid < need ? grid : need;
  grid               = grid < 1 ? 1 : grid;
  kCloudKnn<K, SELF><<<unsigned(grid), 128, 0, s>>>(a);
  return cudaGetLastError();
}

template <int K>
cudaError_t launchKnnK(const CloudQueryArgs& a, bool self, int numSms, cudaStream_t s)
{
  return self ? launchKnnKS<K, true>(a, numSms, s) : launchKnnKS<K, false>(a, numSms, s);
}

// inv[cloud index] = leaf position
__global__ void kInvertOrder(const float4* __restrict__ pts, int64_t n, uint32_t* __restrict__ inv)
{
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
    inv[__float_as_uint(pts[j].w)] = uint32_t(j);
  }
}

// self queries of a caller's list of cloud indices: sort keys = their leaf positions, values = the
// caller's row; an index out of range is reported (ST_INPUT) and replaced by 0
__global__ void kSelfKeys(const int64_t* __restrict__ ids, int64_t m, const uint32_t* __restrict__ inv, int64_t n,
                          uint32_t* __restrict__ keys, uint32_t* __restrict__ rows, int* __restrict__ status)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t id = ids[i];
    const bool    ok = id >= 0 && id < n;
    if (!ok) {
      atomicOr(status, ST_INPUT);
    }
    keys[i] = inv[ok ? id : 0];
    rows[i] = uint32_t(i);
  }
}

inline unsigned blocksFor(int64_t n, int t) { return unsigned((n + t - 1) / t); }

} // namespace

namespace {

// 3 x depth + 1 stack entries: a 4-wide node pushes at most 3 siblings per level besides the one
// the walk descends into
constexpr int kMaxCloudDepth = (EBG_STACK_DEPTH - 1) / 3;

// stream-ordered build workspace, released in order on the stream when the build returns
struct Workspace
{
  cudaStream_t       s;
  std::vector<void*> held;
  explicit Workspace(cudaStream_t st) : s(st) {}
  ~Workspace()
  {
    for (void* p : held) {
      cudaFreeAsync(p, s);
    }
  }
  template <class T>
  T* get(size_t count)
  {
    void* p = nullptr;
    if (cudaMallocAsync(&p, std::max<size_t>(count * sizeof(T), 16), s) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    held.push_back(p);
    return static_cast<T*>(p);
  }
};

// The balanced tree: runs of L sorted points, grouped four at a time, level by level.
cudaError_t buildBalanced(const float4* leafPts, int64_t n, int L, Workspace& ws, CloudTree& tree, cudaStream_t s)
{
  const int     T       = 256;
  const int64_t nLeaves = (n + L - 1) / L;
  int64_t       levelNodes[64];
  int           nl = 0;
  for (int64_t c = nLeaves; c > 1 && nl < 64;) {
    c                = (c + 3) / 4;
    levelNodes[nl++] = c;
  }
  int64_t total = 0;
  for (int l = 0; l < nl; l++) {
    total += levelNodes[l];
  }
  float* boxA = ws.get<float>(6 * size_t(nLeaves));
  float* boxB = ws.get<float>(6 * size_t(nl > 0 ? levelNodes[0] : 1));
  if (!boxA || !boxB) {
    return cudaErrorMemoryAllocation;
  }
  if (cudaMalloc(reinterpret_cast<void**>(&tree.nodes), size_t(std::max<int64_t>(total, 1)) * sizeof(EbgNode4)) !=
      cudaSuccess) {
    cudaGetLastError();
    tree.nodes = nullptr;
    return cudaErrorMemoryAllocation;
  }
  kLeafBoxes<<<blocksFor(nLeaves, T), T, 0, s>>>(leafPts, n, L, nLeaves, boxA);
  // node index base of level l (1..nl) counts the levels above it
  int64_t base[65];
  int64_t acc = 0;
  for (int l = nl; l >= 1; l--) {
    base[l] = acc;
    acc += levelNodes[l - 1];
  }
  float*  cur    = boxA;
  float*  nxt    = boxB;
  int64_t nChild = nLeaves;
  for (int l = 1; l <= nl; l++) {
    const int64_t nn = levelNodes[l - 1];
    kTreeLevel<<<blocksFor(nn, T), T, 0, s>>>(nn, nChild, cur, l == 1 ? 1 : 0, l == 1 ? 0 : base[l - 1], L, n,
                                             tree.nodes, base[l], nxt);
    std::swap(cur, nxt);
    nChild = nn;
  }
  cudaMemcpyAsync(tree.rootBox, cur, 6 * sizeof(float), cudaMemcpyDeviceToHost, s);
  tree.numNodes = total;
  tree.depth    = nl;
  tree.radix    = false;
  return cudaGetLastError();
}

// The radix tree (kCloudSplit, kCloudBoxes).  Sets fallback (and builds nothing) when the tree
// would need more than kMaxCloudDepth levels or more nodes than the workspace holds: n / max(1,
// L / 4) + 64.  A node has at least two children, so a tree never has more than n - 1 nodes (the
// bound for L < 8); Morton-ordered clouds need about n / (1.4 L) (leaves average about 0.7 L
// points, two to four per node), a fifth of the workspace.
cudaError_t buildRadix(const float4* leafPts, const uint32_t* keys, int64_t n, int L, Workspace& ws, CloudTree& tree,
                       cudaStream_t s, bool& fallback)
{
  const int64_t  per        = std::max(1, L / 4);
  const uint32_t cap        = uint32_t(std::min<int64_t>(n / per + 64, int64_t(1) << 29));
  CloudTask*     tasks[2]   = {ws.get<CloudTask>(cap), ws.get<CloudTask>(cap)};
  uint32_t*      parentSlot = ws.get<uint32_t>(cap);
  EbgNode4*      built      = ws.get<EbgNode4>(cap);
  uint32_t*      counters   = ws.get<uint32_t>(4); // nodes, next tasks, overflow
  float*         rootDev    = ws.get<float>(6);
  if (!tasks[0] || !tasks[1] || !parentSlot || !built || !counters || !rootDev) {
    fallback = true;
    return cudaSuccess;
  }
  const CloudTask root{0u, uint32_t(n), 0u};
  const uint32_t  init[4] = {1u, 0u, 0u, 0u};
  cudaMemcpyAsync(tasks[0], &root, sizeof(root), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(counters, init, sizeof(init), cudaMemcpyHostToDevice, s);
  // level l holds nodes [start[l], start[l + 1])
  std::vector<uint32_t> start = {0u, 1u};
  uint32_t              count = 1;
  int                   cur   = 0;
  while (count > 0) {
    if (int(start.size()) - 1 > kMaxCloudDepth) {
      fallback = true;
      return cudaSuccess;
    }
    cudaMemsetAsync(counters + 1, 0, sizeof(uint32_t), s);
    kCloudSplit<<<blocksFor(count, 128), 128, 0, s>>>(tasks[cur], count, keys, leafPts, L, built, tasks[1 - cur],
                                                      counters, parentSlot, cap,
                                                      reinterpret_cast<int*>(counters + 2));
    uint32_t hc[3];
    cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      return e;
    }
    if (hc[2] != 0u) {
      fallback = true;
      return cudaSuccess;
    }
    count = hc[1];
    if (count > 0) {
      start.push_back(hc[0]);
    }
    cur = 1 - cur;
  }
  const int depth = int(start.size()) - 1;
  for (int l = depth - 1; l >= 0; l--) {
    const uint32_t b = start[l], e = start[l + 1];
    kCloudBoxes<<<blocksFor(e - b, 128), 128, 0, s>>>(built, b, e, parentSlot, rootDev);
  }
  const int64_t total = start.back();
  if (cudaMalloc(reinterpret_cast<void**>(&tree.nodes), size_t(total) * sizeof(EbgNode4)) != cudaSuccess) {
    cudaGetLastError();
    tree.nodes = nullptr;
    return cudaErrorMemoryAllocation;
  }
  cudaMemcpyAsync(tree.nodes, built, size_t(total) * sizeof(EbgNode4), cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(tree.rootBox, rootDev, 6 * sizeof(float), cudaMemcpyDeviceToHost, s);
  tree.numNodes = total;
  tree.depth    = depth;
  tree.radix    = true;
  return cudaGetLastError();
}

} // namespace

cudaError_t buildCloud(const float* points, int64_t n, int L, bool balanced, float4* leafPts, CloudTree& tree,
                       cudaStream_t s)
{
  const int T = 256;
  Workspace ws(s);
  uint32_t* box     = ws.get<uint32_t>(6);
  uint32_t* keysIn  = ws.get<uint32_t>(size_t(n));
  uint32_t* keysOut = ws.get<uint32_t>(size_t(n));
  uint32_t* idsIn   = ws.get<uint32_t>(size_t(n));
  uint32_t* idsOut  = ws.get<uint32_t>(size_t(n));
  size_t    tb      = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, keysIn, keysOut, idsIn, idsOut, int(n), 0, 30, s);
  void* sortTemp = ws.get<char>(tb);
  if (!box || !keysIn || !keysOut || !idsIn || !idsOut || !sortTemp) {
    return cudaErrorMemoryAllocation;
  }
  // box init: lo = fkey(+max) (atomicMin), hi = fkey(-max) (atomicMax)
  const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  cudaMemcpyAsync(box, init, sizeof(init), cudaMemcpyHostToDevice, s);
  kBounds<<<unsigned(std::min<int64_t>(blocksFor(n, T), 4096)), T, 0, s>>>(points, n, box);
  kCloudKeys<<<blocksFor(n, T), T, 0, s>>>(points, n, box, keysIn, idsIn);
  cub::DeviceRadixSort::SortPairs(sortTemp, tb, keysIn, keysOut, idsIn, idsOut, int(n), 0, 30, s);
  kGatherLeaves<<<blocksFor(n, T), T, 0, s>>>(points, idsOut, n, leafPts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    return e;
  }
  if (n > L && !balanced) {
    bool fallback = false;
    e             = buildRadix(leafPts, keysOut, n, L, ws, tree, s, fallback);
    if (e != cudaSuccess || !fallback) {
      return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
    }
  }
  e = buildBalanced(leafPts, n, L, ws, tree, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}

cudaError_t launchCloudKnn(const CloudQueryArgs& a, int kTemplate, int numSms, cudaStream_t s, bool self)
{
  switch (kTemplate) {
  case 1:
    return launchKnnK<1>(a, self, numSms, s);
  case 2:
    return launchKnnK<2>(a, self, numSms, s);
  case 4:
    return launchKnnK<4>(a, self, numSms, s);
  case 8:
    return launchKnnK<8>(a, self, numSms, s);
  case 16:
    return launchKnnK<16>(a, self, numSms, s);
  default:
    return launchKnnK<32>(a, self, numSms, s);
  }
}

void launchInvertOrder(const float4* pts, int64_t n, uint32_t* inv, cudaStream_t s)
{
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 8192);
  kInvertOrder<<<unsigned(blocks < 1 ? 1 : blocks), 256, 0, s>>>(pts, n, inv);
}

void launchSelfKeys(const int64_t* ids, int64_t m, const uint32_t* inv, int64_t n, uint32_t* keys, uint32_t* rows,
                    int* status, cudaStream_t s)
{
  const int64_t blocks = std::min<int64_t>((m + 255) / 256, 8192);
  kSelfKeys<<<unsigned(blocks < 1 ? 1 : blocks), 256, 0, s>>>(ids, m, inv, n, keys, rows, status);
}

} // namespace ebg
