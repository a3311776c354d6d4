// Device build of a mesh's Morton 4-wide BVH and its leaf-ordered records (sm_100a).
//
// The same tree family as the host Morton build (mesh_host.cpp): triangles sorted by the 63-bit
// Morton code of their centroid (21 bits per axis over the centroids' box), every range split at
// the highest bit in which its first and last codes differ, 4-wide nodes made by repeatedly
// splitting the child of largest box area, leaves of at most leafSize triangles.  On the device:
//   1. per triangle: FP64 box and centroid, the centroids' box (warp-reduced atomics on
//      order-preserving integer keys), the Morton code; CUB radix sort of (code, triangle);
//   2. the binary radix tree of the sorted codes, each internal node found independently from the
//      common-prefix lengths of its neighbours (equal codes are told apart by position), so its
//      split is the highest differing bit of its range -- the host's Morton split;
//   3. FP64 node boxes bottom-up: each triangle walks to the root and the second of two siblings to
//      arrive computes the parent (an atomic counter per node, no waiting);
//   4. the 4-wide tree top-down, one launch per level: each node expands its largest-area children
//      up to four, as the host does; leaves and nodes get their indices from atomic counters;
//   5. leaf-ordered triangle records (the FP32 hot and sign records, the FP64 lane records, the DCEL
//      normals, areas), and the oriented box of every leaf and node (one block per range).
// The pseudonormals come from the host build's routine or from normals_gpu.cu (both bit-identical
// to the reference's DCEL).  Results do not depend on the tree's shape, so a mesh built here
// answers exactly as a host-built one.
// 6. Refit (moved vertices, either build's tree): pseudonormals, records and oriented boxes again,
//    and every node's child boxes from its children's ranges of leaf positions.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>
#include <math_constants.h>

#include "capi_common.h"
#include "capi_internal.h"
#include "ebg_device.cuh"
#include "mesh_build_gpu.h"
#include "mesh_host.h"

namespace ebg {

namespace {

constexpr uint32_t NONE = 0xffffffffu;

// order-preserving map of a double onto uint64 (for atomic min / max)
__device__ __forceinline__ unsigned long long dkey(double x)
{
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dval(unsigned long long k)
{
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double(static_cast<long long>(b));
}
__host__ double hostDval(unsigned long long k)
{
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double                   d;
  std::memcpy(&d, &b, sizeof(d));
  return d;
}

// FP64 reductions over a warp or a block (one shared slot per warp)
struct WarpGroup
{
  __device__ int    rank() const { return threadIdx.x & 31; }
  __device__ int    size() const { return 32; }
  __device__ double sum(double v) const
  {
    for (int off = 16; off > 0; off >>= 1) {
      v += __shfl_xor_sync(FULL, v, off);
    }
    return v;
  }
  __device__ double min(double v) const
  {
    for (int off = 16; off > 0; off >>= 1) {
      v = fmin(v, __shfl_xor_sync(FULL, v, off));
    }
    return v;
  }
  __device__ double max(double v) const { return -min(-v); }
};

struct BlockGroup
{
  double*           red; // one slot per warp
  __device__ int    rank() const { return threadIdx.x; }
  __device__ int    size() const { return blockDim.x; }
  __device__ double combine(double v, bool isMin) const
  {
    v = isMin ? WarpGroup().min(v) : WarpGroup().sum(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
      red[threadIdx.x >> 5] = v;
    }
    __syncthreads();
    double r = isMin ? DBL_MAX : 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); w++) {
      r = isMin ? fmin(r, red[w]) : r + red[w];
    }
    return r;
  }
  __device__ double sum(double v) const { return combine(v, false); }
  __device__ double min(double v) const { return combine(v, true); }
  __device__ double max(double v) const { return -combine(-v, true); }
};


__device__ __forceinline__ uint64_t spread21(uint64_t x)
{
  x &= 0x1fffff;
  x = (x | x << 32) & 0x1f00000000ffffULL;
  x = (x | x << 16) & 0x1f0000ff0000ffULL;
  x = (x | x << 8) & 0x100f00f00f00f00fULL;
  x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
  x = (x | x << 2) & 0x1249249249249249ULL;
  return x;
}

// 1a. triangle boxes and centroids; bounds: [0..2] centroid lo, [3..5] centroid hi, [6..8] box lo,
// [9..11] box hi, as dkey values
__global__ void kTriBounds(const double* __restrict__ V, const int32_t* __restrict__ F, int64_t nt,
                           double* __restrict__ boxLo, double* __restrict__ boxHi, double* __restrict__ cen,
                           unsigned long long* __restrict__ bounds)
{
  const int lane = threadIdx.x & 31;
  for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < nt; base += int64_t(gridDim.x) * blockDim.x) {
    const int64_t f     = base + threadIdx.x;
    const bool    valid = f < nt;
    double        c[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    if (valid) {
      for (int a = 0; a < 3; a++) {
        const double x0 = V[3 * int64_t(F[3 * f]) + a], x1 = V[3 * int64_t(F[3 * f + 1]) + a],
                     x2 = V[3 * int64_t(F[3 * f + 2]) + a];
        lo[a]           = fmin(x0, fmin(x1, x2));
        hi[a]           = fmax(x0, fmax(x1, x2));
        c[a]            = (x0 + x1 + x2) / 3.0;
        boxLo[3 * f + a] = lo[a];
        boxHi[3 * f + a] = hi[a];
        cen[3 * f + a]   = c[a];
      }
    }
    // warp-reduce the twelve keys, then one atomic each per warp
    unsigned long long k[12];
    for (int a = 0; a < 3; a++) {
      k[a]     = valid ? dkey(c[a]) : ~0ull;
      k[3 + a] = valid ? dkey(c[a]) : 0ull;
      k[6 + a] = valid ? dkey(lo[a]) : ~0ull;
      k[9 + a] = valid ? dkey(hi[a]) : 0ull;
    }
    for (int j = 0; j < 12; j++) {
      const bool isMin = (j < 3) || (j >= 6 && j < 9);
      for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(FULL, k[j], off);
        k[j]                       = isMin ? (o < k[j] ? o : k[j]) : (o > k[j] ? o : k[j]);
      }
      if (lane == 0) {
        if (isMin) {
          atomicMin(bounds + j, k[j]);
        }
        else {
          atomicMax(bounds + j, k[j]);
        }
      }
    }
  }
}

// 1b. Morton codes of the centroids over their box (the host build's codes exactly)
__global__ void kTriMorton(const double* __restrict__ cen, int64_t nt, const unsigned long long* __restrict__ bounds,
                           uint64_t* __restrict__ codes, uint32_t* __restrict__ ids)
{
  double cl[3], ext[3];
  for (int a = 0; a < 3; a++) {
    cl[a]  = dval(bounds[a]);
    ext[a] = dval(bounds[3 + a]) - cl[a];
  }
  for (int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; f < nt; f += int64_t(gridDim.x) * blockDim.x) {
    uint64_t c = 0;
    for (int a = 0; a < 3; a++) {
      const double   u = ext[a] > 0 ? (cen[3 * f + a] - cl[a]) / ext[a] : 0.0;
      const uint64_t q = uint64_t(fmin(fmax(u * 2097151.0, 0.0), 2097151.0));
      c |= spread21(q) << (2 - a);
    }
    codes[f] = c;
    ids[f]   = uint32_t(f);
  }
}

// 2. binary radix tree over the n sorted codes: internal node i in [0, n-1) gets its children
// (leaf = position | EBG_LEAF_BIT), its range [first, last] and is the parent of its children
__device__ __forceinline__ int prefixLen(const uint64_t* __restrict__ k, int64_t n, int64_t i, int64_t j)
{
  if (j < 0 || j >= n) {
    return -1;
  }
  const uint64_t a = k[i], b = k[j];
  return a != b ? __clzll(static_cast<long long>(a ^ b)) : 64 + __clz(static_cast<int>(uint32_t(i) ^ uint32_t(j)));
}

__global__ void kRadixTree(const uint64_t* __restrict__ k, int64_t n, uint32_t* __restrict__ left,
                           uint32_t* __restrict__ right, uint32_t* __restrict__ first, uint32_t* __restrict__ last,
                           uint32_t* __restrict__ parentI, uint32_t* __restrict__ parentL, int* __restrict__ err)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n - 1; i += int64_t(gridDim.x) * blockDim.x) {
    const int d    = prefixLen(k, n, i, i + 1) - prefixLen(k, n, i, i - 1) > 0 ? 1 : -1;
    const int dmin = prefixLen(k, n, i, i - d);
    int64_t   lmax = 2;
    while (prefixLen(k, n, i, i + lmax * d) > dmin) {
      lmax *= 2;
    }
    int64_t l = 0;
    for (int64_t t = lmax / 2; t >= 1; t /= 2) {
      if (prefixLen(k, n, i, i + (l + t) * d) > dmin) {
        l += t;
      }
    }
    const int64_t j     = i + l * d;
    const int     dnode = prefixLen(k, n, i, j);
    int64_t       s     = 0;
    for (int64_t t = (l + 1) / 2;; t = (t + 1) / 2) {
      if (prefixLen(k, n, i, i + (s + t) * d) > dnode) {
        s += t;
      }
      if (t == 1) {
        break;
      }
    }
    const int64_t g  = i + s * d + (d < 0 ? -1 : 0);
    const int64_t lo = i < j ? i : j, hi = i < j ? j : i;
    if (lo < 0 || hi >= n || g < lo || g + 1 > hi) {
      atomicOr(err, 4); // not a valid split: leave this node unwritten and report
      continue;
    }
    const uint32_t L = (lo == g) ? (EBG_LEAF_BIT | uint32_t(g)) : uint32_t(g);
    const uint32_t R = (hi == g + 1) ? (EBG_LEAF_BIT | uint32_t(g + 1)) : uint32_t(g + 1);
    left[i]  = L;
    right[i] = R;
    first[i] = uint32_t(lo);
    last[i]  = uint32_t(hi);
    if (L & EBG_LEAF_BIT) {
      parentL[L & ~EBG_LEAF_BIT] = uint32_t(i);
    }
    else {
      parentI[L] = uint32_t(i);
    }
    if (R & EBG_LEAF_BIT) {
      parentL[R & ~EBG_LEAF_BIT] = uint32_t(i);
    }
    else {
      parentI[R] = uint32_t(i);
    }
  }
}

// 3. FP64 boxes bottom-up.  Leaf boxes are the sorted triangles' boxes; an internal node's box is
// written by whichever of its two children's walks arrives second (the first leaves).
__device__ __forceinline__ void childBox(uint32_t ref, const double* leafLo, const double* leafHi,
                                         const double* nodeLo, const double* nodeHi, double* lo, double* hi)
{
  const double* l = (ref & EBG_LEAF_BIT) ? leafLo + 3 * size_t(ref & ~EBG_LEAF_BIT) : nodeLo + 3 * size_t(ref);
  const double* h = (ref & EBG_LEAF_BIT) ? leafHi + 3 * size_t(ref & ~EBG_LEAF_BIT) : nodeHi + 3 * size_t(ref);
  for (int a = 0; a < 3; a++) {
    lo[a] = __ldcg(l + a);
    hi[a] = __ldcg(h + a);
  }
}

__device__ __forceinline__ bool validRef(uint32_t ref, int64_t n)
{
  return (ref & EBG_LEAF_BIT) ? int64_t(ref & ~EBG_LEAF_BIT) < n : int64_t(ref) < n - 1;
}

__global__ void kRefit(int64_t n, const uint32_t* __restrict__ ids, const double* __restrict__ triLo,
                       const double* __restrict__ triHi, double* __restrict__ leafLo, double* __restrict__ leafHi,
                       const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                       const uint32_t* __restrict__ parentI, const uint32_t* __restrict__ parentL, double* nodeLo,
                       double* nodeHi, uint32_t* arrivals, int* __restrict__ err)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t f = ids[i];
    for (int a = 0; a < 3; a++) {
      leafLo[3 * i + a] = triLo[3 * size_t(f) + a];
      leafHi[3 * i + a] = triHi[3 * size_t(f) + a];
    }
    if (n == 1) {
      continue;
    }
    __threadfence();
    uint32_t p = parentL[i];
    // at most n - 1 ancestors
    for (int64_t step = 0; step < n; step++) {
      if (int64_t(p) >= n - 1 || !validRef(left[p], n) || !validRef(right[p], n)) {
        atomicOr(err, 8); // an unset or invalid link: stop and report
        break;
      }
      if (atomicAdd(arrivals + p, 1u) == 0u) {
        break; // the sibling's walk will write p
      }
      __threadfence();
      double l0[3], h0[3], l1[3], h1[3];
      childBox(left[p], leafLo, leafHi, nodeLo, nodeHi, l0, h0);
      childBox(right[p], leafLo, leafHi, nodeLo, nodeHi, l1, h1);
      for (int a = 0; a < 3; a++) {
        nodeLo[3 * size_t(p) + a] = fmin(l0[a], l1[a]);
        nodeHi[3 * size_t(p) + a] = fmax(h0[a], h1[a]);
      }
      __threadfence();
      if (p == 0) {
        break;
      }
      p = parentI[p];
    }
  }
}

struct TreeView
{
  int64_t         n; // triangles (leaves of the binary tree)
  const uint32_t* left;
  const uint32_t* right;
  const uint32_t* first;
  const uint32_t* last;
  const double*   nodeLo;
  const double*   nodeHi;
  const double*   leafLo;
  const double*   leafHi;
};

__device__ __forceinline__ uint32_t refCount(const TreeView& t, uint32_t ref)
{
  return (ref & EBG_LEAF_BIT) ? 1u : t.last[ref] - t.first[ref] + 1u;
}
// 2 (dx dy + dy dz + dz dx) with every operation rounded on its own, as the host build computes it
__device__ __forceinline__ double boxArea(const double* lo, const double* hi)
{
  const double dx = __dsub_rn(hi[0], lo[0]), dy = __dsub_rn(hi[1], lo[1]), dz = __dsub_rn(hi[2], lo[2]);
  return __dmul_rn(2.0, __dadd_rn(__dadd_rn(__dmul_rn(dx, dy), __dmul_rn(dy, dz)), __dmul_rn(dz, dx)));
}
__device__ __forceinline__ double refArea(const TreeView& t, uint32_t ref)
{
  double lo[3], hi[3];
  childBox(ref, t.leafLo, t.leafHi, t.nodeLo, t.nodeHi, lo, hi);
  return boxArea(lo, hi);
}

__device__ __forceinline__ float rdown(double x) { return __double2float_rd(x); }
__device__ __forceinline__ float rup(double x) { return __double2float_ru(x); }

// 4. one level of the 4-wide tree: frontier[i] = (binary ref, node index)
__global__ void kCollapse(const TreeView t, const uint2* __restrict__ frontier, uint32_t count, int leafSize,
                          EbgNode4* __restrict__ nodes, uint2* __restrict__ next, uint32_t* __restrict__ counters,
                          uint32_t* __restrict__ leafFirst, uint32_t* __restrict__ leafCount,
                          uint32_t* __restrict__ nodeFirst, uint32_t* __restrict__ nodeEnd,
                          uint32_t* __restrict__ nodeParent, uint32_t maxNodes, uint32_t maxLeaves, int* overflow)
{
  // counters: [0] nodes emitted so far, [1] leaves, [2] next frontier size
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < count; w += gridDim.x * blockDim.x) {
    const uint2 fr   = frontier[w];
    uint32_t    m[4] = {fr.x, NONE, NONE, NONE};
    int         nc   = 1;
    while (nc < 4) {
      int    pick = -1;
      double best = -1.0;
      for (int i = 0; i < nc; i++) {
        if (!(m[i] & EBG_LEAF_BIT) && refCount(t, m[i]) > uint32_t(leafSize)) {
          const double ar = refArea(t, m[i]);
          if (pick < 0 || ar > best) {
            pick = i;
            best = ar;
          }
        }
      }
      if (pick < 0) {
        break;
      }
      const uint32_t b = m[pick];
      m[pick]          = t.left[b];
      m[nc++]          = t.right[b];
    }
    bool bad = false;
    for (int i = 0; i < nc; i++) {
      bad = bad || !validRef(m[i], t.n);
    }
    if (bad || fr.y >= maxNodes) {
      atomicOr(overflow, 16);
      continue;
    }
    EbgNode4& nd = nodes[fr.y];
    for (int k = 0; k < 4; k++) {
      if (k >= nc) {
        nd.lox[k] = nd.loy[k] = nd.loz[k] = __int_as_float(0x7f800000);
        nd.hix[k] = nd.hiy[k] = nd.hiz[k] = -__int_as_float(0x7f800000);
        nd.child[k] = 0;
        nd.count[k] = 0;
        continue;
      }
      double lo[3], hi[3];
      childBox(m[k], t.leafLo, t.leafHi, t.nodeLo, t.nodeHi, lo, hi);
      nd.lox[k]            = rdown(lo[0]);
      nd.loy[k]            = rdown(lo[1]);
      nd.loz[k]            = rdown(lo[2]);
      nd.hix[k]            = rup(hi[0]);
      nd.hiy[k]            = rup(hi[1]);
      nd.hiz[k]            = rup(hi[2]);
      const uint32_t cnt   = refCount(t, m[k]);
      const uint32_t first = (m[k] & EBG_LEAF_BIT) ? (m[k] & ~EBG_LEAF_BIT) : t.first[m[k]];
      if (cnt <= uint32_t(leafSize)) {
        const uint32_t id = atomicAdd(counters + 1, 1u);
        if (id >= maxLeaves) {
          atomicOr(overflow, 1);
          nd.child[k] = 0;
          nd.count[k] = 0;
          continue;
        }
        nd.child[k]   = EBG_LEAF_BIT | first;
        nd.count[k]   = cnt | (id << EBG_COUNT_BITS);
        leafFirst[id] = first;
        leafCount[id] = cnt;
      }
      else {
        const uint32_t id = atomicAdd(counters + 0, 1u);
        if (id >= maxNodes) {
          atomicOr(overflow, 2);
          nd.child[k] = 0;
          nd.count[k] = 0;
          continue;
        }
        nd.child[k]    = id;
        nd.count[k]    = 0;
        nodeFirst[id]  = first;
        nodeEnd[id]    = first + cnt;
        nodeParent[id] = fr.y * 4u + uint32_t(k);
        const uint32_t q = atomicAdd(counters + 2, 1u);
        next[q]          = make_uint2(m[k], id);
      }
    }
  }
}

// 2-3 (SAH).  The binary tree of the host's binned-SAH build, level by level, one block per node
// range [b, e) of the current order: its FP64 box and centroid bounds; for each axis with extent,
// 32 centroid bins holding counts and FP64 triangle boxes (per-warp copies merged in warp order); the
// split of least cost A_L N_L + A_R N_R (the first minimum over axis, then bin); a stable partition
// of the range by bin.  Host and device compute the same doubles, so the tree is the host's.  A range
// of at most leafSize triangles keeps no children (the collapse makes it a leaf); a single triangle is
// a leaf reference.
struct SahTask
{
  uint32_t node, b, e;
};

constexpr int SAH_BINS    = 32;
constexpr int SAH_THREADS = 128;
constexpr int SAH_WARPS   = SAH_THREADS / 32;

__device__ __forceinline__ int sahBin(double c, double cl, double k)
{
  const int bi = int(__dmul_rn(__dsub_rn(c, cl), k));
  return bi < 0 ? 0 : (bi > SAH_BINS - 1 ? SAH_BINS - 1 : bi);
}

// The split of least SAH cost over the merged bins (cnt[axis][bin], box keys[axis][bin][6]): the first
// minimum over axis, then bin, among splits with both sides non-empty; axis -1 if none.
__device__ void sahBestSplit(const uint32_t (&cnt)[3][SAH_BINS], const unsigned long long (&box)[3][SAH_BINS][6],
                             const double k[3], int& outAxis, int& outBin)
{
  double bestCost = CUDART_INF;
  int    bestAxis = -1, bestBin = -1;
  for (int a = 0; a < 3; a++) {
    if (k[a] == 0.0) {
      continue;
    }
    double   rightArea[SAH_BINS];
    uint32_t rightCnt[SAH_BINS];
    double   al[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, ah[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    uint32_t c     = 0;
    for (int i = SAH_BINS - 1; i > 0; i--) {
      if (cnt[a][i] > 0) {
        for (int x = 0; x < 3; x++) {
          al[x] = fmin(al[x], dval(box[a][i][x]));
          ah[x] = fmax(ah[x], dval(box[a][i][3 + x]));
        }
      }
      c += cnt[a][i];
      rightArea[i] = c > 0 ? boxArea(al, ah) : 0.0;
      rightCnt[i]  = c;
    }
    double   ll[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, lh[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    uint32_t lc    = 0;
    for (int i = 0; i < SAH_BINS - 1; i++) {
      if (cnt[a][i] > 0) {
        for (int x = 0; x < 3; x++) {
          ll[x] = fmin(ll[x], dval(box[a][i][x]));
          lh[x] = fmax(lh[x], dval(box[a][i][3 + x]));
        }
      }
      lc += cnt[a][i];
      if (lc == 0 || rightCnt[i + 1] == 0) {
        continue;
      }
      const double cost =
        __dadd_rn(__dmul_rn(boxArea(ll, lh), double(lc)), __dmul_rn(rightArea[i + 1], double(rightCnt[i + 1])));
      if (cost < bestCost) {
        bestCost = cost;
        bestAxis = a;
        bestBin  = i;
      }
    }
  }
  outAxis = bestAxis;
  outBin  = bestBin;
}

// The two children of node `node` over [b, m) and [m, e): a single triangle is a leaf reference, a
// longer range a new internal node and a task of the next level.
__device__ void sahEmitChildren(uint32_t node, uint32_t b, uint32_t m, uint32_t e, uint32_t* left, uint32_t* right,
                                SahTask* next, uint32_t* counters, uint32_t maxNodes, int* err)
{
  uint32_t       ref[2];
  const uint32_t cb[2] = {b, m}, ce[2] = {m, e};
  for (int c = 0; c < 2; c++) {
    if (ce[c] - cb[c] == 1) {
      ref[c] = EBG_LEAF_BIT | cb[c];
    }
    else {
      const uint32_t id = atomicAdd(counters + 0, 1u);
      if (id >= maxNodes) {
        atomicOr(err, 32);
        ref[c] = EBG_LEAF_BIT | cb[c];
        continue;
      }
      ref[c]                            = id;
      next[atomicAdd(counters + 1, 1u)] = SahTask{id, cb[c], ce[c]};
    }
  }
  left[node]  = ref[0];
  right[node] = ref[1];
}

// Block-level binning of [b, e) (centroid bins along every axis with k != 0): per-warp bins in
// shared memory, merged in warp order into bcnt[0] / bbox[0].  Ends synchronised.
__device__ void sahBinRange(const uint32_t* __restrict__ ids, uint32_t b, uint32_t e, const double* __restrict__ cen,
                            const double* __restrict__ triLo, const double* __restrict__ triHi, const double cl[3],
                            const double k[3], uint32_t (&bcnt)[SAH_WARPS][3][SAH_BINS],
                            unsigned long long (&bbox)[SAH_WARPS][3][SAH_BINS][6])
{
  const int warp = threadIdx.x >> 5;
  for (int q = threadIdx.x; q < SAH_WARPS * 3 * SAH_BINS; q += SAH_THREADS) {
    const int w = q / (3 * SAH_BINS), r = q % (3 * SAH_BINS), a = r / SAH_BINS, bi = r % SAH_BINS;
    bcnt[w][a][bi] = 0;
    for (int c = 0; c < 3; c++) {
      bbox[w][a][bi][c]     = ~0ull;
      bbox[w][a][bi][3 + c] = 0ull;
    }
  }
  __syncthreads();
  for (uint32_t i = b + threadIdx.x; i < e; i += SAH_THREADS) {
    const size_t p = ids[i];
    for (int a = 0; a < 3; a++) {
      if (k[a] == 0.0) {
        continue;
      }
      const int bi = sahBin(cen[3 * p + a], cl[a], k[a]);
      atomicAdd(&bcnt[warp][a][bi], 1u);
      for (int c = 0; c < 3; c++) {
        atomicMin(&bbox[warp][a][bi][c], dkey(triLo[3 * p + c]));
        atomicMax(&bbox[warp][a][bi][3 + c], dkey(triHi[3 * p + c]));
      }
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < 3 * SAH_BINS; q += SAH_THREADS) {
    const int a = q / SAH_BINS, bi = q % SAH_BINS;
    for (int w = 1; w < SAH_WARPS; w++) {
      bcnt[0][a][bi] += bcnt[w][a][bi];
      for (int c = 0; c < 3; c++) {
        bbox[0][a][bi][c]     = min(bbox[0][a][bi][c], bbox[w][a][bi][c]);
        bbox[0][a][bi][3 + c] = max(bbox[0][a][bi][3 + c], bbox[w][a][bi][3 + c]);
      }
    }
  }
  __syncthreads();
}

// Block-level stable partition of ids[b, e) by (bin along ax <= bin): the left elements to
// tmp[dstL ...], the right ones to tmp[dstR ...], each side in its original order.  wl, wr: one
// shared slot per warp.  Ends synchronised.
__device__ void sahPartitionRange(const uint32_t* __restrict__ ids, uint32_t* __restrict__ tmp, uint32_t b,
                                  uint32_t e, uint32_t dstL, uint32_t dstR, const double* __restrict__ cen, double cla,
                                  double ka, int ax, int bin, uint32_t* wl, uint32_t* wr)
{
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t  offL = 0, offR = 0;
  for (uint32_t base = b; base < e; base += SAH_THREADS) {
    const uint32_t i     = base + threadIdx.x;
    const bool     valid = i < e;
    const uint32_t p     = valid ? ids[i] : 0u;
    const bool     isL   = valid && sahBin(cen[3 * size_t(p) + ax], cla, ka) <= bin;
    const unsigned bl    = __ballot_sync(FULL, isL);
    const unsigned br    = __ballot_sync(FULL, valid && !isL);
    if (lane == 0) {
      wl[warp] = __popc(bl);
      wr[warp] = __popc(br);
    }
    __syncthreads();
    uint32_t pl = offL, pr = offR, tl = 0, tr = 0;
    for (int w = 0; w < SAH_WARPS; w++) {
      if (w < warp) {
        pl += wl[w];
        pr += wr[w];
      }
      tl += wl[w];
      tr += wr[w];
    }
    const unsigned below = (1u << lane) - 1u;
    if (valid) {
      tmp[isL ? dstL + pl + __popc(bl & below) : dstR + pr + __popc(br & below)] = p;
    }
    offL += tl;
    offR += tr;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(SAH_THREADS) kSahLevel(const SahTask* __restrict__ tasks, uint32_t numTasks,
                                                         uint32_t* __restrict__ ids, uint32_t* __restrict__ tmp,
                                                         const double* __restrict__ triLo,
                                                         const double* __restrict__ triHi,
                                                         const double* __restrict__ cen, int leafSize,
                                                         uint32_t* __restrict__ left, uint32_t* __restrict__ right,
                                                         uint32_t* __restrict__ first, uint32_t* __restrict__ last,
                                                         double* __restrict__ nodeLo, double* __restrict__ nodeHi,
                                                         SahTask* __restrict__ next, uint32_t* __restrict__ counters,
                                                         uint32_t maxNodes, uint32_t bigMin, int* __restrict__ err)
{
  // per warp, axis and bin: count, and the bin's box as order-preserving keys (3 lo, 3 hi)
  __shared__ uint32_t           bcnt[SAH_WARPS][3][SAH_BINS];
  __shared__ unsigned long long bbox[SAH_WARPS][3][SAH_BINS][6];
  __shared__ double             red[SAH_WARPS];
  __shared__ int                sAxis, sBin;
  __shared__ uint32_t           wl[SAH_WARPS], wr[SAH_WARPS];
  const BlockGroup              g{red};

  for (uint32_t t = blockIdx.x; t < numTasks; t += gridDim.x) {
    const SahTask tk = tasks[t];
    const uint32_t b = tk.b, e = tk.e, n = e - b;
    if (n > bigMin) {
      continue; // a long range: the chunked kernels below take it
    }
    // the range's box and its centroids' bounds
    double lo[3], hi[3], cl[3], ch[3];
    for (int a = 0; a < 3; a++) {
      lo[a] = cl[a] = DBL_MAX;
      hi[a] = ch[a] = -DBL_MAX;
    }
    for (uint32_t i = b + threadIdx.x; i < e; i += SAH_THREADS) {
      const size_t p = ids[i];
      for (int a = 0; a < 3; a++) {
        lo[a] = fmin(lo[a], triLo[3 * p + a]);
        hi[a] = fmax(hi[a], triHi[3 * p + a]);
        cl[a] = fmin(cl[a], cen[3 * p + a]);
        ch[a] = fmax(ch[a], cen[3 * p + a]);
      }
    }
    for (int a = 0; a < 3; a++) {
      lo[a] = g.min(lo[a]);
      hi[a] = g.max(hi[a]);
      cl[a] = g.min(cl[a]);
      ch[a] = g.max(ch[a]);
    }
    if (threadIdx.x == 0) {
      for (int a = 0; a < 3; a++) {
        nodeLo[3 * size_t(tk.node) + a] = lo[a];
        nodeHi[3 * size_t(tk.node) + a] = hi[a];
      }
      first[tk.node] = b;
      last[tk.node]  = e - 1;
    }
    if (n <= uint32_t(leafSize)) {
      continue;
    }
    double k[3];
    for (int a = 0; a < 3; a++) {
      const double ext = __dsub_rn(ch[a], cl[a]);
      k[a]             = ext > 0.0 ? __ddiv_rn(double(SAH_BINS), ext) : 0.0;
    }
    sahBinRange(ids, b, e, cen, triLo, triHi, cl, k, bcnt, bbox);
    // the cheapest split: thread 0 scans the axes in order, as the host does
    if (threadIdx.x == 0) {
      sahBestSplit(bcnt[0], bbox[0], k, sAxis, sBin);
    }
    __syncthreads();
    const int ax = sAxis, bin = sBin;
    uint32_t  m  = b + n / 2; // every centroid the same point: halve
    if (ax >= 0) {
      // stable partition into tmp, then back
      uint32_t nl = 0;
      for (int i = 0; i <= bin; i++) {
        nl += bcnt[0][ax][i];
      }
      sahPartitionRange(ids, tmp, b, e, b, b + nl, cen, cl[ax], k[ax], ax, bin, wl, wr);
      for (uint32_t i = b + threadIdx.x; i < e; i += SAH_THREADS) {
        ids[i] = tmp[i];
      }
      m = b + nl;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      sahEmitChildren(tk.node, b, m, e, left, right, next, counters, maxNodes, err);
    }
    __syncthreads();
  }
}

// The ranges longer than SAH_BIG triangles: one entry per range, one per SAH_CHUNK-triangle piece,
// the same steps spread over many blocks (bounds, bins, split, stable partition by piece offsets);
// merged piece results are exact (sums of counts, minima and maxima), so the split is the single
// block's.
constexpr uint32_t SAH_BIG   = 32768;
constexpr uint32_t SAH_CHUNK = 8192;

struct SahBig
{
  uint32_t node, b, e, c0, nc; // the task, its span, its first piece and piece count
  int      ax, bin;
  uint32_t nl;
  double   cl[3], k[3];
};
struct SahChunk
{
  uint32_t big, b, e;
};
struct SahBins
{
  uint32_t           cnt[3][SAH_BINS];
  unsigned long long box[3][SAH_BINS][6];
};

__global__ void __launch_bounds__(SAH_THREADS) kSahChunkBounds(const SahChunk* __restrict__ chunks, uint32_t numChunks,
                                                               const uint32_t* __restrict__ ids,
                                                               const double* __restrict__ triLo,
                                                               const double* __restrict__ triHi,
                                                               const double* __restrict__ cen, double* __restrict__ part)
{
  __shared__ double red[SAH_WARPS];
  const BlockGroup  g{red};
  for (uint32_t c = blockIdx.x; c < numChunks; c += gridDim.x) {
    const SahChunk ck = chunks[c];
    double         v[12];
    for (int a = 0; a < 3; a++) {
      v[a] = v[6 + a] = DBL_MAX;
      v[3 + a] = v[9 + a] = -DBL_MAX;
    }
    for (uint32_t i = ck.b + threadIdx.x; i < ck.e; i += SAH_THREADS) {
      const size_t p = ids[i];
      for (int a = 0; a < 3; a++) {
        v[a]     = fmin(v[a], triLo[3 * p + a]);
        v[3 + a] = fmax(v[3 + a], triHi[3 * p + a]);
        v[6 + a] = fmin(v[6 + a], cen[3 * p + a]);
        v[9 + a] = fmax(v[9 + a], cen[3 * p + a]);
      }
    }
    for (int a = 0; a < 3; a++) {
      v[a]     = g.min(v[a]);
      v[3 + a] = g.max(v[3 + a]);
      v[6 + a] = g.min(v[6 + a]);
      v[9 + a] = g.max(v[9 + a]);
    }
    if (threadIdx.x == 0) {
      for (int q = 0; q < 12; q++) {
        part[12 * size_t(c) + q] = v[q];
      }
    }
    __syncthreads();
  }
}

__global__ void kSahBigBounds(SahBig* __restrict__ bigs, uint32_t numBig, const double* __restrict__ part,
                              uint32_t* __restrict__ first, uint32_t* __restrict__ last, double* __restrict__ nodeLo,
                              double* __restrict__ nodeHi)
{
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < numBig; t += gridDim.x * blockDim.x) {
    SahBig& bg = bigs[t];
    double  v[12];
    for (int a = 0; a < 3; a++) {
      v[a] = v[6 + a] = DBL_MAX;
      v[3 + a] = v[9 + a] = -DBL_MAX;
    }
    for (uint32_t c = bg.c0; c < bg.c0 + bg.nc; c++) {
      const double* pc = part + 12 * size_t(c);
      for (int a = 0; a < 3; a++) {
        v[a]     = fmin(v[a], pc[a]);
        v[3 + a] = fmax(v[3 + a], pc[3 + a]);
        v[6 + a] = fmin(v[6 + a], pc[6 + a]);
        v[9 + a] = fmax(v[9 + a], pc[9 + a]);
      }
    }
    for (int a = 0; a < 3; a++) {
      nodeLo[3 * size_t(bg.node) + a] = v[a];
      nodeHi[3 * size_t(bg.node) + a] = v[3 + a];
      bg.cl[a]                        = v[6 + a];
      const double ext                = __dsub_rn(v[9 + a], v[6 + a]);
      bg.k[a]                         = ext > 0.0 ? __ddiv_rn(double(SAH_BINS), ext) : 0.0;
    }
    first[bg.node] = bg.b;
    last[bg.node]  = bg.e - 1;
  }
}

__global__ void __launch_bounds__(SAH_THREADS) kSahChunkBins(const SahChunk* __restrict__ chunks, uint32_t numChunks,
                                                             const SahBig* __restrict__ bigs,
                                                             const uint32_t* __restrict__ ids,
                                                             const double* __restrict__ triLo,
                                                             const double* __restrict__ triHi,
                                                             const double* __restrict__ cen, SahBins* __restrict__ out)
{
  __shared__ uint32_t           bcnt[SAH_WARPS][3][SAH_BINS];
  __shared__ unsigned long long bbox[SAH_WARPS][3][SAH_BINS][6];
  for (uint32_t c = blockIdx.x; c < numChunks; c += gridDim.x) {
    const SahChunk ck = chunks[c];
    const SahBig&  bg = bigs[ck.big];
    const double   cl[3] = {bg.cl[0], bg.cl[1], bg.cl[2]}, k[3] = {bg.k[0], bg.k[1], bg.k[2]};
    sahBinRange(ids, ck.b, ck.e, cen, triLo, triHi, cl, k, bcnt, bbox);
    for (int q = threadIdx.x; q < 3 * SAH_BINS; q += SAH_THREADS) {
      const int a = q / SAH_BINS, bi = q % SAH_BINS;
      out[c].cnt[a][bi] = bcnt[0][a][bi];
      for (int x = 0; x < 6; x++) {
        out[c].box[a][bi][x] = bbox[0][a][bi][x];
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(SAH_THREADS) kSahBigSplit(SahBig* __restrict__ bigs, uint32_t numBig,
                                                            const SahBins* __restrict__ bins)
{
  __shared__ uint32_t           cnt[3][SAH_BINS];
  __shared__ unsigned long long box[3][SAH_BINS][6];
  __shared__ int                sAxis, sBin;
  for (uint32_t t = blockIdx.x; t < numBig; t += gridDim.x) {
    SahBig& bg = bigs[t];
    for (int q = threadIdx.x; q < 3 * SAH_BINS; q += SAH_THREADS) {
      const int          a = q / SAH_BINS, bi = q % SAH_BINS;
      uint32_t           n = 0;
      unsigned long long v[6] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull};
      for (uint32_t c = bg.c0; c < bg.c0 + bg.nc; c++) {
        n += bins[c].cnt[a][bi];
        for (int x = 0; x < 3; x++) {
          v[x]     = min(v[x], bins[c].box[a][bi][x]);
          v[3 + x] = max(v[3 + x], bins[c].box[a][bi][3 + x]);
        }
      }
      cnt[a][bi] = n;
      for (int x = 0; x < 6; x++) {
        box[a][bi][x] = v[x];
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const double k[3] = {bg.k[0], bg.k[1], bg.k[2]};
      sahBestSplit(cnt, box, k, sAxis, sBin);
      uint32_t nl = 0;
      if (sAxis >= 0) {
        for (int i = 0; i <= sBin; i++) {
          nl += cnt[sAxis][i];
        }
      }
      bg.ax  = sAxis;
      bg.bin = sBin;
      bg.nl  = nl;
    }
    __syncthreads();
  }
}

// each piece's left-element count, then each range's pieces' offsets in piece order
__global__ void __launch_bounds__(SAH_THREADS) kSahChunkCount(const SahChunk* __restrict__ chunks, uint32_t numChunks,
                                                              const SahBig* __restrict__ bigs,
                                                              const uint32_t* __restrict__ ids,
                                                              const double* __restrict__ cen,
                                                              uint32_t* __restrict__ chunkL)
{
  for (uint32_t c = blockIdx.x; c < numChunks; c += gridDim.x) {
    const SahChunk ck = chunks[c];
    const SahBig&  bg = bigs[ck.big];
    uint32_t       nL = 0;
    if (bg.ax >= 0) {
      for (uint32_t base = ck.b; base < ck.e; base += SAH_THREADS) {
        const uint32_t i   = base + threadIdx.x;
        const bool     isL = i < ck.e && sahBin(cen[3 * size_t(ids[i]) + bg.ax], bg.cl[bg.ax], bg.k[bg.ax]) <= bg.bin;
        nL += uint32_t(__syncthreads_count(isL));
      }
    }
    if (threadIdx.x == 0) {
      chunkL[c] = nL;
    }
    __syncthreads();
  }
}

__global__ void kSahBigOffsets(const SahBig* __restrict__ bigs, uint32_t numBig, const SahChunk* __restrict__ chunks,
                               const uint32_t* __restrict__ chunkL, uint32_t* __restrict__ offL,
                               uint32_t* __restrict__ offR)
{
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < numBig; t += gridDim.x * blockDim.x) {
    const SahBig& bg = bigs[t];
    uint32_t      l = 0, r = 0;
    for (uint32_t c = bg.c0; c < bg.c0 + bg.nc; c++) {
      offL[c] = l;
      offR[c] = r;
      l += chunkL[c];
      r += (chunks[c].e - chunks[c].b) - chunkL[c];
    }
  }
}

__global__ void __launch_bounds__(SAH_THREADS) kSahChunkScatter(const SahChunk* __restrict__ chunks,
                                                                uint32_t numChunks, const SahBig* __restrict__ bigs,
                                                                const uint32_t* __restrict__ ids,
                                                                uint32_t* __restrict__ tmp,
                                                                const double* __restrict__ cen,
                                                                const uint32_t* __restrict__ offL,
                                                                const uint32_t* __restrict__ offR)
{
  __shared__ uint32_t wl[SAH_WARPS], wr[SAH_WARPS];
  for (uint32_t c = blockIdx.x; c < numChunks; c += gridDim.x) {
    const SahChunk ck = chunks[c];
    const SahBig&  bg = bigs[ck.big];
    if (bg.ax < 0) {
      continue;
    }
    sahPartitionRange(ids, tmp, ck.b, ck.e, bg.b + offL[c], bg.b + bg.nl + offR[c], cen, bg.cl[bg.ax], bg.k[bg.ax],
                      bg.ax, bg.bin, wl, wr);
  }
}

__global__ void kSahChunkCopy(const SahChunk* __restrict__ chunks, uint32_t numChunks, const SahBig* __restrict__ bigs,
                              uint32_t* __restrict__ ids, const uint32_t* __restrict__ tmp)
{
  for (uint32_t c = blockIdx.x; c < numChunks; c += gridDim.x) {
    const SahChunk ck = chunks[c];
    if (bigs[ck.big].ax < 0) {
      continue;
    }
    for (uint32_t i = ck.b + threadIdx.x; i < ck.e; i += blockDim.x) {
      ids[i] = tmp[i];
    }
  }
}

__global__ void kSahBigChildren(const SahBig* __restrict__ bigs, uint32_t numBig, uint32_t* __restrict__ left,
                                uint32_t* __restrict__ right, SahTask* __restrict__ next,
                                uint32_t* __restrict__ counters, uint32_t maxNodes, int* __restrict__ err)
{
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < numBig; t += gridDim.x * blockDim.x) {
    const SahBig&  bg = bigs[t];
    const uint32_t m  = bg.ax >= 0 ? bg.b + bg.nl : bg.b + (bg.e - bg.b) / 2;
    sahEmitChildren(bg.node, bg.b, m, bg.e, left, right, next, counters, maxNodes, err);
  }
}

__global__ void kIota(uint32_t* __restrict__ ids, int64_t n)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    ids[i] = uint32_t(i);
  }
}

__global__ void kGatherLeafBoxes(int64_t n, const uint32_t* __restrict__ ids, const double* __restrict__ triLo,
                                 const double* __restrict__ triHi, double* __restrict__ leafLo,
                                 double* __restrict__ leafHi)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t f = ids[i];
    for (int a = 0; a < 3; a++) {
      leafLo[3 * i + a] = triLo[3 * size_t(f) + a];
      leafHi[3 * i + a] = triHi[3 * size_t(f) + a];
    }
  }
}

// 5a. leaf-ordered records
__global__ void kRecords(const double* __restrict__ V, const int32_t* __restrict__ F,
                         const double* __restrict__ triN, const double* __restrict__ cornerVN,
                         const double* __restrict__ edgeN, const uint32_t* __restrict__ ids, int64_t nt,
                         EbgTriHot* __restrict__ hot, EbgTriSign* __restrict__ sign, double* __restrict__ tri64,
                         int32_t* __restrict__ triId, double* __restrict__ dcelN, double* __restrict__ area)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nt; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t f = ids[i];
    triId[i]        = int32_t(f);
    const double* a = V + 3 * int64_t(F[3 * f]);
    const double* b = V + 3 * int64_t(F[3 * f + 1]);
    const double* c = V + 3 * int64_t(F[3 * f + 2]);
    const double  ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double  ac[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    EbgTriHot     h;
    h.v0x  = float(a[0]);
    h.v0y  = float(a[1]);
    h.v0z  = float(a[2]);
    h.abx  = float(ab[0]);
    h.aby  = float(ab[1]);
    h.abz  = float(ab[2]);
    h.acx  = float(ac[0]);
    h.acy  = float(ac[1]);
    h.acz  = float(ac[2]);
    h.ab2  = float(__dadd_rn(__dadd_rn(__dmul_rn(ab[0], ab[0]), __dmul_rn(ab[1], ab[1])), __dmul_rn(ab[2], ab[2])));
    h.abac = float(__dadd_rn(__dadd_rn(__dmul_rn(ab[0], ac[0]), __dmul_rn(ab[1], ac[1])), __dmul_rn(ab[2], ac[2])));
    h.ac2  = float(__dadd_rn(__dadd_rn(__dmul_rn(ac[0], ac[0]), __dmul_rn(ac[1], ac[1])), __dmul_rn(ac[2], ac[2])));
    hot[i] = h;
    EbgTriSign s;
    s.nx   = float(triN[3 * f]);
    s.ny   = float(triN[3 * f + 1]);
    s.nz   = float(triN[3 * f + 2]);
    s.pad0 = s.pad1 = s.pad2 = 0.f;
    for (int k = 0; k < 9; k++) {
      s.vn[k] = float(cornerVN[9 * f + k]);
      s.en[k] = float(edgeN[9 * f + k]);
    }
    sign[i]   = s;
    double* t = tri64 + 30 * i;
    for (int k = 0; k < 3; k++) {
      t[k]     = a[k];
      t[3 + k] = b[k];
      t[6 + k] = c[k];
      t[9 + k] = triN[3 * f + k];
    }
    for (int k = 0; k < 9; k++) {
      t[12 + k] = cornerVN[9 * f + k];
      t[21 + k] = edgeN[9 * f + k];
    }
    // the DCEL face normal: the Triangle normal normalised again (multiply by the reciprocal)
    const double* tn = triN + 3 * f;
    const double  is = __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(tn[0], tn[0]), __dmul_rn(tn[1], tn[1])),
                                                           __dmul_rn(tn[2], tn[2]))));
    for (int k = 0; k < 3; k++) {
      dcelN[3 * i + k] = __dmul_rn(is, tn[k]);
    }
    const double cx = ab[1] * ac[2] - ab[2] * ac[1], cy = ab[2] * ac[0] - ab[0] * ac[2],
                 cz = ab[0] * ac[1] - ab[1] * ac[0];
    area[i] = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
  }
}

// 5b. oriented box of the triangles at sorted positions [first, end).  The same construction as
// the host build (area-weighted mean normal, in-plane principal axis, padded extents) in FP64, in
// three passes over the range's vertices: (1) normal sum, area and axis-aligned box; (2) in-plane
// mean and covariance; (3) extents along the box's axes.  A range of at most SMALL_RANGE triangles
// (every leaf, most nodes) is one warp's; a larger one is cut into CHUNK-triangle pieces spread over
// blocks, whose partial results are combined per range in chunk order.  Every range's axis-aligned
// box is kept too (the child boxes of a refit come from it).
constexpr uint32_t SMALL_RANGE = 2048;
constexpr uint32_t CHUNK       = 4096;

// pass 1 over [b, e) of this thread's share: normal sum, area, axis-aligned box
template <class G>
__device__ void obbPass1(const double* __restrict__ tri64, uint32_t b, uint32_t e, const G& g, double n[3],
                         double& area, double lo[3], double hi[3])
{
  n[0] = n[1] = n[2] = 0;
  area               = 0;
  for (int a = 0; a < 3; a++) {
    lo[a] = DBL_MAX;
    hi[a] = -DBL_MAX;
  }
  for (uint32_t i = b + g.rank(); i < e; i += g.size()) {
    const double* t     = tri64 + 30 * size_t(i);
    const double  e1[3] = {t[3] - t[0], t[4] - t[1], t[5] - t[2]};
    const double  e2[3] = {t[6] - t[0], t[7] - t[1], t[8] - t[2]};
    const double  cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    for (int a = 0; a < 3; a++) {
      n[a] += cr[a];
      for (int c = 0; c < 3; c++) {
        lo[a] = fmin(lo[a], t[3 * c + a]);
        hi[a] = fmax(hi[a], t[3 * c + a]);
      }
    }
    area += sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  }
  for (int a = 0; a < 3; a++) {
    n[a]  = g.sum(n[a]);
    lo[a] = g.min(lo[a]);
    hi[a] = g.max(hi[a]);
  }
  area = g.sum(area);
}

// the box normal n (the mean normal, or the box's thinnest axis when the normals nearly cancel)
// and an in-plane frame t1, t2
__device__ void obbFrame(double n[3], double area, const double lo[3], const double hi[3], double t1[3], double t2[3])
{
  double ln = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  if (!(ln > 0.5 * area) || !(ln > 0)) {
    int ax = 0;
    for (int a = 1; a < 3; a++) {
      if (hi[a] - lo[a] < hi[ax] - lo[ax]) {
        ax = a;
      }
    }
    n[0] = n[1] = n[2] = 0;
    n[ax]              = 1;
    ln                 = 1;
  }
  for (int a = 0; a < 3; a++) {
    n[a] /= ln;
  }
  if (fabs(n[0]) < 0.9) {
    t1[0] = 0;
    t1[1] = n[2];
    t1[2] = -n[1];
  }
  else {
    t1[0] = -n[2];
    t1[1] = 0;
    t1[2] = n[0];
  }
  const double l1 = sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
  for (int a = 0; a < 3; a++) {
    t1[a] /= l1;
  }
  t2[0] = n[1] * t1[2] - n[2] * t1[1];
  t2[1] = n[2] * t1[0] - n[0] * t1[2];
  t2[2] = n[0] * t1[1] - n[1] * t1[0];
}

// pass 2: vertex sums in the frame, about (ox, oy) for accuracy: sx, sy, sxx, syy, sxy
template <class G>
__device__ void obbPass2(const double* __restrict__ tri64, uint32_t b, uint32_t e, const G& g, const double t1[3],
                         const double t2[3], double ox, double oy, double m[5])
{
  double sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0;
  for (uint32_t i = b + g.rank(); i < e; i += g.size()) {
    const double* t = tri64 + 30 * size_t(i);
    for (int c = 0; c < 3; c++) {
      const double* p = t + 3 * c;
      const double  x = p[0] * t1[0] + p[1] * t1[1] + p[2] * t1[2] - ox;
      const double  y = p[0] * t2[0] + p[1] * t2[1] + p[2] * t2[2] - oy;
      sx += x;
      sy += y;
      sxx += x * x;
      syy += y * y;
      sxy += x * y;
    }
  }
  m[0] = g.sum(sx);
  m[1] = g.sum(sy);
  m[2] = g.sum(sxx);
  m[3] = g.sum(syy);
  m[4] = g.sum(sxy);
}

// the in-plane principal axis u and w = n x u from pass 2's sums over cn vertices
__device__ void obbPrincipal(const double m[5], double cn, const double n[3], const double t1[3], const double t2[3],
                             double u[3], double w[3])
{
  const double mx = m[0] / cn, my = m[1] / cn;
  const double cxx = m[2] / cn - mx * mx, cyy = m[3] / cn - my * my, cxy = m[4] / cn - mx * my;
  const double th  = 0.5 * atan2(2 * cxy, cxx - cyy);
  for (int a = 0; a < 3; a++) {
    u[a] = cos(th) * t1[a] + sin(th) * t2[a];
  }
  w[0] = n[1] * u[2] - n[2] * u[1];
  w[1] = n[2] * u[0] - n[0] * u[2];
  w[2] = n[0] * u[1] - n[1] * u[0];
}

// pass 3: extents of the vertices along n, u, w
template <class G>
__device__ void obbPass3(const double* __restrict__ tri64, uint32_t b, uint32_t e, const G& g, const double n[3],
                         const double u[3], const double w[3], double mn[3], double mx[3])
{
  for (int a = 0; a < 3; a++) {
    mn[a] = DBL_MAX;
    mx[a] = -DBL_MAX;
  }
  for (uint32_t i = b + g.rank(); i < e; i += g.size()) {
    const double* t = tri64 + 30 * size_t(i);
    for (int c = 0; c < 3; c++) {
      const double* p     = t + 3 * c;
      const double  pr[3] = {p[0] * n[0] + p[1] * n[1] + p[2] * n[2], p[0] * u[0] + p[1] * u[1] + p[2] * u[2],
                             p[0] * w[0] + p[1] * w[1] + p[2] * w[2]};
      for (int a = 0; a < 3; a++) {
        mn[a] = fmin(mn[a], pr[a]);
        mx[a] = fmax(mx[a], pr[a]);
      }
    }
  }
  for (int a = 0; a < 3; a++) {
    mn[a] = g.min(mn[a]);
    mx[a] = g.max(mx[a]);
  }
}

// the padded box, whether it is worth testing (at most half the axis-aligned box's volume), and the
// axis-aligned box itself
__device__ void obbStore(const double n[3], const double u[3], const double w[3], const double mn[3],
                         const double mx[3], const double lo[3], const double hi[3], double pad, EbgObb* out,
                         uint8_t* useful, double* aabb)
{
  EbgObb o;
  o.nx  = float(n[0]);
  o.ny  = float(n[1]);
  o.nz  = float(n[2]);
  o.dn  = float(0.5 * (mn[0] + mx[0]));
  o.ux  = float(u[0]);
  o.uy  = float(u[1]);
  o.uz  = float(u[2]);
  o.du  = float(0.5 * (mn[1] + mx[1]));
  o.vx  = float(w[0]);
  o.vy  = float(w[1]);
  o.vz  = float(w[2]);
  o.dv  = float(0.5 * (mn[2] + mx[2]));
  o.hn  = rup(0.5 * (mx[0] - mn[0]) + pad);
  o.hu  = rup(0.5 * (mx[1] - mn[1]) + pad);
  o.hv  = rup(0.5 * (mx[2] - mn[2]) + pad);
  o.pad = 0.f;
  *out  = o;
  if (useful) {
    const double obbVol  = 8.0 * double(o.hn) * double(o.hu) * double(o.hv);
    const double aabbVol = (hi[0] - lo[0] + 2 * pad) * (hi[1] - lo[1] + 2 * pad) * (hi[2] - lo[2] + 2 * pad);
    *useful              = (aabbVol > 0 ? obbVol / aabbVol : 1.0) <= 0.5 ? 1 : 0;
  }
  if (aabb) {
    for (int a = 0; a < 3; a++) {
      aabb[a]     = lo[a];
      aabb[3 + a] = hi[a];
    }
  }
}

// the ranges of at most SMALL_RANGE triangles, [rFirst[r], rEnd[r]) or rFirst[r] + rCount[r]: a warp each
__global__ void __launch_bounds__(128) kRangeObbsSmall(const double* __restrict__ tri64,
                                                       const uint32_t* __restrict__ rFirst,
                                                       const uint32_t* __restrict__ rEnd,
                                                       const uint32_t* __restrict__ rCount, int64_t numRanges,
                                                       double pad, EbgObb* __restrict__ out,
                                                       uint8_t* __restrict__ useful, double* __restrict__ aabb)
{
  const int64_t   nWarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const WarpGroup g;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < numRanges; r += nWarps) {
    const uint32_t b = rFirst[r];
    const uint32_t e = rEnd ? rEnd[r] : b + rCount[r];
    if (e - b > SMALL_RANGE) {
      continue;
    }
    double n[3], area, lo[3], hi[3], t1[3], t2[3], m[5], u[3], w[3], mn[3], mx[3];
    obbPass1(tri64, b, e, g, n, area, lo, hi);
    obbFrame(n, area, lo, hi, t1, t2);
    const double* t0 = tri64 + 30 * size_t(b);
    const double  ox = t0[0] * t1[0] + t0[1] * t1[1] + t0[2] * t1[2], oy = t0[0] * t2[0] + t0[1] * t2[1] + t0[2] * t2[2];
    obbPass2(tri64, b, e, g, t1, t2, ox, oy, m);
    obbPrincipal(m, 3.0 * double(e - b), n, t1, t2, u, w);
    obbPass3(tri64, b, e, g, n, u, w, mn, mx);
    if (g.rank() == 0) {
      obbStore(n, u, w, mn, mx, lo, hi, pad, out + r, useful ? useful + r : nullptr, aabb ? aabb + 6 * r : nullptr);
    }
  }
}

// the larger ranges: one entry per range, one per CHUNK-triangle piece of it
struct ObbRange
{
  uint32_t r, b, e, c0, nc; // range index, its span, its first chunk and chunk count
};
struct ObbChunk
{
  uint32_t lr, b, e; // large-range entry, the piece's span
};
struct ObbFrameState
{
  double n[3], t1[3], t2[3], u[3], w[3], lo[3], hi[3], ox, oy;
};

template <int PASS>
__global__ void __launch_bounds__(128) kObbChunks(const double* __restrict__ tri64, const ObbChunk* __restrict__ chunks,
                                                  uint32_t numChunks, const ObbFrameState* __restrict__ frames,
                                                  double* __restrict__ part)
{
  __shared__ double red[4];
  const BlockGroup  g{red};
  for (uint32_t c = blockIdx.x; c < numChunks; c += gridDim.x) {
    const ObbChunk ch = chunks[c];
    double*        pc = part + 10 * size_t(c);
    if (PASS == 1) {
      double n[3], area, lo[3], hi[3];
      obbPass1(tri64, ch.b, ch.e, g, n, area, lo, hi);
      if (threadIdx.x == 0) {
        for (int a = 0; a < 3; a++) {
          pc[a]     = n[a];
          pc[4 + a] = lo[a];
          pc[7 + a] = hi[a];
        }
        pc[3] = area;
      }
    }
    else if (PASS == 2) {
      const ObbFrameState& f = frames[ch.lr];
      double               m[5];
      obbPass2(tri64, ch.b, ch.e, g, f.t1, f.t2, f.ox, f.oy, m);
      if (threadIdx.x == 0) {
        for (int k = 0; k < 5; k++) {
          pc[k] = m[k];
        }
      }
    }
    else {
      const ObbFrameState& f = frames[ch.lr];
      double               mn[3], mx[3];
      obbPass3(tri64, ch.b, ch.e, g, f.n, f.u, f.w, mn, mx);
      if (threadIdx.x == 0) {
        for (int a = 0; a < 3; a++) {
          pc[a]     = mn[a];
          pc[3 + a] = mx[a];
        }
      }
    }
    __syncthreads();
  }
}

template <int PASS>
__global__ void kObbRanges(const double* __restrict__ tri64, const ObbRange* __restrict__ ranges, uint32_t numLarge,
                           const double* __restrict__ part, ObbFrameState* __restrict__ frames, double pad,
                           EbgObb* __restrict__ out, uint8_t* __restrict__ useful, double* __restrict__ aabb)
{
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < numLarge; l += gridDim.x * blockDim.x) {
    const ObbRange rg = ranges[l];
    ObbFrameState& f  = frames[l];
    if (PASS == 1) {
      double n[3] = {0, 0, 0}, area = 0, lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
      for (uint32_t c = rg.c0; c < rg.c0 + rg.nc; c++) {
        const double* pc = part + 10 * size_t(c);
        for (int a = 0; a < 3; a++) {
          n[a] += pc[a];
          lo[a] = fmin(lo[a], pc[4 + a]);
          hi[a] = fmax(hi[a], pc[7 + a]);
        }
        area += pc[3];
      }
      obbFrame(n, area, lo, hi, f.t1, f.t2);
      for (int a = 0; a < 3; a++) {
        f.n[a]  = n[a];
        f.lo[a] = lo[a];
        f.hi[a] = hi[a];
      }
      const double* t0 = tri64 + 30 * size_t(rg.b);
      f.ox             = t0[0] * f.t1[0] + t0[1] * f.t1[1] + t0[2] * f.t1[2];
      f.oy             = t0[0] * f.t2[0] + t0[1] * f.t2[1] + t0[2] * f.t2[2];
    }
    else if (PASS == 2) {
      double m[5] = {0, 0, 0, 0, 0};
      for (uint32_t c = rg.c0; c < rg.c0 + rg.nc; c++) {
        for (int k = 0; k < 5; k++) {
          m[k] += part[10 * size_t(c) + k];
        }
      }
      obbPrincipal(m, 3.0 * double(rg.e - rg.b), f.n, f.t1, f.t2, f.u, f.w);
    }
    else {
      double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
      for (uint32_t c = rg.c0; c < rg.c0 + rg.nc; c++) {
        for (int a = 0; a < 3; a++) {
          mn[a] = fmin(mn[a], part[10 * size_t(c) + a]);
          mx[a] = fmax(mx[a], part[10 * size_t(c) + 3 + a]);
        }
      }
      obbStore(f.n, f.u, f.w, mn, mx, f.lo, f.hi, pad, out + rg.r, useful ? useful + rg.r : nullptr,
               aabb ? aabb + 6 * size_t(rg.r) : nullptr);
    }
  }
}

__global__ void kNodeObbFlags(const uint8_t* __restrict__ useful, const uint32_t* __restrict__ nodeParent,
                              uint32_t numNodes, EbgNode4* __restrict__ nodes)
{
  for (uint32_t j = 1 + blockIdx.x * blockDim.x + threadIdx.x; j < numNodes; j += gridDim.x * blockDim.x) {
    if (useful[j]) {
      const uint32_t ps = nodeParent[j];
      nodes[ps >> 2].count[ps & 3u] = EBG_NODE_HAS_OBB;
    }
  }
}

// 6. refit (moved vertices, same tree): each node's four child boxes, rounded outward to FP32, from
// the axis-aligned boxes of the children's ranges (leafAabb per leaf id, nodeAabb per node; 6 doubles
// each), and an interior slot's oriented-box flag from `useful`.
__global__ void kSlotBoxes(const double* __restrict__ leafAabb, const double* __restrict__ nodeAabb,
                           const uint8_t* __restrict__ useful, uint32_t numNodes, uint32_t numLeaves,
                           EbgNode4* __restrict__ nodes)
{
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < 4 * numNodes; q += gridDim.x * blockDim.x) {
    EbgNode4&      nd  = nodes[q >> 2];
    const int      k   = int(q & 3u);
    const uint32_t c   = nd.child[k];
    const uint32_t cnt = nd.count[k];
    const double*  bx;
    if (c & EBG_LEAF_BIT) {
      const uint32_t leaf = cnt >> EBG_COUNT_BITS;
      if (leaf >= numLeaves) {
        continue;
      }
      bx = leafAabb + 6 * size_t(leaf);
    }
    else if (c != 0 && c < numNodes) {
      bx                  = nodeAabb + 6 * size_t(c);
      nd.count[k]         = useful[c] ? EBG_NODE_HAS_OBB : 0u;
    }
    else {
      continue; // an empty slot (node 0 is the root, never a child)
    }
    nd.lox[k] = rdown(bx[0]);
    nd.loy[k] = rdown(bx[1]);
    nd.loz[k] = rdown(bx[2]);
    nd.hix[k] = rup(bx[3]);
    nd.hiy[k] = rup(bx[4]);
    nd.hiz[k] = rup(bx[5]);
  }
}

// the normals of the FP64 records (leaf order) back in soup order: out = [face 3N | corner 9N | edge 9N]
__global__ void kGatherNormals(const double* __restrict__ tri64, const int32_t* __restrict__ triId, int64_t n,
                               double* __restrict__ out)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t f = triId[i];
    const double* t = tri64 + 30 * i;
    for (int k = 0; k < 3; k++) {
      out[3 * f + k] = t[9 + k];
    }
    for (int k = 0; k < 9; k++) {
      out[3 * n + 9 * f + k]  = t[12 + k];
      out[12 * n + 9 * f + k] = t[21 + k];
    }
  }
}

__global__ void kAllFinite(const double* __restrict__ v, int64_t n, int* __restrict__ bad)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    if (!isfinite(v[i])) {
      *bad = 1;
    }
  }
}

inline unsigned gridFor(int64_t n, int t, int64_t cap = 1 << 20)
{
  int64_t g = (n + t - 1) / t;
  g         = g < cap ? g : cap;
  return unsigned(g < 1 ? 1 : g);
}

// Oriented boxes (and, with aabb, the axis-aligned boxes) of nr ranges of leaf positions,
// [first[r], end[r]) or first[r] + count[r], device arrays.  With mayBeLong the range arrays are
// read back once to find the ranges of more than SMALL_RANGE triangles and cut them into chunks
// (the call then synchronises s).
ebg_status rangeObbs(const double* tri64, const uint32_t* first, const uint32_t* end, const uint32_t* count,
                     uint32_t nr, bool mayBeLong, double pad, EbgObb* out, uint8_t* useful, double* aabb, int numSms,
                     cudaStream_t s)
{
  if (nr == 0) {
    return EBG_OK;
  }
  kRangeObbsSmall<<<gridFor(nr, 4, 1 << 20), 128, 0, s>>>(tri64, first, end, count, nr, pad, out, useful, aabb);
  if (!mayBeLong) {
    return EBG_OK;
  }
  std::vector<uint32_t> hf(nr), he(nr);
  cudaMemcpyAsync(hf.data(), first, 4 * size_t(nr), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(he.data(), end ? end : count, 4 * size_t(nr), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("oriented boxes: ") + cudaGetErrorString(cudaGetLastError()));
  }
  std::vector<ObbRange> lr;
  std::vector<ObbChunk> ch;
  for (uint32_t r = 0; r < nr; r++) {
    const uint32_t b = hf[r], e = end ? he[r] : hf[r] + he[r];
    if (e - b <= SMALL_RANGE) {
      continue;
    }
    ObbRange x{r, b, e, uint32_t(ch.size()), 0u};
    for (uint32_t c = b; c < e; c += CHUNK) {
      ch.push_back(ObbChunk{uint32_t(lr.size()), c, std::min(c + CHUNK, e)});
      x.nc++;
    }
    lr.push_back(x);
  }
  if (lr.empty()) {
    return EBG_OK;
  }
  const uint32_t nl = uint32_t(lr.size()), nc = uint32_t(ch.size());
  ObbRange*      dR = nullptr;
  ObbChunk*      dC = nullptr;
  ObbFrameState* dF = nullptr;
  double*        dP = nullptr;
  const bool ok = cudaMallocAsync((void**)&dR, sizeof(ObbRange) * nl, s) == cudaSuccess &&
                  cudaMallocAsync((void**)&dC, sizeof(ObbChunk) * nc, s) == cudaSuccess &&
                  cudaMallocAsync((void**)&dF, sizeof(ObbFrameState) * nl, s) == cudaSuccess &&
                  cudaMallocAsync((void**)&dP, 80 * size_t(nc), s) == cudaSuccess;
  if (ok) {
    cudaMemcpyAsync(dR, lr.data(), sizeof(ObbRange) * nl, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dC, ch.data(), sizeof(ObbChunk) * nc, cudaMemcpyHostToDevice, s);
    const unsigned gc = gridFor(nc, 1, int64_t(numSms) * 8), gr = gridFor(nl, 128);
    kObbChunks<1><<<gc, 128, 0, s>>>(tri64, dC, nc, dF, dP);
    kObbRanges<1><<<gr, 128, 0, s>>>(tri64, dR, nl, dP, dF, pad, out, useful, aabb);
    kObbChunks<2><<<gc, 128, 0, s>>>(tri64, dC, nc, dF, dP);
    kObbRanges<2><<<gr, 128, 0, s>>>(tri64, dR, nl, dP, dF, pad, out, useful, aabb);
    kObbChunks<3><<<gc, 128, 0, s>>>(tri64, dC, nc, dF, dP);
    kObbRanges<3><<<gr, 128, 0, s>>>(tri64, dR, nl, dP, dF, pad, out, useful, aabb);
  }
  for (void* p : {(void*)dR, (void*)dC, (void*)dF, (void*)dP}) {
    if (p) {
      cudaFreeAsync(p, s);
    }
  }
  if (!ok) {
    cudaGetLastError();
    return setError(EBG_ERR_NO_MEMORY, "oriented-box workspace");
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? EBG_OK : setError(EBG_ERR_CUDA, std::string("oriented boxes: ") + cudaGetErrorString(e));
}

} // namespace

ebg_status buildMeshOnDevice(ebg_mesh* m, const double* V, int64_t nv, const int32_t* F, int64_t nt, int build,
                             int leafSize, double* outLo, double* outHi, cudaStream_t s, bool normalsOnDevice)
{
  const int64_t n = nt;
  std::vector<void*> tmp;
  auto alloc = [&](void** p, size_t bytes) -> bool {
    if (cudaMallocAsync(p, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
      return false;
    }
    tmp.push_back(*p);
    return true;
  };
  auto freeTmp = [&]() {
    for (void* p : tmp) {
      cudaFreeAsync(p, s);
    }
    tmp.clear();
  };
  struct Guard
  {
    std::function<void()> f;
    ~Guard() { f(); }
  } guard{freeTmp};

  double *dV = nullptr, *dTriN = nullptr, *dVN = nullptr, *dEN = nullptr, *triLo = nullptr, *triHi = nullptr,
         *cen = nullptr, *leafLo = nullptr, *leafHi = nullptr, *nodeLo = nullptr, *nodeHi = nullptr, *area = nullptr;
  int32_t*            dF     = nullptr;
  unsigned long long* bounds = nullptr;
  uint64_t *          codesIn = nullptr, *codesOut = nullptr;
  uint32_t *idsIn = nullptr, *ids = nullptr, *left = nullptr, *right = nullptr, *first = nullptr, *last = nullptr,
           *parentI = nullptr, *parentL = nullptr, *arrivals = nullptr, *counters = nullptr, *leafFirst = nullptr,
           *leafCount = nullptr, *nodeFirst = nullptr, *nodeEnd = nullptr, *nodeParent = nullptr;
  uint2*   frontier[2] = {nullptr, nullptr};
  uint8_t* useful      = nullptr;
  int*     overflow    = nullptr;
  const size_t N = size_t(n), NI = size_t(std::max<int64_t>(n - 1, 1));
  bool ok = alloc((void**)&dV, 24 * size_t(nv)) && alloc((void**)&dF, 12 * N) && alloc((void**)&dTriN, 24 * N) &&
            alloc((void**)&dVN, 72 * N) && alloc((void**)&dEN, 72 * N) && alloc((void**)&triLo, 24 * N) &&
            alloc((void**)&triHi, 24 * N) && alloc((void**)&cen, 24 * N) && alloc((void**)&leafLo, 24 * N) &&
            alloc((void**)&leafHi, 24 * N) && alloc((void**)&nodeLo, 24 * NI) && alloc((void**)&nodeHi, 24 * NI) &&
            alloc((void**)&area, 8 * N) && alloc((void**)&bounds, 12 * 8) && alloc((void**)&codesIn, 8 * N) &&
            alloc((void**)&codesOut, 8 * N) && alloc((void**)&idsIn, 4 * N) && alloc((void**)&ids, 4 * N) &&
            alloc((void**)&left, 4 * NI) && alloc((void**)&right, 4 * NI) && alloc((void**)&first, 4 * NI) &&
            alloc((void**)&last, 4 * NI) && alloc((void**)&parentI, 4 * NI) && alloc((void**)&parentL, 4 * N) &&
            alloc((void**)&arrivals, 4 * NI) && alloc((void**)&counters, 16) && alloc((void**)&leafFirst, 4 * N) &&
            alloc((void**)&leafCount, 4 * N) && alloc((void**)&nodeFirst, 4 * N) && alloc((void**)&nodeEnd, 4 * N) &&
            alloc((void**)&nodeParent, 4 * N) && alloc((void**)&frontier[0], 8 * N) &&
            alloc((void**)&frontier[1], 8 * N) && alloc((void**)&useful, N) && alloc((void**)&overflow, 4);
  if (!ok) {
    return setError(EBG_ERR_NO_MEMORY, "device build workspace");
  }
  cudaMemcpyAsync(dV, V, 24 * size_t(nv), cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(dF, F, 12 * N, cudaMemcpyHostToDevice, s);
  if (normalsOnDevice) {
    const ebg_status rc = pseudonormalsOnDevice(dV, nv, dF, nt, dTriN, dVN, dEN, s);
    if (rc != EBG_OK) {
      return rc;
    }
  }
  else {
    cudaMemcpyAsync(dTriN, m->triN.data(), 24 * N, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dVN, m->cornerVN.data(), 72 * N, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dEN, m->edgeN.data(), 72 * N, cudaMemcpyHostToDevice, s);
  }
  {
    unsigned long long init[12];
    for (int j = 0; j < 12; j++) {
      const bool isMin = (j < 3) || (j >= 6 && j < 9);
      init[j]          = isMin ? ~0ull : 0ull;
    }
    cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, s);
  }
  cudaMemsetAsync(arrivals, 0, 4 * NI, s);
  cudaMemsetAsync(parentI, 0xff, 4 * NI, s);
  cudaMemsetAsync(left, 0xff, 4 * NI, s);
  cudaMemsetAsync(right, 0xff, 4 * NI, s);
  cudaMemsetAsync(parentL, 0xff, 4 * N, s);
  cudaMemsetAsync(counters, 0, 16, s);
  cudaMemsetAsync(overflow, 0, 4, s);
  cudaMemsetAsync(useful, 0, N, s);

  // 1. boxes, bounds, codes, sort
  kTriBounds<<<gridFor(n, 256, 8192), 256, 0, s>>>(dV, dF, n, triLo, triHi, cen, bounds);
  if (build == EBG_BUILD_SAH) {
    // 2-3 (SAH): the binary tree top-down, one launch per level, in place of codes, sort and refit
    const size_t maxTasks = N / 2 + 1;
    SahTask*     tasks[2] = {nullptr, nullptr};
    if (!alloc((void**)&tasks[0], sizeof(SahTask) * maxTasks) || !alloc((void**)&tasks[1], sizeof(SahTask) * maxTasks)) {
      return setError(EBG_ERR_NO_MEMORY, "device build workspace");
    }
    kIota<<<gridFor(n, 256), 256, 0, s>>>(ids, n);
    if (n > leafSize) {
      const SahTask  root{0u, 0u, uint32_t(n)};
      const uint32_t init[2] = {1u, 0u};
      cudaMemcpyAsync(tasks[0], &root, sizeof(root), cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(counters, init, sizeof(init), cudaMemcpyHostToDevice, s);
      uint32_t count  = 1;
      int      cur    = 0;
      bool     mayBig = uint64_t(n) > SAH_BIG;
      for (int level = 0; count > 0; level++) {
        if (level > 256) {
          return setError(EBG_ERR_INVALID, "device SAH build: tree deeper than 256 levels");
        }
        // the level's long ranges (only the first few levels have any), cut into pieces
        std::vector<SahBig>   bigs;
        std::vector<SahChunk> chunks;
        if (mayBig) {
          std::vector<SahTask> ht(count);
          cudaMemcpyAsync(ht.data(), tasks[cur], sizeof(SahTask) * count, cudaMemcpyDeviceToHost, s);
          if (cudaStreamSynchronize(s) != cudaSuccess) {
            return setError(EBG_ERR_CUDA, std::string("device SAH build: ") + cudaGetErrorString(cudaGetLastError()));
          }
          for (const SahTask& t : ht) {
            if (t.e - t.b <= SAH_BIG) {
              continue;
            }
            SahBig bg{};
            bg.node = t.node;
            bg.b    = t.b;
            bg.e    = t.e;
            bg.c0   = uint32_t(chunks.size());
            for (uint32_t c = t.b; c < t.e; c += SAH_CHUNK) {
              chunks.push_back(SahChunk{uint32_t(bigs.size()), c, std::min(c + SAH_CHUNK, t.e)});
              bg.nc++;
            }
            bg.ax = -1;
            bigs.push_back(bg);
          }
          mayBig = !bigs.empty(); // ranges only shrink
        }
        cudaMemsetAsync(counters + 1, 0, 4, s);
        kSahLevel<<<gridFor(count, 1, 1 << 16), SAH_THREADS, 0, s>>>(
          tasks[cur], count, ids, idsIn, triLo, triHi, cen, leafSize, left, right, first, last, nodeLo, nodeHi,
          tasks[1 - cur], counters, uint32_t(NI), bigs.empty() ? UINT32_MAX : SAH_BIG, overflow);
        if (!bigs.empty()) {
          const uint32_t nb = uint32_t(bigs.size()), nc = uint32_t(chunks.size());
          SahBig*        dBig = nullptr;
          SahChunk*      dCh  = nullptr;
          double*        part = nullptr;
          SahBins*       bins = nullptr;
          uint32_t *     cL = nullptr, *oL = nullptr, *oR = nullptr;
          if (!alloc((void**)&dBig, sizeof(SahBig) * nb) || !alloc((void**)&dCh, sizeof(SahChunk) * nc) ||
              !alloc((void**)&part, 96 * size_t(nc)) || !alloc((void**)&bins, sizeof(SahBins) * nc) ||
              !alloc((void**)&cL, 4 * size_t(nc)) || !alloc((void**)&oL, 4 * size_t(nc)) ||
              !alloc((void**)&oR, 4 * size_t(nc))) {
            return setError(EBG_ERR_NO_MEMORY, "device SAH build workspace");
          }
          cudaMemcpyAsync(dBig, bigs.data(), sizeof(SahBig) * nb, cudaMemcpyHostToDevice, s);
          cudaMemcpyAsync(dCh, chunks.data(), sizeof(SahChunk) * nc, cudaMemcpyHostToDevice, s);
          const unsigned gb = gridFor(nb, 128);
          kSahChunkBounds<<<nc, SAH_THREADS, 0, s>>>(dCh, nc, ids, triLo, triHi, cen, part);
          kSahBigBounds<<<gb, 128, 0, s>>>(dBig, nb, part, first, last, nodeLo, nodeHi);
          kSahChunkBins<<<nc, SAH_THREADS, 0, s>>>(dCh, nc, dBig, ids, triLo, triHi, cen, bins);
          kSahBigSplit<<<nb, SAH_THREADS, 0, s>>>(dBig, nb, bins);
          kSahChunkCount<<<nc, SAH_THREADS, 0, s>>>(dCh, nc, dBig, ids, cen, cL);
          kSahBigOffsets<<<gb, 128, 0, s>>>(dBig, nb, dCh, cL, oL, oR);
          kSahChunkScatter<<<nc, SAH_THREADS, 0, s>>>(dCh, nc, dBig, ids, idsIn, cen, oL, oR);
          kSahChunkCopy<<<nc, 256, 0, s>>>(dCh, nc, dBig, ids, idsIn);
          kSahBigChildren<<<gb, 128, 0, s>>>(dBig, nb, left, right, tasks[1 - cur], counters, uint32_t(NI), overflow);
        }
        uint32_t hc[2];
        cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) {
          return setError(EBG_ERR_CUDA, std::string("device SAH build: ") + cudaGetErrorString(cudaGetLastError()));
        }
        count = hc[1];
        cur   = 1 - cur;
      }
    }
    kGatherLeafBoxes<<<gridFor(n, 256), 256, 0, s>>>(n, ids, triLo, triHi, leafLo, leafHi);
  }
  else {
  kTriMorton<<<gridFor(n, 256), 256, 0, s>>>(cen, n, bounds, codesIn, idsIn);
  size_t sortBytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sortBytes, codesIn, codesOut, idsIn, ids, int(n), 0, 63, s);
  void* sortTemp = nullptr;
  if (!alloc(&sortTemp, sortBytes)) {
    return setError(EBG_ERR_NO_MEMORY, "device build sort workspace");
  }
  if (cub::DeviceRadixSort::SortPairs(sortTemp, sortBytes, codesIn, codesOut, idsIn, ids, int(n), 0, 63, s) !=
      cudaSuccess) {
    return setError(EBG_ERR_CUDA, "device build sort failed");
  }

  // 2-3. binary radix tree and its boxes
  if (n > 1) {
    kRadixTree<<<gridFor(n - 1, 256), 256, 0, s>>>(codesOut, n, left, right, first, last, parentI, parentL, overflow);
  }
  kRefit<<<gridFor(n, 256), 256, 0, s>>>(n, ids, triLo, triHi, leafLo, leafHi, left, right, parentI, parentL, nodeLo,
                                         nodeHi, arrivals, overflow);
  }

  // root box (the whole mesh)
  unsigned long long hb[12];
  cudaMemcpyAsync(hb, bounds, sizeof(hb), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("device build: ") + cudaGetErrorString(cudaGetLastError()));
  }
  for (int a = 0; a < 3; a++) {
    outLo[a] = hostDval(hb[6 + a]);
    outHi[a] = hostDval(hb[9 + a]);
  }
  {
    int ov = 0;
    cudaMemcpy(&ov, overflow, 4, cudaMemcpyDeviceToHost);
    if (ov != 0) {
      return setError(EBG_ERR_INVALID, "device build: inconsistent radix tree (code " + std::to_string(ov) + ")");
    }
  }

  // 4. the 4-wide tree, level by level (node 0 = the binary root)
  uint32_t numNodes = 0, numLeaves = 0;
  int      depth    = 1;
  const uint32_t maxNodes = uint32_t(std::max<int64_t>(n, 1)), maxLeaves = uint32_t(std::min<int64_t>(n, EBG_MAX_LEAVES));
  EbgNode4*      dNodesTmp = nullptr;
  if (!alloc((void**)&dNodesTmp, sizeof(EbgNode4) * size_t(maxNodes))) {
    return setError(EBG_ERR_NO_MEMORY, "device build node workspace");
  }
  if (n > leafSize) {
    const uint2 root = make_uint2(0u, 0u);
    cudaMemcpyAsync(frontier[0], &root, sizeof(root), cudaMemcpyHostToDevice, s);
    const uint32_t init[3] = {1u, 0u, 0u};
    cudaMemcpyAsync(counters, init, sizeof(init), cudaMemcpyHostToDevice, s);
    const uint32_t nf = 0u, nl = 0u;
    cudaMemcpyAsync(nodeFirst, &nf, 4, cudaMemcpyHostToDevice, s);
    const uint32_t ne = uint32_t(n);
    cudaMemcpyAsync(nodeEnd, &ne, 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(nodeParent, &nl, 4, cudaMemcpyHostToDevice, s);
    TreeView tv{n, left, right, first, last, nodeLo, nodeHi, leafLo, leafHi};
    uint32_t count = 1;
    int      cur   = 0;
    for (int level = 1; count > 0; level++) {
      if (level > 64) {
        return setError(EBG_ERR_INVALID, "device build: tree deeper than 64 levels");
      }
      cudaMemsetAsync(counters + 2, 0, 4, s);
      kCollapse<<<gridFor(count, 128, 1 << 16), 128, 0, s>>>(tv, frontier[cur], count, leafSize, dNodesTmp,
                                                                frontier[1 - cur], counters, leafFirst, leafCount,
                                                                nodeFirst, nodeEnd, nodeParent, maxNodes, maxLeaves,
                                                                overflow);
      uint32_t hc[3];
      cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, s);
      if (cudaStreamSynchronize(s) != cudaSuccess) {
        return setError(EBG_ERR_CUDA, std::string("device build: ") + cudaGetErrorString(cudaGetLastError()));
      }
      count = hc[2];
      cur   = 1 - cur;
      depth = level + 1;
    }
    uint32_t hc[2];
    int      ov = 0;
    cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&ov, overflow, 4, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    if (ov != 0) {
      return setError(EBG_ERR_TOO_LARGE, "device build: too many nodes or leaves");
    }
    numNodes  = hc[0];
    numLeaves = hc[1];
  }
  else {
    numLeaves = 1;
    const uint32_t lf = 0u, lc = uint32_t(n);
    cudaMemcpyAsync(leafFirst, &lf, 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(leafCount, &lc, 4, cudaMemcpyHostToDevice, s);
  }
  if (3 * depth + 4 > EBG_STACK_DEPTH) {
    return setError(EBG_ERR_INVALID, "BVH too deep for the traversal stack (depth " + std::to_string(depth) + ")");
  }

  // 5. the mesh's device arrays: nodes, records, oriented boxes
  auto keep = [&](void** p, size_t bytes) { return cudaMalloc(p, std::max<size_t>(bytes, 16)) == cudaSuccess; };
  if (!keep(&m->dNodes, sizeof(EbgNode4) * std::max<size_t>(numNodes, 1)) || !keep(&m->dHot, sizeof(EbgTriHot) * N) ||
      !keep(&m->dSign, sizeof(EbgTriSign) * N) || !keep(&m->dTri64, 240 * N) || !keep(&m->dTriId, 4 * N) ||
      !keep(&m->dObb, sizeof(EbgObb) * numLeaves) || !keep(&m->dNodeObb, sizeof(EbgObb) * std::max<size_t>(numNodes, 1)) ||
      !keep(&m->dDcelN, 24 * N) || !keep((void**)&m->dF, 12 * N) || !keep((void**)&m->dLeafFirst, 4 * size_t(numLeaves)) ||
      !keep((void**)&m->dLeafCount, 4 * size_t(numLeaves)) ||
      !keep((void**)&m->dNodeFirst, 4 * std::max<size_t>(numNodes, 1)) ||
      !keep((void**)&m->dNodeEnd, 4 * std::max<size_t>(numNodes, 1))) {
    cudaGetLastError();
    return setError(EBG_ERR_NO_MEMORY, "device allocation for the mesh");
  }
  cudaMemcpyAsync(m->dF, dF, 12 * N, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(m->dLeafFirst, leafFirst, 4 * size_t(numLeaves), cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(m->dLeafCount, leafCount, 4 * size_t(numLeaves), cudaMemcpyDeviceToDevice, s);
  if (numNodes > 0) {
    cudaMemcpyAsync(m->dNodeFirst, nodeFirst, 4 * size_t(numNodes), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(m->dNodeEnd, nodeEnd, 4 * size_t(numNodes), cudaMemcpyDeviceToDevice, s);
  }
  kRecords<<<gridFor(n, 256), 256, 0, s>>>(dV, dF, dTriN, dVN, dEN, ids, n, static_cast<EbgTriHot*>(m->dHot),
                                           static_cast<EbgTriSign*>(m->dSign), static_cast<double*>(m->dTri64),
                                           static_cast<int32_t*>(m->dTriId), static_cast<double*>(m->dDcelN), area);
  double scale = 0;
  for (int a = 0; a < 3; a++) {
    scale = std::max(scale, std::max(std::fabs(outLo[a]), std::fabs(outHi[a])));
  }
  const double pad = 2e-6 * std::max(scale, 1e-30);
  // leaves hold at most EBG_MAX_LEAF triangles; nodes near the root span most of the mesh
  const double* t64 = static_cast<const double*>(m->dTri64);
  ebg_status    orc = rangeObbs(t64, leafFirst, nullptr, leafCount, numLeaves, false, pad,
                                static_cast<EbgObb*>(m->dObb), nullptr, nullptr, m->numSms, s);
  if (orc == EBG_OK && numNodes > 0) {
    orc = rangeObbs(t64, nodeFirst, nodeEnd, nullptr, numNodes, true, pad, static_cast<EbgObb*>(m->dNodeObb), useful,
                    nullptr, m->numSms, s);
  }
  if (orc != EBG_OK) {
    return orc;
  }
  if (numNodes > 0) {
    kNodeObbFlags<<<gridFor(numNodes, 256), 256, 0, s>>>(useful, nodeParent, numNodes, dNodesTmp);
    cudaMemcpyAsync(m->dNodes, dNodesTmp, sizeof(EbgNode4) * size_t(numNodes), cudaMemcpyDeviceToDevice, s);
  }
  // the cumulative area table stays on the host (the seed trainer's band sampler reads it)
  m->areaCdf.resize(N);
  cudaMemcpyAsync(m->areaCdf.data(), area, 8 * N, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("device build: ") + cudaGetErrorString(cudaGetLastError()));
  }
  for (size_t i = 1; i < N; i++) {
    m->areaCdf[i] += m->areaCdf[i - 1];
  }
  m->info.num_nodes  = numNodes;
  m->info.num_leaves = numLeaves;
  m->info.depth      = depth;
  m->view.root_ref   = n > leafSize ? 0u : (EBG_LEAF_BIT | 0u);
  m->view.root_count = n > leafSize ? 0u : uint32_t(n);
  return EBG_OK;
}

} // namespace ebg

namespace ebg {

ebg_status refitMeshOnDevice(ebg_mesh* m, const double* V, bool vOnDevice, int64_t nv, double* outLo, double* outHi,
                             cudaStream_t s)
{
  const int64_t n = m->info.num_triangles;
  const size_t  N = size_t(n);
  if (m->dF == nullptr) {
    return setError(EBG_ERR_INVALID, "mesh has no topology kept for refitting");
  }
  std::vector<void*> tmp;
  auto alloc = [&](void** p, size_t bytes) -> bool {
    if (cudaMallocAsync(p, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    tmp.push_back(*p);
    return true;
  };
  struct Guard
  {
    std::vector<void*>& t;
    cudaStream_t        st;
    ~Guard()
    {
      for (void* p : t) {
        cudaFreeAsync(p, st);
      }
      cudaStreamSynchronize(st);
    }
  } guard{tmp, s};
  const uint32_t numNodes  = uint32_t(m->info.num_nodes);
  const uint32_t numLeaves = uint32_t(m->info.num_leaves);
  double *dV = nullptr, *dTriN = nullptr, *dVN = nullptr, *dEN = nullptr, *triLo = nullptr, *triHi = nullptr,
         *cen = nullptr, *area = nullptr;
  unsigned long long* bounds = nullptr;
  uint8_t*            useful = nullptr;
  int*                bad    = nullptr;
  double *            leafAabb = nullptr, *nodeAabb = nullptr;
  bool ok = alloc((void**)&dTriN, 24 * N) && alloc((void**)&dVN, 72 * N) && alloc((void**)&dEN, 72 * N) &&
            alloc((void**)&triLo, 24 * N) && alloc((void**)&triHi, 24 * N) && alloc((void**)&cen, 24 * N) &&
            alloc((void**)&area, 8 * N) && alloc((void**)&bounds, 12 * 8) &&
            alloc((void**)&useful, std::max<size_t>(numNodes, 1)) && alloc((void**)&bad, 4) &&
            alloc((void**)&leafAabb, 48 * size_t(numLeaves)) && alloc((void**)&nodeAabb, 48 * size_t(numNodes));
  if (ok && !vOnDevice) {
    ok = alloc((void**)&dV, 24 * size_t(nv)) &&
         cudaMemcpyAsync(dV, V, 24 * size_t(nv), cudaMemcpyHostToDevice, s) == cudaSuccess;
  }
  if (!ok) {
    return setError(EBG_ERR_NO_MEMORY, "refit workspace");
  }
  const double* v = vOnDevice ? V : dV;
  cudaMemsetAsync(bad, 0, 4, s);
  cudaMemsetAsync(useful, 0, std::max<size_t>(numNodes, 1), s);
  kAllFinite<<<gridFor(3 * nv, 256, 4096), 256, 0, s>>>(v, 3 * nv, bad);
  int hbad = 0;
  cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("refit: ") + cudaGetErrorString(cudaGetLastError()));
  }
  if (hbad != 0) {
    return setError(EBG_ERR_INVALID, "non-finite vertex coordinate");
  }
  // the pseudonormals of the moved soup (fails, leaving the mesh untouched, on degenerate triangles)
  const ebg_status rc = pseudonormalsOnDevice(v, nv, m->dF, n, dTriN, dVN, dEN, s);
  if (rc != EBG_OK) {
    return rc;
  }
  {
    unsigned long long init[12];
    for (int j = 0; j < 12; j++) {
      const bool isMin = (j < 3) || (j >= 6 && j < 9);
      init[j]          = isMin ? ~0ull : 0ull;
    }
    cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, s);
  }
  kTriBounds<<<gridFor(n, 256, 8192), 256, 0, s>>>(v, m->dF, n, triLo, triHi, cen, bounds);
  unsigned long long hb[12];
  cudaMemcpyAsync(hb, bounds, sizeof(hb), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("refit: ") + cudaGetErrorString(cudaGetLastError()));
  }
  for (int a = 0; a < 3; a++) {
    outLo[a] = hostDval(hb[6 + a]);
    outHi[a] = hostDval(hb[9 + a]);
  }
  kRecords<<<gridFor(n, 256), 256, 0, s>>>(v, m->dF, dTriN, dVN, dEN, reinterpret_cast<const uint32_t*>(m->dTriId), n,
                                           static_cast<EbgTriHot*>(m->dHot), static_cast<EbgTriSign*>(m->dSign),
                                           static_cast<double*>(m->dTri64), static_cast<int32_t*>(m->dTriId),
                                           static_cast<double*>(m->dDcelN), area);
  double scale = 0;
  for (int a = 0; a < 3; a++) {
    scale = std::max(scale, std::max(std::fabs(outLo[a]), std::fabs(outHi[a])));
  }
  const double pad = 2e-6 * std::max(scale, 1e-30);
  const double* t64 = static_cast<const double*>(m->dTri64);
  ebg_status    orc = rangeObbs(t64, m->dLeafFirst, nullptr, m->dLeafCount, numLeaves, false, pad,
                                static_cast<EbgObb*>(m->dObb), nullptr, leafAabb, m->numSms, s);
  if (orc == EBG_OK && numNodes > 0) {
    orc = rangeObbs(t64, m->dNodeFirst, m->dNodeEnd, nullptr, numNodes, true, pad, static_cast<EbgObb*>(m->dNodeObb),
                    useful, nodeAabb, m->numSms, s);
  }
  if (orc != EBG_OK) {
    return orc;
  }
  if (numNodes > 0) {
    kSlotBoxes<<<gridFor(4 * int64_t(numNodes), 256), 256, 0, s>>>(leafAabb, nodeAabb, useful, numNodes, numLeaves,
                                                                   static_cast<EbgNode4*>(m->dNodes));
  }
  std::vector<double> cdf(N);
  cudaMemcpyAsync(cdf.data(), area, 8 * N, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("refit: ") + cudaGetErrorString(cudaGetLastError()));
  }
  for (size_t i = 1; i < N; i++) {
    cdf[i] += cdf[i - 1];
  }
  m->areaCdf.swap(cdf);
  return EBG_OK;
}

} // namespace ebg

namespace ebg {

void launchGatherNormals(const double* tri64, const int32_t* triId, int64_t n, double* out, cudaStream_t s)
{
  kGatherNormals<<<gridFor(n, 256), 256, 0, s>>>(tri64, triId, n, out);
}

} // namespace ebg
