// FP32 mesh signed-distance traversal (sm_100a).
//
// The reference evaluates one point at a time with a stack-based branch-and-bound DFS over a
// K-wide packed BVH (PackedBVH::pruneTraverse, BVHImplem.hpp:1098-1606): pop {node, d2}; skip if
// d2 > bound; leaf -> evaluate its triangles, keeping the signed distance of smallest magnitude
// (strict <, MeshDistanceFunctionsImplem.hpp:480-509); interior -> box distances of the K
// children, sorted far-to-near, pushed if d2 <= bound.
//
// Here one warp traverses a PACKET of 32 queries that were sorted along a Morton curve, so they
// are spatial neighbours:
//  - the warp shares one stack in shared memory (entries carry the child box, so a popped entry is
//    re-tested against every lane's current bound without touching global memory);
//  - every node and triangle is read once per packet with a warp-uniform (broadcast) 16-byte load
//    and tested by all 32 lanes, so control flow never diverges;
//  - a child is pushed when __any_sync says some lane's bound admits it; children are ordered
//    near-first by their distance to the packet centroid;
//  - each lane keeps its own bound (its best squared distance so far), exactly the reference's
//    prune bound for that point;
//  - the leaf test computes only the unsigned squared distance (closest point by Voronoi region);
//    the winning triangle's sign is taken once at the end from the pseudonormal of its closest
//    feature, which is what the reference's per-triangle signed test yields for the minimum;
//  - queries with |d| inside the near-surface band are appended to a list for the FP64
//    re-evaluation (mesh_band64.cu).
// Packets are handed out by an atomic counter, so a warp that drew cheap exterior packets keeps
// working while others finish interior ("blind spot") packets.
#include <cfloat>
#include <cub/device/device_radix_sort.cuh>

#include "ebg_device.cuh"
#include "mesh_kernels.h"
#include "mesh_traverse.cuh"

namespace ebg {

namespace {

// Polls of the wait for a cut's bulk copy before the warp gives up: after the first 64 each
// poll sleeps about 128 ns, so the wait ends within about a tenth of a second, far beyond the
// microseconds a few kilobytes take.
constexpr uint32_t COPY_WAIT_POLLS = 1u << 20;

// True once the mbarrier at shared address `bar` has completed the phase with parity `phase`
// (a non-blocking test).
__device__ __forceinline__ bool mbarDone(uint32_t bar, uint32_t phase)
{
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok)
               : "r"(bar), "r"(phase)
               : "memory");
  return ok != 0;
}

// Every lane of the warp waits until the phase completed, at most COPY_WAIT_POLLS polls each.
__device__ __forceinline__ bool mbarWaitWarp(uint32_t bar, uint32_t phase)
{
  bool done = mbarDone(bar, phase);
  for (uint32_t t = 1; t < COPY_WAIT_POLLS && !done; t++) {
    if (t >= 64) {
      __nanosleep(128);
    }
    done = mbarDone(bar, phase);
  }
  return __all_sync(FULL, done);
}

// SEED: 0 plain, 2 per-query radius hint, 3 per-cell entry cuts and anchors of an attached model
// (cells_kernels.h)
// OCC selects the register budget: 0 = 256-thread blocks, compiler's choice; 1..3 = 128-thread
// blocks with 8, 10, 12 resident blocks per SM (at most 64, 51, 42 registers).
template <int OCC>
struct Bounds
{
  static constexpr int threads = OCC == 0 ? 256 : 128;
  static constexpr int blocks  = OCC == 0 ? 1 : (OCC == 1 ? 8 : (OCC == 2 ? 10 : 12));
};

// TOP: each block copies the tree's first a.top_nodes nodes into shared memory (plain queries only).
// W: node width of the tree a.mesh points at, 4 or 8 (the 8-wide copy: plain or hinted queries).
template <bool STATS, int SEED, int OCC, bool TOP = false, int W = 4>
__global__ void __launch_bounds__(Bounds<OCC>::threads, Bounds<OCC>::blocks) kMeshSdf32(const MeshQueryArgs a)
{
  static_assert(W == 4 || (W == 8 && SEED != 3 && !TOP), "the cuts and the top-tree copy index the 4-wide tree");
  extern __shared__ float4 smem[];
  constexpr int STACK = SEED == 3 ? CUT_STACK_DEPTH : EBG_STACK_DEPTH;
  const int     lane = threadIdx.x & 31;
  float4*       stk  = smem + (threadIdx.x >> 5) * (2 * STACK + 32);
  float4*       lpts = stk + 2 * STACK; // the warp's 32 spread-leaf points
  const EbgMeshView& m = a.mesh;
  const uint64_t numPackets = (uint64_t(a.n) + 31) / 32;

  // the block's copy of the tree's first top_nodes nodes (the device build numbers nodes level by
  // level, so these are the top levels) and their oriented boxes, after the warps' stacks
  const uint32_t topN = TOP ? a.top_nodes : 0u;
  float4*        top  = smem + (blockDim.x >> 5) * (2 * STACK + 32);
  if constexpr (TOP) {
    const float4* gn = reinterpret_cast<const float4*>(m.nodes);
    const float4* go = reinterpret_cast<const float4*>(m.node_obb);
    for (uint32_t i = threadIdx.x; i < topN * (TOP_NODE_BYTES / 16); i += blockDim.x) {
      const uint32_t nI = i / (TOP_NODE_BYTES / 16), w = i - nI * (TOP_NODE_BYTES / 16);
      top[i] = w < 8 ? __ldg(gn + 8 * nI + w) : __ldg(go + 4 * nI + (w - 8));
    }
    __syncthreads();
  }
  const uint32_t topS = uint32_t(__cvta_generic_to_shared(top));

  // seeded packets bring their cell's cut onto the stack with one bulk copy, tracked by the warp's
  // mbarrier (after the stacks and the top nodes' copy); `phase` is the parity of its next phase
  uint32_t bar = 0, phase = 0;
  if constexpr (SEED == 3) {
    uint64_t* bars = reinterpret_cast<uint64_t*>(top + (TOP ? topN * (TOP_NODE_BYTES / 16) : 0u));
    bar            = uint32_t(__cvta_generic_to_shared(bars + (threadIdx.x >> 5)));
    if (lane == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
  }

  // packets come from the work counter `chunk` at a time (the queue chunk the autotuner picks)
  const unsigned long long chunk = a.chunk > 1 ? (unsigned long long)a.chunk : 1ull;
  unsigned long long       pk = 0, pkEnd = 0;
  while (true) {
    if (pk == pkEnd) {
      if (lane == 0) {
        pk = atomicAdd(a.work, chunk);
      }
      pk    = __shfl_sync(FULL, pk, 0);
      pkEnd = pk + chunk;
    }
    if (pk >= numPackets) {
      break;
    }
    const int64_t  pos   = int64_t(pk) * 32 + lane;
    const bool     valid = pos < a.n;
    const int64_t  src   = valid ? pos : a.n - 1;
    const uint32_t id    = a.order ? __ldg(a.order + src) : uint32_t(src);
    const float    px = __ldg(a.points + 3 * size_t(id)), py = __ldg(a.points + 3 * size_t(id) + 1),
                pz = __ldg(a.points + 3 * size_t(id) + 2);

    if (valid && !(isfinite(px) && isfinite(py) && isfinite(pz))) {
      atomicOr(a.status, ST_INPUT);
    }
    constexpr bool SEEDED = SEED != 0;
    float best    = FLT_MAX;
    int   besttri = -1;
    if (SEED == 2) {
      const float r = __ldg(a.hint + id);
      best          = (r > 0.f && r < 1e18f) ? r * r * 1.000004f : FLT_MAX;
    }
    int  startSp = 0;     // entries of a cell's cut on the stack
    bool fromCut = false; // the packet starts from a cell's cut (else at the root)
    int  loaded  = 0;     // entries the cut held
    if (SEED == 3) {
      // the packet's box over its valid lanes, and the cell holding the box's centre
      const float inf = __int_as_float(0x7f800000);
      float       mnx = valid ? px : inf, mny = valid ? py : inf, mnz = valid ? pz : inf;
      float       mxx = valid ? px : -inf, mxy = valid ? py : -inf, mxz = valid ? pz : -inf;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        mnx = fminf(mnx, __shfl_xor_sync(FULL, mnx, o));
        mny = fminf(mny, __shfl_xor_sync(FULL, mny, o));
        mnz = fminf(mnz, __shfl_xor_sync(FULL, mnz, o));
        mxx = fmaxf(mxx, __shfl_xor_sync(FULL, mxx, o));
        mxy = fmaxf(mxy, __shfl_xor_sync(FULL, mxy, o));
        mxz = fmaxf(mxz, __shfl_xor_sync(FULL, mxz, o));
      }
      const SeedCellsView& cv = a.cells;
      const float fx = (0.5f * (mnx + mxx) - cv.lo[0]) * cv.inv[0];
      const float fy = (0.5f * (mny + mxy) - cv.lo[1]) * cv.inv[1];
      const float fz = (0.5f * (mnz + mxz) - cv.lo[2]) * cv.inv[2];
      const float g  = float(cv.g);
      // (NaN coordinates fail these comparisons and keep the packet at the root)
      if (fx >= 0.f && fx < g && fy >= 0.f && fy < g && fz >= 0.f && fz < g) {
        const int ix = min(int(fx), cv.g - 1), iy = min(int(fy), cv.g - 1), iz = min(int(fz), cv.g - 1);
        // the grown cell exactly as the cut builder rounded it
        const bool inside =
          mnx >= __fsub_rd(__fadd_rd(cv.lo[0], float(ix) * cv.size[0]), cv.margin[0]) &&
          mny >= __fsub_rd(__fadd_rd(cv.lo[1], float(iy) * cv.size[1]), cv.margin[1]) &&
          mnz >= __fsub_rd(__fadd_rd(cv.lo[2], float(iz) * cv.size[2]), cv.margin[2]) &&
          mxx <= __fadd_ru(__fadd_ru(cv.lo[0], float(ix + 1) * cv.size[0]), cv.margin[0]) &&
          mxy <= __fadd_ru(__fadd_ru(cv.lo[1], float(iy + 1) * cv.size[1]), cv.margin[1]) &&
          mxz <= __fadd_ru(__fadd_ru(cv.lo[2], float(iz + 1) * cv.size[2]), cv.margin[2]);
        const int64_t cell = (int64_t(iz) * cv.g + iy) * cv.g + ix;
        const int     ne   = inside ? int(__ldg(cv.count + cell)) : 0;
        if (ne > 0) {
          // The cut (32 B per entry, 16-byte aligned at both ends) comes onto the stack by one
          // asynchronous bulk copy while the lanes read the cell's radius and test their anchors.
          // The stack's earlier reads and writes (generic proxy) are ordered before the copy's
          // writes (async proxy) by every lane's proxy fence and the warp barrier.
          const float4*  src   = cv.entries + size_t(cell) * size_t(cv.lmax) * 2;
          const uint32_t bytes = uint32_t(ne) * 32u;
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) {
            const uint32_t dst = uint32_t(__cvta_generic_to_shared(stk));
            asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(bar),
                         "r"(bytes)
                         : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                           dst),
                         "l"(src), "r"(bytes), "r"(bar)
                         : "memory");
          }
          // start below R_C by more than the FP32 error of a triangle distance, so that whatever
          // is found within the bound is nearer than every triangle the cut left out
          const float R = __ldg(cv.radius + cell);
          best          = isfinite(R) ? __fmul_rd(__fmul_rd(R, R), 0.99998f) : FLT_MAX;
          startSp       = ne;
          // the anchor of the lane's own cell (the triangle nearest to that cell's centre, which may
          // be a neighbour of the packet's cell) gives the lane a real distance to start from,
          // usually within a hair of its own nearest
          int anc = -1;
          if (cv.anchor) {
            const float gm = float(cv.g - 1);
            const int   lx = int(fminf(fmaxf((px - cv.lo[0]) * cv.inv[0], 0.f), gm));
            const int   ly = int(fminf(fmaxf((py - cv.lo[1]) * cv.inv[1], 0.f), gm));
            const int   lz = int(fminf(fmaxf((pz - cv.lo[2]) * cv.inv[2], 0.f), gm));
            anc            = __ldg(cv.anchor + (int64_t(lz) * cv.g + ly) * cv.g + lx);
          }
          if (anc >= 0) {
            const float4* h  = reinterpret_cast<const float4*>(m.hot + anc);
            const float4  h0 = __ldg(h), h1 = __ldg(h + 1), h2 = __ldg(h + 2);
            float         s_, t_;
            int           r_;
            const float   dd = triDist2<false>(h0, h1, h2, px, py, pz, s_, t_, r_);
            if (dd <= best) {
              best    = dd;
              besttri = anc;
            }
          }
          // the cut is on the stack once the copy completed the barrier's phase
          if (!mbarWaitWarp(bar, phase)) {
            // give up on the packet and the warp's remaining work; wait (bounded again) for the
            // copy so that no write lands after the warp is gone
            if (lane == 0) {
              atomicOr(a.status, ST_COPY);
            }
            mbarWaitWarp(bar, phase);
            return;
          }
          phase ^= 1u;
          // Keep only the entries some lane can still need.  A lane needs an entry only if the
          // entry's box is within its bound, and every lane lies in the packet's box, so an entry
          // farther from that box than the largest bound is needed by none: 32 entries per step,
          // compacted in place in their order (farthest first).
          float bmax = best;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            bmax = fmaxf(bmax, __shfl_xor_sync(FULL, bmax, o));
          }
          int kept = 0;
#pragma unroll 1
          for (int base = 0; base < ne; base += 32) {
            const int i    = base + lane;
            float4    eA   = make_float4(0.f, 0.f, 0.f, 0.f), eB = eA;
            bool      keep = false;
            if (i < ne) {
              eA   = stk[2 * i];
              eB   = stk[2 * i + 1];
              keep = boxBoxDist2(eA.x, eA.y, eA.z, eB.x, eB.y, eB.z, mnx, mny, mnz, mxx, mxy, mxz) <= bmax;
            }
            const unsigned km = __ballot_sync(FULL, keep);
            __syncwarp(); // every entry of this step is read before any is overwritten
            if (keep) {
              const int r    = kept + __popc(km & ((1u << lane) - 1u));
              stk[2 * r]     = eA;
              stk[2 * r + 1] = eB;
            }
            kept += __popc(km);
            __syncwarp();
          }
          startSp = kept;
          fromCut = true;
          loaded  = ne;
        }
      }
    }
    uint32_t iters = 0;
    int      err   = 0;
    uint32_t cNode = 0, cLeaf = 0, cTri = 0, cFall = 0, cBox = 0;
    uint32_t pPops = 0, pNode = 0, pLeaf = 0, pTri = 0, pBox = 0, pRecs = 0;

#pragma unroll 1
    for (int pass = 0; pass < (SEEDED ? 2 : 1); pass++) {
      if (pass == 1) {
        const bool fail = besttri < 0;
        if (!__any_sync(FULL, fail)) {
          break;
        }
        if (fail) {
          best = FLT_MAX;
          cFall++;
        }
      }
      TraversalCounters tc;
      if (SEED == 3 && pass == 0 && fromCut) {
        traverseFrom<STATS, STACK, TOP, W>(m, px, py, pz, best, besttri, stk, lpts, startSp, iters, err, tc, topS,
                                           topN);
      }
      else {
        traverseMesh<STATS, STACK, TOP, W>(m, px, py, pz, best, besttri, stk, lpts, iters, err, tc, topS, topN);
      }
      cNode += tc.node;
      cLeaf += tc.leaf;
      cTri += tc.tri;
      cBox += tc.box;
      pBox += tc.pbox;
      pPops += tc.pops;
      pNode += tc.pnode;
      pLeaf += tc.pleaf;
      pTri += tc.ptri;
      pRecs += tc.precs;
      if (err) {
        break;
      }
    }

    if (err && lane == 0) {
      atomicOr(a.status, err);
    }
    float dist = FLT_MAX;
    if (besttri >= 0) {
      dist = signedFromWinner(m, uint32_t(besttri), px, py, pz);
    }
    if (valid) {
      a.out_d[id] = dist;
      if (a.out_tri) {
        a.out_tri[id] = besttri >= 0 ? (a.tri_leaf ? besttri : __ldg(m.tri_id + besttri)) : -1;
      }
    }
    if (a.band_flag) {
      // one flag per sorted position; the list is compacted from them in position order
      if (valid) {
        a.band_flag[pos] = uint8_t(besttri >= 0 && fabsf(dist) <= a.band);
      }
    }
    else if (a.band_list) {
      const bool     inb  = valid && besttri >= 0 && fabsf(dist) <= a.band;
      const unsigned mask = __ballot_sync(FULL, inb);
      if (mask) {
        uint32_t base = 0;
        if (lane == 0) {
          base = atomicAdd(a.band_count, uint32_t(__popc(mask)));
        }
        base = __shfl_sync(FULL, base, 0);
        if (inb) {
          const uint32_t r = base + __popc(mask & ((1u << lane) - 1u));
          a.band_list[r]   = uint32_t(pos);
          a.band_d32[r]    = dist;
        }
      }
    }
    if (STATS) {
      if (!valid) {
        cNode = cLeaf = cTri = cFall = cBox = 0;
      }
      atomicAdd(a.stats + 10, (unsigned long long)cBox);
      atomicAdd(a.stats + 0, (unsigned long long)cNode);
      atomicAdd(a.stats + 1, (unsigned long long)cLeaf);
      atomicAdd(a.stats + 2, (unsigned long long)cTri);
      atomicAdd(a.stats + 4, (unsigned long long)cFall);
      if (lane == 0) {
        atomicAdd(a.stats + 5, 1ull);
        atomicAdd(a.stats + 6, (unsigned long long)pPops);
        atomicAdd(a.stats + 7, (unsigned long long)pNode);
        atomicAdd(a.stats + 8, (unsigned long long)pLeaf);
        atomicAdd(a.stats + 9, (unsigned long long)pTri);
        atomicAdd(a.stats + 11, (unsigned long long)pBox);
        atomicAdd(a.stats + 14, (unsigned long long)pRecs);
        if (fromCut) {
          atomicAdd(a.stats + 12, 1ull);
          atomicAdd(a.stats + 13, (unsigned long long)loaded);
        }
      }
    }
    pk++;
  }
}

__global__ void kQueryKeys(const float* __restrict__ pts, int64_t n, float lx, float ly, float lz, float sx, float sy,
                           float sz, uint32_t* __restrict__ keys, uint32_t* __restrict__ ids)
{
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  const float x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
  const float fx = fminf(fmaxf((x - lx) * sx, 0.f), 1023.f);
  const float fy = fminf(fmaxf((y - ly) * sy, 0.f), 1023.f);
  const float fz = fminf(fmaxf((z - lz) * sz, 0.f), 1023.f);
  // NaN coordinates quantise to 0 (fmaxf drops NaN); the traversal kernel reports them (ST_INPUT)
  keys[i] = (spread10(uint32_t(fx)) << 2) | (spread10(uint32_t(fy)) << 1) | spread10(uint32_t(fz));
  ids[i]  = uint32_t(i);
}

template <bool STATS, int SEED, int OCC, bool TOP, int W = 4>
cudaError_t launchOne(const MeshQueryArgs& a, int wpb, int numSms, cudaStream_t s)
{
  if (OCC != 0 && wpb > 4) {
    wpb = 4;
  }
  const int    threads = 32 * wpb;
  const size_t smem    = size_t(wpb) * (2 * (SEED == 3 ? CUT_STACK_DEPTH : EBG_STACK_DEPTH) + 32) * sizeof(float4) +
                      (TOP ? size_t(a.top_nodes) * TOP_NODE_BYTES : 0) + (SEED == 3 ? size_t(wpb) * 8 : 0);
  // resident blocks per SM for each block size and shared-memory size, looked up once (the query
  // path then issues no runtime calls besides its launches, so it can be captured in a CUDA graph)
  static int    cache[9]     = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  static size_t cacheMem[9]  = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int           perSm        = cacheMem[wpb] == smem ? cache[wpb] : 0;
  if (perSm == 0) {
    if (smem > 48 * 1024) {
      const cudaError_t e =
        cudaFuncSetAttribute(kMeshSdf32<STATS, SEED, OCC, TOP, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      if (e != cudaSuccess) {
        return e;
      }
    }
    const cudaError_t e =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kMeshSdf32<STATS, SEED, OCC, TOP, W>, threads, smem);
    if (e != cudaSuccess) {
      return e;
    }
    cache[wpb]    = perSm;
    cacheMem[wpb] = smem;
  }
  perSm               = perSm < 1 ? 1 : perSm;
  const int64_t need  = ((int64_t(a.n) + 31) / 32 + wpb - 1) / wpb;
  int64_t       grid  = int64_t(numSms) * perSm;
  grid                = grid < need ? grid : need;
  grid                = grid < 1 ? 1 : grid;
  kMeshSdf32<STATS, SEED, OCC, TOP, W><<<unsigned(grid), threads, smem, s>>>(a);
  return cudaGetLastError();
}

} // namespace

void launchQueryKeys(const float* points, int64_t n, const float* lo, const float* scale, uint32_t* keys,
                     uint32_t* ids, cudaStream_t s)
{
  const int     threads = 256;
  const int64_t blocks  = (n + threads - 1) / threads;
  kQueryKeys<<<unsigned(blocks), threads, 0, s>>>(points, n, lo[0], lo[1], lo[2], scale[0], scale[1], scale[2], keys,
                                                  ids);
}

template <int SEED, int OCC>
cudaError_t launchStats(const MeshQueryArgs& a, int wpb, int numSms, cudaStream_t s)
{
  if constexpr (SEED != 3) {
    if (a.node_width == 8) {
      return a.stats != nullptr ? launchOne<true, SEED, OCC, false, 8>(a, wpb, numSms, s)
                                : launchOne<false, SEED, OCC, false, 8>(a, wpb, numSms, s);
    }
  }
  if (SEED == 0 && a.top_nodes > 0) {
    return a.stats != nullptr ? launchOne<true, SEED, OCC, SEED == 0>(a, wpb, numSms, s)
                              : launchOne<false, SEED, OCC, SEED == 0>(a, wpb, numSms, s);
  }
  return a.stats != nullptr ? launchOne<true, SEED, OCC, false>(a, wpb, numSms, s)
                            : launchOne<false, SEED, OCC, false>(a, wpb, numSms, s);
}

template <int OCC>
cudaError_t launchSeed(const MeshQueryArgs& a, int wpb, int numSms, cudaStream_t s)
{
  const int mode = a.cells.count != nullptr ? 3 : (a.hint != nullptr ? 2 : 0);
  switch (mode) {
  case 3:
    return launchStats<3, OCC>(a, wpb, numSms, s);
  case 2:
    return launchStats<2, OCC>(a, wpb, numSms, s);
  default:
    return launchStats<0, OCC>(a, wpb, numSms, s);
  }
}

cudaError_t launchMeshSdf32(const MeshQueryArgs& a, int wpb, int numSms, cudaStream_t s, int occupancy)
{
  if (wpb != 1 && wpb != 2 && wpb != 4 && wpb != 8) {
    wpb = 4;
  }
  // occupancy 0 (default) takes the 64-register budget: fastest on B200 in the sweep over
  // budgets and block sizes (full level-8 workload)
  switch (occupancy) {
  case 0:
  case 1:
    return launchSeed<1>(a, wpb, numSms, s);
  case 2:
    return launchSeed<2>(a, wpb, numSms, s);
  case 3:
    return launchSeed<3>(a, wpb, numSms, s);
  default:
    return launchSeed<0>(a, wpb, numSms, s);  // 4: the compiler's own budget (256-thread blocks)
  }
}

} // namespace ebg
