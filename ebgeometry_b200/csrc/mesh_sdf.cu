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

// SEED: 0 plain, 1 learned radius per packet (+ distance to the centroid), 2 per-query radius hint
// OCC selects the register budget: 0 = 256-thread blocks, compiler's choice; 1..3 = 128-thread
// blocks with 8, 10, 12 resident blocks per SM (at most 64, 51, 42 registers).
template <int OCC>
struct Bounds
{
  static constexpr int threads = OCC == 0 ? 256 : 128;
  static constexpr int blocks  = OCC == 0 ? 1 : (OCC == 1 ? 8 : (OCC == 2 ? 10 : 12));
};

template <bool STATS, int SEED, int OCC>
__global__ void __launch_bounds__(Bounds<OCC>::threads, Bounds<OCC>::blocks) kMeshSdf32(const MeshQueryArgs a)
{
  extern __shared__ float4 smem[];
  const int     lane = threadIdx.x & 31;
  float4*       stk  = smem + (threadIdx.x >> 5) * (2 * EBG_STACK_DEPTH + 32);
  float4*       lpts = stk + 2 * EBG_STACK_DEPTH; // the warp's 32 spread-leaf points
  const EbgMeshView& m = a.mesh;
  const uint64_t numPackets = (uint64_t(a.n) + 31) / 32;

  while (true) {
    unsigned long long pk = 0;
    if (lane == 0) {
      pk = atomicAdd(a.work, 1ull);
    }
    pk = __shfl_sync(FULL, pk, 0);
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
    if (SEED == 1) {
      // packet radius at the packet's centre, widened by this lane's distance to that centre (the
      // SDF is 1-Lipschitz), squared and rounded up so FP32 rounding never makes the bound too tight
      const float4 sp = __ldg(a.seed_pk + pk);
      const float  ex = px - sp.x, ey = py - sp.y, ez = pz - sp.z;
      const float  r  = sp.w + sqrtf(fmaf(ex, ex, fmaf(ey, ey, ez * ez))) * 1.000001f;
      best           = (r > 0.f && r < 1e18f) ? r * r * 1.000004f : FLT_MAX;
    }
    uint32_t iters = 0;
    int      err   = 0;
    uint32_t cNode = 0, cLeaf = 0, cTri = 0, cFall = 0, cBox = 0;
    uint32_t pPops = 0, pNode = 0, pLeaf = 0, pTri = 0, pBox = 0;

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
      traverseMesh<STATS>(m, px, py, pz, best, besttri, stk, lpts, iters, err, tc);
      cNode += tc.node;
      cLeaf += tc.leaf;
      cTri += tc.tri;
      cBox += tc.box;
      pBox += tc.pbox;
      pPops += tc.pops;
      pNode += tc.pnode;
      pLeaf += tc.pleaf;
      pTri += tc.ptri;
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
        a.out_tri[id] = besttri >= 0 ? __ldg(m.tri_id + besttri) : -1;
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
      }
    }
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

template <bool STATS, int SEED, int OCC>
cudaError_t launchOne(const MeshQueryArgs& a, int wpb, int numSms, cudaStream_t s)
{
  if (OCC != 0 && wpb > 4) {
    wpb = 4;
  }
  const int    threads = 32 * wpb;
  const size_t smem    = size_t(wpb) * (2 * EBG_STACK_DEPTH + 32) * sizeof(float4);
  // resident blocks per SM for each block size, looked up once (the query path then issues no
  // runtime calls besides its launches, so it can be captured in a CUDA graph)
  static int cache[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int        perSm    = cache[wpb];
  if (perSm == 0) {
    const cudaError_t e =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kMeshSdf32<STATS, SEED, OCC>, threads, smem);
    if (e != cudaSuccess) {
      return e;
    }
    cache[wpb] = perSm;
  }
  perSm               = perSm < 1 ? 1 : perSm;
  const int64_t need  = ((int64_t(a.n) + 31) / 32 + wpb - 1) / wpb;
  int64_t       grid  = int64_t(numSms) * perSm;
  grid                = grid < need ? grid : need;
  grid                = grid < 1 ? 1 : grid;
  kMeshSdf32<STATS, SEED, OCC><<<unsigned(grid), threads, smem, s>>>(a);
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
  return a.stats != nullptr ? launchOne<true, SEED, OCC>(a, wpb, numSms, s) : launchOne<false, SEED, OCC>(a, wpb, numSms, s);
}

template <int OCC>
cudaError_t launchSeed(const MeshQueryArgs& a, int wpb, int numSms, cudaStream_t s)
{
  const int mode = a.seed_pk != nullptr ? 1 : (a.hint != nullptr ? 2 : 0);
  return mode == 1 ? launchStats<1, OCC>(a, wpb, numSms, s)
                   : (mode == 2 ? launchStats<2, OCC>(a, wpb, numSms, s) : launchStats<0, OCC>(a, wpb, numSms, s));
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
