// CSG union of many objects (sm_100a): the reference's BVHUnionIF::value (CSGImplem.hpp:465-501)
// over SphereSDF and Translate(Rotate(TriMeshSDF)) objects, batched.
//
// value(p) = min over objects of object.value(p), with an object-level BVH pruned by the bound
// max(0, best)^2 (an object whose box is farther than the running minimum cannot lower it, and when
// p is inside some object the bound collapses to 0 so only boxes containing p are opened).
//
// One warp traverses a packet of 32 Morton-sorted queries through the object BVH (shared stack, as
// the mesh kernel).  At an object leaf every lane evaluates every object of the leaf:
//   sphere: |p - c| - r;
//   mesh:   the query is moved into the mesh's frame (RotateIF / TranslateIF: local = R (p - t),
//           TransformImplem.hpp:152-225) and the mesh's own BVH is traversed by the same packet,
//           on a second stack region.  The nested traversal is seeded with the lane's running
//           minimum when the local point lies outside the mesh's box (then the point is outside the
//           mesh, and finding no triangle within the bound proves the mesh cannot lower the
//           minimum); inside the box it runs unseeded, because a point inside the mesh can have a
//           large negative distance.
#include <cfloat>

#include "ebg_device.cuh"
#include "mesh_traverse.cuh"
#include "scene_kernels.h"

namespace ebg {

namespace {

constexpr int OUTER_DEPTH = 48; // object-BVH stack entries per warp (builder checks the depth)

// A batched call whose batch sizes did not add up to its point count reads no point.
__device__ __forceinline__ bool batchesValid(const SceneQueryArgs& a)
{
  return a.batches == nullptr || __ldg(a.batch_start + a.num_batches) == a.n;
}


__global__ void __launch_bounds__(128) kSceneValue(const SceneQueryArgs a)
{
  __shared__ float4 smem[4 * (2 * (OUTER_DEPTH + EBG_STACK_DEPTH) + 32)];
  const int         lane  = threadIdx.x & 31;
  float4*           ostk  = smem + (threadIdx.x >> 5) * (2 * (OUTER_DEPTH + EBG_STACK_DEPTH) + 32);
  float4*           istk  = ostk + 2 * OUTER_DEPTH;
  float4*           lpts  = istk + 2 * EBG_STACK_DEPTH; // the warp's 32 spread-leaf points
  const SceneView&  sc    = a.scene;
  const uint64_t    numPk = (uint64_t(a.n) + 31) / 32;
  if (!batchesValid(a)) {
    return;
  }

  // packets come from the work counter `chunk` at a time
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
    if (pk >= numPk) {
      break;
    }
    const int64_t  pos   = int64_t(pk) * 32 + lane;
    const bool     valid = pos < a.n;
    const int64_t  src   = valid ? pos : a.n - 1;
    const uint32_t id    = a.order ? __ldg(a.order + src) : uint32_t(src);
    float*         outp  = nullptr;
    const float*   pp    = scenePoint(a, id, &outp);
    const float    px = __ldg(pp), py = __ldg(pp + 1), pz = __ldg(pp + 2);
    float    best  = __int_as_float(0x7f800000); // +inf, as the reference starts
    uint32_t iters = 0;
    int      err   = 0;
    int      sp    = 1;
    if (lane == 0) {
      ostk[0] = make_float4(sc.root_lo[0], sc.root_lo[1], sc.root_lo[2], __uint_as_float(sc.root_ref));
      ostk[1] = make_float4(sc.root_hi[0], sc.root_hi[1], sc.root_hi[2], __uint_as_float(sc.root_count));
    }
    __syncwarp();
    while (sp > 0) {
      if (++iters > MAX_ITERS) {
        err |= ST_ITERS;
        break;
      }
      --sp;
      const float4 A = ostk[2 * sp], B = ostk[2 * sp + 1];
      const float  bb = fmaxf(best, 0.f);
      const float  bound = bb * bb;
      const float  d2 = boxDist2(A.x, A.y, A.z, B.x, B.y, B.z, px, py, pz);
      if (!__any_sync(FULL, d2 <= bound)) {
        continue;
      }
      const uint32_t ref = __float_as_uint(A.w), cnt = __float_as_uint(B.w) & EBG_COUNT_MASK;
      if (ref & EBG_LEAF_BIT) {
        const uint32_t o0 = ref & ~EBG_LEAF_BIT;
        for (uint32_t oi = o0; oi < o0 + cnt; oi++) {
          const SceneObject& ob = sc.objects[oi];
          if (ob.kind == 0) {
            const float dx = px - ob.t[0], dy = py - ob.t[1], dz = pz - ob.t[2];
            best = fminf(best, sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz))) - ob.radius);
            continue;
          }
          // mesh object: local = R (p - t)
          const float qx = px - ob.t[0], qy = py - ob.t[1], qz = pz - ob.t[2];
          const float lx = fmaf(ob.R[0], qx, fmaf(ob.R[1], qy, ob.R[2] * qz));
          const float ly = fmaf(ob.R[3], qx, fmaf(ob.R[4], qy, ob.R[5] * qz));
          const float lz = fmaf(ob.R[6], qx, fmaf(ob.R[7], qy, ob.R[8] * qz));
          const EbgMeshView& mv = sc.meshes[ob.mesh];
          const bool outsideBox = lx < mv.root_lo[0] || lx > mv.root_hi[0] || ly < mv.root_lo[1] ||
                                  ly > mv.root_hi[1] || lz < mv.root_lo[2] || lz > mv.root_hi[2];
          const bool seeded = outsideBox && best > 0.f && best < 1e18f;
          float      mb     = seeded ? best * best * 1.000004f : FLT_MAX;
          int        bt     = -1;
          TraversalCounters tc;
          traverseMesh<false>(mv, lx, ly, lz, mb, bt, istk, lpts, iters, err, tc);
          if (err) {
            break;
          }
          if (bt >= 0) {
            best = fminf(best, signedFromWinner(mv, uint32_t(bt), lx, ly, lz));
          }
        }
        if (err) {
          break;
        }
      }
      else {
        const EbgNode4& nd = sc.nodes[ref];
        float           key[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const float dk = boxDist2(nd.lox[k], nd.loy[k], nd.loz[k], nd.hix[k], nd.hiy[k], nd.hiz[k], px, py, pz);
          const bool  nk = __any_sync(FULL, dk <= bound) && (nd.child[k] | nd.count[k]) != 0u;
          key[k]         = nk ? __uint_as_float(__reduce_min_sync(FULL, __float_as_uint(dk))) : -1.f;
        }
        const int np = int(key[0] >= 0.f) + int(key[1] >= 0.f) + int(key[2] >= 0.f) + int(key[3] >= 0.f);
        if (sp + np > OUTER_DEPTH) {
          err |= ST_STACK;
          break;
        }
        // lane k (< 4) writes child k into its slot, farther children deeper (ties by slot index)
        if (lane < 4) {
          const float kk = lane == 0 ? key[0] : (lane == 1 ? key[1] : (lane == 2 ? key[2] : key[3]));
          if (kk >= 0.f) {
            int rank = 0;
#pragma unroll
            for (int j = 0; j < 4; j++) {
              rank += int(key[j] >= 0.f && (key[j] > kk || (key[j] == kk && j < lane)));
            }
            float4* e = ostk + 2 * (sp + rank);
            e[0]      = make_float4(nd.lox[lane], nd.loy[lane], nd.loz[lane], __uint_as_float(nd.child[lane]));
            e[1]      = make_float4(nd.hix[lane], nd.hiy[lane], nd.hiz[lane], __uint_as_float(nd.count[lane]));
          }
        }
        sp += np;
        __syncwarp();
        if (err) {
          break;
        }
      }
    }
    if (err && lane == 0) {
      atomicOr(a.status, err);
    }
    if (valid) {
      *outp = best;
      if (a.band_flag) {
        a.band_flag[pos] = uint8_t(fabsf(best) <= a.band);
      }
    }
    pk++;
  }
}

} // namespace

// Sort keys of a batched call: the 30-bit Morton code of each point of every batch, so that the
// points of all batches are ordered together (batches that each cover the whole scene would
// otherwise give packets of points far apart).
__global__ void kSceneBatchKeys(const SceneQueryArgs a, uint32_t* __restrict__ keys, uint32_t* __restrict__ ids)
{
  const SceneView& v = a.scene;
  if (!batchesValid(a)) {
    return;
  }
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < a.n; g += int64_t(gridDim.x) * blockDim.x) {
    float*       outp = nullptr;
    const float* p    = scenePoint(a, uint32_t(g), &outp);
    const float  fx   = fminf(fmaxf((p[0] - v.morton_lo[0]) * v.morton_scale[0], 0.f), 1023.f);
    const float  fy   = fminf(fmaxf((p[1] - v.morton_lo[1]) * v.morton_scale[1], 0.f), 1023.f);
    const float  fz   = fminf(fmaxf((p[2] - v.morton_lo[2]) * v.morton_scale[2], 0.f), 1023.f);
    keys[g] = (spread10(uint32_t(fx)) << 2) | (spread10(uint32_t(fy)) << 1) | spread10(uint32_t(fz));
    ids[g]  = uint32_t(g);
  }
}

// One thread: the exclusive prefix of the batch sizes (at most a few thousand batches).  A negative
// size, or a total other than the caller's, is reported as ST_INPUT and leaves start[nb] != the
// call's point count, which every kernel of the call checks before it reads a point.
__global__ void kSceneBatchStarts(const SceneBatch* __restrict__ b, int32_t nb, int64_t* __restrict__ start,
                                  int* __restrict__ status, int64_t expect)
{
  int64_t acc = 0;
  bool    bad = false;
  for (int32_t i = 0; i < nb; i++) {
    start[i]        = acc;
    const int64_t n = b[i].n;
    bad             = bad || n < 0;
    acc += n > 0 ? n : 0;
  }
  bad       = bad || acc != expect;
  start[nb] = bad ? -1 : acc;
  if (bad) {
    atomicOr(status, ST_INPUT);
  }
}

int sceneOuterDepth() { return OUTER_DEPTH; }

cudaError_t launchSceneBatchKeys(const SceneQueryArgs& a, uint32_t* keys, uint32_t* ids, cudaStream_t s)
{
  int64_t blocks = (a.n + 255) / 256;
  blocks         = blocks < 4096 ? blocks : 4096;
  kSceneBatchKeys<<<unsigned(blocks < 1 ? 1 : blocks), 256, 0, s>>>(a, keys, ids);
  return cudaGetLastError();
}

cudaError_t launchSceneBatchStarts(const SceneBatch* batches, int32_t nb, int64_t* start, int* status,
                                   int64_t expectTotal, cudaStream_t s)
{
  kSceneBatchStarts<<<1, 1, 0, s>>>(batches, nb, start, status, expectTotal);
  return cudaGetLastError();
}

cudaError_t launchSceneValue(const SceneQueryArgs& a, int numSms, cudaStream_t s)
{
  // resident blocks per SM, looked up once (the query then issues only stream-ordered work and can
  // be captured in a CUDA graph)
  static int cached = 0;
  int        perSm  = cached;
  if (perSm == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kSceneValue, 128, 0);
    perSm  = perSm < 1 ? 1 : perSm;
    cached = perSm;
  }
  const int64_t need = ((int64_t(a.n) + 31) / 32 + 3) / 4;
  int64_t       grid = int64_t(numSms) * perSm;
  grid               = grid < need ? grid : need;
  grid               = grid < 1 ? 1 : grid;
  kSceneValue<<<unsigned(grid), 128, 0, s>>>(a);
  return cudaGetLastError();
}

} // namespace ebg
