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

__global__ void __launch_bounds__(128) kSceneValue(const SceneQueryArgs a)
{
  __shared__ float4 smem[4 * (2 * (OUTER_DEPTH + EBG_STACK_DEPTH) + 32)];
  const int         lane  = threadIdx.x & 31;
  float4*           ostk  = smem + (threadIdx.x >> 5) * (2 * (OUTER_DEPTH + EBG_STACK_DEPTH) + 32);
  float4*           istk  = ostk + 2 * OUTER_DEPTH;
  float4*           lpts  = istk + 2 * EBG_STACK_DEPTH; // the warp's 32 spread-leaf points
  const SceneView&  sc    = a.scene;
  const uint64_t    numPk = (uint64_t(a.n) + 31) / 32;

  while (true) {
    unsigned long long pk = 0;
    if (lane == 0) {
      pk = atomicAdd(a.work, 1ull);
    }
    pk = __shfl_sync(FULL, pk, 0);
    if (pk >= numPk) {
      break;
    }
    const int64_t  pos   = int64_t(pk) * 32 + lane;
    const bool     valid = pos < a.n;
    const int64_t  src   = valid ? pos : a.n - 1;
    const uint32_t id    = a.order ? __ldg(a.order + src) : uint32_t(src);
    const float px = __ldg(a.points + 3 * size_t(id)), py = __ldg(a.points + 3 * size_t(id) + 1),
                pz = __ldg(a.points + 3 * size_t(id) + 2);
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
      a.out[id] = best;
    }
  }
}

} // namespace

int sceneOuterDepth() { return OUTER_DEPTH; }

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
