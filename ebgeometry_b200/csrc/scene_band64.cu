// FP64 near-surface pass of the CSG union (sm_100a).  Compiled with -fmad=false, as the mesh band
// pass: the reference evaluates BVHUnionIF<double>::value (CSGImplem.hpp:465-501) in double, and its
// objects' transforms and distances keep their separate multiplies and adds.
//
// A query whose FP32 union value fell inside the band |value| <= band (where the sign of the
// nearest surface is ill-conditioned in FP32) is evaluated again in FP64.  Only objects whose value
// can be the minimum matter: the FP32 value d32 is within delta of the exact one, so the minimum is
// at most d32 + delta, and an object whose box is farther than that cannot reach it.  Each object
// reached is evaluated as the reference does:
//   sphere:          |p - c| - r;
//   mesh instance:   TranslateIF(RotateIF(TriMeshSDF)) -- local = rot(p - t) with RotateIF's
//                    per-axis formulas (TransformImplem.hpp:152-225) -- then the FP64 triangle test
//                    over every triangle within |d32| + delta of the local point (band64.cuh), whose
//                    winner is the mesh's exact value whenever the mesh can hold the minimum (a
//                    winner farther than that is left out: such a mesh cannot).
// The union's value is the minimum over them (std::min, as the reference's evalLeaf).
#include <cfloat>

#include <math_constants.h>

#include "band64.cuh"
#include "ebg_device.cuh"
#include "mesh_traverse.cuh"
#include "scene_kernels.h"

namespace ebg {

namespace {

constexpr int BAND_OUTER = 48; // object-BVH stack entries per warp (the scene builder checks the depth)

__global__ void __launch_bounds__(128, 4) kSceneBand64(const SceneQueryArgs a, float delta)
{
  __shared__ float4 smem[4 * 2 * (BAND_OUTER + EBG_STACK_DEPTH)];
  const int         lane  = threadIdx.x & 31;
  float4*           ostk  = smem + (threadIdx.x >> 5) * (2 * (BAND_OUTER + EBG_STACK_DEPTH));
  float4*           istk  = ostk + 2 * BAND_OUTER;
  const SceneView&  sc    = a.scene;
  if (a.batches != nullptr && __ldg(a.batch_start + a.num_batches) != a.n) {
    return;
  }
  const uint32_t count  = *a.band_count;
  const uint32_t numPk  = (count + 31) / 32;
  const uint32_t warpId = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nWarps = (gridDim.x * blockDim.x) >> 5;

  for (uint32_t pk = warpId; pk < numPk; pk += nWarps) {
    const uint32_t j     = pk * 32 + lane;
    const bool     valid = j < count;
    const uint32_t pos   = a.band_list[valid ? j : count - 1];
    const uint32_t id    = a.order ? a.order[pos] : pos;
    float*         outp  = nullptr;
    const float*   pp    = scenePoint(a, id, &outp);
    const float    px = pp[0], py = pp[1], pz = pp[2];
    const D3       P     = {double(px), double(py), double(pz)};
    const float    d32   = *outp; // the FP32 pass's union value
    // objects whose box is farther than d32 + delta cannot hold the minimum
    const float    ob    = fmaxf(d32 + delta, 0.f) * 1.00001f;
    const float    obound = ob * ob;
    // a mesh that can hold the minimum has |value| <= |d32| + delta
    const float    mr    = (fabsf(d32) * 1.00001f + delta) * 1.000001f;
    double         best  = CUDART_INF;
    uint32_t       iters = 0;
    int            err   = 0;

    int sp = 1;
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
      const float  d2 = boxDist2(A.x, A.y, A.z, B.x, B.y, B.z, px, py, pz);
      if (!__any_sync(FULL, d2 <= obound)) {
        continue;
      }
      const uint32_t ref = __float_as_uint(A.w), cnt = __float_as_uint(B.w) & EBG_COUNT_MASK;
      if (ref & EBG_LEAF_BIT) {
        const uint32_t o0 = ref & ~EBG_LEAF_BIT;
        for (uint32_t oi = o0; oi < o0 + cnt; oi++) {
          const SceneObject64& o = sc.objects64[oi];
          const D3             q = {P.x - o.t[0], P.y - o.t[1], P.z - o.t[2]};
          if (o.kind == 0) {
            best = fmin(best, sqrt(q.x * q.x + q.y * q.y + q.z * q.z) - o.radius);
            continue;
          }
          // RotateIF's point map, axis by axis, in the reference's order of operations
          D3 L = q;
          if (o.axis == 0) {
            L.y = q.y * o.c + q.z * o.s;
            L.z = -q.y * o.s + q.z * o.c;
          }
          else if (o.axis == 1) {
            L.x = q.x * o.c - q.z * o.s;
            L.z = q.x * o.s + q.z * o.c;
          }
          else {
            L.x = q.x * o.c + q.y * o.s;
            L.y = -q.x * o.s + q.y * o.c;
          }
          const EbgMeshView& mv = sc.meshes[sc.objects[oi].mesh];
          // boxes are tested at the FP32 rounding of the local point, `shift` from it
          const float  lx = float(L.x), ly = float(L.y), lz = float(L.z);
          const double ex = L.x - double(lx), ey = L.y - double(ly), ez = L.z - double(lz);
          const float  shift = float(sqrt(ex * ex + ey * ey + ez * ez)) * 1.0001f;
          const float  r     = (mr + 2.f * shift) * 1.000001f;
          float        bound = r * r;
          double       mb    = DBL_MAX;
          int          mbt   = -1;
          band64Mesh<0>(mv, L, lx, ly, lz, shift, bound, mb, mbt, istk, iters, err);
          if (err) {
            break;
          }
          // The packet opens a leaf when any lane needs it and every lane tests its triangles, so a
          // lane can end with a triangle outside its own radius.  Within mr is the mesh's exact
          // value; beyond it the mesh cannot hold the minimum (its value is above d32 + delta, or
          // below d32 - delta, which the minimum is not) and is left out.
          if (mbt >= 0 && fabs(mb) <= double(mr)) {
            best = fmin(best, mb);
          }
        }
        if (err) {
          break;
        }
      }
      else {
        const EbgNode4& nd = sc.nodes[ref];
        for (int k = 0; k < 4; k++) {
          const float dk = boxDist2(nd.lox[k], nd.loy[k], nd.loz[k], nd.hix[k], nd.hiy[k], nd.hiz[k], px, py, pz);
          if (!(__any_sync(FULL, dk <= obound) && (nd.child[k] | nd.count[k]) != 0u)) {
            continue;
          }
          if (sp >= BAND_OUTER) {
            err |= ST_STACK;
            break;
          }
          if (lane == 0) {
            ostk[2 * sp]     = make_float4(nd.lox[k], nd.loy[k], nd.loz[k], __uint_as_float(nd.child[k]));
            ostk[2 * sp + 1] = make_float4(nd.hix[k], nd.hiy[k], nd.hiz[k], __uint_as_float(nd.count[k]));
          }
          sp++;
        }
        __syncwarp();
        if (err) {
          break;
        }
      }
    }
    if (err && lane == 0) {
      atomicOr(a.status, err);
    }
    // no object within reach cannot happen for a value within the band; keep the FP32 value then
    if (valid && best < CUDART_INF) {
      *outp = float(best);
    }
  }
}

} // namespace

cudaError_t launchSceneBand64(const SceneQueryArgs& a, float delta, int numSms, cudaStream_t s)
{
  kSceneBand64<<<unsigned(numSms * 4), 128, 0, s>>>(a, delta);
  return cudaGetLastError();
}

} // namespace ebg
