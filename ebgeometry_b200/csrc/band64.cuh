// FP64 evaluation of mesh triangles for the near-surface passes (sm_100a), shared by the mesh band
// kernel (mesh_band64.cu) and the CSG union's band kernel (scene_band64.cu).  Include it only from
// translation units compiled with -fmad=false: the point-triangle arithmetic keeps the reference's
// separate multiplies and adds in the reference's order.
//
//  - triSd64: a lane-by-lane restatement of the AVX W=4 double path of TriangleSoAT::signedDistance
//    (TriangleSoAImplem.hpp:1029-1180, sign-bit convention of :1076-1082);
//  - dcelFaceSd / dcelFaceUd2: one triangle as a DCEL face, the algorithm of MeshSDF and FlatMeshSDF;
//  - band64Mesh: one packet's FP64 search of a mesh for the triangle of smallest |d| within each
//    lane's bound (strict <, MeshDistanceFunctionsImplem.hpp:492-502).
#ifndef EBG_BAND64_CUH
#define EBG_BAND64_CUH

#include <cfloat>

#include "ebg_device.cuh"
#include "mesh_traverse.cuh"

namespace ebg {

namespace {

struct D3
{
  double x, y, z;
};
__device__ __forceinline__ D3 ld3(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b)
{
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 scl(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double sgnb(double x) { return signbit(x) ? -1.0 : 1.0; }

// tri: v0 v1 v2 n vn0 vn1 vn2 en0 en1 en2 (30 doubles)
__device__ double triSd64(const double* __restrict__ tri, D3 P)
{
  const D3 v0 = ld3(tri), v1 = ld3(tri + 3), v2 = ld3(tri + 6), n = ld3(tri + 9);
  const D3 v21 = sub(v1, v0), v32 = sub(v2, v1), v13 = sub(v0, v2);
  const D3 p1 = sub(P, v0), p2 = sub(P, v1), p3 = sub(P, v2);
  const double s0 = sgnb(dot(cross(v21, n), p1));
  const double s1 = sgnb(dot(cross(v32, n), p2));
  const double s2 = sgnb(dot(cross(v13, n), p3));
  if (fabs((s0 + s1) + s2) >= 2.0) {
    return dot(n, p1);
  }
  const double t1 = dot(p1, v21) / dot(v21, v21);
  const double t2 = dot(p2, v32) / dot(v32, v32);
  const double t3 = dot(p3, v13) / dot(v13, v13);
  const D3     y1 = sub(p1, scl(t1, v21)), y2 = sub(p2, scl(t2, v32)), y3 = sub(p3, scl(t3, v13));

  double bd2 = dot(p1, p1);
  double bs  = sgnb(dot(ld3(tri + 12), p1));
  const double p2d2 = dot(p2, p2), p3d2 = dot(p3, p3);
  if (p2d2 < bd2) {
    bd2 = p2d2;
    bs  = sgnb(dot(ld3(tri + 15), p2));
  }
  if (p3d2 < bd2) {
    bd2 = p3d2;
    bs  = sgnb(dot(ld3(tri + 18), p3));
  }
  const double y1d2 = dot(y1, y1), y2d2 = dot(y2, y2), y3d2 = dot(y3, y3);
  if (t1 > 0.0 && t1 < 1.0 && y1d2 < bd2) {
    bd2 = y1d2;
    bs  = sgnb(dot(ld3(tri + 21), y1));
  }
  if (t2 > 0.0 && t2 < 1.0 && y2d2 < bd2) {
    bd2 = y2d2;
    bs  = sgnb(dot(ld3(tri + 24), y2));
  }
  if (t3 > 0.0 && t3 < 1.0 && y3d2 < bd2) {
    bd2 = y3d2;
    bs  = sgnb(dot(ld3(tri + 27), y3));
  }
  return bs * sqrt(bd2);
}

// ---- one triangle as a DCEL face: the algorithm of MeshSDF and FlatMeshSDF ----------------------
// (FaceT::signedDistance / unsignedDistance2, DCEL_FaceImplem.hpp:388-458; EdgeT, DCEL_EdgeImplem.hpp:
// 283-358; VertexT, DCEL_VertexImplem.hpp:368-380; Polygon2D crossing number,
// Polygon2DImplem.hpp:80-118,164-193).  It differs from the Triangle test above in the last bits:
// the face value is n . (p - centroid) with the DCEL normal, and vertex/edge signs are
// (pseudonormal . delta > 0 ? +1 : -1).

__device__ __forceinline__ D3 add3(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ double len3(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

__device__ __forceinline__ double dcelVertexSd(D3 x, D3 vn, D3 P)
{
  const D3 d = sub(P, x);
  return len3(d) * ((dot(vn, d) > 0.0) ? 1.0 : -1.0);
}

__device__ __forceinline__ D3 dcelCentroid(D3 x0, D3 x1, D3 x2)
{
  const double is = 1.0 / 3.0;
  return scl(is, add3(add3(x0, x1), x2));
}

// crossing number of P projected into the face plane, in the 2D projection that drops the axis of
// largest |n| (the first on ties)
__device__ __forceinline__ bool dcelInside(const D3 (&x)[3], D3 n, D3 c, D3 P)
{
  const double ax = fabs(n.x), ay = fabs(n.y), az = fabs(n.z);
  int          ig = 0;
  if (ay > ax) {
    ig = 1;
  }
  if (az > (ig == 0 ? ax : ay)) {
    ig = 2;
  }
  const D3     q  = sub(P, scl(dot(n, sub(P, c)), n));
  const double qx = ig == 0 ? q.y : q.x, qy = ig == 2 ? q.y : q.z;
  int          cn = 0;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const D3     a = x[i], b = x[(i + 1) % 3];
    const double ax2 = ig == 0 ? a.y : a.x, ay2 = ig == 2 ? a.y : a.z;
    const double bx2 = ig == 0 ? b.y : b.x, by2 = ig == 2 ? b.y : b.z;
    const bool   up = (ay2 <= qy) && (by2 > qy), down = (ay2 > qy) && (by2 <= qy);
    if (up || down) {
      const double t = (qy - ay2) / (by2 - ay2);
      if (qx < ax2 + t * (bx2 - ax2)) {
        cn++;
      }
    }
  }
  return (cn & 1) != 0;
}

// tri: the 30-double record (v0 v1 v2 n vn0 vn1 vn2 en0 en1 en2); fn: the DCEL face normal
__device__ double dcelFaceSd(const double* __restrict__ tri, const double* __restrict__ fn, D3 P)
{
  const D3 x[3] = {ld3(tri), ld3(tri + 3), ld3(tri + 6)};
  const D3 n    = ld3(fn);
  const D3 c    = dcelCentroid(x[0], x[1], x[2]);
  if (dcelInside(x, n, c, P)) {
    return dot(n, sub(P, c));
  }
  double best = CUDART_INF;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const int    j    = (i + 1) % 3;
    const D3     x2x1 = sub(x[j], x[i]);
    const double t    = dot(sub(P, x[i]), x2x1) / dot(x2x1, x2x1);
    double       d;
    if (t <= 0.0) {
      d = dcelVertexSd(x[i], ld3(tri + 12 + 3 * i), P);
    }
    else if (t >= 1.0) {
      d = dcelVertexSd(x[j], ld3(tri + 12 + 3 * j), P);
    }
    else {
      const D3 delta = sub(P, add3(x[i], scl(t, x2x1)));
      d              = ((dot(ld3(tri + 21 + 3 * i), delta) > 0.0) ? 1.0 : -1.0) * len3(delta);
    }
    best = fabs(d) < fabs(best) ? d : best;
  }
  return best;
}

__device__ double dcelFaceUd2(const double* __restrict__ tri, const double* __restrict__ fn, D3 P)
{
  const D3 x[3] = {ld3(tri), ld3(tri + 3), ld3(tri + 6)};
  const D3 n    = ld3(fn);
  const D3 c    = dcelCentroid(x[0], x[1], x[2]);
  if (dcelInside(x, n, c, P)) {
    const double nd = dot(n, sub(P, c));
    return nd * nd;
  }
  double best = CUDART_INF;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const D3 x2x1 = sub(x[(i + 1) % 3], x[i]);
    double   t    = dot(sub(P, x[i]), x2x1) / dot(x2x1, x2x1);
    t             = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
    const D3     delta = sub(P, add3(x[i], scl(t, x2x1)));
    const double d2    = dot(delta, delta);
    best               = d2 < best ? d2 : best;
  }
  return best;
}

// One packet's FP64 search of mesh m.  Each lane has its FP64 point P, the FP32 point (px, py, pz)
// at which boxes are tested (`shift` from P), its squared search bound `bound` (FP32, at the FP32
// point) and its running FP64 result (best, bt: the value of smallest |d| and its triangle, leaf
// order; DBL_MAX / -1 before the first).  Triangles are tested in FP64 with the Triangle test
// (EVAL 0, TriMeshSDF) or the DCEL face (EVAL 1, MeshSDF); each winner shrinks the lane's bound.
// Leaves and nodes are pruned by their axis-aligned and oriented boxes (padded to bound the exact
// distance of every triangle inside from below).  All 32 lanes call it together; `stk` is the
// warp's stack (STACK entries).  The search starts from the `sp0` entries already on the stack
// (a cell's cut, the top entry popped first), or from the root when sp0 is 0.
template <int EVAL, int STACK = EBG_STACK_DEPTH>
__device__ void band64Mesh(const EbgMeshView& m, D3 P, float px, float py, float pz, float shift, float& bound,
                           double& best, int& bt, float4* stk, uint32_t& iters, int& err, int sp0 = 0)
{
  const int lane = threadIdx.x & 31;
  int sp = sp0;
  if (sp0 == 0) {
    sp = 1;
    if (lane == 0) {
      stk[0] = make_float4(m.root_lo[0], m.root_lo[1], m.root_lo[2], __uint_as_float(m.root_ref));
      stk[1] = make_float4(m.root_hi[0], m.root_hi[1], m.root_hi[2], __uint_as_float(m.root_count));
    }
    __syncwarp();
  }
  while (sp > 0) {
    if (++iters > MAX_ITERS) {
      err |= ST_ITERS;
      break;
    }
    --sp;
    const float4 A = stk[2 * sp], B = stk[2 * sp + 1];
    const float  d2 = boxDist2(A.x, A.y, A.z, B.x, B.y, B.z, px, py, pz);
    if (!__any_sync(FULL, d2 <= bound)) {
      continue;
    }
    const uint32_t cntw = __float_as_uint(B.w);
    const uint32_t ref = __float_as_uint(A.w), cnt = cntw & EBG_COUNT_MASK;
    // the leaf's or node's oriented box (padded to bound the exact distance of every triangle
    // inside from below) before its triangles or children
    const EbgObb* obx = (ref & EBG_LEAF_BIT) ? m.obb + (cntw >> EBG_COUNT_BITS)
                                             : ((cntw & EBG_NODE_HAS_OBB) ? m.node_obb + ref : nullptr);
    if (obx != nullptr) {
      const float4* ob = reinterpret_cast<const float4*>(obx);
      if (!__any_sync(FULL, obbDist2(__ldg(ob), __ldg(ob + 1), __ldg(ob + 2), __ldg(ob + 3), px, py, pz) <= bound)) {
        continue;
      }
    }
    if (ref & EBG_LEAF_BIT) {
      const uint32_t t0 = ref & ~EBG_LEAF_BIT;
      for (uint32_t tt = t0; tt < t0 + cnt; ++tt) {
        const double d = EVAL == 0 ? triSd64(m.tri64 + 30 * size_t(tt), P)
                                   : dcelFaceSd(m.tri64 + 30 * size_t(tt), m.dcel_n + 3 * size_t(tt), P);
        // strict < as the reference's leaf loop, ties to the lower leaf position (the winner is
        // then independent of the traversal order)
        if (fabs(d) < fabs(best) || (fabs(d) == fabs(best) && int(tt) < bt)) {
          best = d;
          bt   = int(tt);
          // shrink the bound to the FP64 winner (with the same relative margin), measured at the
          // FP32 point where the boxes are tested
          const float rb = (float(fabs(d)) + shift) * 1.000001f + 1e-30f;
          bound          = fminf(bound, rb * rb);
        }
      }
    }
    else {
      const EbgNode4& nd = m.nodes[ref];
      int             o[4], np = 0;
      float           key[4];
      for (int k = 0; k < 4; k++) {
        const float dk = boxDist2(nd.lox[k], nd.loy[k], nd.loz[k], nd.hix[k], nd.hiy[k], nd.hiz[k], px, py, pz);
        // empty slot: child 0 and count 0 (node 0 is the root and never a child)
        if (__any_sync(FULL, dk <= bound) && (nd.child[k] | nd.count[k]) != 0u) {
          o[np]   = k;
          key[np] = dk;
          np++;
        }
      }
      // per-lane keys differ, so order by lane 0's distance (any fixed order is correct)
      for (int i = 0; i < np; i++) {
        key[i] = __shfl_sync(FULL, key[i], 0);
      }
      for (int i = 1; i < np; i++) {
        for (int q = i; q > 0 && key[q - 1] < key[q]; q--) {
          const float tk = key[q];
          key[q]         = key[q - 1];
          key[q - 1]     = tk;
          const int to   = o[q];
          o[q]           = o[q - 1];
          o[q - 1]       = to;
        }
      }
      for (int i = 0; i < np; i++) {
        if (sp >= STACK) {
          err |= ST_STACK;
          break;
        }
        const int k = o[i];
        if (lane == 0) {
          stk[2 * sp]     = make_float4(nd.lox[k], nd.loy[k], nd.loz[k], __uint_as_float(nd.child[k]));
          stk[2 * sp + 1] = make_float4(nd.hix[k], nd.hiy[k], nd.hiz[k], __uint_as_float(nd.count[k]));
        }
        sp++;
      }
      __syncwarp();
      if (err) {
        break;
      }
    }
  }
}

} // namespace

} // namespace ebg

#endif
