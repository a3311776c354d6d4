// FP64 near-surface re-evaluation (sm_100a).  Compiled with -fmad=false: the point-triangle
// arithmetic below keeps the reference's separate multiplies and adds in the reference's order.
//
// Queries whose FP32 distance fell inside the band |d| <= band (default 1e-4 x the mesh's bounding
// box diagonal, where the sign is ill-conditioned) are re-evaluated here with the reference's own
// FP64 triangle test -- a lane-by-lane restatement of the AVX W=4 double path of
// TriangleSoAT::signedDistance (TriangleSoAImplem.hpp:1029-1180) -- over every triangle whose FP32
// (outward-rounded) box lies within |d32| + delta of the point, keeping the value of smallest
// magnitude with strict < (MeshDistanceFunctionsImplem.hpp:492-502).  delta covers the FP32
// distance error, so the FP64 winner is never pruned; leaves and nodes are also pruned by their
// oriented boxes, which bound the exact distance to every triangle inside from below.  Packets of 32 band queries share one
// traversal stack exactly as in the FP32 kernel.
#include <cfloat>

#include <math_constants.h>

#include "ebg_device.cuh"
#include "mesh_kernels.h"
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

// Eight 128-thread blocks per SM (at most 64 registers, a few spills): the FP64 test is latency
// bound, and the extra warps outweigh the spills (12 % faster than 90 registers and five blocks).
// EVAL 0: the reference's Triangle/TriangleSoA test (TriMeshSDF); 1: the DCEL face (MeshSDF).
template <int EVAL>
__global__ void __launch_bounds__(128, 8) kMeshBand64(const MeshQueryArgs a, float delta)
{
  __shared__ float4  smem[4 * 2 * EBG_STACK_DEPTH];
  const int          lane  = threadIdx.x & 31;
  float4*            stk   = smem + (threadIdx.x >> 5) * (2 * EBG_STACK_DEPTH);
  const EbgMeshView& m     = a.mesh;
  const uint32_t     count = *a.band_count;
  const uint32_t     numPk = (count + 31) / 32;
  const uint32_t     warpId = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t     nWarps = (gridDim.x * blockDim.x) >> 5;

  for (uint32_t pk = warpId; pk < numPk; pk += nWarps) {
    const uint32_t j     = pk * 32 + lane;
    const bool     valid = j < count;
    const uint32_t jj    = valid ? j : count - 1;
    const uint32_t pos   = a.band_list[jj];
    const uint32_t id    = a.order ? a.order[pos] : pos;
    // the FP64 point: the caller's own when it passed FP64, else its FP32 point
    const D3       P     = a.points64 ? D3{a.points64[3 * size_t(id)], a.points64[3 * size_t(id) + 1],
                                          a.points64[3 * size_t(id) + 2]}
                                      : D3{double(a.points[3 * size_t(id)]), double(a.points[3 * size_t(id) + 1]),
                                           double(a.points[3 * size_t(id) + 2])};
    const float    px = a.points[3 * size_t(id)], py = a.points[3 * size_t(id) + 1], pz = a.points[3 * size_t(id) + 2];
    const float    d32 = a.band_d32 ? a.band_d32[jj] : a.out_d[id]; // the FP32 pass's distance
    // Boxes are tested at the FP32 point, `shift` from the FP64 point.  The mesh is within
    // |d32| + delta of the FP32 point (delta covers the FP32 distance error near the surface, the
    // relative term far from it), so the FP64 winner is within |d32| + delta + shift of the FP64
    // point and within |d32| + delta + 2 shift of the FP32 point.
    const double   ex = P.x - double(px), ey = P.y - double(py), ez = P.z - double(pz);
    const float    shift = float(sqrt(ex * ex + ey * ey + ez * ez)) * 1.0001f;
    float          r   = (fabsf(d32) * 1.00001f + delta + 2.f * shift) * 1.000001f;
    float          bound = r * r;
    double         best  = DBL_MAX;
    int            bt    = -1;
    uint32_t       iters = 0;
    int            err   = 0;

    int sp = 1;
    if (lane == 0) {
      stk[0] = make_float4(m.root_lo[0], m.root_lo[1], m.root_lo[2], __uint_as_float(m.root_ref));
      stk[1] = make_float4(m.root_hi[0], m.root_hi[1], m.root_hi[2], __uint_as_float(m.root_count));
    }
    __syncwarp();
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
          if (sp >= EBG_STACK_DEPTH) {
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
    if (err && lane == 0) {
      atomicOr(a.status, err);
    }
    if (valid && a.out_d64 != nullptr) {
      a.out_d64[id] = bt >= 0 ? best : double(d32);
    }
    if (valid && bt >= 0) {
      a.out_d[id] = float(best);
      if (a.out_tri) {
        a.out_tri[id] = m.tri_id[bt];
      }
    }
  }
}

// FlatMeshSDF (MeshT::DirectSignedDistance2, DCEL_MeshImplem.hpp:574-595): every face, the first
// in soup order with the smallest unsigned distance^2 wins, and its signed distance is the value.
// One query per thread; the block walks the triangles (leaf order) through shared-memory tiles of
// their vertices and DCEL normals and keeps the lexicographic minimum of (d^2, soup index).
constexpr int FLAT_TILE = 64;

__global__ void __launch_bounds__(128) kMeshFlat64(const EbgMeshView m, int64_t numTris, const double* __restrict__ pts,
                                                   int64_t n, double* __restrict__ out, int32_t* __restrict__ outTri,
                                                   int* __restrict__ status)
{
  __shared__ double  sv[FLAT_TILE][12];
  __shared__ int32_t sid[FLAT_TILE];
  for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < n; base += int64_t(gridDim.x) * blockDim.x) {
    const int64_t q     = base + threadIdx.x;
    const bool    valid = q < n;
    const D3      P     = valid ? D3{pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]} : D3{0.0, 0.0, 0.0};
    const bool    finite = isfinite(P.x) && isfinite(P.y) && isfinite(P.z);
    if (valid && !finite) {
      atomicOr(status, ST_INPUT);
    }
    double        best  = CUDART_INF;
    int32_t       bsoup = INT32_MAX;
    int64_t       bpos  = -1;
    for (int64_t t0 = 0; t0 < numTris; t0 += FLAT_TILE) {
      __syncthreads();
      for (int k = threadIdx.x; k < FLAT_TILE * 12; k += blockDim.x) {
        const int64_t tt = t0 + k / 12;
        const int     c  = k % 12;
        sv[k / 12][c]    = tt < numTris ? (c < 9 ? m.tri64[30 * tt + c] : m.dcel_n[3 * tt + (c - 9)]) : 0.0;
      }
      for (int k = threadIdx.x; k < FLAT_TILE; k += blockDim.x) {
        sid[k] = t0 + k < numTris ? m.tri_id[t0 + k] : INT32_MAX;
      }
      __syncthreads();
      const int cnt = int(numTris - t0 < FLAT_TILE ? numTris - t0 : FLAT_TILE);
      for (int k = 0; k < cnt; k++) {
        const double d2 = dcelFaceUd2(sv[k], sv[k] + 9, P);
        if (d2 < best || (d2 == best && sid[k] < bsoup)) {
          best  = d2;
          bsoup = sid[k];
          bpos  = t0 + k;
        }
      }
    }
    if (valid) {
      // a non-finite point (reported through the status word) gets NaN
      out[q] = (finite && bpos >= 0) ? dcelFaceSd(m.tri64 + 30 * bpos, m.dcel_n + 3 * bpos, P) : CUDART_NAN;
      if (outTri) {
        outTri[q] = (finite && bpos >= 0) ? bsoup : -1;
      }
    }
  }
}

} // namespace

cudaError_t launchMeshFlat64(const EbgMeshView& m, int64_t numTris, const double* pts, int64_t n, double* out,
                             int32_t* outTri, int* status, int numSms, cudaStream_t s)
{
  int64_t blocks = (n + 127) / 128;
  blocks         = blocks < int64_t(numSms) * 16 ? blocks : int64_t(numSms) * 16;
  kMeshFlat64<<<unsigned(blocks < 1 ? 1 : blocks), 128, 0, s>>>(m, numTris, pts, n, out, outTri, status);
  return cudaGetLastError();
}

namespace {
__global__ void kDoubleToFloat(const double* __restrict__ in, float* __restrict__ out, int64_t count)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x) {
    out[i] = float(in[i]);
  }
}
} // namespace

void launchDoubleToFloat(const double* in, float* out, int64_t count, cudaStream_t s)
{
  int64_t blocks = (count + 255) / 256;
  blocks         = blocks < 4096 ? blocks : 4096;
  kDoubleToFloat<<<unsigned(blocks < 1 ? 1 : blocks), 256, 0, s>>>(in, out, count);
}

cudaError_t launchMeshBand64(const MeshQueryArgs& a, float delta, int numSms, cudaStream_t s)
{
  if (a.eval == 1) {
    kMeshBand64<1><<<unsigned(numSms * 8), 128, 0, s>>>(a, delta);
  }
  else {
    kMeshBand64<0><<<unsigned(numSms * 8), 128, 0, s>>>(a, delta);
  }
  return cudaGetLastError();
}

} // namespace ebg
