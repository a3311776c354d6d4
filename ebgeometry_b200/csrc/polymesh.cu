// Meshes of polygon faces (sm_100a): the reference's MeshSDF<T, Meta, K> and FlatMeshSDF<T, Meta> over
// a DCEL whose faces have any number of vertices (MeshDistanceFunctionsImplem.hpp:210-295;
// DCEL_FaceImplem.hpp:379-458; DCEL_EdgeImplem.hpp:283-358; DCEL_VertexImplem.hpp:368-380;
// Polygon2DImplem.hpp:80-118,164-193).  FP64 throughout, compiled without fused multiply-adds, so
// every face value is the reference's own.
//
// Layout in HBM (faces in leaf order; all FP64 unless noted):
//   nodes[num_nodes]        EbgNode4, FP32 boxes rounded outward (the triangle mesh's layout)
//   face[num_faces]         uint2: first corner, corner count
//   face_rec[num_faces][6]  the DCEL normal and the centroid
//   corner[num_corners][9]  the corner's position, its vertex pseudonormal, the pseudonormal of the
//                           edge from it to the next corner
//   face_id[num_faces]      int32: the face's index in the caller's soup
//
// MeshSDF: one warp per 32 Morton-ordered queries, boxes tested in FP32 at the FP32 rounding of the
// point (bound r = (|best| + shift) (1 + 1e-6), shift = |P64 - P32|), faces evaluated in FP64; the
// smallest |d| wins, ties to the lower leaf position.  FlatMeshSDF (MeshT::DirectSignedDistance2,
// DCEL_MeshImplem.hpp:574-595): one thread per point over every face, the first face in soup order
// with the smallest unsigned distance, then its signed distance.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>
#include <math_constants.h>

#include "capi_common.h"
#include "ebg_device.cuh"
#include "ebgeometry_b200.h"
#include "mesh_host.h"
#include "mesh_kernels.h"

namespace ebg {
namespace {

struct PolyView
{
  const EbgNode4* nodes;
  const uint2*    face;
  const double*   faceRec;
  const double*   corner;
  const int32_t*  faceId;
  uint32_t        rootRef, rootCount;
  float           rootLo[3], rootHi[3];
  int64_t         numFaces;
};

struct PolyArgs
{
  PolyView        m;
  const double*   pts64;
  const float*    pts32;
  const uint32_t* order;
  int64_t         n;
  double*         out;
  int32_t*        outFace;
  int*            status;
};

struct P3
{
  double x, y, z;
};
__device__ __forceinline__ P3 ld(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ P3 add(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ P3 scl(double s, P3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double len(P3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

// the crossing number of P projected into the face plane, in the 2D projection that drops the axis
// of largest |n| (the first on ties)
__device__ bool polyInside(const double* __restrict__ cr, uint32_t N, P3 n, P3 c, P3 P)
{
  const double ax = fabs(n.x), ay = fabs(n.y), az = fabs(n.z);
  int          ig = 0;
  if (ay > ax) {
    ig = 1;
  }
  if (az > (ig == 0 ? ax : ay)) {
    ig = 2;
  }
  const P3     q  = sub(P, scl(dot(n, sub(P, c)), n));
  const double qx = ig == 0 ? q.y : q.x, qy = ig == 2 ? q.y : q.z;
  int          cn = 0;
  for (uint32_t i = 0; i < N; i++) {
    const double* a   = cr + 9 * size_t(i);
    const double* b   = cr + 9 * size_t(i + 1 == N ? 0 : i + 1);
    const double  ax2 = ig == 0 ? a[1] : a[0], ay2 = ig == 2 ? a[1] : a[2];
    const double  bx2 = ig == 0 ? b[1] : b[0], by2 = ig == 2 ? b[1] : b[2];
    const bool    up = (ay2 <= qy) && (by2 > qy), down = (ay2 > qy) && (by2 <= qy);
    if (up || down) {
      const double t = (qy - ay2) / (by2 - ay2);
      if (qx < ax2 + t * (bx2 - ax2)) {
        cn++;
      }
    }
  }
  return (cn & 1) != 0;
}

__device__ __forceinline__ double vertexSd(P3 x, P3 vn, P3 P)
{
  const P3 d = sub(P, x);
  return len(d) * ((dot(vn, d) > 0.0) ? 1.0 : -1.0);
}

// FaceT::signedDistance of the face at leaf position f
__device__ double polyFaceSd(const PolyView& m, uint32_t f, P3 P)
{
  const uint2   fc = m.face[f];
  const double* fr = m.faceRec + 6 * size_t(f);
  const double* cr = m.corner + 9 * size_t(fc.x);
  const P3      n = ld(fr), c = ld(fr + 3);
  if (polyInside(cr, fc.y, n, c, P)) {
    return dot(n, sub(P, c));
  }
  double best = CUDART_INF;
  for (uint32_t i = 0; i < fc.y; i++) {
    const double* a    = cr + 9 * size_t(i);
    const double* b    = cr + 9 * size_t(i + 1 == fc.y ? 0 : i + 1);
    const P3      xi   = ld(a), xj = ld(b);
    const P3      x2x1 = sub(xj, xi);
    const double  t    = dot(sub(P, xi), x2x1) / dot(x2x1, x2x1);
    double        d;
    if (t <= 0.0) {
      d = vertexSd(xi, ld(a + 3), P);
    }
    else if (t >= 1.0) {
      d = vertexSd(xj, ld(b + 3), P);
    }
    else {
      const P3 delta = sub(P, add(xi, scl(t, x2x1)));
      d              = ((dot(ld(a + 6), delta) > 0.0) ? 1.0 : -1.0) * len(delta);
    }
    best = fabs(d) < fabs(best) ? d : best;
  }
  return best;
}

// FaceT::unsignedDistance2 of the face at leaf position f
__device__ double polyFaceUd2(const PolyView& m, uint32_t f, P3 P)
{
  const uint2   fc = m.face[f];
  const double* fr = m.faceRec + 6 * size_t(f);
  const double* cr = m.corner + 9 * size_t(fc.x);
  const P3      n = ld(fr), c = ld(fr + 3);
  if (polyInside(cr, fc.y, n, c, P)) {
    const double nd = dot(n, sub(P, c));
    return nd * nd;
  }
  double best = CUDART_INF;
  for (uint32_t i = 0; i < fc.y; i++) {
    const P3 xi   = ld(cr + 9 * size_t(i));
    const P3 x2x1 = sub(ld(cr + 9 * size_t(i + 1 == fc.y ? 0 : i + 1)), xi);
    double   t    = dot(sub(P, xi), x2x1) / dot(x2x1, x2x1);
    t             = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
    const P3     delta = sub(P, add(xi, scl(t, x2x1)));
    const double d2    = dot(delta, delta);
    best               = d2 < best ? d2 : best;
  }
  return best;
}

__global__ void __launch_bounds__(128) kPolySdf64(const PolyArgs a)
{
  __shared__ float4 smem[4 * 2 * EBG_STACK_DEPTH];
  const int         lane   = threadIdx.x & 31;
  float4*           stk    = smem + (threadIdx.x >> 5) * (2 * EBG_STACK_DEPTH);
  const PolyView&   m      = a.m;
  const int64_t     numPk  = (a.n + 31) / 32;
  const int64_t     warpId = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t     nWarps = (int64_t(gridDim.x) * blockDim.x) >> 5;

  for (int64_t pk = warpId; pk < numPk; pk += nWarps) {
    const int64_t j     = pk * 32 + lane;
    const bool    valid = j < a.n;
    const int64_t jj    = valid ? j : a.n - 1;
    const int64_t id    = a.order ? int64_t(a.order[jj]) : jj;
    const P3      P     = {a.pts64[3 * id], a.pts64[3 * id + 1], a.pts64[3 * id + 2]};
    const float   px = a.pts32[3 * id], py = a.pts32[3 * id + 1], pz = a.pts32[3 * id + 2];
    int           err   = 0;
    if (!(isfinite(P.x) && isfinite(P.y) && isfinite(P.z))) {
      err |= ST_INPUT;
    }
    const double ex = P.x - double(px), ey = P.y - double(py), ez = P.z - double(pz);
    const float  shift = float(sqrt(ex * ex + ey * ey + ez * ez)) * 1.0001f;
    float        bound = __int_as_float(0x7f800000);
    double       best  = CUDART_INF;
    int          bt    = -1;
    uint32_t     iters = 0;

    int sp = 1;
    if (lane == 0) {
      stk[0] = make_float4(m.rootLo[0], m.rootLo[1], m.rootLo[2], __uint_as_float(m.rootRef));
      stk[1] = make_float4(m.rootHi[0], m.rootHi[1], m.rootHi[2], __uint_as_float(m.rootCount));
    }
    __syncwarp();
    while (sp > 0) {
      if (++iters > MAX_ITERS) {
        err |= ST_ITERS;
        break;
      }
      --sp;
      const float4 A    = stk[2 * sp];
      const float4 B    = stk[2 * sp + 1];
      const bool   need = valid && boxDist2(A.x, A.y, A.z, B.x, B.y, B.z, px, py, pz) <= bound;
      if (!__any_sync(FULL, need)) {
        continue;
      }
      const uint32_t ref = __float_as_uint(A.w), cntw = __float_as_uint(B.w);
      if (ref & EBG_LEAF_BIT) {
        const uint32_t f0 = ref & ~EBG_LEAF_BIT, cnt = cntw & EBG_COUNT_MASK;
        if (need) {
          for (uint32_t f = f0; f < f0 + cnt; f++) {
            const double d = polyFaceSd(m, f, P);
            // strict < as the reference's leaf loop, ties to the lower leaf position
            if (fabs(d) < fabs(best) || (fabs(d) == fabs(best) && int(f) < bt)) {
              best               = d;
              bt                 = int(f);
              const float rb     = (float(fabs(d)) + shift) * 1.000001f + 1e-30f;
              bound              = fminf(bound, rb * rb);
            }
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
          if (__any_sync(FULL, valid && dk <= bound) && (nd.child[k] | nd.count[k]) != 0u) {
            o[np]   = k;
            key[np] = dk;
            np++;
          }
        }
        // nearest first by the packet's smallest distance to each child
        for (int i = 0; i < np; i++) {
          key[i] = __uint_as_float(__reduce_min_sync(FULL, __float_as_uint(valid ? key[i] : FLT_MAX)));
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
        if (sp + np > EBG_STACK_DEPTH) {
          err |= ST_STACK;
          break;
        }
        for (int i = 0; i < np; i++) {
          const int k = o[i];
          if (lane == 0) {
            stk[2 * sp]     = make_float4(nd.lox[k], nd.loy[k], nd.loz[k], __uint_as_float(nd.child[k]));
            stk[2 * sp + 1] = make_float4(nd.hix[k], nd.hiy[k], nd.hiz[k], __uint_as_float(nd.count[k]));
          }
          sp++;
        }
        __syncwarp();
      }
    }
    err = __reduce_or_sync(FULL, valid ? err : 0);
    if (err && lane == 0) {
      atomicOr(a.status, err);
    }
    if (valid) {
      a.out[id] = (err & ST_INPUT) && !(isfinite(P.x) && isfinite(P.y) && isfinite(P.z)) ? CUDART_NAN : best;
      if (a.outFace) {
        a.outFace[id] = bt >= 0 ? m.faceId[bt] : -1;
      }
    }
  }
}

__global__ void __launch_bounds__(128) kPolyFlat64(const PolyArgs a)
{
  const PolyView& m = a.m;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.n; i += int64_t(gridDim.x) * blockDim.x) {
    const P3 P = {a.pts64[3 * i], a.pts64[3 * i + 1], a.pts64[3 * i + 2]};
    if (!(isfinite(P.x) && isfinite(P.y) && isfinite(P.z))) {
      atomicOr(a.status, ST_INPUT);
      a.out[i] = CUDART_NAN;
      if (a.outFace) {
        a.outFace[i] = -1;
      }
      continue;
    }
    double  bd2 = CUDART_INF;
    int32_t bid = INT32_MAX;
    int64_t bf  = -1;
    for (int64_t f = 0; f < m.numFaces; f++) {
      const double  d2  = polyFaceUd2(m, uint32_t(f), P);
      const int32_t sid = m.faceId[f];
      // the first face in soup order with the smallest unsigned distance
      if (d2 < bd2 || (d2 == bd2 && sid < bid)) {
        bd2 = d2;
        bid = sid;
        bf  = f;
      }
    }
    a.out[i] = bf >= 0 ? polyFaceSd(m, uint32_t(bf), P) : CUDART_INF;
    if (a.outFace) {
      a.outFace[i] = bf >= 0 ? bid : -1;
    }
  }
}

} // namespace
} // namespace ebg

struct ebg_polymesh
{
  int            device = 0;
  int            numSms = 148;
  ebg::PolyView  view{};
  ebg_mesh_info  info{};
  int64_t        numCorners = 0;
  EbgNode4*      dNodes     = nullptr;
  uint2*         dFace      = nullptr;
  double*        dFaceRec   = nullptr;
  double*        dCorner    = nullptr;
  int32_t*       dFaceId    = nullptr;
  int*           dStatus    = nullptr;
  float          mortonLo[3]    = {0, 0, 0};
  float          mortonScale[3] = {1, 1, 1};
};

using namespace ebg;

namespace {

ebg_status buildPoly(const double* V, int64_t nv, const int64_t* off, const int32_t* idx, int64_t nf,
                     const ebg_build_opts* opts, ebg_polymesh** out)
{
  if (out == nullptr) {
    return setError(EBG_ERR_INVALID, "out handle pointer is null");
  }
  *out = nullptr;
  if (V == nullptr || off == nullptr || idx == nullptr || nv <= 0 || nf <= 0) {
    return setError(EBG_ERR_INVALID, "polygon mesh needs vertices and at least one face");
  }
  if (nf >= int64_t(EBG_LEAF_BIT) || nv > int64_t(INT32_MAX) || off[nf] > int64_t(UINT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "mesh too large (faces < 2^31, vertices < 2^31, corners < 2^32)");
  }
  if (off[0] != 0) {
    return setError(EBG_ERR_INVALID, "face offsets must start at 0");
  }
  for (int64_t f = 0; f < nf; f++) {
    const int64_t b = off[f], e = off[f + 1];
    if (e - b < 3) {
      return setError(EBG_ERR_INVALID, "face " + std::to_string(f) + " has fewer than three vertices");
    }
    for (int64_t k = b; k < e; k++) {
      if (idx[k] < 0 || idx[k] >= nv) {
        return setError(EBG_ERR_INVALID, "face " + std::to_string(f) + " references a vertex out of range");
      }
      for (int64_t q = b; q < k; q++) {
        if (idx[q] == idx[k]) {
          return setError(EBG_ERR_INVALID, "face " + std::to_string(f) + " visits a vertex twice");
        }
      }
    }
  }
  for (int64_t i = 0; i < 3 * nv; i++) {
    if (!std::isfinite(V[i])) {
      return setError(EBG_ERR_INVALID, "non-finite vertex coordinate");
    }
  }
  const int build    = opts ? opts->build : EBG_BUILD_SAH;
  const int leafSize = (opts && opts->leaf_size > 0) ? opts->leaf_size : 4;
  int       device   = (opts && opts->device >= 0) ? opts->device : -1;
  if (build != EBG_BUILD_SAH && build != EBG_BUILD_MORTON) {
    return setError(EBG_ERR_INVALID, "unknown build method");
  }
  if (opts && (opts->flags & EBG_BUILD_ON_DEVICE)) {
    return setError(EBG_ERR_INVALID, "polygon meshes are built on the host");
  }
  DeviceGuard guard;
  if (device >= 0) {
    if (cudaSetDevice(device) != cudaSuccess) {
      return setError(EBG_ERR_NOT_FOUND, "cannot select CUDA device " + std::to_string(device));
    }
  }
  else if (cudaGetDevice(&device) != cudaSuccess) {
    return setError(EBG_ERR_NOT_FOUND, "no CUDA device");
  }
  keepPoolMemory();
  std::string         msg;
  std::vector<double> faceN, cen, cornerVN, edgeN;
  if (!computePolygonNormals(V, nv, off, idx, nf, faceN, cen, cornerVN, edgeN, msg)) {
    return setError(EBG_ERR_INVALID, msg);
  }
  // face boxes and the tree
  std::vector<double> lo(3 * nf), hi(3 * nf);
  for (int64_t f = 0; f < nf; f++) {
    for (int a = 0; a < 3; a++) {
      double l = DBL_MAX, h = -DBL_MAX;
      for (int64_t k = off[f]; k < off[f + 1]; k++) {
        l = std::min(l, V[3 * int64_t(idx[k]) + a]);
        h = std::max(h, V[3 * int64_t(idx[k]) + a]);
      }
      lo[3 * f + a] = l;
      hi[3 * f + a] = h;
    }
  }
  Bvh4 bvh;
  if (!buildBvh4(lo, hi, cen, build, std::min(leafSize, int(EBG_MAX_LEAF)), bvh, msg)) {
    return setError(EBG_ERR_INVALID, msg);
  }
  // leaf-ordered records
  const int64_t         nc = off[nf];
  std::vector<uint2>    face(nf);
  std::vector<double>   faceRec(6 * nf), corner(9 * size_t(nc));
  std::vector<int32_t>  faceId(nf);
  int64_t               at = 0;
  for (int64_t p = 0; p < nf; p++) {
    const int64_t f = bvh.order[p];
    faceId[p]       = int32_t(f);
    face[p]         = make_uint2(uint32_t(at), uint32_t(off[f + 1] - off[f]));
    for (int a = 0; a < 3; a++) {
      faceRec[6 * p + a]     = faceN[3 * f + a];
      faceRec[6 * p + 3 + a] = cen[3 * f + a];
    }
    for (int64_t k = off[f]; k < off[f + 1]; k++, at++) {
      double* c = &corner[9 * size_t(at)];
      for (int a = 0; a < 3; a++) {
        c[a]     = V[3 * int64_t(idx[k]) + a];
        c[3 + a] = cornerVN[3 * k + a];
        c[6 + a] = edgeN[3 * k + a];
      }
    }
  }
  auto* m   = new ebg_polymesh;
  m->device = device;
  cudaDeviceGetAttribute(&m->numSms, cudaDevAttrMultiProcessorCount, device);
  auto up = [](void** dst, const void* src, size_t bytes) -> bool {
    if (cudaMalloc(dst, std::max<size_t>(bytes, 16)) != cudaSuccess) {
      return false;
    }
    return bytes == 0 || cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  if (!up((void**)&m->dNodes, bvh.nodes.data(), bvh.nodes.size() * sizeof(EbgNode4)) ||
      !up((void**)&m->dFace, face.data(), face.size() * sizeof(uint2)) ||
      !up((void**)&m->dFaceRec, faceRec.data(), faceRec.size() * sizeof(double)) ||
      !up((void**)&m->dCorner, corner.data(), corner.size() * sizeof(double)) ||
      !up((void**)&m->dFaceId, faceId.data(), faceId.size() * sizeof(int32_t)) ||
      cudaMalloc((void**)&m->dStatus, sizeof(int)) != cudaSuccess ||
      cudaMemset(m->dStatus, 0, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    ebg_polymesh_destroy(m);
    return setError(EBG_ERR_NO_MEMORY, "device allocation or upload failed for the polygon mesh");
  }
  PolyView& v  = m->view;
  v.nodes      = m->dNodes;
  v.face       = m->dFace;
  v.faceRec    = m->dFaceRec;
  v.corner     = m->dCorner;
  v.faceId     = m->dFaceId;
  v.rootRef    = bvh.rootRef;
  v.rootCount  = bvh.rootCount;
  v.numFaces   = nf;
  double d2    = 0;
  for (int a = 0; a < 3; a++) {
    v.rootLo[a]       = roundDown(bvh.lo[a]);
    v.rootHi[a]       = roundUp(bvh.hi[a]);
    const double c    = 0.5 * (bvh.lo[a] + bvh.hi[a]);
    const double ext  = std::max(bvh.hi[a] - bvh.lo[a], 1e-30);
    m->mortonLo[a]    = float(c - ext);
    m->mortonScale[a] = float(1024.0 / (2.0 * ext));
    m->info.lo[a]     = bvh.lo[a];
    m->info.hi[a]     = bvh.hi[a];
    d2 += (bvh.hi[a] - bvh.lo[a]) * (bvh.hi[a] - bvh.lo[a]);
  }
  m->numCorners         = nc;
  m->info.num_triangles = nf;
  m->info.num_vertices  = nv;
  m->info.num_nodes     = int64_t(bvh.nodes.size());
  m->info.num_leaves    = bvh.numLeaves;
  m->info.depth         = bvh.depth;
  m->info.leaf_size     = leafSize;
  m->info.diagonal      = std::sqrt(d2);
  m->info.device_bytes  = int64_t(bvh.nodes.size() * sizeof(EbgNode4) + size_t(nf) * (8 + 48 + 4) + size_t(nc) * 72);
  *out                  = m;
  return EBG_OK;
}

// MeshSDF (flat = false) or FlatMeshSDF (flat = true) on device arrays, asynchronous on s
ebg_status polyQuery(const ebg_polymesh* m, const double* pts, int64_t n, double* out, int32_t* outFace, bool flat,
                     cudaStream_t s)
{
  PolyArgs a{};
  a.m       = m->view;
  a.pts64   = pts;
  a.n       = n;
  a.out     = out;
  a.outFace = outFace;
  a.status  = m->dStatus;
  if (flat) {
    const int64_t blocks = std::min<int64_t>((n + 127) / 128, int64_t(m->numSms) * 16);
    kPolyFlat64<<<unsigned(std::max<int64_t>(blocks, 1)), 128, 0, s>>>(a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? EBG_OK : setError(EBG_ERR_CUDA, std::string("polygon flat launch: ") + cudaGetErrorString(e));
  }
  std::vector<void*> ws;
  auto get = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMallocAsync(&p, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    ws.push_back(p);
    return p;
  };
  auto*  p32  = static_cast<float*>(get(12 * size_t(n)));
  auto*  kin  = static_cast<uint32_t*>(get(4 * size_t(n)));
  auto*  kout = static_cast<uint32_t*>(get(4 * size_t(n)));
  auto*  iin  = static_cast<uint32_t*>(get(4 * size_t(n)));
  auto*  ord  = static_cast<uint32_t*>(get(4 * size_t(n)));
  size_t tb   = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, iin, ord, int(n), 0, 30, s);
  void* tmp = get(tb);
  if (!p32 || !kin || !kout || !iin || !ord || !tmp) {
    for (void* p : ws) {
      cudaFreeAsync(p, s);
    }
    return setError(EBG_ERR_NO_MEMORY, "polygon query workspace");
  }
  launchDoubleToFloat(pts, p32, 3 * n, s);
  launchQueryKeys(p32, n, m->mortonLo, m->mortonScale, kin, iin, s);
  cub::DeviceRadixSort::SortPairs(tmp, tb, kin, kout, iin, ord, int(n), 0, 30, s);
  a.pts32 = p32;
  a.order = ord;
  kPolySdf64<<<unsigned(m->numSms * 8), 128, 0, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  for (void* p : ws) {
    cudaFreeAsync(p, s);
  }
  return e == cudaSuccess ? EBG_OK : setError(EBG_ERR_CUDA, std::string("polygon query launch: ") + cudaGetErrorString(e));
}

ebg_status polyCheck(const ebg_polymesh* m, cudaStream_t s)
{
  int st = 0;
  if (cudaMemcpyAsync(&st, m->dStatus, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  if (st != 0) {
    cudaMemsetAsync(m->dStatus, 0, sizeof(int), s);
    cudaStreamSynchronize(s);
    if (st & ST_INPUT) {
      return setError(EBG_ERR_INVALID, "non-finite query coordinate");
    }
    return setError(EBG_ERR_TRAVERSAL, "traversal stack or iteration bound reached");
  }
  return EBG_OK;
}

ebg_status polyDevice(const ebg_polymesh* m, const double* pts, int64_t n, double* out, int32_t* face, void* stream,
                      bool flat)
{
  if (m == nullptr || n < 0 || (n > 0 && (pts == nullptr || out == nullptr))) {
    return setError(EBG_ERR_INVALID, "bad polygon mesh query arguments");
  }
  if (n > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 points per call");
  }
  if (n == 0) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  return polyQuery(m, pts, n, out, face, flat, static_cast<cudaStream_t>(stream));
}

ebg_status polyHost(const ebg_polymesh* m, const double* pts, int64_t n, double* out, int32_t* face, void* stream,
                    bool flat)
{
  if (m == nullptr || n < 0 || (n > 0 && (pts == nullptr || out == nullptr))) {
    return setError(EBG_ERR_INVALID, "bad polygon mesh query arguments");
  }
  if (n > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 points per call");
  }
  if (n == 0) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  cudaStream_t s  = static_cast<cudaStream_t>(stream);
  double *     dp = nullptr, *dd = nullptr;
  int32_t*     df = nullptr;
  bool ok = cudaMallocAsync((void**)&dp, 24 * size_t(n), s) == cudaSuccess &&
            cudaMallocAsync((void**)&dd, 8 * size_t(n), s) == cudaSuccess &&
            (face == nullptr || cudaMallocAsync((void**)&df, 4 * size_t(n), s) == cudaSuccess);
  ebg_status rc = ok ? EBG_OK : setError(EBG_ERR_NO_MEMORY, "device buffers for the host call");
  if (rc == EBG_OK) {
    cudaMemcpyAsync(dp, pts, 24 * size_t(n), cudaMemcpyHostToDevice, s);
    rc = polyQuery(m, dp, n, dd, df, flat, s);
  }
  if (rc == EBG_OK) {
    cudaMemcpyAsync(out, dd, 8 * size_t(n), cudaMemcpyDeviceToHost, s);
    if (face) {
      cudaMemcpyAsync(face, df, 4 * size_t(n), cudaMemcpyDeviceToHost, s);
    }
  }
  for (void* p : {(void*)dp, (void*)dd, (void*)df}) {
    if (p) {
      cudaFreeAsync(p, s);
    }
  }
  cudaGetLastError();
  const ebg_status cs = polyCheck(m, s);
  return rc != EBG_OK ? rc : cs;
}

} // namespace

extern "C" {

ebg_status ebg_polymesh_create(const double*         vertices,
                               int64_t               num_vertices,
                               const int64_t*        face_offsets,
                               const int32_t*        face_vertices,
                               int64_t               num_faces,
                               const ebg_build_opts* opts,
                               ebg_polymesh**        out)
{
  return buildPoly(vertices, num_vertices, face_offsets, face_vertices, num_faces, opts, out);
}

ebg_status ebg_polymesh_create_from_file(const char* path, const ebg_build_opts* opts, ebg_polymesh** out)
{
  if (out == nullptr) {
    return setError(EBG_ERR_INVALID, "out handle pointer is null");
  }
  *out          = nullptr;
  ebg_soup*  sp = nullptr;
  ebg_status rc = ebg_soup_read(path, &sp);
  if (rc != EBG_OK) {
    return rc;
  }
  int64_t nv = 0, nf = 0, nc = 0;
  ebg_soup_sizes(sp, &nv, &nf);
  ebg_soup_num_corners(sp, &nc);
  std::vector<double>  V(3 * size_t(nv));
  std::vector<int64_t> off(size_t(nf) + 1);
  std::vector<int32_t> idx(static_cast<size_t>(nc));
  rc = ebg_soup_copy_polygons(sp, V.data(), off.data(), idx.data());
  ebg_soup_destroy(sp);
  if (rc != EBG_OK) {
    return rc;
  }
  return buildPoly(V.data(), nv, off.data(), idx.data(), nf, opts, out);
}

ebg_status ebg_compute_polygon_normals(const double* vertices, int64_t num_vertices, const int64_t* face_offsets,
                                       const int32_t* face_vertices, int64_t num_faces, double* face_normals,
                                       double* centroids, double* corner_vertex_normals, double* edge_normals)
{
  if (vertices == nullptr || face_offsets == nullptr || face_vertices == nullptr || num_vertices <= 0 ||
      num_faces <= 0 || face_offsets[0] != 0) {
    return setError(EBG_ERR_INVALID, "bad polygon soup");
  }
  for (int64_t f = 0; f < num_faces; f++) {
    if (face_offsets[f + 1] - face_offsets[f] < 3) {
      return setError(EBG_ERR_INVALID, "face " + std::to_string(f) + " has fewer than three vertices");
    }
    for (int64_t k = face_offsets[f]; k < face_offsets[f + 1]; k++) {
      if (face_vertices[k] < 0 || face_vertices[k] >= num_vertices) {
        return setError(EBG_ERR_INVALID, "face " + std::to_string(f) + " references a vertex out of range");
      }
    }
  }
  std::vector<double> fn, c, vn, en;
  std::string         msg;
  if (!computePolygonNormals(vertices, num_vertices, face_offsets, face_vertices, num_faces, fn, c, vn, en, msg)) {
    return setError(EBG_ERR_INVALID, msg);
  }
  for (auto [dst, src] : {std::pair<double*, const std::vector<double>*>{face_normals, &fn}, {centroids, &c},
                          {corner_vertex_normals, &vn}, {edge_normals, &en}}) {
    if (dst) {
      std::memcpy(dst, src->data(), src->size() * sizeof(double));
    }
  }
  return EBG_OK;
}

ebg_status ebg_polymesh_destroy(ebg_polymesh* m)
{
  if (m == nullptr) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  cudaFree(m->dNodes);
  cudaFree(m->dFace);
  cudaFree(m->dFaceRec);
  cudaFree(m->dCorner);
  cudaFree(m->dFaceId);
  cudaFree(m->dStatus);
  delete m;
  return EBG_OK;
}

ebg_status ebg_polymesh_get_info(const ebg_polymesh* m, ebg_mesh_info* info, int64_t* num_corners)
{
  if (m == nullptr || info == nullptr) {
    return setError(EBG_ERR_INVALID, "null argument");
  }
  *info = m->info;
  if (num_corners) {
    *num_corners = m->numCorners;
  }
  return EBG_OK;
}

ebg_status ebg_polymesh_get_normals(const ebg_polymesh* m, double* face_normals, double* centroids,
                                    double* corner_vertex_normals, double* edge_normals)
{
  if (m == nullptr) {
    return setError(EBG_ERR_INVALID, "null mesh");
  }
  const int64_t nf = m->info.num_triangles, nc = m->numCorners;
  DeviceGuard   guard;
  cudaSetDevice(m->device);
  std::vector<uint2>   face(nf);
  std::vector<double>  rec(6 * size_t(nf)), corner(9 * size_t(nc));
  std::vector<int32_t> id(nf);
  if (cudaMemcpy(face.data(), m->dFace, 8 * size_t(nf), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(rec.data(), m->dFaceRec, 48 * size_t(nf), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(corner.data(), m->dCorner, 72 * size_t(nc), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(id.data(), m->dFaceId, 4 * size_t(nf), cudaMemcpyDeviceToHost) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  // soup order: face f's corners follow the faces before it
  std::vector<int64_t> first(size_t(nf) + 1, 0);
  for (int64_t p = 0; p < nf; p++) {
    first[size_t(id[p]) + 1] = face[p].y;
  }
  for (int64_t f = 0; f < nf; f++) {
    first[f + 1] += first[f];
  }
  for (int64_t p = 0; p < nf; p++) {
    const int64_t f = id[p];
    for (int a = 0; a < 3; a++) {
      if (face_normals) {
        face_normals[3 * f + a] = rec[6 * p + a];
      }
      if (centroids) {
        centroids[3 * f + a] = rec[6 * p + 3 + a];
      }
    }
    for (uint32_t k = 0; k < face[p].y; k++) {
      const double* c = &corner[9 * size_t(face[p].x + k)];
      for (int a = 0; a < 3; a++) {
        if (corner_vertex_normals) {
          corner_vertex_normals[3 * (first[f] + k) + a] = c[3 + a];
        }
        if (edge_normals) {
          edge_normals[3 * (first[f] + k) + a] = c[6 + a];
        }
      }
    }
  }
  return EBG_OK;
}

ebg_status ebg_polymesh_signed_distance(const ebg_polymesh* m, const double* points_dev, int64_t n, double* out_dev,
                                        int32_t* closest_face_dev, void* stream)
{
  return polyDevice(m, points_dev, n, out_dev, closest_face_dev, stream, false);
}

ebg_status ebg_polymesh_signed_distance_host(const ebg_polymesh* m, const double* points_host, int64_t n,
                                             double* out_host, int32_t* closest_face_host, void* stream)
{
  return polyHost(m, points_host, n, out_host, closest_face_host, stream, false);
}

ebg_status ebg_polymesh_signed_distance_flat(const ebg_polymesh* m, const double* points_dev, int64_t n,
                                             double* out_dev, int32_t* closest_face_dev, void* stream)
{
  return polyDevice(m, points_dev, n, out_dev, closest_face_dev, stream, true);
}

ebg_status ebg_polymesh_signed_distance_flat_host(const ebg_polymesh* m, const double* points_host, int64_t n,
                                                  double* out_host, int32_t* closest_face_host, void* stream)
{
  return polyHost(m, points_host, n, out_host, closest_face_host, stream, true);
}

ebg_status ebg_polymesh_check_status(const ebg_polymesh* m, void* stream)
{
  if (m == nullptr) {
    return setError(EBG_ERR_INVALID, "null mesh");
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  return polyCheck(m, static_cast<cudaStream_t>(stream));
}

} // extern "C"
