// C ABI of the mesh path: handle lifetime, host build + upload, and the query pipeline
//   Morton keys -> radix sort (query coherence) -> FP32 packet traversal -> FP64 band pass.
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cuda_runtime.h>

#include "capi_common.h"
#include "capi_internal.h"
#include "ebg_device.cuh"
#include "ebgeometry_b200.h"
#include "mesh_build_gpu.h"
#include "mesh_host.h"
#include "mesh_kernels.h"
#include "seed_kernels.h"

using namespace ebg;

namespace {

// Oriented box of the triangles at leaf positions [first, end) (see EbgObb): n = area-weighted
// mean face normal (the smallest extent axis of their AABB if the normals nearly cancel), u =
// principal in-plane direction of their vertices, extents from the vertex projections, padded by
// `pad` so FP32 evaluation of the box distance never exceeds the FP64 distance to a triangle
// inside.  Returns the box's volume over the AABB's (how much tighter it is).
double obbOfRange(const double* V, const int32_t* F, const std::vector<uint32_t>& order, uint32_t first, uint32_t end,
                  double pad, EbgObb& o)
{
  auto vert = [&](uint32_t i, int c) { return V + 3 * int64_t(F[3 * int64_t(order[i]) + c]); };
  double n[3] = {0, 0, 0}, area = 0, lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (uint32_t i = first; i < end; i++) {
    const double* p0 = vert(i, 0);
    const double* p1 = vert(i, 1);
    const double* p2 = vert(i, 2);
    const double  e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const double  e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    const double  cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    for (int a = 0; a < 3; a++) {
      n[a] += cr[a];
    }
    area += std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    for (const double* p : {p0, p1, p2}) {
      for (int a = 0; a < 3; a++) {
        lo[a] = std::min(lo[a], p[a]);
        hi[a] = std::max(hi[a], p[a]);
      }
    }
  }
  double ln = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  if (!(ln > 0.5 * area) || !(ln > 0)) {
    int ax = 0;
    for (int a = 1; a < 3; a++) {
      if (hi[a] - lo[a] < hi[ax] - lo[ax]) {
        ax = a;
      }
    }
    n[0] = n[1] = n[2] = 0;
    n[ax] = 1;
    ln    = 1;
  }
  for (int a = 0; a < 3; a++) {
    n[a] /= ln;
  }
  // a first in-plane axis t1 (any perpendicular), then the principal direction in that plane
  double t1[3];
  if (std::fabs(n[0]) < 0.9) {
    t1[0] = 0;
    t1[1] = n[2];
    t1[2] = -n[1];
  }
  else {
    t1[0] = -n[2];
    t1[1] = 0;
    t1[2] = n[0];
  }
  const double l1 = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
  for (int a = 0; a < 3; a++) {
    t1[a] /= l1;
  }
  const double t2[3] = {n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0]};
  const double cnt   = 3.0 * double(end - first);
  double       mx = 0, my = 0;
  for (uint32_t i = first; i < end; i++) {
    for (int c = 0; c < 3; c++) {
      const double* p = vert(i, c);
      mx += p[0] * t1[0] + p[1] * t1[1] + p[2] * t1[2];
      my += p[0] * t2[0] + p[1] * t2[1] + p[2] * t2[2];
    }
  }
  mx /= cnt;
  my /= cnt;
  double sxx = 0, syy = 0, sxy = 0;
  for (uint32_t i = first; i < end; i++) {
    for (int c = 0; c < 3; c++) {
      const double* p = vert(i, c);
      const double  x = p[0] * t1[0] + p[1] * t1[1] + p[2] * t1[2] - mx;
      const double  y = p[0] * t2[0] + p[1] * t2[1] + p[2] * t2[2] - my;
      sxx += x * x;
      syy += y * y;
      sxy += x * y;
    }
  }
  const double th   = 0.5 * std::atan2(2 * sxy, sxx - syy);
  const double u[3] = {std::cos(th) * t1[0] + std::sin(th) * t2[0], std::cos(th) * t1[1] + std::sin(th) * t2[1],
                       std::cos(th) * t1[2] + std::sin(th) * t2[2]};
  const double w[3] = {n[1] * u[2] - n[2] * u[1], n[2] * u[0] - n[0] * u[2], n[0] * u[1] - n[1] * u[0]};
  double       mn[3] = {1e300, 1e300, 1e300}, mxx[3] = {-1e300, -1e300, -1e300};
  for (uint32_t i = first; i < end; i++) {
    for (int c = 0; c < 3; c++) {
      const double* p     = vert(i, c);
      const double  pr[3] = {p[0] * n[0] + p[1] * n[1] + p[2] * n[2], p[0] * u[0] + p[1] * u[1] + p[2] * u[2],
                             p[0] * w[0] + p[1] * w[1] + p[2] * w[2]};
      for (int a = 0; a < 3; a++) {
        mn[a]  = std::min(mn[a], pr[a]);
        mxx[a] = std::max(mxx[a], pr[a]);
      }
    }
  }
  // the box centre's offset along each axis, and the half-extents
  o.nx  = float(n[0]);
  o.ny  = float(n[1]);
  o.nz  = float(n[2]);
  o.dn  = float(0.5 * (mn[0] + mxx[0]));
  o.ux  = float(u[0]);
  o.uy  = float(u[1]);
  o.uz  = float(u[2]);
  o.du  = float(0.5 * (mn[1] + mxx[1]));
  o.vx  = float(w[0]);
  o.vy  = float(w[1]);
  o.vz  = float(w[2]);
  o.dv  = float(0.5 * (mn[2] + mxx[2]));
  o.hn  = roundUp(0.5 * (mxx[0] - mn[0]) + pad);
  o.hu  = roundUp(0.5 * (mxx[1] - mn[1]) + pad);
  o.hv  = roundUp(0.5 * (mxx[2] - mn[2]) + pad);
  o.pad = 0.f;
  const double obbVol  = 8.0 * double(o.hn) * double(o.hu) * double(o.hv);
  const double aabbVol = (hi[0] - lo[0] + 2 * pad) * (hi[1] - lo[1] + 2 * pad) * (hi[2] - lo[2] + 2 * pad);
  return aabbVol > 0 ? obbVol / aabbVol : 1.0;
}

// Oriented boxes of every leaf and every interior node.  An interior node's box is flagged in its
// parent's slot (EBG_NODE_HAS_OBB) only when its volume is at most half the axis-aligned box's, so
// the traversal spends the extra test where it can prune.
void computeObbs(const double* V, const int32_t* F, Bvh4& bvh, std::vector<EbgObb>& leafObb, std::vector<EbgObb>& nodeObb)
{
  double scale = 0;
  for (int a = 0; a < 3; a++) {
    scale = std::max(scale, std::max(std::fabs(bvh.lo[a]), std::fabs(bvh.hi[a])));
  }
  const double pad = 2e-6 * std::max(scale, 1e-30);
  const size_t nl  = bvh.leafFirst.size();
  leafObb.resize(nl);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t l = 0; l < int64_t(nl); l++) {
    obbOfRange(V, F, bvh.order, bvh.leafFirst[l], bvh.leafFirst[l] + bvh.leafCount[l], pad, leafObb[l]);
  }
  const size_t       nn = bvh.nodes.size();
  std::vector<char>  useful(nn, 0);
  nodeObb.resize(std::max<size_t>(nn, 1));
  std::memset(nodeObb.data(), 0, nodeObb.size() * sizeof(EbgObb));
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t j = 0; j < int64_t(nn); j++) {
    useful[j] = obbOfRange(V, F, bvh.order, bvh.nodeFirst[j], bvh.nodeEnd[j], pad, nodeObb[j]) <= 0.5;
  }
  for (size_t j = 0; j < nn; j++) {
    EbgNode4& nd = bvh.nodes[j];
    for (int k = 0; k < 4; k++) {
      const uint32_t c = nd.child[k];
      if (!(c & EBG_LEAF_BIT) && c != 0 && useful[c]) {
        nd.count[k] = EBG_NODE_HAS_OBB;
      }
    }
  }
}

// The mesh's bounding box in its view (FP32 root box, query-ordering domain) and summary.
void setMeshBounds(ebg_mesh* m, const double* lo, const double* hi)
{
  EbgMeshView& v = m->view;
  for (int a = 0; a < 3; a++) {
    v.root_lo[a] = roundDown(lo[a]);
    v.root_hi[a] = roundUp(hi[a]);
    // Morton domain for query ordering: the mesh box grown to twice its extent about its centre
    const double c    = 0.5 * (lo[a] + hi[a]);
    const double ext  = std::max(hi[a] - lo[a], 1e-30);
    v.morton_lo[a]    = float(c - ext);
    v.morton_scale[a] = float(1024.0 / (2.0 * ext));
  }
  double d2 = 0;
  for (int a = 0; a < 3; a++) {
    m->info.lo[a] = lo[a];
    m->info.hi[a] = hi[a];
    d2 += (hi[a] - lo[a]) * (hi[a] - lo[a]);
  }
  m->info.diagonal = std::sqrt(d2);
}

// The device view and the summary of a mesh whose device arrays are in place (either build).
ebg_status finishMesh(ebg_mesh* m, int64_t nv, int64_t nt, int leafSize, const double* lo, const double* hi,
                      ebg_mesh** out)
{
  if (cudaMalloc(reinterpret_cast<void**>(&m->dStatus), sizeof(int)) != cudaSuccess ||
      cudaMemset(m->dStatus, 0, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    ebg_mesh_destroy(m);
    return setError(EBG_ERR_NO_MEMORY, "device allocation for the mesh status");
  }
  EbgMeshView& v = m->view;
  v.nodes        = static_cast<const EbgNode4*>(m->dNodes);
  v.hot          = static_cast<const EbgTriHot*>(m->dHot);
  v.sign         = static_cast<const EbgTriSign*>(m->dSign);
  v.tri64        = static_cast<const double*>(m->dTri64);
  v.tri_id       = static_cast<const int32_t*>(m->dTriId);
  v.obb          = static_cast<const EbgObb*>(m->dObb);
  v.node_obb     = static_cast<const EbgObb*>(m->dNodeObb);
  v.dcel_n       = static_cast<const double*>(m->dDcelN);
  setMeshBounds(m, lo, hi);
  ebg_mesh_info& inf = m->info;
  inf.num_triangles  = nt;
  inf.num_vertices   = nv;
  inf.leaf_size      = leafSize;
  const size_t N     = size_t(nt);
  inf.device_bytes = int64_t(size_t(std::max<int64_t>(inf.num_nodes, 1)) * (sizeof(EbgNode4) + sizeof(EbgObb) + 8) +
                             size_t(inf.num_leaves) * (sizeof(EbgObb) + 8) +
                             N * (sizeof(EbgTriHot) + sizeof(EbgTriSign) + 33 * sizeof(double) + 4 + 12));
  *out             = m;
  return EBG_OK;
}

ebg_status buildMesh(const double*         V,
                     int64_t               nv,
                     const int32_t*        F,
                     int64_t               nt,
                     const double*         givenVN,
                     const double*         givenEN,
                     const ebg_build_opts* opts,
                     ebg_mesh**            out)
{
  if (out == nullptr) {
    return setError(EBG_ERR_INVALID, "out handle pointer is null");
  }
  *out = nullptr;
  if (V == nullptr || F == nullptr || nv <= 0 || nt <= 0) {
    return setError(EBG_ERR_INVALID, "mesh needs at least one vertex and one triangle");
  }
  if (nt >= int64_t(EBG_LEAF_BIT) || nv > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "mesh too large (triangles < 2^31, vertices < 2^31)");
  }
  for (int64_t i = 0; i < 3 * nt; i++) {
    if (F[i] < 0 || F[i] >= nv) {
      return setError(EBG_ERR_INVALID, "triangle corner index out of range");
    }
  }
  for (int64_t i = 0; i < 3 * nv; i++) {
    if (!std::isfinite(V[i])) {
      return setError(EBG_ERR_INVALID, "non-finite vertex coordinate");
    }
  }
  const int build    = opts ? opts->build : EBG_BUILD_SAH;
  const int leafSize = (opts && opts->leaf_size > 0) ? opts->leaf_size : 8;
  int       device   = (opts && opts->device >= 0) ? opts->device : -1;
  if (build != EBG_BUILD_SAH && build != EBG_BUILD_MORTON) {
    return setError(EBG_ERR_INVALID, "unknown build method");
  }
  if (leafSize > int(EBG_MAX_LEAF)) {
    return setError(EBG_ERR_INVALID, "leaf_size must be at most " + std::to_string(EBG_MAX_LEAF));
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
  auto* m   = new ebg_mesh;
  m->device = device;
  cudaDeviceGetAttribute(&m->numSms, cudaDevAttrMultiProcessorCount, device);

  std::string msg;
  if (givenVN != nullptr && givenEN != nullptr) {
    m->cornerVN.assign(givenVN, givenVN + 9 * nt);
    m->edgeN.assign(givenEN, givenEN + 9 * nt);
    m->triN.resize(3 * nt);
    for (int64_t f = 0; f < nt; f++) {
      const double* a = V + 3 * int64_t(F[3 * f]);
      const double* b = V + 3 * int64_t(F[3 * f + 1]);
      const double* c = V + 3 * int64_t(F[3 * f + 2]);
      const double  u[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
      const double  w[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
      const double  x[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
      const double  l    = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
      if (!(l > 0.0)) {
        delete m;
        return setError(EBG_ERR_INVALID, "degenerate (zero-area) triangle in the soup");
      }
      const double is = 1.0 / l;
      for (int k = 0; k < 3; k++) {
        m->triN[3 * f + k] = is * x[k];
      }
    }
  }
  const bool onDevice    = opts && (opts->flags & EBG_BUILD_ON_DEVICE);
  const bool givenNormal = givenVN != nullptr && givenEN != nullptr;
  if (!givenNormal && !onDevice && !computePseudonormals(V, nv, F, nt, m->triN, m->cornerVN, m->edgeN, msg)) {
    delete m;
    return setError(EBG_ERR_INVALID, msg);
  }

  if (onDevice) {
    cudaStream_t bs = nullptr;
    if (cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking) != cudaSuccess) {
      delete m;
      return setError(EBG_ERR_CUDA, "stream for the device build");
    }
    double           lo[3], hi[3];
    const ebg_status rc = buildMeshOnDevice(m, V, nv, F, nt, build, leafSize, lo, hi, bs, !givenNormal);
    cudaStreamDestroy(bs);
    std::vector<double>().swap(m->triN);
    std::vector<double>().swap(m->cornerVN);
    std::vector<double>().swap(m->edgeN);
    if (rc != EBG_OK) {
      const std::string keep = ebg_last_error();
      ebg_mesh_destroy(m);
      return setError(rc, keep);
    }
    return finishMesh(m, nv, nt, leafSize, lo, hi, out);
  }

  // primitive boxes / centroids
  std::vector<double> lo(3 * nt), hi(3 * nt), cen(3 * nt);
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < nt; f++) {
    for (int a = 0; a < 3; a++) {
      const double x0 = V[3 * int64_t(F[3 * f]) + a], x1 = V[3 * int64_t(F[3 * f + 1]) + a],
                   x2 = V[3 * int64_t(F[3 * f + 2]) + a];
      lo[3 * f + a]  = std::min(x0, std::min(x1, x2));
      hi[3 * f + a]  = std::max(x0, std::max(x1, x2));
      cen[3 * f + a] = (x0 + x1 + x2) / 3.0;
    }
  }
  Bvh4 bvh;
  if (!buildBvh4(lo, hi, cen, build, leafSize, bvh, msg)) {
    delete m;
    return setError(EBG_ERR_INVALID, msg);
  }

  // leaf-ordered triangle records
  const size_t            N = size_t(nt);
  std::vector<EbgTriHot>  hot(N);
  std::vector<EbgTriSign> sign(N);
  std::vector<double>     tri64(30 * N);
  std::vector<double>     dcelN(3 * N);
  std::vector<int32_t>    triId(N);
  m->areaCdf.resize(N);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(N); i++) {
    const int64_t f = bvh.order[i];
    triId[i]        = int32_t(f);
    const double* a = V + 3 * int64_t(F[3 * f]);
    const double* b = V + 3 * int64_t(F[3 * f + 1]);
    const double* c = V + 3 * int64_t(F[3 * f + 2]);
    const double  ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double  ac[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    EbgTriHot&    h     = hot[i];
    h.v0x = float(a[0]);
    h.v0y = float(a[1]);
    h.v0z = float(a[2]);
    h.abx = float(ab[0]);
    h.aby = float(ab[1]);
    h.abz = float(ab[2]);
    h.acx = float(ac[0]);
    h.acy = float(ac[1]);
    h.acz = float(ac[2]);
    {
      const double cx = ab[1] * ac[2] - ab[2] * ac[1], cy = ab[2] * ac[0] - ab[0] * ac[2],
                   cz = ab[0] * ac[1] - ab[1] * ac[0];
      m->areaCdf[i] = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
    }
    h.ab2  = float(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2]);
    h.abac = float(ab[0] * ac[0] + ab[1] * ac[1] + ab[2] * ac[2]);
    h.ac2  = float(ac[0] * ac[0] + ac[1] * ac[1] + ac[2] * ac[2]);
    EbgTriSign& s = sign[i];
    s.nx          = float(m->triN[3 * f]);
    s.ny          = float(m->triN[3 * f + 1]);
    s.nz          = float(m->triN[3 * f + 2]);
    s.pad0 = s.pad1 = s.pad2 = 0.f;
    for (int k = 0; k < 9; k++) {
      s.vn[k] = float(m->cornerVN[9 * f + k]);
      s.en[k] = float(m->edgeN[9 * f + k]);
    }
    double* t = &tri64[30 * size_t(i)];
    for (int k = 0; k < 3; k++) {
      t[k]     = a[k];
      t[3 + k] = b[k];
      t[6 + k] = c[k];
      t[9 + k] = m->triN[3 * f + k];
    }
    for (int k = 0; k < 9; k++) {
      t[12 + k] = m->cornerVN[9 * f + k];
      t[21 + k] = m->edgeN[9 * f + k];
    }
    {
      // the DCEL face normal: the Triangle normal normalised again (a multiply by the reciprocal)
      const double* tn = &m->triN[3 * f];
      const double  is = 1.0 / std::sqrt(tn[0] * tn[0] + tn[1] * tn[1] + tn[2] * tn[2]);
      for (int k = 0; k < 3; k++) {
        dcelN[3 * size_t(i) + k] = is * tn[k];
      }
    }
  }

  for (size_t i = 1; i < N; i++) {
    m->areaCdf[i] += m->areaCdf[i - 1];
  }
  std::vector<EbgObb> obb, nodeObb;
  computeObbs(V, F, bvh, obb, nodeObb);
  // upload
  auto up = [&](void** dst, const void* src, size_t bytes) -> bool {
    if (cudaMalloc(dst, std::max<size_t>(bytes, 16)) != cudaSuccess) {
      return false;
    }
    return bytes == 0 || cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  const size_t nodeBytes = bvh.nodes.size() * sizeof(EbgNode4);
  if (!up(&m->dNodes, bvh.nodes.data(), nodeBytes) || !up(&m->dHot, hot.data(), N * sizeof(EbgTriHot)) ||
      !up(&m->dSign, sign.data(), N * sizeof(EbgTriSign)) || !up(&m->dTri64, tri64.data(), 30 * N * sizeof(double)) ||
      !up(&m->dTriId, triId.data(), N * sizeof(int32_t)) ||
      !up(&m->dObb, obb.data(), obb.size() * sizeof(EbgObb)) ||
      !up(&m->dNodeObb, nodeObb.data(), nodeObb.size() * sizeof(EbgObb)) ||
      !up(&m->dDcelN, dcelN.data(), dcelN.size() * sizeof(double)) ||
      !up((void**)&m->dF, F, 3 * N * sizeof(int32_t)) ||
      !up((void**)&m->dLeafFirst, bvh.leafFirst.data(), bvh.leafFirst.size() * sizeof(uint32_t)) ||
      !up((void**)&m->dLeafCount, bvh.leafCount.data(), bvh.leafCount.size() * sizeof(uint32_t)) ||
      !up((void**)&m->dNodeFirst, bvh.nodeFirst.data(), bvh.nodeFirst.size() * sizeof(uint32_t)) ||
      !up((void**)&m->dNodeEnd, bvh.nodeEnd.data(), bvh.nodeEnd.size() * sizeof(uint32_t))) {
    cudaGetLastError();
    ebg_mesh_destroy(m);
    return setError(EBG_ERR_NO_MEMORY, "device allocation or upload failed for the mesh");
  }

  // every normal now lives in the FP64 records on the device (ebg_mesh_get_normals reads them there)
  std::vector<double>().swap(m->triN);
  std::vector<double>().swap(m->cornerVN);
  std::vector<double>().swap(m->edgeN);
  m->info.num_nodes  = int64_t(bvh.nodes.size());
  m->info.num_leaves = bvh.numLeaves;
  m->info.depth      = bvh.depth;
  m->view.root_ref   = bvh.rootRef;
  m->view.root_count = bvh.rootCount;
  return finishMesh(m, nv, nt, leafSize, bvh.lo, bvh.hi, out);
}

struct Workspace
{
  cudaStream_t      s;
  std::vector<void*> ptrs;
  bool              ok = true;
  explicit Workspace(cudaStream_t st) : s(st) {}
  template <class T>
  T* get(size_t count)
  {
    void* p = nullptr;
    if (ok && cudaMallocAsync(&p, std::max<size_t>(count * sizeof(T), 16), s) == cudaSuccess) {
      ptrs.push_back(p);
      return static_cast<T*>(p);
    }
    ok = false;
    return nullptr;
  }
  ~Workspace()
  {
    for (void* p : ptrs) {
      cudaFreeAsync(p, s);
    }
  }
};

} // namespace

ebg_status ebg::meshQuery(const ebg_mesh*       m,
                          const float*          pts,
                          int64_t               n,
                          float*                outD,
                          int32_t*              outTri,
                          const ebg_query_opts* opts,
                          unsigned long long*   statsDev,
                          cudaStream_t          s,
                          const double*         pts64,
                          double*               out64,
                          int                   evalKind,
                          bool                  triLeafOrder)
{
  if (n > int64_t(INT32_MAX)) {
    return setError(EBG_ERR_TOO_LARGE, "at most 2^31-1 points per call");
  }
  const bool sort   = !(opts && opts->no_sort);
  // an FP64 result re-evaluates every query in FP64 (the band covers all distances)
  const bool fp64all = out64 != nullptr;
  const bool band64  = fp64all || !(opts && opts->no_fp64_band);
  const int  wpb    = (opts && opts->warps_per_block > 0) ? opts->warps_per_block
                                                          : (m->tunedWpb > 0 ? m->tunedWpb : 4);
  const int  occ    = (opts && opts->occupancy > 0) ? opts->occupancy : m->tunedOccupancy;
  double     band   = fp64all ? double(INFINITY) : ((opts && opts->band > 0) ? opts->band : 1e-4 * fp32ErrorScale(m));
  const ebg_seed* seed = opts ? opts->seed : nullptr;
  if (seed && seed->device != m->device) {
    return setError(EBG_ERR_INVALID, "seed model lives on another device than the mesh");
  }
  // a model seeds the traversal through the entry cuts it was attached with (ebg_seed_attach)
  if (seed && !(m->cellsSeed == seed && m->dCellCount != nullptr)) {
    return setError(EBG_ERR_INVALID, "the seed model is not attached to this mesh (ebg_seed_attach)");
  }
  // node width of the FP32 traversal: the cuts index the 4-wide tree, so seeded queries keep it
  const int askedWidth = (opts && opts->node_width > 0) ? opts->node_width : 0;
  if (askedWidth != 0 && askedWidth != 4 && askedWidth != 8) {
    return setError(EBG_ERR_INVALID, "node_width must be 0, 4 or 8");
  }
  if (askedWidth == 8 && !m->hasWide) {
    return setError(EBG_ERR_INVALID, "node_width 8 needs the mesh's 8-wide copy (ebg_mesh_widen)");
  }
  const int width = seed ? 4 : (askedWidth ? askedWidth : (m->tunedWidth == 8 && m->hasWide ? 8 : 4));

  // optional per-phase events (ev[0] start, [1] after ordering, [2] after traversal, [3] end)
  ebg_phase_timings* tm = opts ? opts->timings : nullptr;
  cudaEvent_t        ev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (tm) {
    for (auto& e : ev) {
      cudaEventCreate(&e);
    }
    cudaEventRecord(ev[0], s);
  }
  struct EventGuard
  {
    cudaEvent_t* ev;
    ~EventGuard()
    {
      for (int i = 0; i < 4; i++) {
        if (ev[i]) {
          cudaEventDestroy(ev[i]);
        }
      }
    }
  } evGuard{ev};

  Workspace ws(s);
  uint32_t* order = nullptr;
  if (sort) {
    uint32_t* keysIn  = ws.get<uint32_t>(n);
    uint32_t* keysOut = ws.get<uint32_t>(n);
    uint32_t* idsIn   = ws.get<uint32_t>(n);
    order             = ws.get<uint32_t>(n);
    if (!ws.ok) {
      return setError(EBG_ERR_NO_MEMORY, "query workspace allocation failed");
    }
    launchQueryKeys(pts, n, m->view.morton_lo, m->view.morton_scale, keysIn, idsIn, s);
    size_t tempBytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, keysIn, keysOut, idsIn, order, int(n), 0, 30, s);
    void* temp = ws.get<char>(tempBytes);
    if (!ws.ok) {
      return setError(EBG_ERR_NO_MEMORY, "sort workspace allocation failed");
    }
    if (cub::DeviceRadixSort::SortPairs(temp, tempBytes, keysIn, keysOut, idsIn, order, int(n), 0, 30, s) !=
        cudaSuccess) {
      return setError(EBG_ERR_CUDA, "query sort failed");
    }
  }
  // The band list: the traversal flags each sorted position, and a compaction of the flags gives
  // the list in position (Morton) order, so that each FP64 packet holds 32 neighbouring queries.
  // (Appending from the traversal lists them in completion order, which interleaves thousands of
  // packets in flight.)
  unsigned long long* counters = ws.get<unsigned long long>(2); // [0] packets, [1] band count (u32)
  uint32_t*           bandList = band64 ? ws.get<uint32_t>(n) : nullptr;
  uint8_t*            bandFlag = band64 ? ws.get<uint8_t>(n) : nullptr;
  size_t              selBytes = 0;
  void*               selTemp  = nullptr;
  if (band64) {
    cub::DeviceSelect::Flagged(nullptr, selBytes, thrust::counting_iterator<uint32_t>(0u), bandFlag, bandList,
                               reinterpret_cast<uint32_t*>(counters + 1), int(n), s);
    selTemp = ws.get<char>(selBytes);
  }
  if (!ws.ok) {
    return setError(EBG_ERR_NO_MEMORY, "query workspace allocation failed");
  }
  cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), s);
  if (tm) {
    cudaEventRecord(ev[1], s);
  }

  MeshQueryArgs a{};
  a.mesh       = m->view;
  a.points     = pts;
  a.points64   = pts64;
  a.out_d64    = out64;
  a.eval       = evalKind;
  a.order      = order;
  a.hint       = (seed == nullptr && opts) ? opts->radius_hint : nullptr;
  a.n          = n;
  a.out_d      = outD;
  a.out_tri    = outTri;
  a.tri_leaf   = triLeafOrder ? 1 : 0;
  a.band       = float(band);
  a.band_list  = bandList;
  a.band_count = reinterpret_cast<uint32_t*>(counters + 1);
  a.band_d32   = nullptr;
  a.band_flag  = bandFlag;
  a.work       = counters;
  a.status     = m->dStatus;
  a.stats      = statsDev;
  a.chunk      = (opts && opts->queue_chunk > 0) ? opts->queue_chunk : (m->tunedChunk > 0 ? m->tunedChunk : 1);
  if (seed) {
    a.cells = m->cellsView;
  }
  a.top_nodes = topNodesFor(m, opts, seed != nullptr);
  if (width == 8) {
    // the 8-wide copy's nodes (the FP64 pass below reads the 4-wide tree again)
    a.mesh       = m->view8;
    a.node_width = 8;
    a.top_nodes  = 0;
  }
  if (launchMeshSdf32(a, wpb, m->numSms, s, occ) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("traversal launch failed: ") + cudaGetErrorString(cudaGetLastError()));
  }
  a.mesh       = m->view;
  a.node_width = 4;
  if (tm) {
    cudaEventRecord(ev[2], s);
  }
  if (band64) {
    if (cub::DeviceSelect::Flagged(selTemp, selBytes, thrust::counting_iterator<uint32_t>(0u), bandFlag, bandList,
                                   a.band_count, int(n), s) != cudaSuccess) {
      return setError(EBG_ERR_CUDA, "band list compaction failed");
    }
    // delta bounds the FP32 distance error: 2e-6 of the mesh's diagonal, or of its coordinates'
    // magnitude for a mesh far from the origin (about 17 FP32 roundings of either)
    const float delta = float(2e-6 * fp32ErrorScale(m)) + 1e-30f;
    if (launchMeshBand64(a, delta, m->numSms, s) != cudaSuccess) {
      return setError(EBG_ERR_CUDA, "band launch failed");
    }
    if (statsDev) {
      cudaMemcpyAsync(statsDev + 3, counters + 1, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s);
    }
  }
  if (tm) {
    cudaEventRecord(ev[3], s);
    if (cudaEventSynchronize(ev[3]) != cudaSuccess) {
      return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    }
    cudaEventElapsedTime(&tm->order_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&tm->traverse_ms, ev[1], ev[2]);
    cudaEventElapsedTime(&tm->band_ms, ev[2], ev[3]);
    cudaEventElapsedTime(&tm->total_ms, ev[0], ev[3]);
  }
  return EBG_OK;
}


void ebg::dropWide(ebg_mesh* m)
{
  cudaFree(m->dNodes8);
  cudaFree(m->dNodeObb8);
  m->dNodes8    = nullptr;
  m->dNodeObb8  = nullptr;
  m->hasWide    = false;
  m->numNodes8  = 0;
  m->depth8     = 0;
  m->tunedWidth = 0;
  m->view8      = EbgMeshView{};
}

extern "C" {

ebg_status ebg_mesh_create(const double*         vertices,
                           int64_t               num_vertices,
                           const int32_t*        triangles,
                           int64_t               num_triangles,
                           const ebg_build_opts* opts,
                           ebg_mesh**            out)
{
  return buildMesh(vertices, num_vertices, triangles, num_triangles, nullptr, nullptr, opts, out);
}

ebg_status ebg_mesh_create_with_normals(const double*         vertices,
                                        int64_t               num_vertices,
                                        const int32_t*        triangles,
                                        int64_t               num_triangles,
                                        const double*         corner_vertex_normals,
                                        const double*         edge_normals,
                                        const ebg_build_opts* opts,
                                        ebg_mesh**            out)
{
  if (corner_vertex_normals == nullptr || edge_normals == nullptr) {
    return setError(EBG_ERR_INVALID, "normal arrays are null");
  }
  return buildMesh(vertices, num_vertices, triangles, num_triangles, corner_vertex_normals, edge_normals, opts, out);
}

ebg_status ebg_compute_pseudonormals(const double*  vertices,
                                     int64_t        num_vertices,
                                     const int32_t* triangles,
                                     int64_t        num_triangles,
                                     double*        face_normals,
                                     double*        corner_vertex_normals,
                                     double*        edge_normals)
{
  if (vertices == nullptr || triangles == nullptr || num_vertices <= 0 || num_triangles <= 0 ||
      face_normals == nullptr || corner_vertex_normals == nullptr || edge_normals == nullptr) {
    return setError(EBG_ERR_INVALID, "null buffer or empty mesh");
  }
  for (int64_t i = 0; i < 3 * num_triangles; i++) {
    if (triangles[i] < 0 || triangles[i] >= num_vertices) {
      return setError(EBG_ERR_INVALID, "triangle corner index out of range");
    }
  }
  std::vector<double> tn, vn, en;
  std::string         msg;
  if (!computePseudonormals(vertices, num_vertices, triangles, num_triangles, tn, vn, en, msg)) {
    return setError(EBG_ERR_INVALID, msg);
  }
  std::memcpy(face_normals, tn.data(), tn.size() * sizeof(double));
  std::memcpy(corner_vertex_normals, vn.data(), vn.size() * sizeof(double));
  std::memcpy(edge_normals, en.data(), en.size() * sizeof(double));
  return EBG_OK;
}

ebg_status ebg_mesh_destroy(ebg_mesh* m)
{
  if (m == nullptr) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  cudaFree(m->dNodes);
  cudaFree(m->dHot);
  cudaFree(m->dSign);
  cudaFree(m->dTri64);
  cudaFree(m->dTriId);
  cudaFree(m->dObb);
  cudaFree(m->dNodeObb);
  cudaFree(m->dDcelN);
  cudaFree(m->dStatus);
  cudaFree(m->dF);
  cudaFree(m->dLeafFirst);
  cudaFree(m->dLeafCount);
  cudaFree(m->dNodeFirst);
  cudaFree(m->dNodeEnd);
  dropCells(m);
  dropWide(m);
  delete m;
  return EBG_OK;
}

static ebg_status meshRefit(ebg_mesh* m, const double* vertices, bool onDevice, int64_t nv, void* stream)
{
  if (m == nullptr || vertices == nullptr) {
    return setError(EBG_ERR_INVALID, "null mesh or vertex array");
  }
  if (nv != m->info.num_vertices) {
    return setError(EBG_ERR_INVALID, "refit needs the mesh's own vertex count (" + std::to_string(m->info.num_vertices) +
                                         "), got " + std::to_string(nv));
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the entry cuts were cut from the old boxes; they would no longer hold every near triangle
  cudaStreamSynchronize(s);
  dropCells(m);
  dropWide(m); // the copy holds the old boxes
  double       lo[3], hi[3];
  const ebg_status rc = refitMeshOnDevice(m, vertices, onDevice, nv, lo, hi, s);
  if (rc != EBG_OK) {
    return rc;
  }
  setMeshBounds(m, lo, hi);
  return EBG_OK;
}

ebg_status ebg_mesh_refit(ebg_mesh* m, const double* vertices_host, int64_t num_vertices, void* stream)
{
  return meshRefit(m, vertices_host, false, num_vertices, stream);
}

ebg_status ebg_mesh_refit_device(ebg_mesh* m, const double* vertices_dev, int64_t num_vertices, void* stream)
{
  return meshRefit(m, vertices_dev, true, num_vertices, stream);
}

ebg_status ebg_mesh_get_info(const ebg_mesh* m, ebg_mesh_info* info)
{
  if (m == nullptr || info == nullptr) {
    return setError(EBG_ERR_INVALID, "null argument");
  }
  *info = m->info;
  return EBG_OK;
}

ebg_status ebg_mesh_get_normals(const ebg_mesh* m, double* fn, double* vn, double* en)
{
  if (m == nullptr) {
    return setError(EBG_ERR_INVALID, "null mesh");
  }
  if (!fn && !vn && !en) {
    return EBG_OK;
  }
  // the FP64 records hold every normal (leaf order); gather them into soup order on the device
  DeviceGuard  guard;
  cudaSetDevice(m->device);
  const size_t N  = size_t(m->info.num_triangles);
  double*      dN = nullptr;
  if (cudaMalloc(&dN, 21 * 8 * N) != cudaSuccess) {
    cudaGetLastError();
    return setError(EBG_ERR_NO_MEMORY, "device buffer for the normals");
  }
  launchGatherNormals(static_cast<const double*>(m->dTri64), static_cast<const int32_t*>(m->dTriId), int64_t(N), dN,
                      nullptr);
  bool ok = cudaGetLastError() == cudaSuccess;
  ok      = ok && (!fn || cudaMemcpy(fn, dN, 24 * N, cudaMemcpyDeviceToHost) == cudaSuccess);
  ok      = ok && (!vn || cudaMemcpy(vn, dN + 3 * N, 72 * N, cudaMemcpyDeviceToHost) == cudaSuccess);
  ok      = ok && (!en || cudaMemcpy(en, dN + 12 * N, 72 * N, cudaMemcpyDeviceToHost) == cudaSuccess);
  cudaFree(dN);
  if (!ok) {
    return setError(EBG_ERR_CUDA, std::string("reading the normals: ") + cudaGetErrorString(cudaGetLastError()));
  }
  return EBG_OK;
}

ebg_status ebg_mesh_signed_distance(const ebg_mesh*       m,
                                    const float*          points_dev,
                                    int64_t               n,
                                    float*                dist_dev,
                                    int32_t*              closest_tri_dev,
                                    const ebg_query_opts* opts,
                                    void*                 stream)
{
  if (m == nullptr || n < 0 || (n > 0 && (points_dev == nullptr || dist_dev == nullptr))) {
    return setError(EBG_ERR_INVALID, "null mesh/buffer or negative count");
  }
  if (n == 0) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  return meshQuery(m, points_dev, n, dist_dev, closest_tri_dev, opts, nullptr, static_cast<cudaStream_t>(stream));
}

ebg_status ebg_mesh_signed_distance_host(const ebg_mesh*       m,
                                         const float*          points_host,
                                         int64_t               n,
                                         float*                dist_host,
                                         int32_t*              closest_tri_host,
                                         const ebg_query_opts* opts,
                                         void*                 stream)
{
  if (m == nullptr || n < 0 || (n > 0 && (points_host == nullptr || dist_host == nullptr))) {
    return setError(EBG_ERR_INVALID, "null mesh/buffer or negative count");
  }
  if (n == 0) {
    return EBG_OK;
  }
  DeviceGuard  guard;
  cudaSetDevice(m->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaMemsetAsync(m->dStatus, 0, sizeof(int), s);
  // Large calls go in chunks on several streams, so that a chunk's copies in and out overlap its
  // neighbours' traversals (results are per point, so chunking changes none of them).  Calls that
  // ask for phase timings run as one piece.
  const int64_t pieces = (opts && opts->timings) ? 1 : std::min<int64_t>(8, n / (int64_t(1) << 21));
  ebg_status    rc     = EBG_OK;
  {
    Workspace ws(s);
    float*    dp = ws.get<float>(3 * n);
    float*    dd = ws.get<float>(n);
    int32_t*  dt = closest_tri_host ? ws.get<int32_t>(n) : nullptr;
    if (!ws.ok) {
      return setError(EBG_ERR_NO_MEMORY, "device buffers for the host call");
    }
    if (pieces <= 1) {
      cudaMemcpyAsync(dp, points_host, 3 * n * sizeof(float), cudaMemcpyHostToDevice, s);
      rc = meshQuery(m, dp, n, dd, dt, opts, nullptr, s);
      if (rc == EBG_OK) {
        cudaMemcpyAsync(dist_host, dd, n * sizeof(float), cudaMemcpyDeviceToHost, s);
        if (dt) {
          cudaMemcpyAsync(closest_tri_host, dt, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        }
      }
    }
    else {
      // streams the chunks take turns on: with more of them, one chunk's traversal tail and
      // per-chunk passes overlap its neighbours' work (level-8 host call: 121.9 ms with 2 streams,
      // 116.5 with 3, 114.2 with 4)
      constexpr int NS = 4;
      cudaStream_t  aux[NS] = {};
      cudaEvent_t   ev[NS + 1] = {};
      bool          ok = true;
      for (int i = 0; i < NS; i++) {
        ok = ok && cudaStreamCreateWithFlags(&aux[i], cudaStreamNonBlocking) == cudaSuccess;
      }
      for (int i = 0; i < NS + 1; i++) {
        ok = ok && cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) == cudaSuccess;
      }
      if (ok) {
        // the chunks start after what the caller queued on s (including the buffers' allocation)
        cudaEventRecord(ev[0], s);
        for (int i = 0; i < NS; i++) {
          cudaStreamWaitEvent(aux[i], ev[0], 0);
        }
        // Chunk sizes: equal pieces, or for calls of at least 64 M points a ramp -- 1, 2 and 4 units,
        // pieces of about 8 units, then 4, 2 and 1 units (a unit is 1/64 of the call) -- so that the
        // first chunk's copy in and the last chunk's copy out, which nothing overlaps, are short.
        // Every chunk but the last is a multiple of 32 points.
        std::vector<int64_t> sizes;
        auto round32 = [](int64_t x) { return (x + 31) / 32 * 32; };
        if (n >= (int64_t(1) << 26)) {
          const int64_t u = round32((n + 63) / 64);
          for (int64_t f : {1, 2, 4}) {
            sizes.push_back(f * u);
          }
          const int64_t mid   = (n - 14 * u) / 32 * 32;
          const int64_t m     = std::max<int64_t>(1, (mid + 8 * u - 1) / (8 * u));
          const int64_t piece = round32((mid + m - 1) / m);
          for (int64_t left = mid; left > 0; left -= piece) {
            sizes.push_back(std::min(piece, left));
          }
          sizes.push_back(4 * u);
          sizes.push_back(2 * u);
          sizes.push_back(n - 13 * u - mid);
        }
        else {
          const int64_t chunk = round32((n + pieces - 1) / pieces);
          for (int64_t left = n; left > 0; left -= chunk) {
            sizes.push_back(std::min(chunk, left));
          }
        }
        int64_t off = 0;
        for (size_t c = 0; c < sizes.size() && rc == EBG_OK; off += sizes[c], c++) {
          const int64_t  cnt = sizes[c];
          cudaStream_t   st  = aux[c % NS];
          ebg_query_opts o   = opts ? *opts : ebg_query_opts{};
          if (o.radius_hint) {
            o.radius_hint += off;
          }
          cudaMemcpyAsync(dp + 3 * off, points_host + 3 * off, 3 * cnt * sizeof(float), cudaMemcpyHostToDevice, st);
          rc = meshQuery(m, dp + 3 * off, cnt, dd + off, dt ? dt + off : nullptr, &o, nullptr, st);
          if (rc == EBG_OK) {
            cudaMemcpyAsync(dist_host + off, dd + off, cnt * sizeof(float), cudaMemcpyDeviceToHost, st);
            if (dt) {
              cudaMemcpyAsync(closest_tri_host + off, dt + off, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
            }
          }
        }
        // s resumes (and frees the buffers) once every stream is done
        for (int i = 0; i < NS; i++) {
          cudaEventRecord(ev[i + 1], aux[i]);
          cudaStreamWaitEvent(s, ev[i + 1], 0);
        }
      }
      else {
        rc = setError(EBG_ERR_CUDA, "streams for the chunked host call");
      }
      for (int i = 0; i < NS + 1; i++) {
        if (ev[i]) {
          cudaEventDestroy(ev[i]);
        }
      }
      for (int i = 0; i < NS; i++) {
        if (aux[i]) {
          cudaStreamDestroy(aux[i]);
        }
      }
    }
  }
  if (rc != EBG_OK) {
    cudaStreamSynchronize(s);
    return rc;
  }
  return ebg_check_status(m, stream);
}

} // extern "C"

namespace {

// FP64 points in, FP64 distances out: the FP32 copy of the points drives the traversal, the FP64
// pass evaluates every query with evaluator evalKind (0 Triangle test, 1 DCEL face).
ebg_status meshQuery64(const ebg_mesh*       m,
                       const double*         points_dev,
                       int64_t               n,
                       double*               dist_dev,
                       int32_t*              closest_tri_dev,
                       const ebg_query_opts* opts,
                       void*                 stream,
                       int                   evalKind)
{
  if (m == nullptr || n < 0 || (n > 0 && (points_dev == nullptr || dist_dev == nullptr))) {
    return setError(EBG_ERR_INVALID, "null mesh/buffer or negative count");
  }
  if (n == 0) {
    return EBG_OK;
  }
  DeviceGuard  guard;
  cudaSetDevice(m->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Workspace    ws(s);
  float*       p32 = ws.get<float>(3 * n);
  float*       d32 = ws.get<float>(n);
  if (!ws.ok) {
    return setError(EBG_ERR_NO_MEMORY, "FP32 copy of the FP64 points");
  }
  launchDoubleToFloat(points_dev, p32, 3 * n, s);
  return meshQuery(m, p32, n, d32, closest_tri_dev, opts, nullptr, s, points_dev, dist_dev, evalKind);
}

// FlatMeshSDF: every triangle for every point (FP64, DCEL face algorithm).
ebg_status meshFlat64(const ebg_mesh*       m,
                      const double*         points_dev,
                      int64_t               n,
                      double*               dist_dev,
                      int32_t*              closest_tri_dev,
                      const ebg_query_opts* opts,
                      void*                 stream,
                      int                   evalKind)
{
  (void)opts;
  (void)evalKind;
  if (m == nullptr || n < 0 || (n > 0 && (points_dev == nullptr || dist_dev == nullptr))) {
    return setError(EBG_ERR_INVALID, "null mesh/buffer or negative count");
  }
  if (n == 0) {
    return EBG_OK;
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  if (launchMeshFlat64(m->view, m->info.num_triangles, points_dev, n, dist_dev, closest_tri_dev, m->dStatus,
                       m->numSms, static_cast<cudaStream_t>(stream)) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, std::string("brute-force launch failed: ") + cudaGetErrorString(cudaGetLastError()));
  }
  return EBG_OK;
}

using Entry64 = ebg_status (*)(const ebg_mesh*, const double*, int64_t, double*, int32_t*, const ebg_query_opts*,
                               void*, int);

// Host-buffer form of an FP64 entry: copies in, evaluates, copies out, synchronises.
ebg_status hostCall64(Entry64               fn,
                      int                   evalKind,
                      const ebg_mesh*       m,
                      const double*         points_host,
                      int64_t               n,
                      double*               dist_host,
                      int32_t*              closest_tri_host,
                      const ebg_query_opts* opts,
                      void*                 stream)
{
  if (m == nullptr || n < 0 || (n > 0 && (points_host == nullptr || dist_host == nullptr))) {
    return setError(EBG_ERR_INVALID, "null mesh/buffer or negative count");
  }
  if (n == 0) {
    return EBG_OK;
  }
  DeviceGuard  guard;
  cudaSetDevice(m->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaMemsetAsync(m->dStatus, 0, sizeof(int), s);
  ebg_status rc;
  {
    Workspace ws(s);
    double*   dp = ws.get<double>(3 * n);
    double*   dd = ws.get<double>(n);
    int32_t*  dt = closest_tri_host ? ws.get<int32_t>(n) : nullptr;
    if (!ws.ok) {
      return setError(EBG_ERR_NO_MEMORY, "device buffers for the host call");
    }
    cudaMemcpyAsync(dp, points_host, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s);
    rc = fn(m, dp, n, dd, dt, opts, stream, evalKind);
    if (rc == EBG_OK) {
      cudaMemcpyAsync(dist_host, dd, n * sizeof(double), cudaMemcpyDeviceToHost, s);
      if (dt) {
        cudaMemcpyAsync(closest_tri_host, dt, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
      }
    }
  }
  if (rc != EBG_OK) {
    return rc;
  }
  return ebg_check_status(m, stream);
}

} // namespace

extern "C" {

ebg_status ebg_mesh_signed_distance_f64(const ebg_mesh*       m,
                                        const double*         points_dev,
                                        int64_t               n,
                                        double*               dist_dev,
                                        int32_t*              closest_tri_dev,
                                        const ebg_query_opts* opts,
                                        void*                 stream)
{
  return meshQuery64(m, points_dev, n, dist_dev, closest_tri_dev, opts, stream, 0);
}

ebg_status ebg_mesh_signed_distance_f64_host(const ebg_mesh*       m,
                                             const double*         points_host,
                                             int64_t               n,
                                             double*               dist_host,
                                             int32_t*              closest_tri_host,
                                             const ebg_query_opts* opts,
                                             void*                 stream)
{
  return hostCall64(meshQuery64, 0, m, points_host, n, dist_host, closest_tri_host, opts, stream);
}

ebg_status ebg_mesh_signed_distance_dcel_f64(const ebg_mesh*       m,
                                             const double*         points_dev,
                                             int64_t               n,
                                             double*               dist_dev,
                                             int32_t*              closest_tri_dev,
                                             const ebg_query_opts* opts,
                                             void*                 stream)
{
  return meshQuery64(m, points_dev, n, dist_dev, closest_tri_dev, opts, stream, 1);
}

ebg_status ebg_mesh_signed_distance_dcel_f64_host(const ebg_mesh*       m,
                                                  const double*         points_host,
                                                  int64_t               n,
                                                  double*               dist_host,
                                                  int32_t*              closest_tri_host,
                                                  const ebg_query_opts* opts,
                                                  void*                 stream)
{
  return hostCall64(meshQuery64, 1, m, points_host, n, dist_host, closest_tri_host, opts, stream);
}

ebg_status ebg_mesh_signed_distance_flat_f64(const ebg_mesh* m,
                                             const double*   points_dev,
                                             int64_t         n,
                                             double*         dist_dev,
                                             int32_t*        closest_tri_dev,
                                             void*           stream)
{
  return meshFlat64(m, points_dev, n, dist_dev, closest_tri_dev, nullptr, stream, 0);
}

ebg_status ebg_mesh_signed_distance_flat_f64_host(const ebg_mesh* m,
                                                  const double*   points_host,
                                                  int64_t         n,
                                                  double*         dist_host,
                                                  int32_t*        closest_tri_host,
                                                  void*           stream)
{
  return hostCall64(meshFlat64, 0, m, points_host, n, dist_host, closest_tri_host, nullptr, stream);
}

ebg_status ebg_mesh_signed_distance_stats(const ebg_mesh*       m,
                                          const float*          points_dev,
                                          int64_t               n,
                                          float*                dist_dev,
                                          const ebg_query_opts* opts,
                                          ebg_query_stats*      stats,
                                          void*                 stream)
{
  if (m == nullptr || stats == nullptr || n < 0 || (n > 0 && (points_dev == nullptr || dist_dev == nullptr))) {
    return setError(EBG_ERR_INVALID, "null argument or negative count");
  }
  std::memset(stats, 0, sizeof(*stats));
  if (n == 0) {
    return EBG_OK;
  }
  DeviceGuard  guard;
  cudaSetDevice(m->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ebg_status   rc;
  constexpr int      NSTAT    = 15;
  unsigned long long host[NSTAT] = {};
  {
    Workspace           ws(s);
    unsigned long long* dev = ws.get<unsigned long long>(NSTAT);
    if (!ws.ok) {
      return setError(EBG_ERR_NO_MEMORY, "stats buffer");
    }
    cudaMemsetAsync(dev, 0, NSTAT * sizeof(unsigned long long), s);
    rc = meshQuery(m, points_dev, n, dist_dev, nullptr, opts, dev, s);
    if (rc == EBG_OK) {
      cudaMemcpyAsync(host, dev, sizeof(host), cudaMemcpyDeviceToHost, s);
    }
  }
  if (rc != EBG_OK) {
    return rc;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  stats->nodes_visited    = int64_t(host[0]);
  stats->leaves_visited   = int64_t(host[1]);
  stats->triangles_tested = int64_t(host[2]);
  stats->band_queries     = int64_t(host[3] & 0xffffffffull);
  stats->seed_fallbacks   = int64_t(host[4]);
  stats->packets          = int64_t(host[5]);
  stats->packet_pops      = int64_t(host[6]);
  stats->packet_nodes     = int64_t(host[7]);
  stats->packet_leaves    = int64_t(host[8]);
  stats->packet_triangles = int64_t(host[9]);
  stats->boxes_tested     = int64_t(host[10]);
  stats->packet_boxes     = int64_t(host[11]);
  stats->cut_packets      = int64_t(host[12]);
  stats->cut_entries      = int64_t(host[13]);
  stats->packet_triangle_records = int64_t(host[14]);
  return ebg_check_status(m, stream);
}

ebg_status ebg_mesh_autotune(ebg_mesh*       m,
                             const float*    sample_points_dev,
                             int64_t         n,
                             const ebg_seed* seed,
                             int32_t*        best_occupancy,
                             int32_t*        best_warps_per_block,
                             int32_t*        best_queue_chunk,
                             int32_t*        best_node_width,
                             float*          best_ms,
                             void*           stream)
{
  if (m == nullptr || sample_points_dev == nullptr || n < 32) {
    return setError(EBG_ERR_INVALID, "autotune needs a mesh and at least 32 sample points");
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  float*       out = nullptr;
  cudaStream_t s   = static_cast<cudaStream_t>(stream);
  if (cudaMallocAsync(reinterpret_cast<void**>(&out), size_t(n) * sizeof(float), s) != cudaSuccess) {
    cudaGetLastError();
    return setError(EBG_ERR_NO_MEMORY, "autotune output buffer");
  }
  // the traversal time of one candidate: the best of two timed runs after a warm-up run
  auto timeOne = [&](int o, int w, int c, float& ms, int width = 4) -> ebg_status {
    ebg_query_opts    q{};
    ebg_phase_timings t{};
    q.occupancy       = o;
    q.warps_per_block = w;
    q.queue_chunk     = c;
    q.node_width      = width;
    q.no_fp64_band    = 1;
    q.seed            = seed;
    ms                = INFINITY;
    for (int rep = 0; rep < 3; rep++) {
      q.timings           = &t;
      const ebg_status rc = meshQuery(m, sample_points_dev, n, out, nullptr, &q, nullptr, s);
      if (rc != EBG_OK) {
        return rc;
      }
      if (rep > 0) {
        ms = std::min(ms, t.traverse_ms);
      }
    }
    return EBG_OK;
  };
  float     bestMs = INFINITY;
  int       bestO = 1, bestW = 4, bestC = 1;
  const int occs[] = {1, 4, 2};
  const int wpbs[] = {2, 4, 8};
  for (int o : occs) {
    for (int w : wpbs) {
      if (o != 4 && w > 4) {
        continue;
      }
      float            ms = INFINITY;
      const ebg_status rc = timeOne(o, w, 1, ms);
      if (rc != EBG_OK) {
        cudaFreeAsync(out, s);
        return rc;
      }
      if (ms < bestMs) {
        bestMs = ms;
        bestO  = o;
        bestW  = w;
      }
    }
  }
  for (int c : {2, 4}) {
    float            ms = INFINITY;
    const ebg_status rc = timeOne(bestO, bestW, c, ms);
    if (rc != EBG_OK) {
      cudaFreeAsync(out, s);
      return rc;
    }
    if (ms < bestMs) {
      bestMs = ms;
      bestC  = c;
    }
  }
  // node width: the 8-wide copy at the launch shapes again (its node visits differ), kept when faster
  int bestWidth = 4;
  if (seed == nullptr && m->hasWide && !(m->view.root_ref & EBG_LEAF_BIT)) {
    for (int o : occs) {
      for (int w : wpbs) {
        if (o != 4 && w > 4) {
          continue;
        }
        float            ms = INFINITY;
        const ebg_status rc = timeOne(o, w, bestC, ms, 8);
        if (rc != EBG_OK) {
          cudaFreeAsync(out, s);
          return rc;
        }
        if (ms < bestMs) {
          bestMs    = ms;
          bestO     = o;
          bestW     = w;
          bestWidth = 8;
        }
      }
    }
  }
  cudaFreeAsync(out, s);
  cudaStreamSynchronize(s);
  m->tunedOccupancy = bestO;
  m->tunedWpb       = bestW;
  m->tunedChunk     = bestC;
  m->tunedWidth     = bestWidth;
  if (best_occupancy) {
    *best_occupancy = bestO;
  }
  if (best_warps_per_block) {
    *best_warps_per_block = bestW;
  }
  if (best_queue_chunk) {
    *best_queue_chunk = bestC;
  }
  if (best_node_width) {
    *best_node_width = bestWidth;
  }
  if (best_ms) {
    *best_ms = bestMs;
  }
  return EBG_OK;
}

ebg_status ebg_mesh_widen(ebg_mesh* m, int64_t* num_nodes8, int32_t* depth8)
{
  if (m == nullptr) {
    return setError(EBG_ERR_INVALID, "null mesh");
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  if (!m->hasWide) {
    if (m->view.root_ref & EBG_LEAF_BIT) {
      // a single leaf: nothing to widen, the 8-wide traversal meets the same root
      m->view8   = m->view;
      m->hasWide = true;
    }
    else {
      const size_t          nn = size_t(m->info.num_nodes);
      std::vector<EbgNode4> n4(nn);
      std::vector<EbgObb>   o4(nn);
      if (cudaMemcpy(n4.data(), m->dNodes, nn * sizeof(EbgNode4), cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMemcpy(o4.data(), m->dNodeObb, nn * sizeof(EbgObb), cudaMemcpyDeviceToHost) != cudaSuccess) {
        return setError(EBG_ERR_CUDA, std::string("widen: reading the tree: ") + cudaGetErrorString(cudaGetLastError()));
      }
      std::vector<EbgNode8> n8;
      std::vector<EbgObb>   o8;
      int                   d8 = 0;
      std::string           msg;
      if (!widenBvh8(n4, o4, m->info.num_triangles, m->info.num_leaves, n8, o8, d8, msg)) {
        return setError(msg.find("too deep") != std::string::npos ? EBG_ERR_TOO_LARGE : EBG_ERR_INVALID, msg);
      }
      if (cudaMalloc(&m->dNodes8, n8.size() * sizeof(EbgNode8)) != cudaSuccess ||
          cudaMalloc(&m->dNodeObb8, o8.size() * sizeof(EbgObb)) != cudaSuccess) {
        cudaGetLastError();
        dropWide(m);
        return setError(EBG_ERR_NO_MEMORY, "widen: device allocation for the 8-wide nodes");
      }
      if (cudaMemcpy(m->dNodes8, n8.data(), n8.size() * sizeof(EbgNode8), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(m->dNodeObb8, o8.data(), o8.size() * sizeof(EbgObb), cudaMemcpyHostToDevice) != cudaSuccess) {
        const std::string e = cudaGetErrorString(cudaGetLastError());
        dropWide(m);
        return setError(EBG_ERR_CUDA, "widen: uploading the 8-wide nodes: " + e);
      }
      // the root keeps its box and index 0; the kernels read EbgNode8 records through these
      m->view8          = m->view;
      m->view8.nodes    = static_cast<const EbgNode4*>(m->dNodes8);
      m->view8.node_obb = static_cast<const EbgObb*>(m->dNodeObb8);
      m->numNodes8      = int64_t(n8.size());
      m->depth8         = d8;
      m->hasWide        = true;
    }
  }
  if (num_nodes8) {
    *num_nodes8 = m->numNodes8;
  }
  if (depth8) {
    *depth8 = m->depth8;
  }
  return EBG_OK;
}

ebg_status ebg_mesh_value(const ebg_mesh* m, double x, double y, double z, double* value)
{
  if (m == nullptr || value == nullptr) {
    return setError(EBG_ERR_INVALID, "null argument");
  }
  // one point, evaluated in FP64 like the reference's value()
  const double   p[3] = {x, y, z};
  ebg_query_opts o{};
  o.no_sort = 1;
  return ebg_mesh_signed_distance_f64_host(m, p, 1, value, nullptr, &o, nullptr);
}

ebg_status ebg_check_status(const ebg_mesh* m, void* stream)
{
  if (m == nullptr) {
    return setError(EBG_ERR_INVALID, "null mesh");
  }
  DeviceGuard guard;
  cudaSetDevice(m->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int          st = 0;
  if (cudaMemcpyAsync(&st, m->dStatus, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    return setError(EBG_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
  }
  if (st != 0) {
    cudaMemsetAsync(m->dStatus, 0, sizeof(int), s);
    if (st & ST_INPUT) {
      return setError(EBG_ERR_INVALID, "non-finite query coordinate");
    }
    return setError(EBG_ERR_TRAVERSAL, "traversal stopped early (status " + std::to_string(st) + ")");
  }
  return EBG_OK;
}

} // extern "C"
