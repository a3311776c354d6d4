// Host-side preprocessing for the mesh path (C++17, OpenMP tasks for the tree build).
//
// 1. Pseudonormals.  The reference reaches TriMeshSDF through Soup::soupToDCEL and
//    MeshT::reconcile(Angle) (SoupImplem.hpp:149-227, DCEL_MeshImplem.hpp:304-366), then copies
//    per face the normals into a Triangle (MeshDistanceFunctionsImplem.hpp:429-452).  The result
//    is reproduced here without building a half-edge structure, keeping the reference's
//    floating-point operation order so the normals agree bit for bit:
//      - DCEL face normal: (x2-x0) x (x2-x1), normalised twice (FaceT::computeNormal and then
//        reconcile's normalizeNormalVector, DCEL_FaceImplem.hpp:71-79,136-166); division is a
//        multiply by the reciprocal (Vec3T::operator/, VecImplem.hpp:303-309);
//      - the Triangle's own face normal, recomputed by Triangle::setVertexPositions, normalised
//        once (TriangleImplem.hpp:45-57,94-106); it is the one the distance test uses;
//      - edge normal: normalize(n_face + n_pair_face) (DCEL_EdgeImplem.hpp:128-165);
//      - vertex normal: sum over the vertex's faces in facet order of alpha * n_face, alpha the
//        subtended angle acos(clamp(e1.e2)), then normalised (DCEL_VertexImplem.hpp:190-~290).
// 2. A 4-wide BVH: binned SAH (32 bins, cost A_L N_L + A_R N_R, the reference's
//    BinnedSAHPartitioner / SAH2WaySplit, BVH.hpp:521-734) or a Morton split (highest differing
//    bit of 63-bit codes), each node taking up to four children by repeatedly splitting its
//    largest-area child.  Leaves hold at most leafSize primitives.
#include "mesh_host.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>

namespace ebg {

namespace {

struct V3
{
  double x, y, z;
};
inline V3 ld3(const double* p) { return {p[0], p[1], p[2]}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double len(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline V3 divs(V3 a, double s)
{
  const double is = 1.0 / s;
  return {is * a.x, is * a.y, is * a.z};
}
inline void st3(double* p, V3 a)
{
  p[0] = a.x;
  p[1] = a.y;
  p[2] = a.z;
}

} // namespace

float roundDown(double x)
{
  float f = static_cast<float>(x);
  if (static_cast<double>(f) > x) {
    f = std::nextafter(f, -std::numeric_limits<float>::infinity());
  }
  return f;
}

float roundUp(double x)
{
  float f = static_cast<float>(x);
  if (static_cast<double>(f) < x) {
    f = std::nextafter(f, std::numeric_limits<float>::infinity());
  }
  return f;
}

bool computePseudonormals(const double*        V,
                          int64_t              nv,
                          const int32_t*       F,
                          int64_t              nt,
                          std::vector<double>& triN,
                          std::vector<double>& cornerVN,
                          std::vector<double>& edgeN,
                          std::string&         msg)
{
  triN.assign(3 * nt, 0.0);
  cornerVN.assign(9 * nt, 0.0);
  edgeN.assign(9 * nt, 0.0);
  std::vector<double> faceN(3 * nt);

  bool degenerate = false;
#pragma omp parallel for schedule(static) reduction(|| : degenerate)
  for (int64_t f = 0; f < nt; f++) {
    const V3 x0 = ld3(V + 3 * int64_t(F[3 * f])), x1 = ld3(V + 3 * int64_t(F[3 * f + 1])),
             x2 = ld3(V + 3 * int64_t(F[3 * f + 2]));
    const V3     c = cross(sub(x2, x0), sub(x2, x1));
    const double l = len(c);
    if (!(l > 0.0)) {
      degenerate = true;
      continue;
    }
    const V3 once = divs(c, l);
    st3(&triN[3 * f], once);
    st3(&faceN[3 * f], divs(once, len(once)));
  }
  if (degenerate) {
    msg = "degenerate (zero-area) triangle in the soup";
    return false;
  }

  // Faces around each vertex, in facet order (a stable counting sort): the order the reference's
  // DCEL vertex keeps its faces in (soupToDCEL adds them facet by facet, SoupImplem.hpp:204-207).
  std::vector<int64_t> start(nv + 1, 0);
  for (int64_t i = 0; i < 3 * nt; i++) {
    start[int64_t(F[i]) + 1]++;
  }
  for (int64_t v = 0; v < nv; v++) {
    start[v + 1] += start[v];
  }
  std::vector<int64_t> fill(start.begin(), start.end() - 1);
  std::vector<int64_t> around(3 * nt); // entries f * 3 + corner
  for (int64_t f = 0; f < nt; f++) {
    for (int k = 0; k < 3; k++) {
      around[fill[F[3 * f + k]]++] = 3 * f + k;
    }
  }

  // Edge pseudonormals: the pair of half-edge (a -> b) of face f is the half-edge (b -> a) of the
  // other face around a that also holds b.
  bool nonManifold = false;
#pragma omp parallel for schedule(static) reduction(|| : nonManifold)
  for (int64_t f = 0; f < nt; f++) {
    for (int i = 0; i < 3; i++) {
      const int32_t a = F[3 * f + i], b = F[3 * f + (i + 1) % 3];
      int64_t       pair = -1, found = 0;
      for (int64_t e = start[a]; e < start[a + 1]; e++) {
        const int64_t g = around[e] / 3;
        if (g == f) {
          continue;
        }
        for (int k = 0; k < 3; k++) {
          if (F[3 * g + k] == b) {
            found++;
            pair = g;
          }
        }
      }
      if (found > 1) {
        nonManifold = true;
      }
      V3 n = ld3(&faceN[3 * f]);
      if (pair >= 0) {
        n = {n.x + faceN[3 * pair], n.y + faceN[3 * pair + 1], n.z + faceN[3 * pair + 2]};
      }
      const double l = len(n);
      st3(&edgeN[9 * f + 3 * i], (l > std::numeric_limits<double>::epsilon()) ? divs(n, l) : V3{0, 0, 0});
    }
  }
  if (nonManifold) {
    msg = "non-manifold edge (shared by more than two triangles)";
    return false;
  }

  // Angle-weighted vertex normals: each corner's alpha * n_face in parallel, then each vertex sums
  // its corners in facet order with the reference's operation order (m_normal += alpha * n).
  std::vector<double> contrib(9 * nt);
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < nt; f++) {
    const int32_t a = F[3 * f], b = F[3 * f + 1], c = F[3 * f + 2];
    // neighbours of each corner in half-edge loop order: a:(b,c) b:(a,c) c:(b,a)
    const int32_t corner[3] = {a, b, c}, n1[3] = {b, a, b}, n2[3] = {c, c, a};
    const V3      fn        = ld3(&faceN[3 * f]);
    for (int k = 0; k < 3; k++) {
      const V3 x0 = ld3(V + 3 * int64_t(corner[k]));
      V3       e1 = sub(ld3(V + 3 * int64_t(n1[k])), x0);
      V3       e2 = sub(ld3(V + 3 * int64_t(n2[k])), x0);
      e1          = divs(e1, len(e1));
      e2          = divs(e2, len(e2));
      const double alpha = std::acos(std::clamp(dot(e1, e2), -1.0, 1.0));
      contrib[9 * f + 3 * k + 0] = alpha * fn.x;
      contrib[9 * f + 3 * k + 1] = alpha * fn.y;
      contrib[9 * f + 3 * k + 2] = alpha * fn.z;
    }
  }
  std::vector<double> vn(3 * nv, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < nv; v++) {
    double x = 0.0, y = 0.0, z = 0.0;
    for (int64_t e = start[v]; e < start[v + 1]; e++) {
      const double* c = &contrib[3 * around[e]];
      x += c[0];
      y += c[1];
      z += c[2];
    }
    const V3     n = {x, y, z};
    const double l = len(n);
    st3(&vn[3 * v], (l > std::numeric_limits<double>::epsilon()) ? divs(n, l) : n);
  }
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < nt; f++) {
    for (int k = 0; k < 3; k++) {
      std::memcpy(&cornerVN[9 * f + 3 * k], &vn[3 * int64_t(F[3 * f + k])], 3 * sizeof(double));
    }
  }
  return true;
}

// ---------------------------------------------------------------------------------------------
// Polygon faces: the same DCEL rules for faces of any vertex count.

bool computePolygonNormals(const double*        V,
                           int64_t              nv,
                           const int64_t*       off,
                           const int32_t*       idx,
                           int64_t              nf,
                           std::vector<double>& faceN,
                           std::vector<double>& centroid,
                           std::vector<double>& cornerVN,
                           std::vector<double>& edgeN,
                           std::string&         msg)
{
  const int64_t nc = off[nf];
  faceN.assign(3 * nf, 0.0);
  centroid.assign(3 * nf, 0.0);
  cornerVN.assign(3 * nc, 0.0);
  edgeN.assign(3 * nc, 0.0);
  auto vx = [&](int64_t corner) { return ld3(V + 3 * int64_t(idx[corner])); };

  // face normal: (x2 - x0) x (x2 - x1) of the first vertex triple (i, i+1, i+2) that spans a plane,
  // normalised twice (FaceT::computeNormal, then reconcile's normalizeNormalVector); centroid: the
  // vertex sum times 1/N (DCEL_FaceImplem.hpp:71-79,121-166)
  bool degenerate = false;
#pragma omp parallel for schedule(static) reduction(|| : degenerate)
  for (int64_t f = 0; f < nf; f++) {
    const int64_t b = off[f], N = off[f + 1] - off[f];
    V3            c{0, 0, 0};
    double        l = 0;
    for (int64_t i = 0; i < N; i++) {
      const V3 x0 = vx(b + i), x1 = vx(b + (i + 1) % N), x2 = vx(b + (i + 2) % N);
      c = cross(sub(x2, x0), sub(x2, x1));
      l = len(c);
      if (l > 0.0) {
        break;
      }
    }
    if (!(l > 0.0)) {
      degenerate = true;
      continue;
    }
    const V3 once = divs(c, l);
    st3(&faceN[3 * f], divs(once, len(once)));
    V3 s{0, 0, 0};
    for (int64_t i = 0; i < N; i++) {
      const V3 x = vx(b + i);
      s          = {s.x + x.x, s.y + x.y, s.z + x.z};
    }
    st3(&centroid[3 * f], divs(s, double(N)));
  }
  if (degenerate) {
    msg = "degenerate face (no three vertices span a plane)";
    return false;
  }

  // faces around each vertex in facet order (soupToDCEL adds them facet by facet)
  std::vector<int64_t> start(nv + 1, 0);
  for (int64_t i = 0; i < nc; i++) {
    start[int64_t(idx[i]) + 1]++;
  }
  for (int64_t v = 0; v < nv; v++) {
    start[v + 1] += start[v];
  }
  std::vector<int64_t> fill(start.begin(), start.end() - 1);
  std::vector<int64_t> around(nc); // entries: the corner
  std::vector<int64_t> faceOf(nc);
  for (int64_t f = 0; f < nf; f++) {
    for (int64_t k = off[f]; k < off[f + 1]; k++) {
      around[fill[idx[k]]++] = k;
      faceOf[k]              = f;
    }
  }

  // edge normals: the pair of half-edge (a -> b) is a half-edge (b -> a) of a face around a
  // (Soup::reconcilePairEdgesDCEL, SoupImplem.hpp:229-262); normalize(n_face + n_pair)
  bool nonManifold = false;
#pragma omp parallel for schedule(static) reduction(|| : nonManifold)
  for (int64_t f = 0; f < nf; f++) {
    const int64_t b = off[f], N = off[f + 1] - off[f];
    for (int64_t i = 0; i < N; i++) {
      const int32_t a = idx[b + i], e = idx[b + (i + 1) % N];
      int64_t       pair = -1, found = 0;
      for (int64_t s2 = start[a]; s2 < start[a + 1]; s2++) {
        const int64_t g = faceOf[around[s2]];
        const int64_t gb = off[g], gn = off[g + 1] - off[g];
        for (int64_t j = 0; j < gn; j++) {
          if (idx[gb + j] == e && idx[gb + (j + 1) % gn] == a) {
            found++;
            pair = g;
          }
        }
      }
      if (found > 1) {
        nonManifold = true;
      }
      V3 n = ld3(&faceN[3 * f]);
      if (pair >= 0) {
        n = {n.x + faceN[3 * pair], n.y + faceN[3 * pair + 1], n.z + faceN[3 * pair + 2]};
      }
      const double l = len(n);
      st3(&edgeN[3 * (b + i)], (l > std::numeric_limits<double>::epsilon()) ? divs(n, l) : V3{0, 0, 0});
    }
  }
  if (nonManifold) {
    msg = "non-manifold edge (shared by more than two faces)";
    return false;
  }

  // angle-weighted vertex normals: the angle at each corner between its two neighbours in the
  // face's loop, alpha * n_face summed over the vertex's faces in facet order, then normalised
  std::vector<double> contrib(3 * nc);
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < nf; f++) {
    const int64_t b = off[f], N = off[f + 1] - off[f];
    const V3      fn = ld3(&faceN[3 * f]);
    for (int64_t k = 0; k < N; k++) {
      const V3 x0 = vx(b + k);
      V3       e1 = sub(vx(b + (k + N - 1) % N), x0);
      V3       e2 = sub(vx(b + (k + 1) % N), x0);
      e1          = divs(e1, len(e1));
      e2          = divs(e2, len(e2));
      const double alpha = std::acos(std::clamp(dot(e1, e2), -1.0, 1.0));
      contrib[3 * (b + k) + 0] = alpha * fn.x;
      contrib[3 * (b + k) + 1] = alpha * fn.y;
      contrib[3 * (b + k) + 2] = alpha * fn.z;
    }
  }
  std::vector<double> vn(3 * nv, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < nv; v++) {
    double x = 0.0, y = 0.0, z = 0.0;
    for (int64_t e = start[v]; e < start[v + 1]; e++) {
      const double* c = &contrib[3 * around[e]];
      x += c[0];
      y += c[1];
      z += c[2];
    }
    const V3     n = {x, y, z};
    const double l = len(n);
    st3(&vn[3 * v], (l > std::numeric_limits<double>::epsilon()) ? divs(n, l) : n);
  }
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nc; k++) {
    std::memcpy(&cornerVN[3 * k], &vn[3 * int64_t(idx[k])], 3 * sizeof(double));
  }
  return true;
}

// ---------------------------------------------------------------------------------------------
// 4-wide BVH build

namespace {

struct Box
{
  double lo[3] = {std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                  std::numeric_limits<double>::infinity()};
  double hi[3] = {-std::numeric_limits<double>::infinity(), -std::numeric_limits<double>::infinity(),
                  -std::numeric_limits<double>::infinity()};
  void   grow(const double* l, const double* h)
  {
    for (int a = 0; a < 3; a++) {
      lo[a] = std::min(lo[a], l[a]);
      hi[a] = std::max(hi[a], h[a]);
    }
  }
  void grow(const Box& b) { grow(b.lo, b.hi); }
  double area() const
  {
    if (!(hi[0] >= lo[0])) {
      return 0.0;
    }
    const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return 2.0 * (dx * dy + dy * dz + dz * dx);
  }
};

struct Builder
{
  const std::vector<double>& lo;
  const std::vector<double>& hi;
  const std::vector<double>& cen;
  std::vector<uint64_t>      morton;
  int                        build;
  int                        leafSize;
  std::vector<uint32_t>&     idx;
  std::vector<EbgNode4>&     nodes;
  std::atomic<uint32_t>      nodeCount{0};
  std::vector<uint32_t>*     leafFirst = nullptr;
  std::vector<uint32_t>*     leafCount = nullptr;
  std::vector<uint32_t>*     nodeFirst = nullptr;
  std::vector<uint32_t>*     nodeEnd   = nullptr;
  std::atomic<int>           maxDepth{0};
  std::atomic<int64_t>       leaves{0};

  Builder(const std::vector<double>& l, const std::vector<double>& h, const std::vector<double>& c, int b, int ls,
          std::vector<uint32_t>& i, std::vector<EbgNode4>& n)
    : lo(l), hi(h), cen(c), build(b), leafSize(ls), idx(i), nodes(n)
  {}

  Box rangeBox(uint32_t b, uint32_t e) const
  {
    Box box;
    for (uint32_t i = b; i < e; i++) {
      box.grow(&lo[3 * size_t(idx[i])], &hi[3 * size_t(idx[i])]);
    }
    return box;
  }

  // Splits [b,e) in two; returns the split position (b < m < e).
  uint32_t split(uint32_t b, uint32_t e)
  {
    const uint32_t n = e - b;
    if (build == 1) {
      // Morton: codes are sorted; split where the highest differing bit flips.
      const uint64_t cb = morton[b], ce = morton[e - 1];
      if (cb == ce) {
        return b + n / 2;
      }
      const int      bit  = 63 - __builtin_clzll(cb ^ ce);
      const uint64_t mask = ~((uint64_t(1) << bit) - 1);
      const uint64_t pivot = (ce & mask);
      uint32_t       lo_i = b, hi_i = e - 1;
      while (lo_i < hi_i) {
        const uint32_t mid = lo_i + (hi_i - lo_i) / 2;
        if ((morton[mid] & mask) >= pivot) {
          hi_i = mid;
        }
        else {
          lo_i = mid + 1;
        }
      }
      return (lo_i > b && lo_i < e) ? lo_i : b + n / 2;
    }

    // Binned SAH over centroids.
    double cl[3] = {1e300, 1e300, 1e300}, ch[3] = {-1e300, -1e300, -1e300};
    for (uint32_t i = b; i < e; i++) {
      const double* c = &cen[3 * size_t(idx[i])];
      for (int a = 0; a < 3; a++) {
        cl[a] = std::min(cl[a], c[a]);
        ch[a] = std::max(ch[a], c[a]);
      }
    }
    constexpr int NB       = 32;
    double        bestCost = std::numeric_limits<double>::infinity();
    int           bestAxis = -1, bestBin = -1;
    for (int a = 0; a < 3; a++) {
      const double ext = ch[a] - cl[a];
      if (!(ext > 0.0)) {
        continue;
      }
      Box      bins[NB];
      uint32_t cnt[NB] = {0};
      const double k   = NB / ext;
      for (uint32_t i = b; i < e; i++) {
        const size_t p  = idx[i];
        int          bi = int((cen[3 * p + a] - cl[a]) * k);
        bi              = std::min(std::max(bi, 0), NB - 1);
        bins[bi].grow(&lo[3 * p], &hi[3 * p]);
        cnt[bi]++;
      }
      double   rightArea[NB];
      uint32_t rightCnt[NB];
      Box      acc;
      uint32_t c = 0;
      for (int i = NB - 1; i > 0; i--) {
        acc.grow(bins[i]);
        c += cnt[i];
        rightArea[i] = acc.area();
        rightCnt[i]  = c;
      }
      Box      left;
      uint32_t lc = 0;
      for (int i = 0; i < NB - 1; i++) {
        left.grow(bins[i]);
        lc += cnt[i];
        if (lc == 0 || rightCnt[i + 1] == 0) {
          continue;
        }
        const double cost = left.area() * lc + rightArea[i + 1] * rightCnt[i + 1];
        if (cost < bestCost) {
          bestCost = cost;
          bestAxis = a;
          bestBin  = i;
        }
      }
    }
    if (bestAxis >= 0) {
      const double ext = ch[bestAxis] - cl[bestAxis];
      const double k   = NB / ext;
      // stable, so the order inside each side (and with it every leaf's triangle order) is the
      // order it had, exactly as the device build's partition keeps it
      auto         mid = std::stable_partition(idx.begin() + b, idx.begin() + e, [&](uint32_t p) {
        int bi = int((cen[3 * size_t(p) + bestAxis] - cl[bestAxis]) * k);
        bi     = std::min(std::max(bi, 0), NB - 1);
        return bi <= bestBin;
      });
      const uint32_t m = uint32_t(mid - idx.begin());
      if (m > b && m < e) {
        return m;
      }
    }
    // No SAH split has both sides non-empty only when every centroid is the same point (on any
    // axis with extent, the lowest and highest centroids fall in the first and last bins): halve.
    return b + n / 2;
  }

  // Builds the interior node for [b,e) into nodes[self] (count > leafSize).
  void node(uint32_t self, uint32_t b, uint32_t e, int depth)
  {
    struct R
    {
      uint32_t b, e;
      double   area;
    };
    R   ch[4];
    int nc = 1;
    ch[0]  = {b, e, rangeBox(b, e).area()};
    while (nc < 4) {
      int pick = -1;
      for (int i = 0; i < nc; i++) {
        if (ch[i].e - ch[i].b > uint32_t(leafSize) && (pick < 0 || ch[i].area > ch[pick].area)) {
          pick = i;
        }
      }
      if (pick < 0) {
        break;
      }
      const uint32_t m = split(ch[pick].b, ch[pick].e);
      const R        l{ch[pick].b, m, rangeBox(ch[pick].b, m).area()};
      const R        r{m, ch[pick].e, rangeBox(m, ch[pick].e).area()};
      ch[pick]  = l;
      ch[nc++]  = r;
    }
    EbgNode4& nd       = nodes[self];
    (*nodeFirst)[self] = b;
    (*nodeEnd)[self]   = e;
    for (int k = 0; k < 4; k++) {
      nd.lox[k] = nd.loy[k] = nd.loz[k] = std::numeric_limits<float>::infinity();
      nd.hix[k] = nd.hiy[k] = nd.hiz[k] = -std::numeric_limits<float>::infinity();
      nd.child[k] = 0;
      nd.count[k] = 0;
    }
    uint32_t childNode[4] = {0, 0, 0, 0};
    for (int k = 0; k < nc; k++) {
      const Box bx = rangeBox(ch[k].b, ch[k].e);
      nd.lox[k]    = roundDown(bx.lo[0]);
      nd.loy[k]    = roundDown(bx.lo[1]);
      nd.loz[k]    = roundDown(bx.lo[2]);
      nd.hix[k]    = roundUp(bx.hi[0]);
      nd.hiy[k]    = roundUp(bx.hi[1]);
      nd.hiz[k]    = roundUp(bx.hi[2]);
      const uint32_t cnt = ch[k].e - ch[k].b;
      if (cnt <= uint32_t(leafSize)) {
        const uint32_t id = uint32_t(leaves.fetch_add(1));
        nd.child[k]       = EBG_LEAF_BIT | ch[k].b;
        nd.count[k]       = cnt | (id << EBG_COUNT_BITS);
        (*leafFirst)[id]  = ch[k].b;
        (*leafCount)[id]  = cnt;
        int d = depth + 1;
        int cur = maxDepth.load();
        while (d > cur && !maxDepth.compare_exchange_weak(cur, d)) {
        }
      }
      else {
        childNode[k] = nodeCount.fetch_add(1);
        nd.child[k]  = childNode[k];
        nd.count[k]  = 0;
      }
    }
    for (int k = 0; k < nc; k++) {
      if (childNode[k] != 0) {
        const uint32_t cb = ch[k].b, ce = ch[k].e, cn = childNode[k];
        if (ce - cb > 4096) {
#pragma omp task firstprivate(cb, ce, cn, depth)
          node(cn, cb, ce, depth + 1);
        }
        else {
          node(cn, cb, ce, depth + 1);
        }
      }
    }
  }
};

inline uint64_t spread21(uint64_t x)
{
  x &= 0x1fffff;
  x = (x | x << 32) & 0x1f00000000ffffULL;
  x = (x | x << 16) & 0x1f0000ff0000ffULL;
  x = (x | x << 8) & 0x100f00f00f00f00fULL;
  x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
  x = (x | x << 2) & 0x1249249249249249ULL;
  return x;
}

} // namespace

bool buildBvh4(const std::vector<double>& boxLo,
               const std::vector<double>& boxHi,
               const std::vector<double>& centroid,
               int                        build,
               int                        leafSize,
               Bvh4&                      out,
               std::string&               msg)
{
  const size_t n = boxLo.size() / 3;
  if (n == 0) {
    msg = "empty primitive list";
    return false;
  }
  if (leafSize < 1 || leafSize > EBG_MAX_LEAF) {
    msg = "leaf size must be in [1, 32]";
    return false;
  }
  if (n >= size_t(EBG_LEAF_BIT)) {
    msg = "too many primitives";
    return false;
  }
  out.order.resize(n);
  std::iota(out.order.begin(), out.order.end(), 0u);
  Box all;
  for (size_t i = 0; i < n; i++) {
    all.grow(&boxLo[3 * i], &boxHi[3 * i]);
  }
  for (int a = 0; a < 3; a++) {
    out.lo[a] = all.lo[a];
    out.hi[a] = all.hi[a];
  }

  // every interior node has at least two children, so there are fewer interior nodes than leaves
  std::vector<EbgNode4> nodes(std::max<size_t>(1, n));
  Builder               B(boxLo, boxHi, centroid, build, leafSize, out.order, nodes);

  if (build == 1) {
    // Morton codes of the centroids (21 bits per axis, SFC::Morton's resolution, SFC.hpp:61-96).
    double cl[3] = {1e300, 1e300, 1e300}, ch[3] = {-1e300, -1e300, -1e300};
    for (size_t i = 0; i < n; i++) {
      for (int a = 0; a < 3; a++) {
        cl[a] = std::min(cl[a], centroid[3 * i + a]);
        ch[a] = std::max(ch[a], centroid[3 * i + a]);
      }
    }
    std::vector<uint64_t> code(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); i++) {
      uint64_t c = 0;
      for (int a = 0; a < 3; a++) {
        const double ext = ch[a] - cl[a];
        const double u   = ext > 0 ? (centroid[3 * i + a] - cl[a]) / ext : 0.0;
        const uint64_t q = uint64_t(std::min(std::max(u * 2097151.0, 0.0), 2097151.0));
        c |= spread21(q) << (2 - a);
      }
      code[i] = c;
    }
    std::sort(out.order.begin(), out.order.end(), [&](uint32_t p, uint32_t q) {
      return code[p] < code[q] || (code[p] == code[q] && p < q);
    });
    B.morton.resize(n);
    for (size_t i = 0; i < n; i++) {
      B.morton[i] = code[out.order[i]];
    }
  }

  // leaf ids: at most one leaf per primitive
  out.leafFirst.assign(n, 0);
  out.leafCount.assign(n, 0);
  B.leafFirst = &out.leafFirst;
  B.leafCount = &out.leafCount;
  out.nodeFirst.assign(n, 0);
  out.nodeEnd.assign(n, 0);
  B.nodeFirst = &out.nodeFirst;
  B.nodeEnd   = &out.nodeEnd;
  if (n <= size_t(leafSize)) {
    out.rootRef   = EBG_LEAF_BIT | 0u;
    out.rootCount = uint32_t(n);  // leaf id 0
    out.depth     = 1;
    out.numLeaves = 1;
    out.leafFirst.assign(1, 0);
    out.leafCount.assign(1, uint32_t(n));
    out.nodes.clear();
    out.nodeFirst.clear();
    out.nodeEnd.clear();
    return true;
  }
  B.nodeCount = 1;
#pragma omp parallel
#pragma omp single
  B.node(0, 0, uint32_t(n), 1);

  nodes.resize(B.nodeCount.load());
  out.nodeFirst.resize(nodes.size());
  out.nodeEnd.resize(nodes.size());
  out.nodes     = std::move(nodes);
  out.rootRef   = 0;
  out.rootCount = 0;
  out.depth     = B.maxDepth.load();
  out.numLeaves = B.leaves.load();
  out.leafFirst.resize(size_t(out.numLeaves));
  out.leafCount.resize(size_t(out.numLeaves));
  if (out.numLeaves > int64_t(EBG_MAX_LEAVES)) {
    msg = "too many leaves (at most 2^26)";
    return false;
  }
  if (3 * out.depth + 4 > EBG_STACK_DEPTH) {
    msg = "BVH too deep for the traversal stack (depth " + std::to_string(out.depth) + ")";
    return false;
  }
  return true;
}

} // namespace ebg
