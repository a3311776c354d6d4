// Oracle harness: thin extern "C" wrappers around the UNMODIFIED reference library
// (rmrsk/EBGeometry, header-only C++17), compiled from the reference's own headers by
// oracle/Makefile into oracle/_ref/.  This file is test infrastructure: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm load the resulting
// shared library, and only as the checker or as the timed CPU baseline.
//
// The reference has no batched API (every query is one virtual call, see
// Source/EBGeometry_ImplicitFunction.hpp:51-60), so the batch loops below are the caller-side
// loops the reference's own examples and integrations write (Examples/MeshSDF/main.cpp,
// Integrations/AMReX/MeshSDF/main.cpp), wrapped in an OpenMP parallel-for.
//
// Mesh ingest goes through Soup::soupToDCEL (Source/EBGeometry_SoupImplem.hpp:149-227), exactly
// the path the reference's parsers take, so every pseudonormal is the reference's own.

#include <EBGeometry.hpp>

#include <omp.h>

#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <random>
#include <string>
#include <vector>

using namespace EBGeometry;

namespace {

using Vec3d = Vec3T<double>;
using Vec3f = Vec3T<float>;
using MeshD = DCEL::MeshT<double, short>;

// TriMeshSDF<double, short, 4, 4>: the 4-wide BVH / 4-wide SoA configuration the mesh
// workloads are specified with (Source/EBGeometry_MeshDistanceFunctions.hpp:309-489).
using TriSDF44 = TriMeshSDF<double, short, 4, 4>;
// The ISA-default K/W the reference picks for the host (Source/EBGeometry_BVH.hpp:89-111).
using TriSDFDef = TriMeshSDF<double, short, BVH::DefaultBranchingRatio<double>(), TriangleSoA::DefaultWidth<double>()>;

using Cloud = PointCloudBVH<float, std::size_t>;
using Grid  = PointCloudHashGrid<float, std::size_t>;

struct RefMesh
{
  std::shared_ptr<MeshD>                  mesh;
  std::shared_ptr<TriSDF44>               sdf44;
  std::shared_ptr<TriSDFDef>              sdfdef;
  std::shared_ptr<FlatMeshSDF<double, short>> flat;
  std::shared_ptr<MeshSDF<double, short, 4>>  dcel;
};

std::shared_ptr<MeshD>
makeMesh(const double* V, int64_t nv, const int64_t* F, int64_t nf)
{
  std::vector<Vec3d> verts(nv);
  for (int64_t i = 0; i < nv; i++) {
    verts[i] = Vec3d(V[3 * i + 0], V[3 * i + 1], V[3 * i + 2]);
  }
  std::vector<std::vector<size_t>> facets(nf);
  for (int64_t f = 0; f < nf; f++) {
    facets[f] = {size_t(F[3 * f + 0]), size_t(F[3 * f + 1]), size_t(F[3 * f + 2])};
  }
  auto mesh = std::make_shared<MeshD>();
  Soup::soupToDCEL(*mesh, verts, facets, "oracle");
  return mesh;
}

// The same from a polygon soup: face f is idx[off[f] .. off[f+1]).
std::shared_ptr<MeshD>
makePolyMesh(const double* V, int64_t nv, const int64_t* off, const int64_t* idx, int64_t nf)
{
  std::vector<Vec3d> verts(nv);
  for (int64_t i = 0; i < nv; i++) {
    verts[i] = Vec3d(V[3 * i + 0], V[3 * i + 1], V[3 * i + 2]);
  }
  std::vector<std::vector<size_t>> facets(nf);
  for (int64_t f = 0; f < nf; f++) {
    for (int64_t k = off[f]; k < off[f + 1]; k++) {
      facets[f].push_back(size_t(idx[k]));
    }
  }
  auto mesh = std::make_shared<MeshD>();
  Soup::soupToDCEL(*mesh, verts, facets, "oracle");
  return mesh;
}

BVH::Build
buildOf(int b)
{
  switch (b) {
  case 1:
    return BVH::Build::Morton;
  case 2:
    return BVH::Build::TopDown;
  default:
    return BVH::Build::SAH;
  }
}

} // namespace

extern "C" {

int
ref_omp_max_threads()
{
  return omp_get_max_threads();
}

// --- meshes -----------------------------------------------------------------------------------

// Builds the reference TriMeshSDF from a vertex/triangle soup.  a_kind: 0 = <double,short,4,4>,
// 1 = ISA-default K/W, 2 = FlatMeshSDF only (brute force, no BVH), 3 = MeshSDF<double,short,4>
// (BVH over the DCEL faces, MeshDistanceFunctionsImplem.hpp:249-295).  a_build: 0 SAH, 1 Morton,
// 2 TopDown.  a_maxLeafGroups follows TriMeshSDF(mesh, build, maxLeafGroups).
void*
ref_mesh_create(const double* V, int64_t nv, const int64_t* F, int64_t nf, int a_kind, int a_build, int a_maxLeafGroups)
{
  auto* h = new RefMesh;
  h->mesh = makeMesh(V, nv, F, nf);
  if (a_kind == 0) {
    h->sdf44 = std::make_shared<TriSDF44>(h->mesh, buildOf(a_build), size_t(a_maxLeafGroups));
  }
  else if (a_kind == 1) {
    h->sdfdef = std::make_shared<TriSDFDef>(h->mesh, buildOf(a_build), size_t(a_maxLeafGroups));
  }
  else if (a_kind == 3) {
    h->dcel = std::make_shared<MeshSDF<double, short, 4>>(h->mesh, buildOf(a_build));
  }
  h->flat = std::make_shared<FlatMeshSDF<double, short>>(h->mesh);
  return h;
}

// MeshSDF<double, short, 4> (a_build) and FlatMeshSDF<double, short> over a polygon soup; query
// them with ref_mesh_sdf (a_which 2 and 1).
void*
ref_polymesh_create(const double* V, int64_t nv, const int64_t* off, const int64_t* idx, int64_t nf, int a_build)
{
  auto* h = new RefMesh;
  h->mesh = makePolyMesh(V, nv, off, idx, nf);
  h->dcel = std::make_shared<MeshSDF<double, short, 4>>(h->mesh, buildOf(a_build));
  h->flat = std::make_shared<FlatMeshSDF<double, short>>(h->mesh);
  return h;
}

// The DCEL quantities of a mesh in face order: normal and centroid per face; per corner in
// gatherVertices() order the vertex normal, and in gatherEdges() order the half-edge normal.
int
ref_polymesh_normals(void* a_h, double* faceN, double* centroid, double* vertN, double* edgeN)
{
  auto*       h     = static_cast<RefMesh*>(a_h);
  const auto& faces = h->mesh->getFaces();
  int64_t     at    = 0;
  for (size_t f = 0; f < faces.size(); f++) {
    const auto& n = faces[f]->getNormal();
    const auto& c = faces[f]->getCentroid();
    for (int a = 0; a < 3; a++) {
      faceN[3 * f + a]    = n[a];
      centroid[3 * f + a] = c[a];
    }
    const auto verts = faces[f]->gatherVertices();
    const auto edges = faces[f]->gatherEdges();
    for (size_t k = 0; k < verts.size(); k++, at++) {
      const auto& vn = verts[k]->getNormal();
      const auto& en = edges[k]->getNormal();
      for (int a = 0; a < 3; a++) {
        vertN[3 * at + a] = vn[a];
        edgeN[3 * at + a] = en[a];
      }
    }
  }
  return 0;
}

// Parser::readIntoDCEL of a file of any faces: vertices, face offsets and vertex indices.  Call
// with null buffers first for the counts.
int
ref_read_polysoup(const char* a_file, double* V, int64_t* nv, int64_t* off, int64_t* idx, int64_t* nf, int64_t* nc)
{
  auto mesh = Parser::readIntoDCEL<double, short>(std::string(a_file));
  if (!mesh) {
    return -1;
  }
  const auto& verts = mesh->getVertices();
  const auto& faces = mesh->getFaces();
  std::map<const void*, int64_t> index;
  for (size_t i = 0; i < verts.size(); i++) {
    index[verts[i].get()] = int64_t(i);
    if (V != nullptr) {
      for (int c = 0; c < 3; c++) {
        V[3 * i + c] = verts[i]->getPosition()[c];
      }
    }
  }
  int64_t at = 0;
  if (off != nullptr) {
    off[0] = 0;
  }
  for (size_t f = 0; f < faces.size(); f++) {
    const auto fv = faces[f]->gatherVertices();
    for (const auto& v : fv) {
      if (idx != nullptr) {
        idx[at] = index[v.get()];
      }
      at++;
    }
    if (off != nullptr) {
      off[f + 1] = at;
    }
  }
  *nv = int64_t(verts.size());
  *nf = int64_t(faces.size());
  *nc = at;
  return 0;
}

void
ref_mesh_destroy(void* a_h)
{
  delete static_cast<RefMesh*>(a_h);
}

// Signed distance of n points (xyz interleaved, double) through the virtual value() entry point.
// a_which: 0 = the TriMeshSDF built above, 1 = FlatMeshSDF (DCEL brute force), 2 = the MeshSDF.
int
ref_mesh_sdf(void* a_h, const double* P, int64_t n, double* out, int a_which, int a_threads)
{
  auto*                        h = static_cast<RefMesh*>(a_h);
  const ImplicitFunction<double>* f = nullptr;
  if (a_which == 1) {
    f = h->flat.get();
  }
  else if (a_which == 2) {
    f = h->dcel.get();
  }
  else if (h->sdf44) {
    f = h->sdf44.get();
  }
  else if (h->sdfdef) {
    f = h->sdfdef.get();
  }
  if (f == nullptr) {
    return -1;
  }
  const int nt = a_threads > 0 ? a_threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nt)
  for (int64_t i = 0; i < n; i++) {
    out[i] = f->value(Vec3d(P[3 * i + 0], P[3 * i + 1], P[3 * i + 2]));
  }
  return 0;
}

// Single-point calls through the virtual value() (the per-point drop-in surface), used to time the
// reference exactly the way its integrations call it.
double
ref_mesh_value1(void* a_h, double x, double y, double z)
{
  auto* h = static_cast<RefMesh*>(a_h);
  if (h->sdf44) {
    return h->sdf44->value(Vec3d(x, y, z));
  }
  return h->sdfdef->value(Vec3d(x, y, z));
}

int
ref_mesh_face_normals(void* a_h, double* faceN, double* vertN, double* edgeN)
{
  // Pseudonormals exactly as TriMeshSDF(mesh, ...) takes them
  // (MeshDistanceFunctionsImplem.hpp:429-452): per face, the triangle's own face normal (recomputed
  // by Triangle::setVertexPositions, TriangleImplem.hpp:45-57,94-106), the three vertex normals in
  // gatherVertices() order and the three half-edge normals in gatherEdges() order.
  auto*       h     = static_cast<RefMesh*>(a_h);
  const auto& faces = h->mesh->getFaces();
  for (size_t f = 0; f < faces.size(); f++) {
    const auto verts = faces[f]->gatherVertices();
    const auto edges = faces[f]->gatherEdges();
    Triangle<double, short> tri;
    tri.setVertexPositions({verts[0]->getPosition(), verts[1]->getPosition(), verts[2]->getPosition()});
    const auto& n = tri.getNormal();
    for (int c = 0; c < 3; c++) {
      faceN[3 * f + c] = n[c];
    }
    for (int v = 0; v < 3; v++) {
      const auto& vn = verts[v]->getNormal();
      const auto& en = edges[v]->getNormal();
      for (int c = 0; c < 3; c++) {
        vertN[9 * f + 3 * v + c] = vn[c];
        edgeN[9 * f + 3 * v + c] = en[c];
      }
    }
  }
  return 0;
}

// Scalar Triangle::signedDistance (TriangleImplem.hpp:143-190) with caller-given normals: the
// known-answer cases of Tests/TestTriangle.cpp run through this.
double
ref_triangle_sd(const double* v, const double* vn, const double* en, const double* p)
{
  Triangle<double, short> tri({Vec3d(v[0], v[1], v[2]), Vec3d(v[3], v[4], v[5]), Vec3d(v[6], v[7], v[8])});
  tri.setVertexNormals({Vec3d(vn[0], vn[1], vn[2]), Vec3d(vn[3], vn[4], vn[5]), Vec3d(vn[6], vn[7], vn[8])});
  tri.setEdgeNormals({Vec3d(en[0], en[1], en[2]), Vec3d(en[3], en[4], en[5]), Vec3d(en[6], en[7], en[8])});
  return tri.signedDistance(Vec3d(p[0], p[1], p[2]));
}

// TriangleSoAT<double,4>::signedDistance over 1..4 triangles (TriangleSoAImplem.hpp:72-1195): the
// SIMD lane kernel TriMeshSDF actually runs.
double
ref_trisoa4_sd(int count, const double* v, const double* vn, const double* en, const double* p)
{
  std::vector<Triangle<double, short>> tris(count);
  for (int t = 0; t < count; t++) {
    const double* a = v + 9 * t;
    const double* b = vn + 9 * t;
    const double* c = en + 9 * t;
    tris[t].setVertexPositions({Vec3d(a[0], a[1], a[2]), Vec3d(a[3], a[4], a[5]), Vec3d(a[6], a[7], a[8])});
    tris[t].setVertexNormals({Vec3d(b[0], b[1], b[2]), Vec3d(b[3], b[4], b[5]), Vec3d(b[6], b[7], b[8])});
    tris[t].setEdgeNormals({Vec3d(c[0], c[1], c[2]), Vec3d(c[3], c[4], c[5]), Vec3d(c[6], c[7], c[8])});
  }
  TriangleSoAT<double, 4> soa;
  soa.pack<short>(tris.data(), uint32_t(count));
  return soa.signedDistance(Vec3d(p[0], p[1], p[2]));
}

// Reads a mesh file through the reference's own parser into a vertex/facet soup (used only to
// turn Tests/data fixtures into committed golden vectors).  Returns the counts; call twice, first
// with null buffers.
int
ref_read_soup(const char* a_file, double* V, int64_t* nv, int64_t* F, int64_t* nf)
{
  auto mesh = Parser::readIntoDCEL<double, short>(std::string(a_file));
  if (!mesh) {
    return -1;
  }
  const auto& verts = mesh->getVertices();
  const auto& faces = mesh->getFaces();
  if (V != nullptr) {
    for (size_t i = 0; i < verts.size(); i++) {
      for (int c = 0; c < 3; c++) {
        V[3 * i + c] = verts[i]->getPosition()[c];
      }
    }
  }
  if (F != nullptr) {
    for (size_t f = 0; f < faces.size(); f++) {
      const auto fv = faces[f]->gatherVertices();
      if (fv.size() != 3) {
        return -2;
      }
      for (int c = 0; c < 3; c++) {
        size_t idx = 0;
        for (size_t i = 0; i < verts.size(); i++) {
          if (verts[i] == fv[c]) {
            idx = i;
            break;
          }
        }
        F[3 * f + c] = int64_t(idx);
      }
    }
  }
  *nv = int64_t(verts.size());
  *nf = int64_t(faces.size());
  return 0;
}

// Random::samplePoints (RandomImplem.hpp:27-44): mt19937_64 + uniform [0,1)^3.
void
ref_sample_points(int64_t n, uint64_t seed, double* out)
{
  const auto pts = Random::samplePoints<double>(size_t(n), seed);
  for (int64_t i = 0; i < n; i++) {
    for (int c = 0; c < 3; c++) {
      out[3 * i + c] = pts[i][c];
    }
  }
}

// The reference test suite's cloud generator (Tests/TestPointCloudBVH.cpp:25-35, makeCloud<float>):
// std::mt19937(seed) with uniform_real_distribution<float>(0, 1), x then y then z per point.
void
ref_make_cloud_mt19937(int64_t n, uint32_t seed, float* out)
{
  std::mt19937                          rng(seed);
  std::uniform_real_distribution<float> dist(0.0f, 1.0f);
  for (int64_t i = 0; i < n; i++) {
    const float x = dist(rng);
    const float y = dist(rng);
    const float z = dist(rng);
    out[3 * i + 0] = x;
    out[3 * i + 1] = y;
    out[3 * i + 2] = z;
  }
}

// --- point clouds -----------------------------------------------------------------------------

void*
ref_cloud_create(const float* P, int64_t n)
{
  std::vector<Vec3f> pos(n);
  std::vector<size_t> meta(n);
  for (int64_t i = 0; i < n; i++) {
    pos[i]  = Vec3f(P[3 * i + 0], P[3 * i + 1], P[3 * i + 2]);
    meta[i] = size_t(i);
  }
  return new Cloud(pos, meta);
}

void
ref_cloud_destroy(void* h)
{
  delete static_cast<Cloud*>(h);
}

// PointCloudBVH::closestPoints (PointCloudBVHImplem.hpp:441-453), the reference's own tie order.
int
ref_cloud_knn(void* a_h, const float* Q, int64_t nq, int k, int64_t* idx, float* d2, int a_threads)
{
  auto*     c  = static_cast<Cloud*>(a_h);
  const int nt = a_threads > 0 ? a_threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
  {
    std::vector<Cloud::Hit> hits(k);
#pragma omp for schedule(dynamic, 1024)
    for (int64_t i = 0; i < nq; i++) {
      const size_t found = c->closestPoints(Vec3f(Q[3 * i], Q[3 * i + 1], Q[3 * i + 2]), size_t(k), hits.data());
      for (int j = 0; j < k; j++) {
        idx[i * k + j] = (size_t(j) < found) ? int64_t(hits[j].index) : -1;
        d2[i * k + j]  = (size_t(j) < found) ? hits[j].distanceSquared : std::numeric_limits<float>::infinity();
      }
    }
  }
  return 0;
}

// The reference's own pruneTraverse (BVHImplem.hpp:1098-1606), inherited by PointCloudBVH, driven
// with a k-best state ordered lexicographically by (d2, index): ties resolve to the lowest index.
// The leaf scan reads the reference's PointSoA squared distances (PointSoAImplem.hpp:60-230).
int
ref_cloud_knn_lex_excl(void* a_h, const float* Q, int64_t nq, int k, int64_t* idx, float* d2, int a_threads,
                       int a_excludeSelf);

int
ref_cloud_knn_lex(void* a_h, const float* Q, int64_t nq, int k, int64_t* idx, float* d2, int a_threads)
{
  return ref_cloud_knn_lex_excl(a_h, Q, nq, k, idx, d2, a_threads, 0);
}

// The same with, when a_excludeSelf is set, query i being cloud point i and excluded from its own
// result (the self queries nearestNeighbors / allNearestNeighbors, PointCloudBVHImplem.hpp:455-507).
int
ref_cloud_knn_lex_excl(void* a_h, const float* Q, int64_t nq, int k, int64_t* idx, float* d2, int a_threads,
                       int a_excludeSelf)
{
  auto*     c  = static_cast<Cloud*>(a_h);
  const int nt = a_threads > 0 ? a_threads : omp_get_max_threads();
  struct State
  {
    int                 k;
    int                 found = 0;
    std::vector<float>  d;
    std::vector<size_t> id;
  };
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nt)
  for (int64_t i = 0; i < nq; i++) {
    const Vec3f q(Q[3 * i], Q[3 * i + 1], Q[3 * i + 2]);
    State       s;
    s.k = k;
    s.d.assign(k, std::numeric_limits<float>::max());
    s.id.assign(k, std::numeric_limits<size_t>::max());
    const auto& groups   = c->getPrimitives();
    const size_t self     = a_excludeSelf ? size_t(i) : std::numeric_limits<size_t>::max();
    auto        evalLeaf = [&groups, &q, self](State& st, size_t off, size_t cnt) noexcept {
      for (size_t g = off; g < off + cnt; g++) {
        const auto dist = groups[g].getDistances2(q);
        for (size_t lane = 0; lane < dist.size(); lane++) {
          const float  dd = dist[lane];
          const size_t ii = groups[g].getMetaData(lane);
          if (ii == self) {
            continue;
          }
          // Padded lanes repeat the last real point; skip duplicates already held.
          bool dup = false;
          for (int j = 0; j < st.found; j++) {
            dup = dup || (st.id[j] == ii);
          }
          if (dup) {
            continue;
          }
          const bool better = (st.found < st.k) || dd < st.d[st.k - 1] || (dd == st.d[st.k - 1] && ii < st.id[st.k - 1]);
          if (!better) {
            continue;
          }
          int slot = (st.found < st.k) ? st.found++ : st.k - 1;
          st.d[slot]  = dd;
          st.id[slot] = ii;
          while (slot > 0 && (st.d[slot] < st.d[slot - 1] || (st.d[slot] == st.d[slot - 1] && st.id[slot] < st.id[slot - 1]))) {
            std::swap(st.d[slot], st.d[slot - 1]);
            std::swap(st.id[slot], st.id[slot - 1]);
            slot--;
          }
        }
      }
    };
    auto bound = [](const State& st) noexcept -> float {
      return (st.found < st.k) ? std::numeric_limits<float>::max() : st.d[st.k - 1];
    };
    c->pruneTraverse(q, s, evalLeaf, bound);
    for (int j = 0; j < k; j++) {
      idx[i * k + j] = (j < s.found) ? int64_t(s.id[j]) : -1;
      d2[i * k + j]  = (j < s.found) ? s.d[j] : std::numeric_limits<float>::infinity();
    }
  }
  return 0;
}

// The reference's own allNearestNeighbors(k) (PointCloudBVHImplem.hpp:488-507): k neighbours of every
// cloud point, itself excluded, in the reference's order (ties in traversal order).
int
ref_cloud_all_nn(void* a_h, int k, int64_t n, int64_t* idx, float* d2)
{
  auto*      c    = static_cast<Cloud*>(a_h);
  const auto hits = c->allNearestNeighbors(size_t(k));
  if (int64_t(hits.size()) != n * k) {
    return -1;
  }
  for (int64_t i = 0; i < n * k; i++) {
    const bool none = hits[i].index == std::numeric_limits<size_t>::max();
    idx[i]          = none ? -1 : int64_t(hits[i].index);
    d2[i]           = none ? std::numeric_limits<float>::infinity() : hits[i].distanceSquared;
  }
  return 0;
}

// --- uniform-grid point clouds ----------------------------------------------------------------

// PointCloudHashGrid(positions, meta, targetPerCell) (PointCloudHashGridImplem.hpp:27-152).
void*
ref_grid_create(const float* P, int64_t n, float a_target)
{
  std::vector<Vec3f>  pos(n);
  std::vector<size_t> meta(n);
  for (int64_t i = 0; i < n; i++) {
    pos[i]  = Vec3f(P[3 * i + 0], P[3 * i + 1], P[3 * i + 2]);
    meta[i] = size_t(i);
  }
  return new Grid(pos, meta, a_target);
}

void
ref_grid_destroy(void* h)
{
  delete static_cast<Grid*>(h);
}

// closestPoints (PointCloudHashGridImplem.hpp:321-333) for a batch of points, or, when a_ids is
// given, nearestNeighbors(ids[i], k) (:349-362); the reference's own order (ties in visiting order).
int
ref_grid_knn(void* a_h, const float* Q, const int64_t* a_ids, int64_t nq, int k, int64_t* idx, float* d2,
             int a_threads)
{
  auto*     g  = static_cast<Grid*>(a_h);
  const int nt = a_threads > 0 ? a_threads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
  {
    std::vector<Grid::Hit> hits(k);
#pragma omp for schedule(dynamic, 1024)
    for (int64_t i = 0; i < nq; i++) {
      const size_t found = a_ids ? g->nearestNeighbors(size_t(a_ids[i]), size_t(k), hits.data())
                                 : g->closestPoints(Vec3f(Q[3 * i], Q[3 * i + 1], Q[3 * i + 2]), size_t(k), hits.data());
      for (int j = 0; j < k; j++) {
        idx[i * k + j] = (size_t(j) < found) ? int64_t(hits[j].index) : -1;
        d2[i * k + j]  = (size_t(j) < found) ? hits[j].distanceSquared : std::numeric_limits<float>::infinity();
      }
    }
  }
  return 0;
}

// allNearestNeighbors(k) (PointCloudHashGridImplem.hpp:364-385).  Rows with fewer than k other
// points keep the reference's default Hit (distanceSquared = float max), reported as -1 / +inf.
int
ref_grid_all_nn(void* a_h, int k, int64_t n, int64_t* idx, float* d2)
{
  auto*      g    = static_cast<Grid*>(a_h);
  const auto hits = g->allNearestNeighbors(size_t(k));
  if (int64_t(hits.size()) != n * k) {
    return -1;
  }
  for (int64_t i = 0; i < n * k; i++) {
    const bool none = hits[i].distanceSquared == std::numeric_limits<float>::max();
    idx[i]          = none ? -1 : int64_t(hits[i].index);
    d2[i]           = none ? std::numeric_limits<float>::infinity() : hits[i].distanceSquared;
  }
  return 0;
}

// --- CSG union --------------------------------------------------------------------------------

struct RefScene
{
  std::shared_ptr<ImplicitFunction<double>>           root;
  std::vector<std::shared_ptr<ImplicitFunction<double>>> prims;
};

// Builds BVHUnion<double, ImplicitFunction<double>, AABB, 4> (CSG.hpp:99-101, CSGImplem.hpp:51-95)
// over spheres (SphereSDF, AnalyticDistanceFunctions.hpp:137-246) and meshes wrapped as
// Translate(Rotate(TriMeshSDF<double,short,4,4>)) (TransformImplem.hpp:38,47,152-225).
//   spheres:   ns x (cx, cy, cz, r)
//   meshes:    nm meshes; mesh m has vertices V + vOff[m]*3 (vCnt[m]) and facets F + fOff[m]*3
//              (fCnt[m]); pose[m] = (angle_deg, axis, tx, ty, tz); bbox[m] = world AABB (lo, hi).
void*
ref_scene_create(int64_t        ns,
                 const double*  spheres,
                 int64_t        nm,
                 const double*  V,
                 const int64_t* vOff,
                 const int64_t* vCnt,
                 const int64_t* F,
                 const int64_t* fOff,
                 const int64_t* fCnt,
                 const double*  pose,
                 const double*  bbox)
{
  using AABB = BoundingVolumes::AABBT<double>;
  auto*             s = new RefScene;
  std::vector<AABB> bvs;
  for (int64_t i = 0; i < ns; i++) {
    const double* sp = spheres + 4 * i;
    s->prims.emplace_back(std::make_shared<SphereSDF<double>>(Vec3d(sp[0], sp[1], sp[2]), sp[3]));
    bvs.emplace_back(Vec3d(sp[0] - sp[3], sp[1] - sp[3], sp[2] - sp[3]), Vec3d(sp[0] + sp[3], sp[1] + sp[3], sp[2] + sp[3]));
  }
  // the meshes are independent objects: build them on all host threads, then add them in order
  std::vector<std::shared_ptr<ImplicitFunction<double>>> built(size_t(nm < 0 ? 0 : nm));
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t m = 0; m < nm; m++) {
    auto mesh = makeMesh(V + 3 * vOff[m], vCnt[m], F + 3 * fOff[m], fCnt[m]);
    std::shared_ptr<ImplicitFunction<double>> sdf = std::make_shared<TriSDF44>(mesh, BVH::Build::SAH, 4);
    const double* ps  = pose + 5 * m;
    sdf               = Rotate<double>(sdf, ps[0], size_t(ps[1]));
    built[size_t(m)]  = Translate<double>(sdf, Vec3d(ps[2], ps[3], ps[4]));
  }
  for (int64_t m = 0; m < nm; m++) {
    s->prims.emplace_back(built[size_t(m)]);
    const double* b = bbox + 6 * m;
    bvs.emplace_back(Vec3d(b[0], b[1], b[2]), Vec3d(b[3], b[4], b[5]));
  }
  s->root = BVHUnion<double, ImplicitFunction<double>, AABB, 4>(s->prims, bvs);
  return s;
}

void
ref_scene_destroy(void* h)
{
  delete static_cast<RefScene*>(h);
}

int
ref_scene_value(void* a_h, const double* P, int64_t n, double* out, int a_brute, int a_threads)
{
  auto*     s  = static_cast<RefScene*>(a_h);
  const int nt = a_threads > 0 ? a_threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nt)
  for (int64_t i = 0; i < n; i++) {
    const Vec3d p(P[3 * i], P[3 * i + 1], P[3 * i + 2]);
    if (a_brute) {
      double v = std::numeric_limits<double>::infinity();
      for (const auto& f : s->prims) {
        v = std::min(v, f->value(p));
      }
      out[i] = v;
    }
    else {
      out[i] = s->root->value(p);
    }
  }
  return 0;
}

} // extern "C"
