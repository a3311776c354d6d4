// C++17 drop-in host classes over the C ABI (include/ebgeometry_b200.h).
//
// They mirror the reference's (rmrsk/EBGeometry) query objects and keep its single-point
// interface -- ImplicitFunction<T>::value(point) / SignedDistanceFunction<T>::signedDistance(point)
// (Source/EBGeometry_ImplicitFunction.hpp:51-60, Source/EBGeometry_SignedDistanceFunction.hpp:53-62)
// -- while adding the batched calls that reach the GPU's throughput:
//
//   EBGeometry::B200::TriMeshSDF     ~ TriMeshSDF<T,Meta,K,W>   (MeshDistanceFunctions.hpp:309-489)
//   EBGeometry::B200::PointCloudBVH  ~ PointCloudBVH<T,Meta,K,W> (PointCloudBVH.hpp:56-350)
//   EBGeometry::B200::SeedModel      the learned pruning radius (no reference counterpart)
//
// Define EBGEOMETRY_B200_WITH_REFERENCE before including this header (with the reference's
// EBGeometry.hpp on the include path) and TriMeshSDF derives from the reference's own
// EBGeometry::SignedDistanceFunction<double>, so it plugs into the reference's CSG unions,
// transforms and integrations unchanged.  Without it, a minimal ImplicitFunction base with the same
// virtual value() is provided.
//
// Errors: constructors and batched calls throw EBGeometry::B200::Error carrying the C status and
// message; value() is noexcept like the reference's and returns NaN if the device call fails.
#ifndef EBGEOMETRY_B200_HPP
#define EBGEOMETRY_B200_HPP

#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/ebgeometry_b200.h"

#ifdef EBGEOMETRY_B200_WITH_REFERENCE
#include <EBGeometry.hpp>
#endif

namespace EBGeometry {
namespace B200 {

class Error : public std::runtime_error
{
public:
  Error(ebg_status s, const std::string& what) : std::runtime_error(what), status(s) {}
  ebg_status status;
};

inline void
check(ebg_status s)
{
  if (s != EBG_OK) {
    throw Error(s, ebg_last_error());
  }
}

#ifdef EBGEOMETRY_B200_WITH_REFERENCE
using Vec3          = EBGeometry::Vec3T<double>;
using ImplicitBase  = EBGeometry::SignedDistanceFunction<double>;
inline double x(const Vec3& p) { return p[0]; }
inline double y(const Vec3& p) { return p[1]; }
inline double z(const Vec3& p) { return p[2]; }
#else
struct Vec3
{
  double v[3];
  Vec3(double a = 0, double b = 0, double c = 0) : v{a, b, c} {}
  double operator[](int i) const { return v[i]; }
};
inline double x(const Vec3& p) { return p[0]; }
inline double y(const Vec3& p) { return p[1]; }
inline double z(const Vec3& p) { return p[2]; }

// Same virtual single-point surface as the reference's ImplicitFunction / SignedDistanceFunction.
class ImplicitBase
{
public:
  virtual ~ImplicitBase() = default;
  virtual double value(const Vec3& a_point) const noexcept { return this->signedDistance(a_point); }
  double operator()(const Vec3& a_point) const noexcept { return this->value(a_point); }
  virtual double signedDistance(const Vec3& a_point) const noexcept = 0;
};
#endif

enum class Build : int32_t
{
  SAH    = EBG_BUILD_SAH,
  Morton = EBG_BUILD_MORTON
};

class SeedModel;

// Signed distance to a watertight triangle mesh; pseudonormals as the reference's DCEL computes them.
class TriMeshSDF : public ImplicitBase
{
public:
  TriMeshSDF(const std::vector<std::array<double, 3>>& a_vertices,
             const std::vector<std::array<int32_t, 3>>& a_triangles,
             Build                                      a_build    = Build::SAH,
             int                                        a_leafSize = 8,
             int                                        a_device   = -1)
  {
    ebg_build_opts o{static_cast<int32_t>(a_build), a_leafSize, a_device, 0};
    check(ebg_mesh_create(&a_vertices[0][0], int64_t(a_vertices.size()), &a_triangles[0][0],
                          int64_t(a_triangles.size()), &o, &m_mesh));
  }
  TriMeshSDF(const TriMeshSDF&) = delete;
  TriMeshSDF& operator=(const TriMeshSDF&) = delete;
  ~TriMeshSDF() override { ebg_mesh_destroy(m_mesh); }

  // ImplicitFunction<T>::value / SignedDistanceFunction<T>::signedDistance for one point
  // (one small synchronous launch per call -- batch where you can).
  double signedDistance(const Vec3& a_point) const noexcept override
  {
    double d = std::numeric_limits<double>::quiet_NaN();
    if (ebg_mesh_value(m_mesh, x(a_point), y(a_point), z(a_point), &d) != EBG_OK) {
      return std::numeric_limits<double>::quiet_NaN();
    }
    return d;
  }

  // Batched signed distances of n host points (xyz float32 interleaved), synchronous.
  void signedDistances(const float* a_pointsHost, size_t a_n, float* a_distHost, const SeedModel* a_seed = nullptr,
                       int32_t* a_closestTriangleHost = nullptr) const;

  // Batched, device buffers, asynchronous on a_stream (a cudaStream_t).
  void signedDistancesDevice(const float* a_pointsDev, size_t a_n, float* a_distDev, void* a_stream = nullptr,
                             const SeedModel* a_seed = nullptr) const;

  // Builds this mesh's per-cell entry cuts from a trained model (ebg_seed_attach); queries passing
  // that model then start from them.  Synchronous.
  void attachSeed(const SeedModel& a_seed, const ebg_attach_opts* a_opts = nullptr);

  // FP64 end to end (the reference's own precision): host points, synchronous.
  void signedDistances(const double* a_pointsHost, size_t a_n, double* a_distHost,
                       int32_t* a_closestTriangleHost = nullptr) const
  {
    ebg_query_opts o{};
    check(ebg_mesh_signed_distance_f64_host(m_mesh, a_pointsHost, int64_t(a_n), a_distHost, a_closestTriangleHost,
                                            &o, nullptr));
  }

  // FP64 end to end, device buffers, asynchronous on a_stream.
  void signedDistancesDevice(const double* a_pointsDev, size_t a_n, double* a_distDev, void* a_stream = nullptr) const
  {
    ebg_query_opts o{};
    check(ebg_mesh_signed_distance_f64(m_mesh, a_pointsDev, int64_t(a_n), a_distDev, nullptr, &o, a_stream));
  }

  // PackedBVH::refit (BVHImplem.hpp:1608-1652) for moved vertices: the same vertices' new
  // positions; the tree keeps its topology, normals and boxes are recomputed on the device.
  void refit(const std::vector<std::array<double, 3>>& a_vertices, void* a_stream = nullptr)
  {
    check(ebg_mesh_refit(m_mesh, &a_vertices[0][0], int64_t(a_vertices.size()), a_stream));
  }

  // The 8-wide copy of the tree (ebg_mesh_widen) for plain queries: taken when the autotuner picks
  // width 8, or when a query's options ask for it.  Same results; a refit drops the copy.
  void widen()
  {
    check(ebg_mesh_widen(m_mesh, nullptr, nullptr));
  }

  ebg_mesh_info info() const
  {
    ebg_mesh_info i{};
    check(ebg_mesh_get_info(m_mesh, &i));
    return i;
  }
  const ebg_mesh* handle() const noexcept { return m_mesh; }

private:
  ebg_mesh* m_mesh = nullptr;
};

// MeshSDF<double,short,K>: the same mesh, each triangle evaluated as a DCEL face (the reference's
// MeshSDF values, which differ from TriMeshSDF's in the last bits).  FP64 end to end.
class MeshSDF : public TriMeshSDF
{
public:
  using TriMeshSDF::TriMeshSDF;
  double signedDistance(const Vec3& a_point) const noexcept override
  {
    const double   p[3] = {x(a_point), y(a_point), z(a_point)};
    double         d    = std::numeric_limits<double>::quiet_NaN();
    ebg_query_opts o{};
    o.no_sort = 1;
    return ebg_mesh_signed_distance_dcel_f64_host(handle(), p, 1, &d, nullptr, &o, nullptr) == EBG_OK
             ? d
             : std::numeric_limits<double>::quiet_NaN();
  }
  // Batched, host buffers (xyz interleaved), synchronous.
  void signedDistances(const double* a_pointsHost, size_t a_n, double* a_distHost) const
  {
    ebg_query_opts o{};
    check(ebg_mesh_signed_distance_dcel_f64_host(handle(), a_pointsHost, int64_t(a_n), a_distHost, nullptr, &o,
                                                 nullptr));
  }
};

// FlatMeshSDF<double,short>: every triangle for every point (the DCEL mesh's default search);
// a ground truth for small meshes.
class FlatMeshSDF : public TriMeshSDF
{
public:
  using TriMeshSDF::TriMeshSDF;
  double signedDistance(const Vec3& a_point) const noexcept override
  {
    const double p[3] = {x(a_point), y(a_point), z(a_point)};
    double       d    = std::numeric_limits<double>::quiet_NaN();
    return ebg_mesh_signed_distance_flat_f64_host(handle(), p, 1, &d, nullptr, nullptr) == EBG_OK
             ? d
             : std::numeric_limits<double>::quiet_NaN();
  }
  void signedDistances(const double* a_pointsHost, size_t a_n, double* a_distHost) const
  {
    check(ebg_mesh_signed_distance_flat_f64_host(handle(), a_pointsHost, int64_t(a_n), a_distHost, nullptr, nullptr));
  }
};

// MeshSDF<double,short,K> over a DCEL of polygon faces (three or more vertices each; face f is
// a_faces[f], counter-clockwise = outward).  The reference's DCEL normals and face algorithm, FP64.
class PolygonMeshSDF : public ImplicitBase
{
public:
  PolygonMeshSDF(const std::vector<std::array<double, 3>>& a_vertices, const std::vector<std::vector<int32_t>>& a_faces,
                 Build a_build = Build::SAH, int a_leafSize = 4, int a_device = -1)
  {
    std::vector<int64_t> off(1, 0);
    std::vector<int32_t> idx;
    for (const auto& f : a_faces) {
      idx.insert(idx.end(), f.begin(), f.end());
      off.push_back(int64_t(idx.size()));
    }
    ebg_build_opts o{static_cast<int32_t>(a_build), a_leafSize, a_device, 0};
    check(ebg_polymesh_create(&a_vertices[0][0], int64_t(a_vertices.size()), off.data(), idx.data(),
                              int64_t(a_faces.size()), &o, &m_mesh));
  }
  // Parser::readIntoDCEL + MeshSDF: a .stl / .obj / .ply / .vtk file of any faces.
  explicit PolygonMeshSDF(const std::string& a_file, Build a_build = Build::SAH, int a_leafSize = 4, int a_device = -1)
  {
    ebg_build_opts o{static_cast<int32_t>(a_build), a_leafSize, a_device, 0};
    check(ebg_polymesh_create_from_file(a_file.c_str(), &o, &m_mesh));
  }
  PolygonMeshSDF(const PolygonMeshSDF&) = delete;
  PolygonMeshSDF& operator=(const PolygonMeshSDF&) = delete;
  ~PolygonMeshSDF() override { ebg_polymesh_destroy(m_mesh); }

  double signedDistance(const Vec3& a_point) const noexcept override
  {
    const double p[3] = {x(a_point), y(a_point), z(a_point)};
    double       d    = std::numeric_limits<double>::quiet_NaN();
    return evalHost(p, 1, &d) == EBG_OK ? d : std::numeric_limits<double>::quiet_NaN();
  }
  // Batched, host buffers (xyz interleaved), synchronous.
  void signedDistances(const double* a_pointsHost, size_t a_n, double* a_distHost) const
  {
    check(evalHost(a_pointsHost, int64_t(a_n), a_distHost));
  }
  const ebg_polymesh* handle() const noexcept { return m_mesh; }

protected:
  virtual ebg_status evalHost(const double* a_p, int64_t a_n, double* a_d) const
  {
    return ebg_polymesh_signed_distance_host(m_mesh, a_p, a_n, a_d, nullptr, nullptr);
  }

private:
  ebg_polymesh* m_mesh = nullptr;
};

// FlatMeshSDF<double,short> over polygon faces: every face for every point.
class PolygonFlatMeshSDF : public PolygonMeshSDF
{
public:
  using PolygonMeshSDF::PolygonMeshSDF;

protected:
  ebg_status evalHost(const double* a_p, int64_t a_n, double* a_d) const override
  {
    return ebg_polymesh_signed_distance_flat_host(handle(), a_p, a_n, a_d, nullptr, nullptr);
  }
};

// The learned pruning radius (trained on the device from the mesh's own exact distances).
class SeedModel
{
public:
  // Trains on a_mesh and attaches the model to it with the default cells.
  explicit SeedModel(TriMeshSDF& a_mesh, const ebg_seed_opts* a_opts = nullptr)
  {
    check(ebg_seed_train(a_mesh.handle(), a_opts, &m_seed, nullptr, nullptr));
    a_mesh.attachSeed(*this);
  }
  explicit SeedModel(const std::string& a_checkpoint, int a_device = -1)
  {
    check(ebg_seed_load(a_checkpoint.c_str(), a_device, &m_seed));
  }
  SeedModel(const SeedModel&) = delete;
  SeedModel& operator=(const SeedModel&) = delete;
  ~SeedModel() { ebg_seed_destroy(m_seed); }
  void save(const std::string& a_path) const { check(ebg_seed_save(m_seed, a_path.c_str())); }
  ebg_seed_report report() const
  {
    ebg_seed_report r{};
    check(ebg_seed_get_report(m_seed, &r));
    return r;
  }
  const ebg_seed* handle() const noexcept { return m_seed; }

private:
  ebg_seed* m_seed = nullptr;
};

inline void
TriMeshSDF::attachSeed(const SeedModel& a_seed, const ebg_attach_opts* a_opts)
{
  check(ebg_seed_attach(m_mesh, a_seed.handle(), a_opts, nullptr, nullptr));
}

inline void
TriMeshSDF::signedDistances(const float* a_pointsHost, size_t a_n, float* a_distHost, const SeedModel* a_seed,
                            int32_t* a_closestTriangleHost) const
{
  ebg_query_opts o{};
  o.seed = a_seed ? a_seed->handle() : nullptr;
  check(ebg_mesh_signed_distance_host(m_mesh, a_pointsHost, int64_t(a_n), a_distHost, a_closestTriangleHost, &o,
                                      nullptr));
}

inline void
TriMeshSDF::signedDistancesDevice(const float* a_pointsDev, size_t a_n, float* a_distDev, void* a_stream,
                                  const SeedModel* a_seed) const
{
  ebg_query_opts o{};
  o.seed = a_seed ? a_seed->handle() : nullptr;
  check(ebg_mesh_signed_distance(m_mesh, a_pointsDev, int64_t(a_n), a_distDev, nullptr, &o, a_stream));
}

// k nearest neighbours; Hit mirrors PointCloudBVH::Hit (PointCloudBVH.hpp:93-97).
class PointCloudBVH
{
public:
  struct Hit
  {
    size_t index;
    float  distanceSquared;
  };

  // Shape of the cloud's tree (ebg_cloud_tree_info).
  struct TreeInfo
  {
    int64_t nodes;
    int     depth;
    bool    radix; // false: the balanced tree
  };

  // a_balanced: fixed runs of a_leafSize Morton-ordered points grouped four at a time instead of
  // the radix tree (EBG_CLOUD_BALANCED); the answers are the same.
  explicit PointCloudBVH(const std::vector<std::array<float, 3>>& a_points, int a_leafSize = 8, int a_device = -1,
                         bool a_balanced = false)
  {
    ebg_build_opts o{0, a_leafSize, a_device, a_balanced ? EBG_CLOUD_BALANCED : 0};
    check(ebg_cloud_create(&a_points[0][0], int64_t(a_points.size()), &o, &m_cloud));
  }
  PointCloudBVH(const PointCloudBVH&) = delete;
  PointCloudBVH& operator=(const PointCloudBVH&) = delete;
  ~PointCloudBVH() { ebg_cloud_destroy(m_cloud); }

  size_t numPoints() const noexcept { return size_t(ebg_cloud_size(m_cloud)); }

  TreeInfo treeInfo() const
  {
    int64_t n = 0;
    int32_t d = 0, r = 0;
    check(ebg_cloud_tree_info(m_cloud, &n, &d, &r));
    return TreeInfo{n, int(d), r != 0};
  }

  // PointCloudBVH::closestPoint / closestPoints for one query (PointCloudBVHImplem.hpp:429-453);
  // returns how many neighbours were found (< k only if the cloud has fewer points).
  Hit closestPoint(const std::array<float, 3>& a_q) const
  {
    Hit h{0, std::numeric_limits<float>::max()};
    closestPoints(a_q, 1, &h);
    return h;
  }
  size_t closestPoints(const std::array<float, 3>& a_q, size_t a_k, Hit* a_out) const
  {
    std::vector<int32_t> idx(a_k);
    std::vector<float>   d2(a_k);
    check(ebg_cloud_knn_host(m_cloud, a_q.data(), 1, int32_t(a_k), idx.data(), d2.data(), nullptr, nullptr));
    size_t found = 0;
    for (size_t j = 0; j < a_k; j++) {
      if (idx[j] >= 0) {
        a_out[found++] = Hit{size_t(idx[j]), d2[j]};
      }
    }
    return found;
  }
  // Batched: idx/d2 are (n x k), host buffers, synchronous.
  void knn(const float* a_queriesHost, size_t a_n, int a_k, int32_t* a_idx, float* a_d2) const
  {
    check(ebg_cloud_knn_host(m_cloud, a_queriesHost, int64_t(a_n), a_k, a_idx, a_d2, nullptr, nullptr));
  }

  // Self queries, the point itself excluded (PointCloudBVHImplem.hpp:455-507).  A neighbour that
  // does not exist keeps the reference's default Hit (index 0, distanceSquared = float max).
  Hit nearestNeighbor(size_t a_point) const
  {
    Hit h{0, std::numeric_limits<float>::max()};
    nearestNeighbors(a_point, 1, &h);
    return h;
  }
  size_t nearestNeighbors(size_t a_point, size_t a_k, Hit* a_out) const
  {
    std::vector<int32_t> idx(a_k);
    std::vector<float>   d2(a_k);
    const int64_t        id = int64_t(a_point);
    check(ebg_cloud_self_knn_points_host(m_cloud, &id, 1, int32_t(a_k), idx.data(), d2.data(), nullptr));
    return collect(idx, d2, a_out);
  }
  std::vector<Hit> allNearestNeighbors(size_t a_k = 1) const
  {
    const size_t         n = numPoints();
    std::vector<int32_t> idx(n * a_k);
    std::vector<float>   d2(n * a_k);
    check(ebg_cloud_self_knn_host(m_cloud, int32_t(a_k), idx.data(), d2.data(), nullptr));
    return rows(idx, d2);
  }

  static size_t collect(const std::vector<int32_t>& a_idx, const std::vector<float>& a_d2, Hit* a_out)
  {
    size_t found = 0;
    for (size_t j = 0; j < a_idx.size(); j++) {
      if (a_idx[j] >= 0) {
        a_out[found++] = Hit{size_t(a_idx[j]), a_d2[j]};
      }
    }
    return found;
  }
  static std::vector<Hit> rows(const std::vector<int32_t>& a_idx, const std::vector<float>& a_d2)
  {
    std::vector<Hit> out(a_idx.size(), Hit{0, std::numeric_limits<float>::max()});
    for (size_t j = 0; j < a_idx.size(); j++) {
      if (a_idx[j] >= 0) {
        out[j] = Hit{size_t(a_idx[j]), a_d2[j]};
      }
    }
    return out;
  }

private:
  ebg_cloud* m_cloud = nullptr;
};

// Drop-in for PointCloudHashGrid<float, size_t> (PointCloudHashGrid.hpp:54-316): a uniform grid
// built on the device; the same queries and results as PointCloudBVH above.
class PointCloudHashGrid
{
public:
  using Hit = PointCloudBVH::Hit;

  explicit PointCloudHashGrid(const std::vector<std::array<float, 3>>& a_points, double a_targetPerCell = 1.0,
                              int a_device = -1)
  {
    check(ebg_grid_create(a_points.empty() ? nullptr : &a_points[0][0], int64_t(a_points.size()), a_targetPerCell,
                          a_device, &m_grid));
  }
  PointCloudHashGrid(const PointCloudHashGrid&) = delete;
  PointCloudHashGrid& operator=(const PointCloudHashGrid&) = delete;
  ~PointCloudHashGrid() { ebg_grid_destroy(m_grid); }

  size_t numPoints() const noexcept { return size_t(ebg_grid_size(m_grid)); }

  // closestPoint / closestPoints (PointCloudHashGridImplem.hpp:309-333)
  Hit closestPoint(const std::array<float, 3>& a_q) const
  {
    Hit h{0, std::numeric_limits<float>::max()};
    closestPoints(a_q, 1, &h);
    return h;
  }
  size_t closestPoints(const std::array<float, 3>& a_q, size_t a_k, Hit* a_out) const
  {
    std::vector<int32_t> idx(a_k);
    std::vector<float>   d2(a_k);
    check(ebg_grid_knn_host(m_grid, a_q.data(), 1, int32_t(a_k), idx.data(), d2.data(), nullptr));
    return PointCloudBVH::collect(idx, d2, a_out);
  }
  void knn(const float* a_queriesHost, size_t a_n, int a_k, int32_t* a_idx, float* a_d2) const
  {
    check(ebg_grid_knn_host(m_grid, a_queriesHost, int64_t(a_n), a_k, a_idx, a_d2, nullptr));
  }

  // nearestNeighbor(s) / allNearestNeighbors (PointCloudHashGridImplem.hpp:335-385)
  Hit nearestNeighbor(size_t a_point) const
  {
    Hit h{0, std::numeric_limits<float>::max()};
    nearestNeighbors(a_point, 1, &h);
    return h;
  }
  size_t nearestNeighbors(size_t a_point, size_t a_k, Hit* a_out) const
  {
    std::vector<int32_t> idx(a_k);
    std::vector<float>   d2(a_k);
    const int64_t        id = int64_t(a_point);
    check(ebg_grid_self_knn_points_host(m_grid, &id, 1, int32_t(a_k), idx.data(), d2.data(), nullptr));
    return PointCloudBVH::collect(idx, d2, a_out);
  }
  std::vector<Hit> allNearestNeighbors(size_t a_k = 1) const
  {
    const size_t         n = numPoints();
    std::vector<int32_t> idx(n * a_k);
    std::vector<float>   d2(n * a_k);
    check(ebg_grid_self_knn_host(m_grid, int32_t(a_k), idx.data(), d2.data(), nullptr));
    return PointCloudBVH::rows(idx, d2);
  }

private:
  ebg_grid* m_grid = nullptr;
};

} // namespace B200
} // namespace EBGeometry

#endif
