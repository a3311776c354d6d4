// A C++ caller of the drop-in classes: builds a mesh from a soup, evaluates signed distances one
// point at a time through the virtual value() the reference's callers use, and in one batched call,
// then a point cloud's nearest neighbours.  Prints "ok" and exits 0 when the single-point and the
// batched values agree.
//
//   g++ -std=c++17 -I<repo> meshsdf_example.cpp -L<repo>/ebgeometry_b200 -lebgb200 -o meshsdf_example
#include <cmath>
#include <cstdio>
#include <vector>

#include "ebgeometry_b200/include/EBGeometry_B200.hpp"

using namespace EBGeometry::B200;

int main()
{
  // an octahedron of radius 1
  const std::vector<std::array<double, 3>> v = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  const std::vector<std::array<int32_t, 3>> f = {{0, 2, 4}, {2, 1, 4}, {1, 3, 4}, {3, 0, 4},
                                                 {2, 0, 5}, {1, 2, 5}, {3, 1, 5}, {0, 3, 5}};
  TriMeshSDF    sdf(v, f);
  const ImplicitBase& asImplicit = sdf; // the reference's interface: virtual value(point)

  std::vector<float> pts;
  for (int i = 0; i < 1000; i++) {
    pts.push_back(float(std::sin(0.7 * i) * 1.5));
    pts.push_back(float(std::cos(1.3 * i) * 1.5));
    pts.push_back(float(std::sin(2.1 * i + 0.3) * 1.5));
  }
  std::vector<float> d(pts.size() / 3);
  sdf.signedDistances(pts.data(), d.size(), d.data());
  // the same points in FP64 end to end: value() is FP64 too, so these agree exactly
  std::vector<double> pts64(pts.begin(), pts.end()), d64(d.size());
  sdf.signedDistances(pts64.data(), d64.size(), d64.data());
  double maxDiff = 0, maxDiff64 = 0;
  for (size_t i = 0; i < d.size(); i += 37) {
    const double one = asImplicit.value(Vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]));
    maxDiff          = std::fmax(maxDiff, std::fabs(one - double(d[i])));
    maxDiff64        = std::fmax(maxDiff64, std::fabs(one - d64[i]));
  }
  // the octahedron's exact signed distance is (|x|+|y|+|z|-1)/sqrt(3) where the closest feature
  // is a face; check the centre
  const double centre = asImplicit.value(Vec3(0, 0, 0));
  // the DCEL-face classes (MeshSDF with a tree, FlatMeshSDF without) agree with each other
  MeshSDF     msdf(v, f);
  FlatMeshSDF flat(v, f);
  double      maxDcel = 0;
  for (size_t i = 0; i < d.size(); i += 37) {
    const Vec3 q(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
    maxDcel = std::fmax(maxDcel, std::fabs(msdf.value(q) - flat.value(q)));
  }

  std::vector<std::array<float, 3>> cloud;
  for (int i = 0; i < 5000; i++) {
    cloud.push_back({float(std::fmod(i * 0.618034, 1.0)), float(std::fmod(i * 0.414214, 1.0)),
                     float(std::fmod(i * 0.732051, 1.0))});
  }
  PointCloudBVH      pc(cloud);
  PointCloudHashGrid grid(cloud);
  const auto         hit = pc.closestPoint(cloud[123]);
  // the grid answers the BVH's queries identically, self queries included
  bool       same = grid.closestPoint(cloud[123]).index == hit.index;
  const auto nnB  = pc.allNearestNeighbors(4);
  const auto nnG  = grid.allNearestNeighbors(4);
  for (size_t i = 0; i < nnB.size(); i++) {
    same = same && nnB[i].index == nnG[i].index && nnB[i].distanceSquared == nnG[i].distanceSquared;
  }
  PointCloudBVH::Hit one[4];
  same = same && pc.nearestNeighbors(77, 4, one) == 4 && one[0].index == nnB[77 * 4].index &&
         grid.nearestNeighbor(77).index == one[0].index;
  // the balanced tree (fixed runs of points) gives the same answers as the default radix tree
  PointCloudBVH balanced(cloud, 8, -1, true);
  const auto    nnBal = balanced.allNearestNeighbors(4);
  for (size_t i = 0; i < nnB.size(); i++) {
    same = same && nnB[i].index == nnBal[i].index && nnB[i].distanceSquared == nnBal[i].distanceSquared;
  }
  same = same && pc.treeInfo().radix && !balanced.treeInfo().radix && pc.treeInfo().depth <= 31;
  // a unit cube of quad faces through the polygon-face MeshSDF and FlatMeshSDF
  const std::vector<std::array<double, 3>> cv = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                                 {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  const std::vector<std::vector<int32_t>>  cf = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4},
                                                 {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
  PolygonMeshSDF     cube(cv, cf);
  PolygonFlatMeshSDF cubeFlat(cv, cf);
  const bool cubeOk = cube.value(Vec3(0.5, 0.5, 0.5)) == -0.5 && cube.value(Vec3(2.0, 0.5, 0.5)) == 1.0 &&
                      cubeFlat.value(Vec3(0.5, 0.5, -1.0)) == 1.0;
  std::printf("batch/single max diff %.3g (FP64 batch: %.3g), centre %.6f (expect %.6f), nearest of point 123: "
              "%zu (d2 %g), grid == BVH: %d, quad cube: %d\n",
              maxDiff, maxDiff64, centre, -1.0 / std::sqrt(3.0), hit.index, double(hit.distanceSquared), int(same),
              int(cubeOk));
  const bool ok = maxDiff <= 1e-6 && maxDiff64 == 0.0 && maxDcel == 0.0 && std::fabs(centre + 1.0 / std::sqrt(3.0)) < 1e-12 &&
                  hit.index == 123 && hit.distanceSquared == 0.f && same && cubeOk;
  std::printf("%s\n", ok ? "ok" : "FAILED");
  return ok ? 0 : 1;
}
