/*
 * ebgeometry_b200 -- C ABI of the B200-native mesh signed-distance / nearest-neighbour /
 * CSG-union query path (sm_100a CUDA kernels behind plain C entry points).
 *
 * The reference (rmrsk/EBGeometry) is a header-only C++ library with no C ABI: its interface is
 * the virtual ImplicitFunction<T>::value(point) (Source/EBGeometry_ImplicitFunction.hpp:51-60)
 * called once per point.  Each entry point below names the reference interface it replaces.
 * The C++ drop-in classes in ebgeometry_b200/include/EBGeometry_B200.hpp wrap this ABI behind the
 * reference's class names and value(point) signature.
 *
 * Conventions
 *  - Every function returns an ebg_status (0 = EBG_OK).  On failure, ebg_last_error() returns a
 *    thread-local message describing the last error on the calling thread.
 *  - Handles are opaque and owned by the caller (create / destroy).
 *  - "_dev" pointers are CUDA device pointers on the handle's device; "_host" entry points take
 *    host pointers and do the host<->device copies themselves.
 *  - stream is a cudaStream_t passed as void* (NULL = the legacy default stream).  Device entry
 *    points are asynchronous on that stream unless stated otherwise; status codes that depend on
 *    device-side checks are reported by the next synchronising call (ebg_check_status).
 *  - Points are float32 xyz triples (interleaved, 12 bytes per point), except in the *_f64 entry
 *    points, which take and return FP64.
 */
#ifndef EBGEOMETRY_B200_H
#define EBGEOMETRY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ebg_status
{
  EBG_OK             = 0,
  EBG_ERR_INVALID    = 1, /* bad argument (null pointer, negative size, k out of range, ...) */
  EBG_ERR_CUDA       = 2, /* a CUDA runtime call failed */
  EBG_ERR_NO_MEMORY  = 3, /* device or host allocation failed */
  EBG_ERR_TRAVERSAL  = 4, /* a kernel hit its stack-depth or iteration bound and stopped early,
                             or (device entry points) a query coordinate was not finite */
  EBG_ERR_NOT_FOUND  = 5, /* the library or a device could not be found */
  EBG_ERR_TOO_LARGE  = 6  /* input exceeds a documented limit */
} ebg_status;

/* Tree builders, mirroring BVH::Build (Source/EBGeometry_BVH.hpp:47-55). */
typedef enum ebg_build
{
  EBG_BUILD_SAH    = 0, /* binned SAH, top-down (BinnedSAHPartitioner, BVH.hpp:715-734) */
  EBG_BUILD_MORTON = 1  /* bottom-up along a Morton curve (bottomUpSortAndPartition, BVHImplem.hpp:207-312) */
} ebg_build;

/* ebg_build_opts.flags */
#define EBG_BUILD_ON_DEVICE 1 /* meshes: build the tree (Morton or SAH, the host build's tree), the
                                 pseudonormals (bit-identical to the DCEL), records and boxes on the GPU */
#define EBG_CLOUD_BALANCED 2  /* point clouds: fixed runs of leaf_size Morton-ordered points grouped four
                                 at a time (a balanced tree) instead of the radix tree; same answers */

typedef struct ebg_build_opts
{
  int32_t build;     /* ebg_build */
  int32_t leaf_size; /* max primitives per leaf (the reference's maxLeafGroups * W); 0 = default 8 */
  int32_t device;    /* CUDA device ordinal; -1 = current device */
  int32_t flags;     /* EBG_BUILD_* flags */
} ebg_build_opts;

typedef struct ebg_soup  ebg_soup;
typedef struct ebg_polymesh ebg_polymesh;
typedef struct ebg_mesh  ebg_mesh;
typedef struct ebg_cloud ebg_cloud;
typedef struct ebg_grid  ebg_grid;
typedef struct ebg_scene ebg_scene;
typedef struct ebg_seed  ebg_seed;

/* Device time of each phase of one query call, from CUDA events recorded on the call's stream. */
typedef struct ebg_phase_timings
{
  float order_ms;    /* Morton keys + radix sort of the points */
  float traverse_ms; /* FP32 packet traversal (+ seed inference when seeded) */
  float band_ms;     /* FP64 near-surface re-evaluation */
  float total_ms;
} ebg_phase_timings;

/* Per-call options of the mesh signed-distance query.  Zero-initialised = defaults. */
typedef struct ebg_query_opts
{
  double             band;            /* |d| below which the FP64 re-evaluation runs; <= 0 -> 1e-4 x the
                                         mesh's diagonal (or x its coordinates' magnitude, for a
                                         mesh far from the origin) */
  int32_t            no_sort;         /* 1: keep the caller's point order (no Morton reordering) */
  int32_t            no_fp64_band;    /* 1: skip the FP64 near-surface re-evaluation */
  const ebg_seed*    seed;            /* learned pruning-radius model (NULL = plain traversal) */
  int32_t            warps_per_block; /* 0 = tuned default */
  int32_t            occupancy;       /* traversal register budget: 0 = default (= 1); 1, 2, 3 = at
                                         most 64, 51, 42 registers per thread (8, 10, 12 blocks of
                                         128 threads per SM; warps_per_block <= 4); 4 = the
                                         compiler's own choice with 256-thread blocks */
  ebg_phase_timings* timings;         /* non-NULL: record events per phase; the call then
                                         synchronises the stream and fills this struct */
  const float*       radius_hint;     /* device, one per point (caller order): an upper bound on
                                         |d| (e.g. a coarser level's distance plus the cell
                                         diagonal) that seeds the pruning radius; <= 0 or non-finite
                                         = no hint for that point.  A hint below the true |d| only
                                         costs a second traversal of that point.  Ignored when
                                         seed is set. */
  int32_t            queue_chunk;     /* packets of 32 queries a warp takes from the device work
                                         queue at a time (mesh and union queries); 0 = tuned
                                         default (1) */
  int32_t            top_nodes;       /* plain mesh queries: each block of the traversal copies the
                                         tree's first top_nodes nodes (the device build numbers them
                                         level by level: 21 = the root and two levels) with their
                                         oriented boxes into shared memory and reads them there;
                                         at most 512; 0 = none (the default, and the faster on the
                                         level-8 workload).  Seeded queries start below the top
                                         levels and ignore it. */
  int32_t            node_width;      /* plain (and radius-hinted) FP32 traversals: 4 = the 4-wide
                                         tree, 8 = the mesh's 8-wide copy (ebg_mesh_widen; without
                                         one: EBG_ERR_INVALID); 0 = the mesh's tuned width (4 until
                                         ebg_mesh_autotune picks 8).  Same results either way;
                                         seeded queries and the FP64 pass read the 4-wide tree.
                                         With 8, top_nodes is ignored. */
} ebg_query_opts;

/* Mesh summary. */
typedef struct ebg_mesh_info
{
  int64_t num_triangles;
  int64_t num_vertices;
  int64_t num_nodes;   /* 4-wide BVH nodes */
  int64_t num_leaves;
  int32_t depth;       /* node levels on the deepest root-to-leaf path */
  int32_t leaf_size;
  double  lo[3], hi[3];
  double  diagonal;    /* |hi - lo| of the vertex bounding box */
  int64_t device_bytes;
} ebg_mesh_info;

/* Counters of one query call (for the roofline and the seed statistics).  Filled when the call
 * is made through a *_stats entry point; all counts are summed over the queries of the call. */
typedef struct ebg_query_stats
{
  int64_t nodes_visited;     /* interior nodes whose child boxes were loaded, per query */
  int64_t leaves_visited;    /* leaves whose triangles were tested, per query */
  int64_t triangles_tested;  /* point-triangle tests, per query */
  int64_t band_queries;      /* queries re-evaluated in FP64 */
  int64_t seed_fallbacks;    /* seeded queries whose predicted radius held no triangle */
  /* per 32-query packet (what the warp actually executes: the union over its lanes) */
  int64_t packets;
  int64_t packet_pops;       /* stack entries popped */
  int64_t packet_nodes;      /* interior nodes whose children were tested */
  int64_t packet_leaves;     /* leaves whose triangles were tested */
  int64_t packet_triangles;  /* point-triangle tests executed by the warp */
  int64_t boxes_tested;      /* oriented leaf/node boxes evaluated, per query */
  int64_t packet_boxes;      /* oriented boxes the warp evaluated */
  int64_t cut_packets;       /* packets that started from a cell's entry cut (ebg_seed_attach) */
  int64_t cut_entries;       /* entries those packets took from their cuts */
  int64_t packet_triangle_records; /* triangle records (48 B each) of the leaves the warps opened */
} ebg_query_stats;

const char* ebg_last_error(void);
const char* ebg_version(void);
int         ebg_device_count(void);

/* Random::samplePoints<double>(n, seed) (RandomImplem.hpp:27-44): the reference's seeded point sets
 * (n points uniform in [0,1)^3, xyz interleaved into out_host), the same points as the reference
 * compiled with GCC.  Host only. */
ebg_status ebg_sample_points(int64_t n, uint64_t seed, double* out_host);

/* ---- triangle meshes: TriMeshSDF (MeshDistanceFunctions.hpp:309-489) -------------------------
 *
 * ebg_mesh_create replaces TriMeshSDF(mesh, build, maxLeafGroups) after Soup::soupToDCEL
 * (MeshDistanceFunctionsImplem.hpp:417-460, SoupImplem.hpp:149-227): it takes a vertex/triangle
 * soup (double xyz, int32 corner indices, counter-clockwise = outward), computes the face, edge
 * and angle-weighted vertex pseudonormals the way the reference's DCEL does, builds the 4-wide BVH
 * on the host and uploads it.  Vertices are not merged (as in soupToDCEL). */
ebg_status ebg_mesh_create(const double*         vertices,
                           int64_t               num_vertices,
                           const int32_t*        triangles,
                           int64_t               num_triangles,
                           const ebg_build_opts* opts,
                           ebg_mesh**            out);

/* Same with caller-given pseudonormals instead of computed ones (the reference's
 * Triangle::setVertexNormals / setEdgeNormals, TriangleImplem.hpp:60-88): per triangle, 3 vertex
 * normals and 3 edge normals (edge i runs from corner i to corner i+1), 9 doubles each. */
ebg_status ebg_mesh_create_with_normals(const double*         vertices,
                                        int64_t               num_vertices,
                                        const int32_t*        triangles,
                                        int64_t               num_triangles,
                                        const double*         corner_vertex_normals,
                                        const double*         edge_normals,
                                        const ebg_build_opts* opts,
                                        ebg_mesh**            out);

/* Host-only: the pseudonormals ebg_mesh_create computes (no device needed).  Per triangle: the
 * face normal (3 doubles; Triangle::computeNormal, TriangleImplem.hpp:94-106), the vertex
 * pseudonormal at each corner (9; angle-weighted, DCEL_VertexImplem.hpp:190-~290) and the
 * pseudonormal of each edge (9; edge i from corner i to i+1, DCEL_EdgeImplem.hpp:128-165). */
ebg_status ebg_compute_pseudonormals(const double*  vertices,
                                     int64_t        num_vertices,
                                     const int32_t* triangles,
                                     int64_t        num_triangles,
                                     double*        face_normals,
                                     double*        corner_vertex_normals,
                                     double*        edge_normals);

ebg_status ebg_mesh_destroy(ebg_mesh* mesh);

/* Moving geometry: PackedBVH::refit (BVHImplem.hpp:1608-1652) for a TriMeshSDF whose vertices have
 * moved.  vertices: the new positions of the same num_vertices vertices (the soup's triangles stay).
 * The tree keeps its topology and leaf order; on the device the pseudonormals (the reference's
 * DCEL rules, as ebg_mesh_create computes them), every triangle record, every box and oriented box
 * are recomputed, so queries after the call answer exactly for the moved mesh -- as fast as a
 * fresh build while the motion keeps the tree's grouping sensible.  Normals given to
 * ebg_mesh_create_with_normals are replaced by computed ones.  Synchronous; work of earlier calls
 * on other streams that reads the mesh must be complete.  Non-finite coordinates or a triangle
 * that became degenerate: EBG_ERR_INVALID, mesh unchanged. */
ebg_status ebg_mesh_refit(ebg_mesh* mesh, const double* vertices_host, int64_t num_vertices, void* stream);
ebg_status ebg_mesh_refit_device(ebg_mesh* mesh, const double* vertices_dev, int64_t num_vertices, void* stream);

/* Mesh files (host only, no device needed): the reading half of Parser::readIntoDCEL
 * (ParserImplem.hpp:1752-1800) for .stl (ASCII or binary), .obj, .ply (ascii or binary, either byte
 * order) and legacy ASCII .vtk POLYDATA, with the reference's rules for which triangles a file
 * yields, then its vertex merging (Soup::compress, SoupImplem.hpp:78-145: equal positions become
 * one vertex, vertices in lexicographic order, facets in file order).  Faces keep their vertex
 * count.  ebg_soup_sizes gives the vertex and face counts; ebg_soup_copy hands a triangle soup out
 * (vertices 3 doubles, triangles 3 int32; EBG_ERR_INVALID when some face is not a triangle);
 * ebg_soup_copy_polygons hands any soup out as face offsets (num_faces + 1 int64, starting at 0)
 * into a list of ebg_soup_num_corners vertex indices. */
ebg_status ebg_soup_read(const char* path, ebg_soup** soup);
ebg_status ebg_soup_sizes(const ebg_soup* soup, int64_t* num_vertices, int64_t* num_faces);
ebg_status ebg_soup_copy(const ebg_soup* soup, double* vertices, int32_t* triangles);
ebg_status ebg_soup_num_corners(const ebg_soup* soup, int64_t* num_corners);
ebg_status ebg_soup_copy_polygons(const ebg_soup* soup, double* vertices, int64_t* face_offsets, int32_t* face_vertices);
ebg_status ebg_soup_destroy(ebg_soup* soup);
/* Parser::readIntoTriangleBVH (ParserImplem.hpp:1893-1903): read + merge + ebg_mesh_create. */
ebg_status ebg_mesh_create_from_file(const char* path, const ebg_build_opts* opts, ebg_mesh** mesh);

/* ---- meshes of polygon faces: MeshSDF / FlatMeshSDF over a DCEL of any faces -------------------
 *
 * ebg_polymesh_create replaces Soup::soupToDCEL + MeshSDF<double, Meta, 4>(mesh, build)
 * (SoupImplem.hpp:149-227, MeshDistanceFunctionsImplem.hpp:249-295) for faces of three or more
 * vertices: face f is face_vertices[face_offsets[f] .. face_offsets[f + 1]) (counter-clockwise =
 * outward; no vertex twice in one face).  The DCEL quantities are the reference's (face normal from
 * the first vertex triple that spans a plane, centroid, angle-weighted vertex and edge
 * pseudonormals); the 4-wide tree (opts: SAH or Morton, leaf_size default 4) is built on the host.
 * Queries are FP64: the DCEL face algorithm (projection into the face plane, crossing-number inside
 * test, else the nearest edge or vertex with its pseudonormal's sign).  closest_face (nullable)
 * receives the winner's soup index.  A face whose vertices span no plane, or an edge of more than
 * two faces: EBG_ERR_INVALID. */
ebg_status ebg_polymesh_create(const double*         vertices,
                               int64_t               num_vertices,
                               const int64_t*        face_offsets,
                               const int32_t*        face_vertices,
                               int64_t               num_faces,
                               const ebg_build_opts* opts,
                               ebg_polymesh**        out);
/* Host-only: the DCEL quantities ebg_polymesh_create computes (no device needed), in soup order
 * as ebg_polymesh_get_normals gives them.  Any output may be null. */
ebg_status ebg_compute_polygon_normals(const double* vertices, int64_t num_vertices, const int64_t* face_offsets,
                                       const int32_t* face_vertices, int64_t num_faces, double* face_normals,
                                       double* centroids, double* corner_vertex_normals, double* edge_normals);
/* Parser::readIntoDCEL + MeshSDF: read + merge (polygon faces kept) + ebg_polymesh_create. */
ebg_status ebg_polymesh_create_from_file(const char* path, const ebg_build_opts* opts, ebg_polymesh** out);
ebg_status ebg_polymesh_destroy(ebg_polymesh* mesh);
/* info->num_triangles holds the face count; num_corners (nullable) the number of face corners. */
ebg_status ebg_polymesh_get_info(const ebg_polymesh* mesh, ebg_mesh_info* info, int64_t* num_corners);
/* The DCEL quantities in soup order: per face normal (3) and centroid (3); per corner (face after
 * face) the vertex pseudonormal (3) and the pseudonormal of the edge to the next corner (3).  Any
 * output may be null. */
ebg_status ebg_polymesh_get_normals(const ebg_polymesh* mesh, double* face_normals, double* centroids,
                                    double* corner_vertex_normals, double* edge_normals);
/* MeshSDF::signedDistance (MeshDistanceFunctionsImplem.hpp:269-295) for n FP64 points; device
 * arrays, asynchronous on stream. */
ebg_status ebg_polymesh_signed_distance(const ebg_polymesh* mesh, const double* points_dev, int64_t n,
                                        double* out_dev, int32_t* closest_face_dev, void* stream);
ebg_status ebg_polymesh_signed_distance_host(const ebg_polymesh* mesh, const double* points_host, int64_t n,
                                             double* out_host, int32_t* closest_face_host, void* stream);
/* FlatMeshSDF::signedDistance (MeshDistanceFunctionsImplem.hpp:219-229, DCEL_MeshImplem.hpp:574-595):
 * every face for every point; the first face in soup order with the smallest unsigned distance. */
ebg_status ebg_polymesh_signed_distance_flat(const ebg_polymesh* mesh, const double* points_dev, int64_t n,
                                             double* out_dev, int32_t* closest_face_dev, void* stream);
ebg_status ebg_polymesh_signed_distance_flat_host(const ebg_polymesh* mesh, const double* points_host, int64_t n,
                                                  double* out_host, int32_t* closest_face_host, void* stream);
/* Synchronises stream; reports a non-finite query point (EBG_ERR_INVALID) or a traversal bound. */
ebg_status ebg_polymesh_check_status(const ebg_polymesh* mesh, void* stream);
ebg_status ebg_mesh_get_info(const ebg_mesh* mesh, ebg_mesh_info* info);

/* Pseudonormals the handle computed (per triangle: face normal 3, vertex normals 9, edge normals 9
 * doubles), for checking against the reference's DCEL. */
ebg_status ebg_mesh_get_normals(const ebg_mesh* mesh, double* face_normals, double* corner_vertex_normals,
                                double* edge_normals);

/* Batched TriMeshSDF::signedDistance (MeshDistanceFunctionsImplem.hpp:480-509) over n points:
 * dist_dev[i] = signed distance of points_dev[3i..3i+2]; closest_tri_dev (nullable) receives the
 * index of the winning triangle in the input soup (getClosestTriangle's metadata,
 * MeshDistanceFunctionsImplem.hpp:511-549).  Asynchronous on stream. */
ebg_status ebg_mesh_signed_distance(const ebg_mesh*       mesh,
                                    const float*          points_dev,
                                    int64_t               n,
                                    float*                dist_dev,
                                    int32_t*              closest_tri_dev,
                                    const ebg_query_opts* opts,
                                    void*                 stream);

/* The same with host buffers: copies points in, evaluates, copies distances out, synchronises. */
ebg_status ebg_mesh_signed_distance_host(const ebg_mesh*       mesh,
                                         const float*          points_host,
                                         int64_t               n,
                                         float*                dist_host,
                                         int32_t*              closest_tri_host,
                                         const ebg_query_opts* opts,
                                         void*                 stream);

/* Batched TriMeshSDF<double>::signedDistance in FP64 end to end (the reference's own precision,
 * MeshDistanceFunctionsImplem.hpp:480-509 with TriangleSoAImplem.hpp:1029-1180): FP64 points in,
 * FP64 distances out.  The FP32 traversal finds each query's candidate bound; every query is then
 * re-evaluated with the reference's FP64 triangle test over all triangles within that bound of the
 * caller's FP64 point, so the result is the reference's value (opts->band and no_fp64_band are
 * ignored).  Asynchronous on stream. */
ebg_status ebg_mesh_signed_distance_f64(const ebg_mesh*       mesh,
                                        const double*         points_dev,
                                        int64_t               n,
                                        double*               dist_dev,
                                        int32_t*              closest_tri_dev,
                                        const ebg_query_opts* opts,
                                        void*                 stream);

/* The same with host buffers (copies in, evaluates, copies out, synchronises). */
ebg_status ebg_mesh_signed_distance_f64_host(const ebg_mesh*       mesh,
                                             const double*         points_host,
                                             int64_t               n,
                                             double*               dist_host,
                                             int32_t*              closest_tri_host,
                                             const ebg_query_opts* opts,
                                             void*                 stream);

/* MeshSDF<double,short,K>::signedDistance (MeshDistanceFunctionsImplem.hpp:269-295): the same FP64
 * query with each triangle evaluated as a DCEL face (FaceT::signedDistance,
 * DCEL_FaceImplem.hpp:388-423: crossing-number inside test in the face's 2D projection, then
 * n . (p - centroid) inside, else the nearest edge or vertex signed by its pseudonormal), which
 * differs from the Triangle test of TriMeshSDF in the last bits.  Keeps the value of smallest |d|
 * (strict <), as MeshSDF's leaf loop does.  Asynchronous on stream. */
ebg_status ebg_mesh_signed_distance_dcel_f64(const ebg_mesh*       mesh,
                                             const double*         points_dev,
                                             int64_t               n,
                                             double*               dist_dev,
                                             int32_t*              closest_tri_dev,
                                             const ebg_query_opts* opts,
                                             void*                 stream);
ebg_status ebg_mesh_signed_distance_dcel_f64_host(const ebg_mesh*       mesh,
                                                  const double*         points_host,
                                                  int64_t               n,
                                                  double*               dist_host,
                                                  int32_t*              closest_tri_host,
                                                  const ebg_query_opts* opts,
                                                  void*                 stream);

/* FlatMeshSDF<double,short>::signedDistance (MeshDistanceFunctionsImplem.hpp:218-228 through
 * MeshT::DirectSignedDistance2, DCEL_MeshImplem.hpp:574-595): no tree; every triangle is tested
 * for every point, the first triangle in soup order with the smallest unsigned distance wins and
 * its DCEL-face signed distance is the value.  O(points x triangles): a ground truth for small
 * meshes.  closest_tri (nullable) receives the winner's soup index.  Asynchronous on stream. */
ebg_status ebg_mesh_signed_distance_flat_f64(const ebg_mesh* mesh,
                                             const double*   points_dev,
                                             int64_t         n,
                                             double*         dist_dev,
                                             int32_t*        closest_tri_dev,
                                             void*           stream);
ebg_status ebg_mesh_signed_distance_flat_f64_host(const ebg_mesh* mesh,
                                                  const double*   points_host,
                                                  int64_t         n,
                                                  double*         dist_host,
                                                  int32_t*        closest_tri_host,
                                                  void*           stream);

/* The same batched query WITHOUT ANY DEVICE ALLOCATION (no counterpart in the reference).  For
 * callers that cannot let a library allocate: AMR codes such as AMReX reserve most of the GPU's memory
 * for their own arena at start-up, so a library's cudaMalloc or stream-ordered allocation can fail
 * inside their embedded-boundary loop, and other codes forbid allocations there for latency.  The
 * per-call workspace comes from a fixed 24 MiB array compiled into the library instead of the memory
 * pool.  Limits: n <= 524,288 points per call (larger n returns EBG_ERR_TOO_LARGE); opts->timings and
 * opts->node_width are ignored (the 4-wide tree is traversed).  The first call on a device (n = 0 is enough) resolves the array's address there, and
 * with lazy module loading (the CUDA default) that is also when the 24 MiB are taken on that device,
 * where they stay until the process exits: make that first call before reserving a memory arena and
 * before capturing a CUDA graph.  cudaDeviceReset on the device invalidates the array; do not call
 * this entry point on a device after resetting it.  All calls on a device share the array, so calls
 * whose work overlaps on the GPU (different streams) race and must be serialised.  Results are those
 * of ebg_mesh_signed_distance (the same launch shape, seed and band handling). */
ebg_status ebg_mesh_signed_distance_noalloc(const ebg_mesh*       mesh,
                                            const float*          points_dev,
                                            int64_t               n,
                                            float*                dist_dev,
                                            int32_t*              closest_tri_dev,
                                            const ebg_query_opts* opts,
                                            void*                 stream);

/* Synchronous variant that also returns traversal counters (slower: counts with atomics). */
ebg_status ebg_mesh_signed_distance_stats(const ebg_mesh*       mesh,
                                          const float*          points_dev,
                                          int64_t               n,
                                          float*                dist_dev,
                                          const ebg_query_opts* opts,
                                          ebg_query_stats*      stats,
                                          void*                 stream);

/* Autotuner (no reference counterpart; the reference fixes its branching ratio and SoA width at
 * compile time, DefaultBranchingRatio, BVH.hpp:89-111, and TriangleSoA::DefaultWidth,
 * TriangleSoA.hpp:55-77): times the traversal's launch shapes -- register budget
 * (ebg_query_opts.occupancy 1..4) x warps per block (2, 4, 8), then the work-queue chunk (1, 2, 4
 * packets per grab) at the fastest shape, then (plain traversal of a mesh with an 8-wide copy,
 * ebg_mesh_widen) the node width 8 against 4 at that shape, with the launch shape re-tuned for
 * width 8 -- on the caller's sample points (device), keeps the fastest as this mesh's default for
 * queries that leave those options at 0, and returns it (best_occupancy / best_warps_per_block /
 * best_queue_chunk / best_node_width, any of them nullable; best_ms = the sample's traversal time).
 * `seed` (nullable) times the seeded traversal of a model attached to the mesh (node width 4).
 * Synchronous. */
ebg_status ebg_mesh_autotune(ebg_mesh*       mesh,
                             const float*    sample_points_dev,
                             int64_t         n,
                             const ebg_seed* seed,
                             int32_t*        best_occupancy,
                             int32_t*        best_warps_per_block,
                             int32_t*        best_queue_chunk,
                             int32_t*        best_node_width,
                             float*          best_ms,
                             void*           stream);

/* The 8-wide copy of the mesh's tree for plain FP32 queries (no reference counterpart: the
 * reference's branching ratio is the compile-time K of BVH.hpp:89-111).  Made on the host from the
 * 4-wide tree: each 8-wide node takes one 4-wide node's children and replaces the largest-area
 * interior child by that child's own children while they fit in eight slots.  Leaves and child
 * boxes are the 4-wide tree's, so queries through it give the same results bit for bit, with fewer
 * levels and more boxes tested per node.  Costs 256 B + 64 B per 8-wide node on the device.
 * num_nodes8 / depth8 (nullable) receive its node count and its levels on the deepest path (leaf
 * level included).  A mesh whose root is a leaf needs no copy (EBG_OK, 0 nodes).  A tree too deep
 * for the 8-wide traversal's stack: EBG_ERR_TOO_LARGE.  ebg_mesh_refit drops the copy (and a
 * tuned width of 8).  Synchronous. */
ebg_status ebg_mesh_widen(ebg_mesh* mesh, int64_t* num_nodes8, int32_t* depth8);

/* ImplicitFunction<T>::value(point) for one point (ImplicitFunction.hpp:51-52): the drop-in
 * single-point call, in FP64 (ebg_mesh_signed_distance_f64_host).  Synchronous; each call is a few
 * tiny launches, so batch where you can. */
ebg_status ebg_mesh_value(const ebg_mesh* mesh, double x, double y, double z, double* value);

/* Blocks until the stream's work for this mesh is done and reports any device-side error
 * (EBG_ERR_TRAVERSAL) recorded by earlier asynchronous calls. */
ebg_status ebg_check_status(const ebg_mesh* mesh, void* stream);

/* ---- point clouds: PointCloudBVH (PointCloudBVH.hpp:56-350) --------------------------------
 *
 * ebg_cloud_create replaces PointCloudBVH(positions, meta) (PointCloudBVHImplem.hpp:27-57): the
 * tree is built on the device (the points in Morton order, a 4-wide tree whose nodes divide their
 * range where the Morton curve jumps, leaves of at most opts->leaf_size points, default 8).  The
 * cloud index of a point is its position in the input array. */
ebg_status ebg_cloud_create(const float* points_host, int64_t n, const ebg_build_opts* opts, ebg_cloud** out);
/* The same from a device array (no host copy); the build runs on stream and is complete on return. */
ebg_status ebg_cloud_create_device(const float* points_dev, int64_t n, const ebg_build_opts* opts, ebg_cloud** out,
                                   void* stream);
ebg_status ebg_cloud_destroy(ebg_cloud* cloud);
int64_t    ebg_cloud_size(const ebg_cloud* cloud);
/* The tree's shape: 4-wide nodes, node levels (0 when the root is a single leaf) and whether it is
 * the radix tree (1) or the balanced tree of fixed runs of leaf_size points (0), which the build
 * falls back to when the radix tree would be deeper than the traversal stack allows. */
ebg_status ebg_cloud_tree_info(const ebg_cloud* cloud, int64_t* num_nodes, int32_t* depth, int32_t* radix);

/* Batched PointCloudBVH::closestPoints (PointCloudBVHImplem.hpp:441-453) / closestPoint (k = 1):
 * for each query the k nearest points in increasing (squared distance, index) order -- equal
 * distances resolve to the LOWEST index -- as int32 indices idx_dev[q*k + j] and float squared
 * distances d2_dev[q*k + j] computed as the reference does ((dx*dx + dy*dy) + dz*dz, dx = q - p,
 * float, no fused multiply-add).  Fewer than k points: the missing entries are index -1 and +inf.
 * 1 <= k <= 32.  opts: only no_sort is used.  Asynchronous on stream. */
ebg_status ebg_cloud_knn(const ebg_cloud*      cloud,
                         const float*          queries_dev,
                         int64_t               num_queries,
                         int32_t               k,
                         int32_t*              idx_dev,
                         float*                d2_dev,
                         const ebg_query_opts* opts,
                         void*                 stream);
/* The same with host buffers (copies in and out, synchronous). */
ebg_status ebg_cloud_knn_host(const ebg_cloud*      cloud,
                              const float*          queries_host,
                              int64_t               num_queries,
                              int32_t               k,
                              int32_t*              idx_host,
                              float*                d2_host,
                              const ebg_query_opts* opts,
                              void*                 stream);
/* Self queries, PointCloudBVH::allNearestNeighbors(k) (PointCloudBVHImplem.hpp:488-507): the k
 * nearest OTHER points of every cloud point (the point itself excluded; another point at the same
 * position is a neighbour at d2 = 0), ordered by (d2, index) -- ties to the lowest index -- into
 * idx_dev / d2_dev (n x k, row = the point's cloud index; missing neighbours: -1 / +inf).  The
 * queries run in the cloud's own leaf order, so a packet starts next to its own leaves.
 * Asynchronous on stream. */
ebg_status ebg_cloud_self_knn(const ebg_cloud* cloud, int32_t k, int32_t* idx_dev, float* d2_dev, void* stream);
/* The same for a list of m cloud indices (nearestNeighbors(point, k), PointCloudBVHImplem.hpp:
 * 470-486); row i answers point_ids_dev[i].  Indices out of range are reported by the next
 * ebg_cloud_check_status as EBG_ERR_INVALID. */
ebg_status ebg_cloud_self_knn_points(const ebg_cloud* cloud,
                                     const int64_t*   point_ids_dev,
                                     int64_t          m,
                                     int32_t          k,
                                     int32_t*         idx_dev,
                                     float*           d2_dev,
                                     void*            stream);
/* ebg_cloud_self_knn_points with host arrays, synchronous (reports device-side errors). */
ebg_status ebg_cloud_self_knn_points_host(const ebg_cloud* cloud,
                                          const int64_t*   point_ids_host,
                                          int64_t          m,
                                          int32_t          k,
                                          int32_t*         idx_host,
                                          float*           d2_host,
                                          void*            stream);
/* ebg_cloud_self_knn with host output arrays (n x k), synchronous. */
ebg_status ebg_cloud_self_knn_host(const ebg_cloud* cloud, int32_t k, int32_t* idx_host, float* d2_host, void* stream);
/* Synchronises stream and reports a device-side error of earlier k-NN calls. */
ebg_status ebg_cloud_check_status(const ebg_cloud* cloud, void* stream);

/* ---- point clouds: PointCloudHashGrid (PointCloudHashGrid.hpp:54-316) -----------------------
 *
 * ebg_grid_create replaces PointCloudHashGrid(positions, meta, targetPerCell)
 * (PointCloudHashGridImplem.hpp:27-152): a dense uniform grid over the cloud's box, cell size
 * cbrt(box volume / n * target_per_cell) (target_per_cell <= 0 means 1), coarsened until the grid
 * has at most 64 + 8 n cells; the points are sorted into their cells on the device.  n = 0 gives an
 * empty grid whose queries find nothing.  Non-finite coordinates are rejected (EBG_ERR_INVALID).
 * The queries are those of PointCloudBVH with the same results: the k nearest points by the same
 * float squared distance, in (d2, index) order -- ties to the lowest index; missing entries -1 and
 * +inf; 1 <= k <= 32.  The reference's grid query orders equal distances by visiting order instead;
 * its distances are the same. */
ebg_status ebg_grid_create(const float* points_host, int64_t n, double target_per_cell, int32_t device, ebg_grid** out);
ebg_status ebg_grid_destroy(ebg_grid* grid);
int64_t    ebg_grid_size(const ebg_grid* grid);
/* Cells per axis and the cell size. */
ebg_status ebg_grid_info(const ebg_grid* grid, int32_t* cells_xyz, double* cell_size);
/* closestPoints / closestPoint (PointCloudHashGridImplem.hpp:309-333) for a batch of points;
 * asynchronous on stream. */
ebg_status ebg_grid_knn(const ebg_grid* grid, const float* queries_dev, int64_t num_queries, int32_t k, int32_t* idx_dev,
                        float* d2_dev, void* stream);
ebg_status ebg_grid_knn_host(const ebg_grid* grid, const float* queries_host, int64_t num_queries, int32_t k,
                             int32_t* idx_host, float* d2_host, void* stream);
/* allNearestNeighbors(k) (PointCloudHashGridImplem.hpp:364-385): every point's k nearest OTHER
 * points, row = cloud index; the queries run in cell order. */
ebg_status ebg_grid_self_knn(const ebg_grid* grid, int32_t k, int32_t* idx_dev, float* d2_dev, void* stream);
ebg_status ebg_grid_self_knn_host(const ebg_grid* grid, int32_t k, int32_t* idx_host, float* d2_host, void* stream);
/* nearestNeighbors(point, k) / nearestNeighbor(point) (PointCloudHashGridImplem.hpp:335-362) for
 * m cloud indices; row i answers point_ids[i].  Indices out of range give a row of -1 / +inf and
 * are reported by the next status check as EBG_ERR_INVALID. */
ebg_status ebg_grid_self_knn_points(const ebg_grid* grid, const int64_t* point_ids_dev, int64_t m, int32_t k,
                                    int32_t* idx_dev, float* d2_dev, void* stream);
ebg_status ebg_grid_self_knn_points_host(const ebg_grid* grid, const int64_t* point_ids_host, int64_t m, int32_t k,
                                         int32_t* idx_host, float* d2_host, void* stream);
/* Synchronises stream and reports a device-side error of earlier grid queries. */
ebg_status ebg_grid_check_status(const ebg_grid* grid, void* stream);

/* ---- CSG union: BVHUnionIF (CSG.hpp:401-468) ------------------------------------------------
 *
 * ebg_scene_create replaces BVHUnion<T, ImplicitFunction<T>, AABB, K>(prims, bvs) (CSG.hpp:99-101,
 * CSGImplem.hpp:51-95) over SphereSDF objects (AnalyticDistanceFunctions.hpp:137-246; spheres[4i..]
 * = centre xyz, radius) and instances Translate(Rotate(mesh, angle, axis), t) of existing mesh
 * handles (TransformImplem.hpp:38-47,152-225; poses[5i..] = angle in degrees, axis 0/1/2, tx, ty,
 * tz).  The object hierarchy is a 4-wide SAH BVH with opts->leaf_size objects per leaf (default 3,
 * the reference's "fewer than K").  Mesh handles must outlive the scene and share its device. */
ebg_status ebg_scene_create(int64_t                num_spheres,
                            const double*          spheres,
                            int64_t                num_meshes,
                            const ebg_mesh* const* meshes,
                            const double*          poses,
                            const ebg_build_opts*  opts,
                            ebg_scene**            out);
ebg_status ebg_scene_destroy(ebg_scene* scene);
int64_t    ebg_scene_num_objects(const ebg_scene* scene);
/* BVHUnionIF::value (CSGImplem.hpp:465-501) at n device points: min over the objects, the object
 * BVH pruned with max(0, best)^2.  FP32 with an FP64 near-surface pass: a point whose FP32 value
 * lies within opts->band (default 1e-4 x the scene box's diagonal, or x the magnitude of the
 * scene's or its meshes' coordinates when larger) of zero is evaluated again in
 * double as the reference does (the sphere distance, RotateIF's per-axis point map with cos / sin in
 * double, the mesh's FP64 triangle test), over the objects that can hold the minimum.  One
 * persistent launch for the whole array.  Asynchronous on stream; opts->no_sort, no_fp64_band and
 * band are used. */
ebg_status ebg_scene_value(const ebg_scene*      scene,
                           const float*          points_dev,
                           int64_t               n,
                           float*                out_dev,
                           const ebg_query_opts* opts,
                           void*                 stream);
/* One batch of ebg_scene_eval_batches: n device points (xyz float32) and n device results. */
typedef struct ebg_batch
{
  const float* points_dev;
  int64_t      n;
  float*       out_dev;
} ebg_batch;
/* Many query batches of uneven length in one call (the reference has no batch API; its callers loop
 * over value(point)): batches_dev is a DEVICE array of num_batches descriptors whose n add up to
 * total_points (a mismatch or a negative n computes nothing and is reported by the next status
 * check as EBG_ERR_TRAVERSAL).  The points of all batches are ordered together along one Morton
 * curve and served by one persistent launch with a device work queue, then the FP64 near-surface
 * pass, as ebg_scene_value.  Only stream-ordered work, so the call
 * can be captured in a CUDA graph. */
ebg_status ebg_scene_eval_batches(const ebg_scene*      scene,
                                  const ebg_batch*      batches_dev,
                                  int32_t               num_batches,
                                  int64_t               total_points,
                                  const ebg_query_opts* opts,
                                  void*                 stream);
ebg_status ebg_scene_value_host(const ebg_scene*      scene,
                                const float*          points_host,
                                int64_t               n,
                                float*                out_host,
                                const ebg_query_opts* opts,
                                void*                 stream);
ebg_status ebg_scene_check_status(const ebg_scene* scene, void* stream);
/* Autotuner of the union query (no reference counterpart): times the work-queue chunk (1, 2, 4, 8
 * packets per grab) on the caller's sample points (device) and keeps the fastest as this scene's
 * default for calls that leave ebg_query_opts.queue_chunk at 0.  best_queue_chunk and best_ms (the
 * sample's call time) nullable.  Synchronous. */
ebg_status ebg_scene_autotune(ebg_scene*   scene,
                              const float* sample_points_dev,
                              int64_t      n,
                              int32_t*     best_queue_chunk,
                              float*       best_ms,
                              void*        stream);

/* ---- learned pruning radius (no counterpart in the reference) --------------------------------
 *
 * A multiresolution hash-grid encoding (16 levels x 2 BF16 features, 2^log2_table entries per
 * level) feeding a 3-hidden-layer, 64-wide ReLU MLP (BF16 weights, FP32 accumulation on the tensor
 * cores) that predicts the signed distance; its calibrated radius (1 + alpha) |prediction| + beta
 * bounds |d|.  Attached to a mesh (ebg_seed_attach below), it bounds |d| over the cells of a grid,
 * and each cell keeps the part of the mesh's tree within that bound; passed as ebg_query_opts.seed,
 * it starts the traversal of every packet of 32 sorted queries there.  Distances stay exact: the
 * radius only prunes, and a query whose radius holds no triangle is traversed again without it. */
typedef struct ebg_seed_opts
{
  int64_t  num_samples;     /* exact training samples: half uniform in the domain, half within
                               +-surface_band of the surface; 0 = 2^25 */
  int32_t  steps;           /* Adam steps; 0 = 2000 */
  int32_t  batch;           /* samples per step; 0 = 2^18 */
  int32_t  log2_table;      /* hash-table entries per level = 2^log2_table; 0 = 19 */
  int32_t  base_resolution; /* grid resolution of the coarsest level; 0 = 16 */
  int32_t  max_resolution;  /* of the finest level; 0 = 1024 */
  float    learning_rate;   /* initial Adam step (decays 10x over the run); 0 = 1e-2 */
  float    surface_band;    /* half-width of the near-surface sample band; 0 = 0.02 */
  float    coverage;        /* fraction of validation points whose radius must hold |d|; 0 = 0.995 */
  uint64_t rng_seed;
  double   lo[3], hi[3];    /* sample / encoding domain; lo == hi -> the mesh box grown 1.25x */
} ebg_seed_opts;

typedef struct ebg_seed_report
{
  float   train_seconds;
  float   final_loss;         /* weighted MSE of the last step */
  float   alpha, beta;        /* radius = (1 + alpha) |prediction| + beta */
  float   coverage;           /* validation fraction with radius >= |d| */
  float   mean_abs_err;       /* |prediction - d| over the validation samples */
  float   far_tau;            /* far-field threshold (0.05) */
  float   max_abs_err_far;    /* max |prediction - d| where |d| > far_tau (the optional surrogate's error) */
  int64_t validation_samples;
  int64_t train_samples;
} ebg_seed_report;

/* Untrained model (random initial parameters) over a domain; used by ebg_seed_train and by
 * gradient checks. */
ebg_status ebg_seed_create(const ebg_seed_opts* opts, ebg_seed** out);
/* Generates num_samples exact signed distances with the mesh path, trains the model on the device
 * with the library's own forward/backward/Adam kernels, calibrates alpha and beta on fresh
 * validation samples and returns the model.  report (nullable) receives the training summary. */
ebg_status ebg_seed_train(const ebg_mesh* mesh, const ebg_seed_opts* opts, ebg_seed** out, ebg_seed_report* report,
                          void* stream);
ebg_status ebg_seed_destroy(ebg_seed* seed);
ebg_status ebg_seed_get_report(const ebg_seed* seed, ebg_seed_report* report);
/* Raw predicted signed distance at n device points (the optional far-field surrogate). */
ebg_status ebg_seed_predict(const ebg_seed* seed, const float* points_dev, int64_t n, float* out_dev, void* stream);
/* Checkpoint of the model (configuration, FP32 tables and MLP parameters, calibration). */
ebg_status ebg_seed_save(const ebg_seed* seed, const char* path);
ebg_status ebg_seed_load(const char* path, int32_t device, ebg_seed** out);
/* Parameter access: table = 16 * 2^log2_table * 2 floats (level-major, [level][entry][feature]),
 * params = the 10,497 MLP floats (W1[64][32], b1, W2[64][64], b2, W3[64][64], b3, w4[64], b4).
 * Either pointer may be null. */
ebg_status ebg_seed_get_params(const ebg_seed* seed, float* table, float* params);
ebg_status ebg_seed_set_params(ebg_seed* seed, const float* table, const float* params);
/* Loss and gradients of one training batch (device samples) with the current parameters, without
 * updating them: loss = sum_i w_i (y_i - d_i)^2 / n, w_i = 1 / (|d_i| + eps)^2.  Outputs are host
 * arrays (grad_table nullable). */
ebg_status ebg_seed_gradients(ebg_seed* seed, const float* points_dev, const float* target_dev, int32_t n, float eps,
                              float* loss, float* grad_table, float* grad_params);

/* Attaching a model to a mesh (no counterpart in the reference; it replaces the root-down start of
 * PackedBVH::pruneTraverse, BVHImplem.hpp:1098-1606, for the packets it covers).
 *
 * A regular grid of cells_per_axis^3 cells covers the model's domain.  For every cell the model's
 * calibrated radius at the cell centre, plus the half-diagonal of the cell grown by margin_cells
 * cells on every side, bounds |d| over that grown cell (R_C); the mesh keeps a CUT of its BVH per
 * cell: at most max_entries subtrees, refined nearest-first from the root, that hold every triangle
 * within R_C of the grown cell, and the cell's ANCHOR, the triangle nearest to the cell centre
 * (found by the mesh path itself).  A query call that passes this model (ebg_query_opts.seed)
 * starts every packet of 32 sorted queries whose box fits a grown cell from that cell's cut, each
 * lane's bound being the smaller of R_C and its distance to the anchor; a query that finds nothing
 * within R_C is traversed again from the root.  Distances are exact whatever the model predicts.
 * Queries passing a model that is not attached to the mesh are rejected (EBG_ERR_INVALID). */
typedef struct ebg_attach_opts
{
  int32_t cells_per_axis; /* <= 512; 0 = 2 cbrt(tree leaves) rounded up to a multiple of 8,
                             within 16..128 (128 for 1.3 M triangles) */
  int32_t max_entries;    /* subtrees per cell, <= 112; 0 = 112 (lowered for deep trees).  Memory:
                             cells * max_entries * 32 B (7.5 GB at 128^3 cells and 112 entries) */
  float   margin_cells;   /* growth of each cell on every side, in cells; <= 0 -> 1.5 */
  int32_t radius_mode;    /* 0 = the model's radius (default); 1 = no radius (cuts ordered by
                             distance only, nothing dropped); 2 = the exact distance at the cell
                             centres from the mesh path (for comparison with the model) */
  int32_t no_anchors;     /* 1: no anchor triangles (the triangle nearest to each cell centre, found
                             by the mesh path, whose distance starts every lane's bound) */
} ebg_attach_opts;

typedef struct ebg_attach_report
{
  int32_t cells_per_axis;
  int32_t max_entries;
  int64_t cells;
  int64_t cut_entries;     /* sum over cells */
  int64_t empty_cells;     /* cells whose cut is empty (every triangle farther than R_C) */
  int64_t device_bytes;    /* entries + counts + radii */
  float   build_ms;        /* device time of the cell radii and cuts */
  float   mean_radius;     /* mean finite R_C */
} ebg_attach_report;

/* Builds the mesh's per-cell cuts from `seed` (replacing any earlier attachment; the model may be
 * destroyed afterwards, the cuts do not refer to it).  ebg_mesh_refit drops the cuts.  Synchronous.
 * report nullable. */
ebg_status ebg_seed_attach(ebg_mesh* mesh, const ebg_seed* seed, const ebg_attach_opts* opts, ebg_attach_report* report,
                           void* stream);
/* Frees the mesh's cuts; later calls passing the model use the per-packet radius. */
ebg_status ebg_seed_detach(ebg_mesh* mesh);

#ifdef __cplusplus
}
#endif

#endif /* EBGEOMETRY_B200_H */
