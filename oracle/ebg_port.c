/*
 * ORACLE -- test infrastructure, not the product.
 *
 * A plain-C restatement of the reference's (rmrsk/EBGeometry) CPU algorithms on the mesh
 * signed-distance / nearest-neighbour / CSG-union query path, used to check the CUDA path on
 * seeded inputs.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it.  Every function names the reference file:line it restates.  Parity of this restatement is
 * pinned against the reference itself (compiled from its headers into oracle/_ref/) and against
 * the known-answer cases of the reference's Tests/ (see tests/test_oracle.py).
 *
 * Compiled with -ffp-contract=off: the reference's arithmetic is written as separate multiplies
 * and adds, and this file keeps exactly that association order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct
{
  double x, y, z;
} v3;

static inline v3 mk(double x, double y, double z)
{
  v3 r = {x, y, z};
  return r;
}
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
/* Vec3T::operator*(T) (VecImplem.hpp:289-292): s * component. */
static inline v3 scale(double s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
/* Vec3T::dot (VecImplem.hpp:485-488): x*x' + y*y' + z*z', left to right. */
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* Vec3T::cross (VecImplem.hpp:372-375). */
static inline v3 cross(v3 a, v3 b)
{
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* Vec3T::length (VecImplem.hpp:492-495). */
static inline double length(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
/* Vec3T::operator/(T) (VecImplem.hpp:303-309): multiply by the reciprocal. */
static inline v3 divs(v3 a, double s)
{
  const double is = 1.0 / s;
  return mk(is * a.x, is * a.y, is * a.z);
}
static inline v3 ld(const double* p) { return mk(p[0], p[1], p[2]); }

/* Sign as the SIMD TriangleSoA paths take it: from the sign bit, so +0 -> +1 and -0 -> -1
 * (TriangleSoAImplem.hpp:1076-1082, the _mm256_or/and with -0.0 mask). */
static inline double sgnbit(double x) { return signbit(x) ? -1.0 : 1.0; }

/*
 * Point-triangle signed distance of one SoA lane, restating the AVX W=4 double path of
 * TriangleSoAT::signedDistance (TriangleSoAImplem.hpp:1029-1180) lane by lane:
 *   s_i = sgn((e_i x n) . p_i); inside iff |s0+s1+s2| >= 2 -> d = n . p1;
 *   else (d2, sign) = first of vertex0..2 then edges 0..2 (t in (0,1)) with strictly smaller d2,
 *   d = sign * sqrt(d2).
 * v: 3 vertices (9 doubles), fn: unit face normal, vn: 3 vertex pseudonormals, en: 3 edge
 * pseudonormals (edge i runs from vertex i to vertex i+1).
 */
double port_triangle_sd(const double* v, const double* fn, const double* vn, const double* en, const double* p)
{
  const v3 P = ld(p), v0 = ld(v), v1 = ld(v + 3), v2 = ld(v + 6), n = ld(fn);
  const v3 v21 = sub(v1, v0), v32 = sub(v2, v1), v13 = sub(v0, v2);
  const v3 p1 = sub(P, v0), p2 = sub(P, v1), p3 = sub(P, v2);

  const double s0 = sgnbit(dot(cross(v21, n), p1));
  const double s1 = sgnbit(dot(cross(v32, n), p2));
  const double s2 = sgnbit(dot(cross(v13, n), p3));
  const double ssum = (s0 + s1) + s2;

  if (fabs(ssum) >= 2.0) {
    return dot(n, p1);
  }

  const double t1 = dot(p1, v21) / dot(v21, v21);
  const double t2 = dot(p2, v32) / dot(v32, v32);
  const double t3 = dot(p3, v13) / dot(v13, v13);
  const v3     y1 = sub(p1, scale(t1, v21));
  const v3     y2 = sub(p2, scale(t2, v32));
  const v3     y3 = sub(p3, scale(t3, v13));

  double best_d2  = dot(p1, p1);
  double best_sgn = sgnbit(dot(ld(vn), p1));
  const double p2d2 = dot(p2, p2), p3d2 = dot(p3, p3);
  if (p2d2 < best_d2) {
    best_d2  = p2d2;
    best_sgn = sgnbit(dot(ld(vn + 3), p2));
  }
  if (p3d2 < best_d2) {
    best_d2  = p3d2;
    best_sgn = sgnbit(dot(ld(vn + 6), p3));
  }
  const double y1d2 = dot(y1, y1), y2d2 = dot(y2, y2), y3d2 = dot(y3, y3);
  if (t1 > 0.0 && t1 < 1.0 && y1d2 < best_d2) {
    best_d2  = y1d2;
    best_sgn = sgnbit(dot(ld(en), y1));
  }
  if (t2 > 0.0 && t2 < 1.0 && y2d2 < best_d2) {
    best_d2  = y2d2;
    best_sgn = sgnbit(dot(ld(en + 3), y2));
  }
  if (t3 > 0.0 && t3 < 1.0 && y3d2 < best_d2) {
    best_d2  = y3d2;
    best_sgn = sgnbit(dot(ld(en + 6), y3));
  }
  return best_sgn * sqrt(best_d2);
}

/*
 * Scalar Triangle::signedDistance (TriangleImplem.hpp:143-190): same geometry, but the sign
 * function maps 0 to -1 and later candidates win ties (each candidate test is "not greater").
 */
double port_triangle_sd_scalar(const double* v, const double* fn, const double* vn, const double* en, const double* p)
{
  const v3 P = ld(p), v0 = ld(v), v1 = ld(v + 3), v2 = ld(v + 6), n = ld(fn);
  const v3 v21 = sub(v1, v0), v32 = sub(v2, v1), v13 = sub(v0, v2);
  const v3 p1 = sub(P, v0), p2 = sub(P, v1), p3 = sub(P, v2);
#define SGN(x) (((x) > 0.0) ? 1.0 : -1.0)
  const double s0 = SGN(dot(cross(v21, n), p1));
  const double s1 = SGN(dot(cross(v32, n), p2));
  const double s2 = SGN(dot(cross(v13, n), p3));
  const double t1 = dot(p1, v21) / dot(v21, v21);
  const double t2 = dot(p2, v32) / dot(v32, v32);
  const double t3 = dot(p3, v13) / dot(v13, v13);
  const v3     y1 = sub(p1, scale(t1, v21)), y2 = sub(p2, scale(t2, v32)), y3 = sub(p3, scale(t3, v13));
  double       ret = 1.79769313486231570815e+308; /* numeric_limits<double>::max() */
  ret = (length(p1) > fabs(ret)) ? ret : length(p1) * SGN(dot(ld(vn), p1));
  ret = (length(p2) > fabs(ret)) ? ret : length(p2) * SGN(dot(ld(vn + 3), p2));
  ret = (length(p3) > fabs(ret)) ? ret : length(p3) * SGN(dot(ld(vn + 6), p3));
  ret = (t1 > 0.0 && t1 < 1.0 && length(y1) < fabs(ret)) ? length(y1) * SGN(dot(ld(en), y1)) : ret;
  ret = (t2 > 0.0 && t2 < 1.0 && length(y2) < fabs(ret)) ? length(y2) * SGN(dot(ld(en + 3), y2)) : ret;
  ret = (t3 > 0.0 && t3 < 1.0 && length(y3) < fabs(ret)) ? length(y3) * SGN(dot(ld(en + 6), y3)) : ret;
#undef SGN
  return (fabs((s0 + s1) + s2) >= 2.0) ? dot(n, p1) : ret;
}

/*
 * Pseudonormals of a triangle soup, restating Soup::soupToDCEL + MeshT::reconcile(Angle)
 * (SoupImplem.hpp:149-227, DCEL_MeshImplem.hpp:304-366) and TriMeshSDF(mesh,...)'s per-face
 * gathering (MeshDistanceFunctionsImplem.hpp:417-460):
 *   triN[f]   -- the Triangle's own face normal, (x2-x0)x(x2-x1) normalised once
 *                (TriangleImplem.hpp:94-106; setVertexPositions recomputes it);
 *   DCEL face normal -- same cross product, normalised twice (FaceT::computeNormal then
 *                reconcile's normalizeNormalVector, DCEL_FaceImplem.hpp:71-79,136-166);
 *   edgeN[f][i] -- half-edge i (vertex i -> i+1): normalize(n_face + n_pairface)
 *                (DCEL_EdgeImplem.hpp:128-165); a boundary edge takes n_face alone;
 *   vertN[v]  -- sum over the vertex's faces, in facet order, of alpha * n_face, alpha the angle
 *                the face subtends at v, then normalised (DCEL_VertexImplem.hpp:190-~290).
 * Vertices are not merged (soupToDCEL keeps the soup's vertex list as is).
 * Returns 0, or -1 when a half-edge's pair cannot be found among more than one candidate.
 */
int port_mesh_normals(const double* V, int64_t nv, const int64_t* F, int64_t nf, double* triN, double* vertN,
                      double* edgeN)
{
  double* faceN = (double*)malloc(sizeof(double) * 3 * (size_t)(nf > 0 ? nf : 1));
  for (int64_t f = 0; f < nf; f++) {
    const v3 x0 = ld(V + 3 * F[3 * f]), x1 = ld(V + 3 * F[3 * f + 1]), x2 = ld(V + 3 * F[3 * f + 2]);
    const v3 c  = cross(sub(x2, x0), sub(x2, x1));
    v3       n1 = divs(c, length(c));
    const v3 tn = n1;
    n1          = divs(n1, length(n1));
    faceN[3 * f + 0] = n1.x;
    faceN[3 * f + 1] = n1.y;
    faceN[3 * f + 2] = n1.z;
    triN[3 * f + 0]  = tn.x;
    triN[3 * f + 1]  = tn.y;
    triN[3 * f + 2]  = tn.z;
  }

  /* Pair half-edges through a sort of (min, max, face, slot) keys. */
  const int64_t ne  = 3 * nf;
  int64_t*      key = (int64_t*)malloc(sizeof(int64_t) * 4 * (size_t)(ne > 0 ? ne : 1));
  for (int64_t f = 0; f < nf; f++) {
    for (int i = 0; i < 3; i++) {
      const int64_t a = F[3 * f + i], b = F[3 * f + (i + 1) % 3];
      int64_t*      k = key + 4 * (3 * f + i);
      k[0] = a < b ? a : b;
      k[1] = a < b ? b : a;
      k[2] = f;
      k[3] = i;
    }
  }
  /* simple heap-free merge sort on 4-tuples (lexicographic on the first two, then face) */
  int64_t* tmp = (int64_t*)malloc(sizeof(int64_t) * 4 * (size_t)(ne > 0 ? ne : 1));
  for (int64_t w = 1; w < ne; w *= 2) {
    for (int64_t lo = 0; lo < ne; lo += 2 * w) {
      int64_t mid = lo + w < ne ? lo + w : ne, hi = lo + 2 * w < ne ? lo + 2 * w : ne;
      int64_t i = lo, j = mid, o = lo;
      while (i < mid || j < hi) {
        int takei;
        if (i >= mid) {
          takei = 0;
        }
        else if (j >= hi) {
          takei = 1;
        }
        else {
          const int64_t* a = key + 4 * i;
          const int64_t* b = key + 4 * j;
          takei = (a[0] < b[0]) || (a[0] == b[0] && (a[1] < b[1] || (a[1] == b[1] && a[2] <= b[2])));
        }
        memcpy(tmp + 4 * o, key + 4 * (takei ? i : j), sizeof(int64_t) * 4);
        o++;
        if (takei) {
          i++;
        }
        else {
          j++;
        }
      }
    }
    int64_t* t = key;
    key        = tmp;
    tmp        = t;
  }
  int rc = 0;
  for (int64_t s = 0; s < ne;) {
    int64_t e = s + 1;
    while (e < ne && key[4 * e] == key[4 * s] && key[4 * e + 1] == key[4 * s + 1]) {
      e++;
    }
    for (int64_t q = s; q < e; q++) {
      const int64_t f = key[4 * q + 2], i = key[4 * q + 3];
      v3            nrm = ld(faceN + 3 * f);
      if (e - s == 2) {
        const int64_t g = key[4 * (q == s ? s + 1 : s) + 2];
        nrm             = add(nrm, ld(faceN + 3 * g));
      }
      else if (e - s > 2) {
        rc = -1;
      }
      const double len = length(nrm);
      const v3     en  = (len > 2.220446049250313e-16) ? divs(nrm, len) : mk(0, 0, 0);
      edgeN[9 * f + 3 * i + 0] = en.x;
      edgeN[9 * f + 3 * i + 1] = en.y;
      edgeN[9 * f + 3 * i + 2] = en.z;
    }
    s = e;
  }

  for (int64_t v = 0; v < nv; v++) {
    vertN[3 * v + 0] = 0.0;
    vertN[3 * v + 1] = 0.0;
    vertN[3 * v + 2] = 0.0;
  }
  for (int64_t f = 0; f < nf; f++) {
    const int64_t a = F[3 * f], b = F[3 * f + 1], c = F[3 * f + 2];
    /* the two neighbours of each corner in half-edge loop order: a:(b,c) b:(a,c) c:(b,a) */
    const int64_t corner[3] = {a, b, c}, n1[3] = {b, a, b}, n2[3] = {c, c, a};
    for (int k = 0; k < 3; k++) {
      const v3 x0 = ld(V + 3 * corner[k]);
      v3       e1 = sub(ld(V + 3 * n1[k]), x0);
      v3       e2 = sub(ld(V + 3 * n2[k]), x0);
      e1          = divs(e1, length(e1));
      e2          = divs(e2, length(e2));
      double cs   = dot(e1, e2);
      cs          = cs < -1.0 ? -1.0 : (cs > 1.0 ? 1.0 : cs);
      const double alpha = acos(cs);
      const v3     w     = scale(alpha, ld(faceN + 3 * f));
      double*      dst   = vertN + 3 * corner[k];
      dst[0] += w.x;
      dst[1] += w.y;
      dst[2] += w.z;
    }
  }
  for (int64_t v = 0; v < nv; v++) {
    const v3     n   = ld(vertN + 3 * v);
    const double len = length(n);
    if (len > 2.220446049250313e-16) {
      const v3 u = divs(n, len);
      vertN[3 * v + 0] = u.x;
      vertN[3 * v + 1] = u.y;
      vertN[3 * v + 2] = u.z;
    }
  }
  free(key);
  free(tmp);
  free(faceN);
  return rc;
}

/*
 * Brute-force mesh signed distance: the min-|d| scan of FlatMeshSDF / TriMeshSDF's leaf loop
 * (MeshDistanceFunctionsImplem.hpp:492-502: keep d if |d| < |best|, strict, so the first found
 * wins a tie) over every triangle in soup order, with the SoA lane kernel above.
 * Also returns the winning triangle (its soup index) when tri_out is non-null.
 */
void port_mesh_sdf_brute(const double* V, const int64_t* F, int64_t nf, const double* triN, const double* vertN,
                         const double* edgeN, const double* P, int64_t n, double* out, int64_t* tri_out)
{
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t q = 0; q < n; q++) {
    double  best = 1.79769313486231570815e+308;
    int64_t bt   = -1;
    for (int64_t f = 0; f < nf; f++) {
      double v[9], vn[9];
      for (int k = 0; k < 3; k++) {
        for (int c = 0; c < 3; c++) {
          v[3 * k + c]  = V[3 * F[3 * f + k] + c];
          vn[3 * k + c] = vertN[3 * F[3 * f + k] + c];
        }
      }
      const double d = port_triangle_sd(v, triN + 3 * f, vn, edgeN + 9 * f, P + 3 * q);
      if (fabs(d) < fabs(best)) {
        best = d;
        bt   = f;
      }
    }
    out[q] = best;
    if (tri_out) {
      tri_out[q] = bt;
    }
  }
}

/*
 * Signed distance to one triangle as a DCEL face, the algorithm of MeshSDF and FlatMeshSDF
 * (FaceT::signedDistance, DCEL_FaceImplem.hpp:388-423), which differs in the last bits from the
 * Triangle/TriangleSoA test above:
 *   - centroid c = ((x0 + x1) + x2) * (1/3) (computeCentroid, :120-133, Vec3T::operator/);
 *   - inside test: the point projected into the face plane, p - n (n.(p - c)) (:370-378), then
 *     the crossing number of its 2D projection that drops the axis of largest |n| (first on
 *     ties) and keeps the other two in increasing order (Polygon2DImplem.hpp:80-118,164-193);
 *   - inside: n.(p - c) with the DCEL face normal n (normalised twice);
 *   - outside: the edge of smallest |d| (strict <, edges in loop order), where an edge gives the
 *     distance to its start vertex for t <= 0, to its end vertex for t >= 1 and to its interior
 *     otherwise, signed by (pseudonormal . delta > 0 ? +1 : -1) (DCEL_EdgeImplem.hpp:283-331,
 *     DCEL_VertexImplem.hpp:368-380).
 * v: 3 vertices in loop order; fn: DCEL face normal; vn: the 3 vertex normals; en: the 3 edge
 * normals (edge i from vertex i to vertex i+1).
 */
static double dcel_vertex_sd(v3 x, v3 vn, v3 p)
{
  const v3     delta = sub(p, x);
  const double dist  = length(delta);
  return dist * ((dot(vn, delta) > 0.0) ? 1.0 : -1.0);
}

static double dcel_edge_sd(v3 x1, v3 x2, v3 en, v3 vn1, v3 vn2, v3 p)
{
  const v3     x2x1 = sub(x2, x1);
  const double t    = dot(sub(p, x1), x2x1) / dot(x2x1, x2x1);
  if (t <= 0.0) {
    return dcel_vertex_sd(x1, vn1, p);
  }
  if (t >= 1.0) {
    return dcel_vertex_sd(x2, vn2, p);
  }
  const v3 delta = sub(p, add(x1, scale(t, x2x1)));
  return ((dot(en, delta) > 0.0) ? 1.0 : -1.0) * length(delta);
}

static double dcel_edge_ud2(v3 x1, v3 x2, v3 p)
{
  const v3 x2x1 = sub(x2, x1);
  double   t    = dot(sub(p, x1), x2x1) / dot(x2x1, x2x1);
  t             = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
  const v3 delta = sub(p, add(x1, scale(t, x2x1)));
  return dot(delta, delta);
}

static v3 dcel_centroid(const v3* x)
{
  const double is = 1.0 / 3.0;
  return scale(is, add(add(x[0], x[1]), x[2]));
}

static int dcel_inside(const v3* x, v3 n, v3 c, v3 p)
{
  const double a[3] = {fabs(n.x), fabs(n.y), fabs(n.z)};
  int          ig   = 0;
  for (int d = 1; d < 3; d++) {
    if (a[d] > a[ig]) {
      ig = d;
    }
  }
  const int xd = ig == 0 ? 1 : 0, yd = ig == 2 ? 1 : 2;
  const v3  q  = sub(p, scale(dot(n, sub(p, c)), n));
  const double qa[3] = {q.x, q.y, q.z};
  int          cn    = 0;
  for (int i = 0; i < 3; i++) {
    const double p1[3] = {x[i].x, x[i].y, x[i].z}, p2[3] = {x[(i + 1) % 3].x, x[(i + 1) % 3].y, x[(i + 1) % 3].z};
    const int up = (p1[yd] <= qa[yd]) && (p2[yd] > qa[yd]), down = (p1[yd] > qa[yd]) && (p2[yd] <= qa[yd]);
    if (up || down) {
      const double t = (qa[yd] - p1[yd]) / (p2[yd] - p1[yd]);
      if (qa[xd] < p1[xd] + t * (p2[xd] - p1[xd])) {
        cn++;
      }
    }
  }
  return cn & 1;
}

double port_dcel_face_sd(const double* v, const double* fn, const double* vn, const double* en, const double* pp)
{
  const v3 x[3] = {ld(v), ld(v + 3), ld(v + 6)}, n = ld(fn), p = ld(pp);
  const v3 c    = dcel_centroid(x);
  if (dcel_inside(x, n, c, p)) {
    return dot(n, sub(p, c));
  }
  double best = INFINITY;
  for (int i = 0; i < 3; i++) {
    const int    j = (i + 1) % 3;
    const double d = dcel_edge_sd(x[i], x[j], ld(en + 3 * i), ld(vn + 3 * i), ld(vn + 3 * j), p);
    best           = fabs(d) < fabs(best) ? d : best;
  }
  return best;
}

/* FaceT::unsignedDistance2 (DCEL_FaceImplem.hpp:425-458). */
double port_dcel_face_ud2(const double* v, const double* fn, const double* pp)
{
  const v3 x[3] = {ld(v), ld(v + 3), ld(v + 6)}, n = ld(fn), p = ld(pp);
  const v3 c    = dcel_centroid(x);
  if (dcel_inside(x, n, c, p)) {
    const double nd = dot(n, sub(p, c));
    return nd * nd;
  }
  double best = INFINITY;
  for (int i = 0; i < 3; i++) {
    const double d2 = dcel_edge_ud2(x[i], x[(i + 1) % 3], p);
    best            = d2 < best ? d2 : best;
  }
  return best;
}

/*
 * FlatMeshSDF::signedDistance with the DCEL mesh's default search (MeshT::DirectSignedDistance2,
 * DCEL_MeshImplem.hpp:574-595): the first face in soup order with the smallest unsigned
 * distance^2, then its signed distance.  triN: the Triangle normals (normalised once); the DCEL
 * face normal is that normalised again.  tri_out (nullable) receives the winning face.
 */
void port_mesh_sdf_flat(const double* V, const int64_t* F, int64_t nf, const double* triN, const double* vertN,
                        const double* edgeN, const double* P, int64_t n, double* out, int64_t* tri_out)
{
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t q = 0; q < n; q++) {
    double  best = INFINITY;
    int64_t bt   = -1;
    double  fnb[3], vb[9], vnb[9];
    for (int64_t f = 0; f < nf; f++) {
      double v[9];
      for (int k = 0; k < 3; k++) {
        for (int c = 0; c < 3; c++) {
          v[3 * k + c] = V[3 * F[3 * f + k] + c];
        }
      }
      const v3 fd = divs(ld(triN + 3 * f), length(ld(triN + 3 * f)));
      const double fn[3] = {fd.x, fd.y, fd.z};
      const double d2    = port_dcel_face_ud2(v, fn, P + 3 * q);
      if (bt < 0 || d2 < best) {
        best = d2;
        bt   = f;
        memcpy(fnb, fn, sizeof(fnb));
        memcpy(vb, v, sizeof(vb));
        for (int k = 0; k < 3; k++) {
          for (int c = 0; c < 3; c++) {
            vnb[3 * k + c] = vertN[3 * F[3 * f + k] + c];
          }
        }
      }
    }
    out[q] = bt >= 0 ? port_dcel_face_sd(vb, fnb, vnb, edgeN + 9 * bt, P + 3 * q) : INFINITY;
    if (tri_out) {
      tri_out[q] = bt;
    }
  }
}

/*
 * Brute-force k nearest neighbours ordered lexicographically by (d2, index) -- the order
 * closestPointBruteForce / bruteForceK (PointCloudBVHImplem.hpp:509-576) give for k = 1 (lowest
 * index on ties) extended to k > 1.  d2 is PointSoAT::getDistances2's float arithmetic
 * (PointSoAImplem.hpp:214-230): dx = q - p, d2 = (dx*dx + dy*dy) + dz*dz, no fused multiply-add.
 * Missing neighbours (k > n) are index -1, d2 = +inf.
 */
void port_knn_brute_excl(const float* P, int64_t n, const float* Q, int64_t nq, int k, int32_t* idx, float* d2,
                         int exclude_self)
{
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t q = 0; q < nq; q++) {
    float   bd[64];
    int32_t bi[64];
    int     found = 0;
    for (int64_t i = 0; i < n; i++) {
      if (exclude_self && i == q) {
        continue;
      }
      const float dx = Q[3 * q + 0] - P[3 * i + 0];
      const float dy = Q[3 * q + 1] - P[3 * i + 1];
      const float dz = Q[3 * q + 2] - P[3 * i + 2];
      const float dd = dx * dx + dy * dy + dz * dz;
      if (found == k && !(dd < bd[k - 1] || (dd == bd[k - 1] && (int32_t)i < bi[k - 1]))) {
        continue;
      }
      int slot = (found < k) ? found++ : k - 1;
      bd[slot] = dd;
      bi[slot] = (int32_t)i;
      while (slot > 0 && (bd[slot] < bd[slot - 1] || (bd[slot] == bd[slot - 1] && bi[slot] < bi[slot - 1]))) {
        float   td = bd[slot];
        int32_t ti = bi[slot];
        bd[slot]     = bd[slot - 1];
        bi[slot]     = bi[slot - 1];
        bd[slot - 1] = td;
        bi[slot - 1] = ti;
        slot--;
      }
    }
    for (int j = 0; j < k; j++) {
      idx[q * k + j] = j < found ? bi[j] : -1;
      d2[q * k + j]  = j < found ? bd[j] : INFINITY;
    }
  }
}

void port_knn_brute(const float* P, int64_t n, const float* Q, int64_t nq, int k, int32_t* idx, float* d2)
{
  port_knn_brute_excl(P, n, Q, nq, k, idx, d2, 0);
}

/*
 * Self queries (nearestNeighbors / allNearestNeighbors, PointCloudBVHImplem.hpp:455-507): query i is
 * cloud point i and is excluded from its own neighbours; same order and tie rule as above.
 */
void port_knn_brute_self(const float* P, int64_t n, int k, int32_t* idx, float* d2)
{
  port_knn_brute_excl(P, n, P, n, k, idx, d2, 1);
}

/* SphereSDF::signedDistance (AnalyticDistanceFunctions.hpp:238-246): |p - c| - r. */
double port_sphere_sd(const double* c, double r, const double* p) { return length(sub(ld(p), ld(c))) - r; }

/*
 * RotateIF::value's point map (TransformImplem.hpp:163-225): the angle is in degrees
 * (theta = angle * pi / 180, pi from Constants.hpp:23) about one axis.
 */
void port_rotate_point(double angle_deg, int axis, const double* p, double* out)
{
  const double theta = angle_deg * 3.14159265358979323846 / 180.0;
  const double c = cos(theta), s = sin(theta);
  const double x = p[0], y = p[1], z = p[2];
  out[0] = x;
  out[1] = y;
  out[2] = z;
  if (axis == 0) {
    out[1] = y * c + z * s;
    out[2] = -y * s + z * c;
  }
  else if (axis == 1) {
    out[0] = x * c - z * s;
    out[2] = x * s + z * c;
  }
  else {
    out[0] = x * c + y * s;
    out[1] = -x * s + y * c;
  }
}

/*
 * Brute-force union of spheres and posed meshes: UnionIF::value's min over every object
 * (CSGImplem.hpp:355-368), each mesh evaluated as Translate(Rotate(mesh)).value(p) =
 * mesh(rotate(p - t)) (TransformImplem.hpp:152-162) with the brute-force mesh distance above.
 * Meshes are given as one concatenated soup with per-mesh vertex and facet offsets/counts and
 * per-mesh pseudonormals (triN/vertN/edgeN concatenated the same way).
 */
void port_scene_brute(int64_t ns, const double* spheres, int64_t nm, const double* V, const int64_t* vOff,
                      const int64_t* fOff, const int64_t* fCnt, const int64_t* F, const double* triN,
                      const double* vertN, const double* edgeN, const double* pose, const double* P, int64_t n,
                      double* out)
{
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t q = 0; q < n; q++) {
    double best = INFINITY;
    for (int64_t s = 0; s < ns; s++) {
      const double v = port_sphere_sd(spheres + 4 * s, spheres[4 * s + 3], P + 3 * q);
      best           = v < best ? v : best;
    }
    for (int64_t m = 0; m < nm; m++) {
      const double* ps = pose + 5 * m;
      const double  t[3] = {P[3 * q] - ps[2], P[3 * q + 1] - ps[3], P[3 * q + 2] - ps[4]};
      double        lp[3];
      port_rotate_point(ps[0], (int)ps[1], t, lp);
      double mbest = 1.79769313486231570815e+308;
      for (int64_t f = fOff[m]; f < fOff[m] + fCnt[m]; f++) {
        double v[9], vn[9];
        for (int k = 0; k < 3; k++) {
          const int64_t vi = vOff[m] + F[3 * f + k];
          for (int c = 0; c < 3; c++) {
            v[3 * k + c]  = V[3 * vi + c];
            vn[3 * k + c] = vertN[3 * vi + c];
          }
        }
        const double d = port_triangle_sd(v, triN + 3 * f, vn, edgeN + 9 * f, lp);
        if (fabs(d) < fabs(mbest)) {
          mbest = d;
        }
      }
      best = mbest < best ? mbest : best;
    }
    out[q] = best;
  }
}
