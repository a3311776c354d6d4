// Device-side packet traversal of one mesh BVH, shared by the mesh SDF kernel and the CSG scene
// kernel (which runs it once per mesh object a packet reaches, on the object-local query points).
#ifndef EBG_MESH_TRAVERSE_CUH
#define EBG_MESH_TRAVERSE_CUH

#include <cfloat>

#include "ebg_device.cuh"

namespace ebg {

// Closest point of triangle (v0, v0+ab, v0+ac) to p by Voronoi region (the standard barycentric
// region tests).  Returns the squared distance; s, t are the barycentric weights of ab and ac of
// the closest point and region is 0 face, 1..3 vertex 0..2, 4 edge 0-1, 5 edge 1-2, 6 edge 2-0.
// Equivalent to the reference's triangle test (TriangleSoAImplem.hpp:1199-1293): its "inside"
// test (all three (e_i x n).p_i of one sign) is the face region, and outside it the minimum over
// vertices and interior edge points is the closest boundary point.
template <bool WANT_REGION>
__device__ __forceinline__ float triDist2(const float4 h0, const float4 h1, const float4 h2, float px, float py,
                                          float pz, float& s, float& t, int& region)
{
  const float apx = px - h0.x, apy = py - h0.y, apz = pz - h0.z;
  const float ab2 = h0.w, abac = h1.w, ac2 = h2.w;
  const float d1 = fmaf(h1.x, apx, fmaf(h1.y, apy, h1.z * apz));
  const float d2 = fmaf(h2.x, apx, fmaf(h2.y, apy, h2.z * apz));
  const float d3 = d1 - ab2, d4 = d2 - abac;
  const float d5 = d1 - abac, d6 = d2 - ac2;
  const float vc = fmaf(d1, d4, -d3 * d2);
  const float vb = fmaf(d5, d2, -d1 * d6);
  const float va = fmaf(d3, d6, -d5 * d4);

  // face region by default; each test below overrides, the highest-priority region last
  float sn = vb, tn = vc, den = va + vb + vc;
  int   r  = 0;
  const float bc1 = d4 - d3, bc2 = d5 - d6;
  if (va <= 0.f && bc1 >= 0.f && bc2 >= 0.f) { // edge 1-2
    sn = bc2;
    tn = bc1;
    den = bc1 + bc2;
    r   = 5;
  }
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) { // edge 2-0 (along ac)
    sn  = 0.f;
    tn  = d2;
    den = d2 - d6;
    r   = 6;
  }
  if (d6 >= 0.f && d5 <= d6) { // vertex 2
    sn  = 0.f;
    tn  = 1.f;
    den = 1.f;
    r   = 3;
  }
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) { // edge 0-1 (along ab)
    sn  = d1;
    tn  = 0.f;
    den = d1 - d3;
    r   = 4;
  }
  if (d3 >= 0.f && d4 <= d3) { // vertex 1
    sn  = 1.f;
    tn  = 0.f;
    den = 1.f;
    r   = 2;
  }
  if (d1 <= 0.f && d2 <= 0.f) { // vertex 0
    sn  = 0.f;
    tn  = 0.f;
    den = 1.f;
    r   = 1;
  }
  const float inv = __fdividef(1.f, den);
  s               = sn * inv;
  t               = tn * inv;
  const float dx  = fmaf(-t, h2.x, fmaf(-s, h1.x, apx));
  const float dy  = fmaf(-t, h2.y, fmaf(-s, h1.y, apy));
  const float dz  = fmaf(-t, h2.z, fmaf(-s, h1.z, apz));
  if (WANT_REGION) {
    region = r;
  }
  return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

__device__ __forceinline__ float signOf(float x) { return signbit(x) ? -1.f : 1.f; }


// Squared distance from p to an oriented box (EbgObb as four float4: n|dn, u|du, v|dv, h), scaled
// down by 4e-6 relative.  The FP32 error of each plane distance n . p - dn is about 1e-7 of |p|,
// which the padding of the half-extents (2e-6 of the mesh's extent) covers near the mesh and the
// relative scaling covers far from it (there the box distance itself is about |p|).
__device__ __forceinline__ float obbDist2(const float4 o0, const float4 o1, const float4 o2, const float4 o3, float px,
                                          float py, float pz)
{
  const float a  = fmaf(o0.x, px, fmaf(o0.y, py, fmaf(o0.z, pz, -o0.w)));
  const float b  = fmaf(o1.x, px, fmaf(o1.y, py, fmaf(o1.z, pz, -o1.w)));
  const float e  = fmaf(o2.x, px, fmaf(o2.y, py, fmaf(o2.z, pz, -o2.w)));
  const float dn = fmaxf(fabsf(a) - o3.x, 0.f), du = fmaxf(fabsf(b) - o3.y, 0.f), dv = fmaxf(fabsf(e) - o3.z, 0.f);
  return fmaf(dn, dn, fmaf(du, du, dv * dv)) * (1.f - 4e-6f);
}

// a[k] for a warp-uniform k without dynamic register-array indexing (which would go to local memory)
__device__ __forceinline__ float sel4(const float (&a)[4], int k)
{
  return k == 0 ? a[0] : (k == 1 ? a[1] : (k == 2 ? a[2] : a[3]));
}
__device__ __forceinline__ uint32_t sel4u(const uint32_t (&a)[4], int k)
{
  return k == 0 ? a[0] : (k == 1 ? a[1] : (k == 2 ? a[2] : a[3]));
}

// Signed distance of p to triangle `tri` (leaf order), sign from the pseudonormal of the closest
// feature (the reference's sign-bit convention, TriangleSoAImplem.hpp:1076-1082: +0 -> +1).
__device__ __forceinline__ float signedFromWinner(const EbgMeshView& m, uint32_t tri, float px, float py, float pz)
{
  const float4* h = reinterpret_cast<const float4*>(m.hot + tri);
  const float4  h0 = __ldg(h), h1 = __ldg(h + 1), h2 = __ldg(h + 2);
  float         s, t;
  int           region;
  const float   d2 = triDist2<true>(h0, h1, h2, px, py, pz, s, t, region);
  const float*  sg = reinterpret_cast<const float*>(m.sign + tri);
  const float   apx = px - h0.x, apy = py - h0.y, apz = pz - h0.z;
  if (region == 0) {
    // face: the reference returns n . (p - v0) itself
    return fmaf(__ldg(sg + 0), apx, fmaf(__ldg(sg + 1), apy, __ldg(sg + 2) * apz));
  }
  const float dx = fmaf(-t, h2.x, fmaf(-s, h1.x, apx));
  const float dy = fmaf(-t, h2.y, fmaf(-s, h1.y, apy));
  const float dz = fmaf(-t, h2.z, fmaf(-s, h1.z, apz));
  // vertex i -> vn[3i..], edge j -> en[3j..]: sign record = n(3) pad vn(9) en(9)
  const int   o  = (region <= 3) ? (4 + 3 * (region - 1)) : (13 + 3 * (region - 4));
  const float sd = fmaf(__ldg(sg + o), dx, fmaf(__ldg(sg + o + 1), dy, __ldg(sg + o + 2) * dz));
  return signOf(sd) * sqrtf(d2);
}


struct TraversalCounters
{
  uint32_t node = 0, leaf = 0, tri = 0, fall = 0, box = 0; // per lane: what this query needed
  uint32_t pops = 0, pnode = 0, pleaf = 0, ptri = 0, pbox = 0; // per packet: what the warp executed
  uint32_t precs = 0;                                             // triangle records of its opened leaves
};

// 16- and 4-byte loads from a shared-memory address (the block's copy of the tree's top nodes).
__device__ __forceinline__ float4 lds4(uint32_t addr)
{
  float4 v;
  asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
  return v;
}

__device__ __forceinline__ float lds1(uint32_t addr)
{
  float v;
  asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}

// Bytes per node in the shared-memory copy of the top of the tree: the 128-byte node line, then
// its 64-byte oriented box.
constexpr uint32_t TOP_NODE_BYTES = 192;

// Packet traversal of mesh m from the `sp` entries already on the warp's stack (the top entry is
// popped first): each lane's best squared distance `best` (its pruning bound, already seeded or
// FLT_MAX) and winning triangle `besttri` (leaf order) are updated.  Children are ordered by their
// smallest distance over the packet's lanes.  `stk` is this warp's stack region (2 float4 per entry,
// STACK entries); `pts` is this warp's 32-entry scratch for the points of the lanes a leaf is spread
// over; `iters` counts loop trips against MAX_ITERS; `err` receives ST_* bits.  With TOP, nodes
// with index below `topN` are read from the block's shared-memory copy at shared address `topS`
// (TOP_NODE_BYTES per node).  W is the tree's node width: 4 (EbgNode4, every kernel) or 8 (the
// optional EbgNode8 copy, m.nodes and m.node_obb then point at the 8-wide arrays; no TOP).  All 32
// lanes must call it together.
template <bool STATS, int STACK, bool TOP = false, int W = 4>
__device__ __forceinline__ void traverseFrom(const EbgMeshView& m, float px, float py, float pz, float& best,
                                             int& besttri, float4* stk, float4* pts, int sp, uint32_t& iters,
                                             int& err, TraversalCounters& cnt_, uint32_t topS = 0,
                                             uint32_t topN = 0)
{
  const int lane = threadIdx.x & 31;
      // a finite bound keeps empty child slots (infinite box distance) off the stack
      best = fminf(best, FLT_MAX);
#pragma unroll 1
      while (sp > 0) {
        if (++iters > MAX_ITERS) {
          err |= ST_ITERS;
          break;
        }
        --sp;
        if (STATS) {
          cnt_.pops++;
        }
        const float4 A    = stk[2 * sp];
        const float4 B    = stk[2 * sp + 1];
        const float  d2   = boxDist2(A.x, A.y, A.z, B.x, B.y, B.z, px, py, pz);
        const bool   need = d2 <= best;
        if (!__any_sync(FULL, need)) {
          continue;
        }
        const uint32_t ref = __float_as_uint(A.w), cntw = __float_as_uint(B.w);
        if (ref & EBG_LEAF_BIT) {
          const uint32_t t0 = ref & ~EBG_LEAF_BIT, cnt = cntw & EBG_COUNT_MASK;
          // the leaf's oriented box (a thin slab on smooth surfaces) before its triangles
          const float4* ob = reinterpret_cast<const float4*>(m.obb + (cntw >> EBG_COUNT_BITS));
          const float4  o0 = __ldg(ob), o1 = __ldg(ob + 1), o2 = __ldg(ob + 2), o3 = __ldg(ob + 3);
          const bool    needObb = need && obbDist2(o0, o1, o2, o3, px, py, pz) <= best;
          if (STATS) {
            cnt_.box += need;
            cnt_.pbox++;
          }
          const unsigned needMask = __ballot_sync(FULL, needObb);
          if (needMask == 0u) {
            continue;
          }
          // Few lanes need the leaf: spread their (lane, triangle) pairs over the warp, 32 / cnt
          // lanes per pass, instead of every lane testing every triangle.  A pass costs about two
          // triangle tests, so this runs when it needs at most cnt / 2 passes (level-8 step:
          // 103.7 ms seeded, 185.4 plain; at most cnt - 2 passes: 104.6, 186.6; at most cnt / 3:
          // 104.7, 186.0).
          const int nNeed  = __popc(needMask);
          const int lpp    = int(c_lanesPer[cnt]);
          const int passes = divSmall(nNeed + lpp - 1, lpp);
          if (STATS && needObb) {
            cnt_.leaf++;
            cnt_.tri += cnt;
          }
          if (STATS) {
            cnt_.pleaf++;
            cnt_.ptri += 2 * passes <= int(cnt) ? uint32_t(passes) : cnt;
            cnt_.precs += cnt;
          }
          if (2 * passes <= int(cnt)) {
            const int rank = __popc(needMask & ((1u << lane) - 1u));
            if (needObb) {
              pts[rank] = make_float4(px, py, pz, 0.f);
            }
            __syncwarp();
            const int     li = divSmall(lane, int(cnt)), ti = lane - li * int(cnt);
            const float4* h  = reinterpret_cast<const float4*>(m.hot + t0 + uint32_t(ti));
#pragma unroll 1
            for (int ps = 0; ps < passes; ps++) {
              const int slot = ps * lpp + li;
              float     dd   = __int_as_float(0x7f800000);
              int       bi   = ti;
              if (li < lpp && slot < nNeed) {
                const float4 q  = pts[slot];
                const float4 h0 = __ldg(h), h1 = __ldg(h + 1), h2 = __ldg(h + 2);
                float        s, t;
                int          r;
                dd = triDist2<false>(h0, h1, h2, q.x, q.y, q.z, s, t, r);
              }
              // minimum of (d2, triangle) over the cnt threads serving one lane; the first thread
              // of the segment ends with it (offsets of cnt or more reach no segment partner)
#pragma unroll
              for (int off = 16; off > 0; off >>= 1) {
                if (off >= int(cnt)) {
                  continue;
                }
                const float od = __shfl_down_sync(FULL, dd, off);
                const int   oi = __shfl_down_sync(FULL, bi, off);
                if (ti + off < int(cnt) && (od < dd || (od == dd && oi < bi))) {
                  dd = od;
                  bi = oi;
                }
              }
              const int  seg  = rank - ps * lpp;
              const bool mine = needObb && seg >= 0 && seg < lpp;
              const int  from = mine ? seg * int(cnt) : 0;
              const float rd = __shfl_sync(FULL, dd, from);
              const int   ri = __shfl_sync(FULL, bi, from);
              // ties go to the lower leaf position, so the winner does not depend on the order
              // in which packets meet the triangles
              if (mine && (rd < best || (rd == best && int(t0) + ri < besttri))) {
                best    = rd;
                besttri = int(t0) + ri;
              }
            }
            __syncwarp();
            continue;
          }
#pragma unroll 1
          for (uint32_t tt = t0; tt < t0 + cnt; ++tt) {
            const float4* h = reinterpret_cast<const float4*>(m.hot + tt);
            const float4  h0 = __ldg(h), h1 = __ldg(h + 1), h2 = __ldg(h + 2);
            float         s, t;
            int           r;
            const float   dd = triDist2<false>(h0, h1, h2, px, py, pz, s, t, r);
            if (dd < best || (dd == best && int(tt) < besttri)) {
              best    = dd;
              besttri = int(tt);
            }
          }
        }
        else if constexpr (W == 8) {
          static_assert(!TOP, "the shared-memory top tree is a 4-wide option");
          // 16 float4 per node: lo.x[8] lo.y[8] lo.z[8] hi.x[8] hi.y[8] hi.z[8] child[8] count[8];
          // the first half's boxes go out before the oriented-box test, which overlaps their latency
          const float4* nd  = reinterpret_cast<const float4*>(m.nodes) + size_t(ref) * 16u;
          float4        lx = __ldg(nd), ly = __ldg(nd + 2), lz = __ldg(nd + 4);
          float4        hx = __ldg(nd + 6), hy = __ldg(nd + 8), hz = __ldg(nd + 10);
          bool          needN = need;
          if (cntw & EBG_NODE_HAS_OBB) {
            const float4* ob = reinterpret_cast<const float4*>(m.node_obb + ref);
            const float4  o0 = __ldg(ob), o1 = __ldg(ob + 1), o2 = __ldg(ob + 2), o3 = __ldg(ob + 3);
            needN            = need && obbDist2(o0, o1, o2, o3, px, py, pz) <= best;
            if (STATS) {
              cnt_.box += need;
              cnt_.pbox++;
            }
            if (!__any_sync(FULL, needN)) {
              continue;
            }
          }
          if (STATS && needN) {
            cnt_.node++;
          }
          if (STATS) {
            cnt_.pnode++;
          }
          float key[8];
#pragma unroll
          for (int h = 0; h < 2; h++) {
            if (h == 1) {
              lx = __ldg(nd + 1), ly = __ldg(nd + 3), lz = __ldg(nd + 5);
              hx = __ldg(nd + 7), hy = __ldg(nd + 9), hz = __ldg(nd + 11);
            }
            const float clx[4] = {lx.x, lx.y, lx.z, lx.w}, cly[4] = {ly.x, ly.y, ly.z, ly.w},
                        clz[4] = {lz.x, lz.y, lz.z, lz.w};
            const float chx[4] = {hx.x, hx.y, hx.z, hx.w}, chy[4] = {hy.x, hy.y, hy.z, hy.w},
                        chz[4] = {hz.x, hz.y, hz.z, hz.w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const float dk = needN ? boxDist2(clx[k], cly[k], clz[k], chx[k], chy[k], chz[k], px, py, pz)
                                     : __int_as_float(0x7f800000);
              const bool  nk = __any_sync(FULL, dk <= best);
              key[4 * h + k] = nk ? __uint_as_float(__reduce_min_sync(FULL, __float_as_uint(dk))) : -1.f;
            }
          }
          int np = 0;
#pragma unroll
          for (int k = 0; k < 8; k++) {
            np += int(key[k] >= 0.f);
          }
          if (sp + np > STACK) {
            err |= ST_STACK;
            break;
          }
          // lane k (< 8) writes child k into its slot, nearest on top, as in the 4-wide case
          if (lane < 8) {
            float kk = key[0];
#pragma unroll
            for (int j = 1; j < 8; j++) {
              kk = lane == j ? key[j] : kk;
            }
            if (kk >= 0.f) {
              int rank = 0;
#pragma unroll
              for (int j = 0; j < 8; j++) {
                rank += int(key[j] >= 0.f && (key[j] > kk || (key[j] == kk && j < lane)));
              }
              float4*      e  = stk + 2 * (sp + rank);
              const float* nf = reinterpret_cast<const float*>(nd) + lane;
              e[0]            = make_float4(__ldg(nf), __ldg(nf + 8), __ldg(nf + 16), __ldg(nf + 48));
              e[1]            = make_float4(__ldg(nf + 24), __ldg(nf + 32), __ldg(nf + 40), __ldg(nf + 56));
            }
          }
          sp += np;
          __syncwarp();
          if (err) {
            break;
          }
        }
        else {
          // the node's loads go out first; the oriented-box test below overlaps their latency
          const float4*  nd    = reinterpret_cast<const float4*>(m.nodes + ref);
          const bool     inTop = TOP && ref < topN; // warp-uniform: the node's copy in shared memory
          const uint32_t ts    = topS + ref * TOP_NODE_BYTES;
          float4         lx, ly, lz, hx, hy, hz;
          if (inTop) {
            lx = lds4(ts), ly = lds4(ts + 16), lz = lds4(ts + 32);
            hx = lds4(ts + 48), hy = lds4(ts + 64), hz = lds4(ts + 80);
          }
          else {
            lx = __ldg(nd), ly = __ldg(nd + 1), lz = __ldg(nd + 2);
            hx = __ldg(nd + 3), hy = __ldg(nd + 4), hz = __ldg(nd + 5);
          }
          // lanes for which the node's own oriented box (all triangles below it) is within bound
          bool needN = need;
          if (cntw & EBG_NODE_HAS_OBB) {
            float4 o0, o1, o2, o3;
            if (inTop) {
              o0 = lds4(ts + 128), o1 = lds4(ts + 144), o2 = lds4(ts + 160), o3 = lds4(ts + 176);
            }
            else {
              const float4* ob = reinterpret_cast<const float4*>(m.node_obb + ref);
              o0 = __ldg(ob), o1 = __ldg(ob + 1), o2 = __ldg(ob + 2), o3 = __ldg(ob + 3);
            }
            needN = need && obbDist2(o0, o1, o2, o3, px, py, pz) <= best;
            if (STATS) {
              cnt_.box += need;
              cnt_.pbox++;
            }
            if (!__any_sync(FULL, needN)) {
              continue;
            }
          }
          if (STATS && needN) {
            cnt_.node++;
          }
          if (STATS) {
            cnt_.pnode++;
          }
          const float   clx[4] = {lx.x, lx.y, lx.z, lx.w}, cly[4] = {ly.x, ly.y, ly.z, ly.w},
                      clz[4] = {lz.x, lz.y, lz.z, lz.w};
          const float chx[4] = {hx.x, hx.y, hx.z, hx.w}, chy[4] = {hy.x, hy.y, hy.z, hy.w},
                      chz[4] = {hz.x, hz.y, hz.z, hz.w};
          float key[4];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            // lanes that ruled the node out cannot gain from its children
            const float dk = needN ? boxDist2(clx[k], cly[k], clz[k], chx[k], chy[k], chz[k], px, py, pz)
                                   : __int_as_float(0x7f800000);
            // an empty slot (child 0, count 0) has an empty box, at +inf: never within the finite bound
            const bool  nk = __any_sync(FULL, dk <= best);
            // uniform ordering key: the child's smallest distance over the packet's lanes (one
            // warp min-reduction; non-negative floats order like their bit patterns); children
            // nobody needs get -1 and are not pushed
            key[k] = nk ? __uint_as_float(__reduce_min_sync(FULL, __float_as_uint(dk))) : -1.f;
          }
          const int np = int(key[0] >= 0.f) + int(key[1] >= 0.f) + int(key[2] >= 0.f) + int(key[3] >= 0.f);
          if (sp + np > STACK) {
            err |= ST_STACK;
            break;
          }
          // lane k (< 4) writes child k straight into its slot: farther children sit deeper, so the
          // nearest is popped first; ties go by slot index (a total order, so slots are distinct).
          // The child's box and words come again from the node's line (an L1 hit), which is cheaper
          // than selecting them out of the registers.
          if (lane < 4) {
            const float kk = sel4(key, lane);
            if (kk >= 0.f) {
              int rank = 0;
#pragma unroll
              for (int j = 0; j < 4; j++) {
                rank += int(key[j] >= 0.f && (key[j] > kk || (key[j] == kk && j < lane)));
              }
              float4* e = stk + 2 * (sp + rank);
              if (inTop) {
                const uint32_t nf = ts + 4 * lane;
                e[0] = make_float4(lds1(nf), lds1(nf + 16), lds1(nf + 32), lds1(nf + 96));
                e[1] = make_float4(lds1(nf + 48), lds1(nf + 64), lds1(nf + 80), lds1(nf + 112));
              }
              else {
                const float* nf = reinterpret_cast<const float*>(nd) + lane;
                e[0]            = make_float4(__ldg(nf), __ldg(nf + 4), __ldg(nf + 8), __ldg(nf + 24));
                e[1]            = make_float4(__ldg(nf + 12), __ldg(nf + 16), __ldg(nf + 20), __ldg(nf + 28));
              }
            }
          }
          sp += np;
          __syncwarp();
          if (err) {
            break;
          }
        }
      }
}

// One packet traversal from the root of mesh m (see traverseFrom).
template <bool STATS, int STACK = EBG_STACK_DEPTH, bool TOP = false, int W = 4>
__device__ __forceinline__ void traverseMesh(const EbgMeshView& m, float px, float py, float pz, float& best,
                                             int& besttri, float4* stk, float4* pts, uint32_t& iters, int& err,
                                             TraversalCounters& cnt_, uint32_t topS = 0, uint32_t topN = 0)
{
  if ((threadIdx.x & 31) == 0) {
    stk[0] = make_float4(m.root_lo[0], m.root_lo[1], m.root_lo[2], __uint_as_float(m.root_ref));
    stk[1] = make_float4(m.root_hi[0], m.root_hi[1], m.root_hi[2], __uint_as_float(m.root_count));
  }
  __syncwarp();
  traverseFrom<STATS, STACK, TOP, W>(m, px, py, pz, best, besttri, stk, pts, 1, iters, err, cnt_, topS, topN);
}

} // namespace ebg

#endif
