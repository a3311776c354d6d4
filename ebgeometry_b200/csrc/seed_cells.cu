// Per-cell entry cuts of a mesh BVH from a learned distance bound (see cells_kernels.h).
#include <cfloat>
#include <cmath>

#include "cells_kernels.h"
#include "ebg_device.cuh"
#include "mesh_traverse.cuh"

namespace ebg {

namespace {

constexpr int CUT_WARPS = 4;

__global__ void kCellCentres(const SeedCellsView v, float* __restrict__ out)
{
  const int64_t cells = int64_t(v.g) * v.g * v.g;
  for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += int64_t(gridDim.x) * blockDim.x) {
    const int ix = int(c % v.g), iy = int((c / v.g) % v.g), iz = int(c / (int64_t(v.g) * v.g));
    out[3 * c]     = v.lo[0] + (float(ix) + 0.5f) * v.size[0];
    out[3 * c + 1] = v.lo[1] + (float(iy) + 0.5f) * v.size[1];
    out[3 * c + 2] = v.lo[2] + (float(iz) + 0.5f) * v.size[2];
  }
}

__global__ void kCellRadius(const float* __restrict__ value, int64_t cells, int mode, float alpha, float beta,
                            float halfDiag, float* __restrict__ radius)
{
  for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += int64_t(gridDim.x) * blockDim.x) {
    float r = __int_as_float(0x7f800000);
    if (mode != 1) {
      const float y = value[c];
      const float a = fabsf(y);
      // the cell-centre bound, then the grown cell's half-diagonal; every step rounded up
      const float rc = mode == 0 ? __fadd_ru(__fmul_ru(1.f + alpha, a), beta) : __fadd_ru(__fmul_ru(a, 1.000002f), 1e-7f);
      r              = isfinite(y) ? __fmul_ru(__fadd_ru(rc, halfDiag), 1.00001f) : r;
    }
    radius[c] = r;
  }
}

// One warp per cell.  The cut lives in shared memory as up to CUT_MAX_ENTRIES slots (entry, key =
// lower bound of the squared distance from the cell centre, expandable flag); each round the warp
// splits the expandable slot of least key into its children within R_C of the grown cell, or marks
// it final when the children would not fit.
__global__ void __launch_bounds__(CUT_WARPS * 32) kCellCuts(const EbgMeshView m, const SeedCellsView v,
                                                            float4* __restrict__ entries, uint32_t* __restrict__ count)
{
  __shared__ float4 sEnt[CUT_WARPS][2 * CUT_MAX_ENTRIES];
  __shared__ float  sKey[CUT_WARPS][CUT_MAX_ENTRIES];
  __shared__ int    sExp[CUT_WARPS][CUT_MAX_ENTRIES];
  const int     lane  = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t cells = int64_t(v.g) * v.g * v.g;
  const int64_t cell  = int64_t(blockIdx.x) * CUT_WARPS + wid;
  if (cell >= cells) {
    return; // the whole warp
  }
  float4* E   = sEnt[wid];
  float*  K   = sKey[wid];
  int*    X   = sExp[wid];
  const int lmax = v.lmax;
  const int ix = int(cell % v.g), iy = int((cell / v.g) % v.g), iz = int(cell / (int64_t(v.g) * v.g));
  const float cx = v.lo[0] + (float(ix) + 0.5f) * v.size[0];
  const float cy = v.lo[1] + (float(iy) + 0.5f) * v.size[1];
  const float cz = v.lo[2] + (float(iz) + 0.5f) * v.size[2];
  // the grown cell, rounded outward
  const float glx = __fsub_rd(__fadd_rd(v.lo[0], float(ix) * v.size[0]), v.margin[0]);
  const float gly = __fsub_rd(__fadd_rd(v.lo[1], float(iy) * v.size[1]), v.margin[1]);
  const float glz = __fsub_rd(__fadd_rd(v.lo[2], float(iz) * v.size[2]), v.margin[2]);
  const float ghx = __fadd_ru(__fadd_ru(v.lo[0], float(ix + 1) * v.size[0]), v.margin[0]);
  const float ghy = __fadd_ru(__fadd_ru(v.lo[1], float(iy + 1) * v.size[1]), v.margin[1]);
  const float ghz = __fadd_ru(__fadd_ru(v.lo[2], float(iz + 1) * v.size[2]), v.margin[2]);
  const float hx = 0.5f * (ghx - glx), hy = 0.5f * (ghy - gly), hz = 0.5f * (ghz - glz);
  const float halfDiag = __fmul_ru(sqrtf(fmaf(hx, hx, fmaf(hy, hy, hz * hz))), 1.00001f);
  const float R        = v.radius[cell];
  const float R2       = isfinite(R) ? __fmul_ru(__fmul_ru(R, R), 1.00002f) : __int_as_float(0x7f800000);

  int cnt = 1;
  if (lane == 0) {
    E[0] = make_float4(m.root_lo[0], m.root_lo[1], m.root_lo[2], __uint_as_float(m.root_ref));
    E[1] = make_float4(m.root_hi[0], m.root_hi[1], m.root_hi[2], __uint_as_float(m.root_count));
    K[0] = boxDist2(m.root_lo[0], m.root_lo[1], m.root_lo[2], m.root_hi[0], m.root_hi[1], m.root_hi[2], cx, cy, cz);
    X[0] = (m.root_ref & EBG_LEAF_BIT) ? 0 : 1;
  }
  __syncwarp();
  if (boxBoxDist2(glx, gly, glz, ghx, ghy, ghz, m.root_lo[0], m.root_lo[1], m.root_lo[2], m.root_hi[0], m.root_hi[1],
                  m.root_hi[2]) > R2) {
    cnt = 0; // the whole mesh is farther than R_C: nothing to cut, the cell's packets start at the root
  }

#pragma unroll 1
  for (int round = 0; round < 16 * CUT_MAX_ENTRIES && cnt > 0; round++) {
    // the expandable slot of least key (ties: lowest slot)
    float bk = __int_as_float(0x7f800000);
    int   bs = -1;
    for (int j = lane; j < cnt; j += 32) {
      if (X[j] && K[j] < bk) {
        bk = K[j];
        bs = j;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float ok = __shfl_xor_sync(FULL, bk, o);
      const int   os = __shfl_xor_sync(FULL, bs, o);
      if (os >= 0 && (bs < 0 || ok < bk || (ok == bk && os < bs))) {
        bk = ok;
        bs = os;
      }
    }
    if (bs < 0) {
      break;
    }
    const uint32_t ref = __float_as_uint(E[2 * bs].w);
    const EbgNode4* nd = m.nodes + ref;
    bool     keep = false;
    float4   ea, eb;
    float    key = 0.f;
    if (lane < 4) {
      const float lx = nd->lox[lane], ly = nd->loy[lane], lz = nd->loz[lane];
      const float hx2 = nd->hix[lane], hy2 = nd->hiy[lane], hz2 = nd->hiz[lane];
      const uint32_t ch = nd->child[lane], cw = nd->count[lane];
      keep = lx <= hx2 && boxBoxDist2(glx, gly, glz, ghx, ghy, ghz, lx, ly, lz, hx2, hy2, hz2) <= R2;
      key  = boxDist2(lx, ly, lz, hx2, hy2, hz2, cx, cy, cz);
      const bool leaf = (ch & EBG_LEAF_BIT) != 0;
      if (keep && (leaf || (cw & EBG_NODE_HAS_OBB))) {
        // the oriented box: a lower bound of the distance from the centre to the triangles below,
        // less the half-diagonal, bounds the distance from any point of the grown cell
        const float4* ob = reinterpret_cast<const float4*>(leaf ? (m.obb + (cw >> EBG_COUNT_BITS)) : (m.node_obb + ch));
        const float od2 = obbDist2(__ldg(ob), __ldg(ob + 1), __ldg(ob + 2), __ldg(ob + 3), cx, cy, cz);
        const float od  = __fsub_rd(__fmul_rd(sqrtf(od2), 0.99999f), halfDiag);
        keep            = od <= 0.f || !isfinite(R2) || __fmul_rd(od, od) <= R2;
        key             = fmaxf(key, od2);
      }
      ea = make_float4(lx, ly, lz, __uint_as_float(ch));
      eb = make_float4(hx2, hy2, hz2, __uint_as_float(cw));
    }
    const unsigned km   = __ballot_sync(FULL, keep) & 0xfu;
    const int      kept = __popc(km);
    __syncwarp(); // every lane has read the slot before it is overwritten
    if (cnt - 1 + kept > lmax) {
      if (lane == 0) {
        X[bs] = 0; // final: its children would not fit
      }
      __syncwarp();
      continue;
    }
    if (kept == 0) {
      // every child is farther than R_C: drop the slot (the last slot moves into it)
      if (lane == 0 && bs != cnt - 1) {
        E[2 * bs]     = E[2 * (cnt - 1)];
        E[2 * bs + 1] = E[2 * (cnt - 1) + 1];
        K[bs]         = K[cnt - 1];
        X[bs]         = X[cnt - 1];
      }
      cnt--;
      __syncwarp();
      continue;
    }
    // kept children: the first replaces the slot, the others are appended
    if (keep) {
      const int r  = __popc(km & ((1u << lane) - 1u));
      const int sl = r == 0 ? bs : cnt + r - 1;
      E[2 * sl]     = ea;
      E[2 * sl + 1] = eb;
      K[sl]         = key;
      X[sl]         = (__float_as_uint(ea.w) & EBG_LEAF_BIT) ? 0 : 1;
    }
    cnt += kept - 1;
    __syncwarp();
  }

  // store farthest first (descending key, ties by descending slot), so the nearest is on top of the
  // stack once the list is copied onto it
  float4* out = entries + size_t(cell) * size_t(lmax) * 2;
  for (int j = lane; j < cnt; j += 32) {
    const float kj   = K[j];
    int         rank = 0;
    for (int i = 0; i < cnt; i++) {
      const float ki = K[i];
      rank += int(ki > kj || (ki == kj && i > j));
    }
    out[2 * rank]     = E[2 * j];
    out[2 * rank + 1] = E[2 * j + 1];
  }
  if (lane == 0) {
    count[cell] = uint32_t(cnt);
  }
}

} // namespace

cudaError_t launchCellCentres(const SeedCellsView& v, float* out, cudaStream_t s)
{
  kCellCentres<<<1024, 256, 0, s>>>(v, out);
  return cudaGetLastError();
}

cudaError_t launchCellRadius(const float* value, int64_t cells, int mode, float alpha, float beta, float halfDiag,
                             float* radius, cudaStream_t s)
{
  kCellRadius<<<1024, 256, 0, s>>>(value, cells, mode, alpha, beta, halfDiag, radius);
  return cudaGetLastError();
}

cudaError_t launchCellCuts(const EbgMeshView& m, const SeedCellsView& v, float4* entries, uint32_t* count,
                           cudaStream_t s)
{
  const int64_t cells  = int64_t(v.g) * v.g * v.g;
  const int64_t blocks = (cells + CUT_WARPS - 1) / CUT_WARPS;
  kCellCuts<<<unsigned(blocks), CUT_WARPS * 32, 0, s>>>(m, v, entries, count);
  return cudaGetLastError();
}

} // namespace ebg
