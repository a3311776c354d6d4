// Learned pruning-radius model (no counterpart in the reference): a multiresolution hash-grid
// encoding (16 levels x 2 BF16 features, 2^log2T entries per level) feeding a 32-64-64-64-1 ReLU
// MLP whose matrix products run on the tensor cores as BF16 x BF16 -> FP32 warp MMAs
// (mma.sync m16n8k16).  Forward, backward and Adam are the kernels below; the exact mesh SDF path
// generates the training labels.
//
// Per warp the MLP works on a tile of 32 samples held in shared memory:
//   forward   H1 = relu(X W1^T + b1), H2 = relu(H1 W2^T + b2), H3 = relu(H2 W3^T + b3),
//             y = H3 w4 + b4                      (X: 32x32 encoding, H: 32x64, BF16 tiles)
//   backward  dH3 = dy w4^T (.) [H3>0]; dW3 += dH3^T H2; dH2 = dH3 W3 (.) [H2>0]; ...; dX = dH1 W1
// The weight-gradient products (dW = dH^T H, K = 32 samples) and the input-gradient products
// (dH_prev = dH W) are also m16n8k16 MMAs; weight gradients are summed per block in shared memory
// and then added to the global FP32 gradient; encoding gradients are scattered to the FP32 table
// gradient with atomics (several samples touch one entry).
#include <cfloat>
#include <cmath>
#include <cstdint>

#include "ebg_device.cuh"
#include "seed_kernels.h"

namespace ebg {

namespace {

constexpr int WARPS = 4;

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ uint32_t pack2(float lo, float hi)
{
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}

__device__ __forceinline__ uint32_t pack2b(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
  __nv_bfloat162 h;
  h.x = lo;
  h.y = hi;
  return *reinterpret_cast<uint32_t*>(&h);
}

// D = A(16x16, row) * B(16x8, col) + D, BF16 inputs, FP32 accumulate.
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float clamp01(float x) { return fminf(fmaxf(x, 0.f), 1.f); }

__device__ __forceinline__ uint32_t gridIndex(const SeedView& v, int l, int cx, int cy, int cz)
{
  const uint32_t T = 1u << v.log2T;
  if (v.dense[l]) {
    const uint32_t r = uint32_t(v.res[l]) + 1u;
    return (uint32_t(cz) * r + uint32_t(cy)) * r + uint32_t(cx);
  }
  return (uint32_t(cx) ^ (uint32_t(cy) * 2654435761u) ^ (uint32_t(cz) * 805459861u)) & (T - 1u);
}

struct Cell
{
  int   ix, iy, iz;
  float fx, fy, fz;
};

__device__ __forceinline__ Cell cellOf(const SeedView& v, int l, float ux, float uy, float uz)
{
  const float N = float(v.res[l]);
  const float x = ux * N, y = uy * N, z = uz * N;
  Cell        c;
  c.ix = min(int(floorf(x)), v.res[l] - 1);
  c.iy = min(int(floorf(y)), v.res[l] - 1);
  c.iz = min(int(floorf(z)), v.res[l] - 1);
  c.fx = x - float(c.ix);
  c.fy = y - float(c.iy);
  c.fz = z - float(c.iz);
  return c;
}

// 32 encoding features of one point (trilinear interpolation of the 8 cell corners per level).
__device__ void encode(const SeedView& v, float px, float py, float pz, float* feat)
{
  const float    ux = clamp01((px - v.lo[0]) * v.scale[0]), uy = clamp01((py - v.lo[1]) * v.scale[1]),
              uz = clamp01((pz - v.lo[2]) * v.scale[2]);
  const uint32_t T = 1u << v.log2T;
  const __nv_bfloat162* tab = reinterpret_cast<const __nv_bfloat162*>(v.table);
#pragma unroll 1
  for (int l = 0; l < SEED_LEVELS; l++) {
    const Cell c  = cellOf(v, l, ux, uy, uz);
    float      f0 = 0.f, f1 = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int   dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
      const float w  = (dx ? c.fx : 1.f - c.fx) * (dy ? c.fy : 1.f - c.fy) * (dz ? c.fz : 1.f - c.fz);
      const uint32_t idx = gridIndex(v, l, c.ix + dx, c.iy + dy, c.iz + dz);
      const float2   e   = __bfloat1622float2(tab[size_t(l) * T + idx]);
      f0 = fmaf(w, e.x, f0);
      f1 = fmaf(w, e.y, f1);
    }
    feat[2 * l]     = f0;
    feat[2 * l + 1] = f1;
  }
}

__device__ void encodeBackward(const SeedView& v, float px, float py, float pz, const float* dfeat, float* gradTable)
{
  const float    ux = clamp01((px - v.lo[0]) * v.scale[0]), uy = clamp01((py - v.lo[1]) * v.scale[1]),
              uz = clamp01((pz - v.lo[2]) * v.scale[2]);
  const uint32_t T = 1u << v.log2T;
#pragma unroll 1
  for (int l = 0; l < SEED_LEVELS; l++) {
    const Cell  c  = cellOf(v, l, ux, uy, uz);
    const float g0 = dfeat[2 * l], g1 = dfeat[2 * l + 1];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int   dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
      const float w  = (dx ? c.fx : 1.f - c.fx) * (dy ? c.fy : 1.f - c.fy) * (dz ? c.fz : 1.f - c.fz);
      const uint32_t idx = gridIndex(v, l, c.ix + dx, c.iy + dy, c.iz + dz);
      // both features of the entry in one vector atomic (global memory, sm_90 and later)
      atomicAdd(reinterpret_cast<float2*>(gradTable + (size_t(l) * T + idx) * 2), make_float2(w * g0, w * g1));
    }
  }
}

// Shared-memory layout of the block's weights (BF16, [out][in] rows) and biases (FP32).
struct SmemWeights
{
  __nv_bfloat16 w1[SEED_WIDTH * SEED_IN];
  __nv_bfloat16 w2[SEED_WIDTH * SEED_WIDTH];
  __nv_bfloat16 w3[SEED_WIDTH * SEED_WIDTH];
  __nv_bfloat16 w4[SEED_WIDTH];
  float         b1[SEED_WIDTH], b2[SEED_WIDTH], b3[SEED_WIDTH];
  float         b4;
};

struct WarpTiles
{
  __nv_bfloat16 x[32 * SEED_IN];
  __nv_bfloat16 h1[32 * SEED_WIDTH], h2[32 * SEED_WIDTH], h3[32 * SEED_WIDTH];
};

__device__ void stageWeights(const float* __restrict__ p, SmemWeights& w)
{
  for (int i = threadIdx.x; i < SEED_WIDTH * SEED_IN; i += blockDim.x) {
    w.w1[i] = __float2bfloat16_rn(p[SEED_W1 + i]);
  }
  for (int i = threadIdx.x; i < SEED_WIDTH * SEED_WIDTH; i += blockDim.x) {
    w.w2[i] = __float2bfloat16_rn(p[SEED_W2 + i]);
    w.w3[i] = __float2bfloat16_rn(p[SEED_W3 + i]);
  }
  for (int i = threadIdx.x; i < SEED_WIDTH; i += blockDim.x) {
    w.w4[i] = __float2bfloat16_rn(p[SEED_W4 + i]);
    w.b1[i] = p[SEED_B1 + i];
    w.b2[i] = p[SEED_B2 + i];
    w.b3[i] = p[SEED_B3 + i];
  }
  if (threadIdx.x == 0) {
    w.b4 = p[SEED_B4];
  }
}

// out[32][64] = relu(in[32][K] W^T + b), BF16 tiles, one warp.
template <int K>
__device__ void layerForward(const __nv_bfloat16* in, const __nv_bfloat16* W, const float* bias, __nv_bfloat16* out,
                             int lane)
{
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; mt++) {
    uint32_t a[K / 16][4];
#pragma unroll
    for (int kc = 0; kc < K / 16; kc++) {
      const __nv_bfloat16* r0 = in + (mt * 16 + g) * K + kc * 16 + 2 * t;
      const __nv_bfloat16* r1 = r0 + 8 * K;
      a[kc][0]                = ld32(r0);
      a[kc][1]                = ld32(r1);
      a[kc][2]                = ld32(r0 + 8);
      a[kc][3]                = ld32(r1 + 8);
    }
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const int n0   = nt * 8 + 2 * t;
      float     c[4] = {bias[n0], bias[n0 + 1], bias[n0], bias[n0 + 1]};
#pragma unroll
      for (int kc = 0; kc < K / 16; kc++) {
        const __nv_bfloat16* wr = W + (nt * 8 + g) * K + kc * 16 + 2 * t;
        mma16816(c, a[kc], ld32(wr), ld32(wr + 8));
      }
      *reinterpret_cast<uint32_t*>(out + (mt * 16 + g) * SEED_WIDTH + n0)     = pack2(fmaxf(c[0], 0.f), fmaxf(c[1], 0.f));
      *reinterpret_cast<uint32_t*>(out + (mt * 16 + g + 8) * SEED_WIDTH + n0) = pack2(fmaxf(c[2], 0.f), fmaxf(c[3], 0.f));
    }
  }
}

// Forward of the 32 samples whose encodings are in tiles.x; returns sample `lane`'s output.
__device__ float mlpForward(const SmemWeights& w, WarpTiles& tl, int lane)
{
  layerForward<SEED_IN>(tl.x, w.w1, w.b1, tl.h1, lane);
  __syncwarp();
  layerForward<SEED_WIDTH>(tl.h1, w.w2, w.b2, tl.h2, lane);
  __syncwarp();
  layerForward<SEED_WIDTH>(tl.h2, w.w3, w.b3, tl.h3, lane);
  __syncwarp();
  float y = w.b4;
#pragma unroll 8
  for (int n = 0; n < SEED_WIDTH; n++) {
    y = fmaf(__bfloat162float(tl.h3[lane * SEED_WIDTH + n]), __bfloat162float(w.w4[n]), y);
  }
  return y;
}

__device__ void storeFeatures(WarpTiles& tl, int lane, const float* feat)
{
#pragma unroll
  for (int k = 0; k < SEED_IN; k += 2) {
    *reinterpret_cast<uint32_t*>(tl.x + lane * SEED_IN + k) = pack2(feat[k], feat[k + 1]);
  }
}

// ---- backward helpers -------------------------------------------------------------------------

// gW[n][k] += sum_m D[m][n] H[m][k]; D FP32 [32][64], H BF16 [32][K]; MMA with M = 64 (n),
// N = K (k), reduction over the 32 samples.
template <int K>
__device__ void weightGrad(const float* D, const __nv_bfloat16* H, float* gW, int lane)
{
  const int g = lane >> 2, t = lane & 3;
#pragma unroll 1
  for (int mt = 0; mt < 4; mt++) {
    uint32_t a[2][4];
#pragma unroll
    for (int kc = 0; kc < 2; kc++) {
      const int n0 = mt * 16 + g, m0 = kc * 16 + 2 * t;
      a[kc][0]     = pack2(D[m0 * SEED_WIDTH + n0], D[(m0 + 1) * SEED_WIDTH + n0]);
      a[kc][1]     = pack2(D[m0 * SEED_WIDTH + n0 + 8], D[(m0 + 1) * SEED_WIDTH + n0 + 8]);
      a[kc][2]     = pack2(D[(m0 + 8) * SEED_WIDTH + n0], D[(m0 + 9) * SEED_WIDTH + n0]);
      a[kc][3]     = pack2(D[(m0 + 8) * SEED_WIDTH + n0 + 8], D[(m0 + 9) * SEED_WIDTH + n0 + 8]);
    }
#pragma unroll
    for (int nt = 0; nt < K / 8; nt++) {
      float     c[4] = {0.f, 0.f, 0.f, 0.f};
      const int k0   = nt * 8 + g;
#pragma unroll
      for (int kc = 0; kc < 2; kc++) {
        const int m0 = kc * 16 + 2 * t;
        const uint32_t b0 = pack2b(H[m0 * K + k0], H[(m0 + 1) * K + k0]);
        const uint32_t b1 = pack2b(H[(m0 + 8) * K + k0], H[(m0 + 9) * K + k0]);
        mma16816(c, a[kc], b0, b1);
      }
      const int n0 = mt * 16 + g, kk = nt * 8 + 2 * t;
      atomicAdd(gW + n0 * K + kk, c[0]);
      atomicAdd(gW + n0 * K + kk + 1, c[1]);
      atomicAdd(gW + (n0 + 8) * K + kk, c[2]);
      atomicAdd(gW + (n0 + 8) * K + kk + 1, c[3]);
    }
  }
}

// gb[n] += sum_m D[m][n]
__device__ void biasGrad(const float* D, float* gb, int lane)
{
  for (int n = lane; n < SEED_WIDTH; n += 32) {
    float s = 0.f;
    for (int m = 0; m < 32; m++) {
      s += D[m * SEED_WIDTH + n];
    }
    atomicAdd(gb + n, s);
  }
}

// P[m][k] = (sum_n D[m][n] W[n][k]) * [H[m][k] > 0]  (mask skipped when H is null); P FP32 with
// row stride ldP; W BF16 [64][K].
template <int K>
__device__ void inputGrad(const float* D, const __nv_bfloat16* W, const __nv_bfloat16* H, float* P, int ldP, int lane)
{
  const int g = lane >> 2, t = lane & 3;
#pragma unroll 1
  for (int mt = 0; mt < 2; mt++) {
    uint32_t a[4][4];
#pragma unroll
    for (int kc = 0; kc < 4; kc++) {
      const float* r0 = D + (mt * 16 + g) * SEED_WIDTH + kc * 16 + 2 * t;
      const float* r1 = r0 + 8 * SEED_WIDTH;
      a[kc][0]        = pack2(r0[0], r0[1]);
      a[kc][1]        = pack2(r1[0], r1[1]);
      a[kc][2]        = pack2(r0[8], r0[9]);
      a[kc][3]        = pack2(r1[8], r1[9]);
    }
#pragma unroll
    for (int nt = 0; nt < K / 8; nt++) {
      float     c[4] = {0.f, 0.f, 0.f, 0.f};
      const int k0   = nt * 8 + g;
#pragma unroll
      for (int kc = 0; kc < 4; kc++) {
        const int      n0 = kc * 16 + 2 * t;
        const uint32_t b0 = pack2b(W[n0 * K + k0], W[(n0 + 1) * K + k0]);
        const uint32_t b1 = pack2b(W[(n0 + 8) * K + k0], W[(n0 + 9) * K + k0]);
        mma16816(c, a[kc], b0, b1);
      }
      const int r = mt * 16 + g, kk = nt * 8 + 2 * t;
      if (H != nullptr) {
        c[0] = __bfloat162float(H[r * K + kk]) > 0.f ? c[0] : 0.f;
        c[1] = __bfloat162float(H[r * K + kk + 1]) > 0.f ? c[1] : 0.f;
        c[2] = __bfloat162float(H[(r + 8) * K + kk]) > 0.f ? c[2] : 0.f;
        c[3] = __bfloat162float(H[(r + 8) * K + kk + 1]) > 0.f ? c[3] : 0.f;
      }
      P[r * ldP + kk]           = c[0];
      P[r * ldP + kk + 1]       = c[1];
      P[(r + 8) * ldP + kk]     = c[2];
      P[(r + 8) * ldP + kk + 1] = c[3];
    }
  }
}

struct TrainSmem
{
  SmemWeights w;
  float       grad[SEED_NPARAM];
  WarpTiles   tiles[WARPS];
  float       d0[WARPS][32 * SEED_WIDTH];
  float       d1[WARPS][32 * SEED_WIDTH];
};

__global__ void __launch_bounds__(WARPS * 32) kSeedTrain(const SeedTrainArgs a)
{
  extern __shared__ __align__(16) unsigned char smraw[];
  TrainSmem&     S    = *reinterpret_cast<TrainSmem*>(smraw);
  const int      lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  stageWeights(a.net.params, S.w);
  for (int i = threadIdx.x; i < SEED_NPARAM; i += blockDim.x) {
    S.grad[i] = 0.f;
  }
  __syncthreads();
  WarpTiles& tl = S.tiles[wid];
  float*     D0 = S.d0[wid];
  float*     D1 = S.d1[wid];
  const int  tiles = (a.batch + 31) / 32;
  float      lossAcc = 0.f;

  for (int tile = blockIdx.x * WARPS + wid; tile < tiles; tile += gridDim.x * WARPS) {
    const int     m     = tile * 32 + lane;
    const bool    valid = m < a.batch;
    const int64_t si    = (a.offset + (valid ? m : 0)) % a.poolSize;
    const float   px = a.points[3 * si], py = a.points[3 * si + 1], pz = a.points[3 * si + 2];
    const float   target = a.target[si];
    float         feat[SEED_IN];
    encode(a.net, px, py, pz, feat);
    storeFeatures(tl, lane, feat);
    __syncwarp();
    const float y = mlpForward(S.w, tl, lane);

    // loss = mean w (y - d)^2, w = 1 / (|d| + eps)^2 (relative error away from the surface)
    const float wgt  = 1.f / ((fabsf(target) + a.eps) * (fabsf(target) + a.eps));
    const float diff = y - target;
    const float dy   = valid ? 2.f * wgt * diff / float(a.batch) : 0.f;
    lossAcc += valid ? wgt * diff * diff : 0.f;

    // output layer: dW4[n] = sum_m H3[m][n] dy_m, db4 = sum_m dy_m, dH3 = dy w4 [H3 > 0]
    for (int n = lane; n < SEED_WIDTH; n += 32) {
      float s = 0.f;
      for (int mm = 0; mm < 32; mm++) {
        s = fmaf(__bfloat162float(tl.h3[mm * SEED_WIDTH + n]), __shfl_sync(FULL, dy, mm), s);
      }
      atomicAdd(S.grad + SEED_W4 + n, s);
    }
    {
      const float sdy = warpSum(dy);
      if (lane == 0) {
        atomicAdd(S.grad + SEED_B4, sdy);
      }
    }
    for (int n = 0; n < SEED_WIDTH; n++) {
      const float h = __bfloat162float(tl.h3[lane * SEED_WIDTH + n]);
      D0[lane * SEED_WIDTH + n] = h > 0.f ? dy * __bfloat162float(S.w.w4[n]) : 0.f;
    }
    __syncwarp();
    weightGrad<SEED_WIDTH>(D0, tl.h2, S.grad + SEED_W3, lane);
    biasGrad(D0, S.grad + SEED_B3, lane);
    inputGrad<SEED_WIDTH>(D0, S.w.w3, tl.h2, D1, SEED_WIDTH, lane);
    __syncwarp();
    weightGrad<SEED_WIDTH>(D1, tl.h1, S.grad + SEED_W2, lane);
    biasGrad(D1, S.grad + SEED_B2, lane);
    inputGrad<SEED_WIDTH>(D1, S.w.w2, tl.h1, D0, SEED_WIDTH, lane);
    __syncwarp();
    weightGrad<SEED_IN>(D0, tl.x, S.grad + SEED_W1, lane);
    biasGrad(D0, S.grad + SEED_B1, lane);
    inputGrad<SEED_IN>(D0, S.w.w1, nullptr, D1, SEED_IN, lane);
    __syncwarp();
    if (valid) {
      encodeBackward(a.net, px, py, pz, D1 + lane * SEED_IN, a.gradTable);
    }
    __syncwarp();
  }
  lossAcc = warpSum(lossAcc);
  if (lane == 0 && lossAcc != 0.f) {
    atomicAdd(a.lossSum, lossAcc);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < SEED_NPARAM; i += blockDim.x) {
    if (S.grad[i] != 0.f) {
      atomicAdd(a.gradParams + i, S.grad[i]);
    }
  }
}

// ---- inference with the activations in registers ---------------------------------------------
//
// The accumulator fragment of m16n8k16 (rows g, g+8; columns 2t, 2t+1 of an 8-wide n-tile) is, for
// two neighbouring n-tiles, exactly the A fragment of a 16-wide k-chunk of the next layer, so the
// hidden activations go from one layer's MMAs to the next without touching shared memory.

constexpr int PK_WARPS = 8;

struct PredSmem
{
  SmemWeights   w;
  __nv_bfloat16 x[PK_WARPS][32 * SEED_IN]; // encodings of the warp's 32 points
};

// c[nt] = bias + A x W^T restricted to n-tile nt, for one 16-row tile (W BF16 [64][K] rows in
// shared memory).
template <int K>
__device__ __forceinline__ void denseRegs(const uint32_t (&a)[K / 16][4], const __nv_bfloat16* W, const float* bias,
                                          float (&c)[8][4], int lane)
{
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    const int n0 = nt * 8 + 2 * t;
    c[nt][0]     = bias[n0];
    c[nt][1]     = bias[n0 + 1];
    c[nt][2]     = bias[n0];
    c[nt][3]     = bias[n0 + 1];
#pragma unroll
    for (int kc = 0; kc < K / 16; kc++) {
      const __nv_bfloat16* wr = W + (nt * 8 + g) * K + kc * 16 + 2 * t;
      mma16816(c[nt], a[kc], ld32(wr), ld32(wr + 8));
    }
  }
}

// ReLU, BF16 rounding and repacking of a layer's accumulators as the next layer's A fragments.
__device__ __forceinline__ void reluToA(const float (&c)[8][4], uint32_t (&a)[4][4])
{
#pragma unroll
  for (int kc = 0; kc < 4; kc++) {
    a[kc][0] = pack2(fmaxf(c[2 * kc][0], 0.f), fmaxf(c[2 * kc][1], 0.f));
    a[kc][1] = pack2(fmaxf(c[2 * kc][2], 0.f), fmaxf(c[2 * kc][3], 0.f));
    a[kc][2] = pack2(fmaxf(c[2 * kc + 1][0], 0.f), fmaxf(c[2 * kc + 1][1], 0.f));
    a[kc][3] = pack2(fmaxf(c[2 * kc + 1][2], 0.f), fmaxf(c[2 * kc + 1][3], 0.f));
  }
}

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// The network on the warp's 32 encodings in xt (row q = sample q); returns row `lane`'s output.
__device__ float mlpRegs(const SmemWeights& w, const __nv_bfloat16* xt, int lane)
{
  const int g = lane >> 2, t = lane & 3;
  // y[mt][h] = this lane's share of row 16 mt + 8 h + g of the output layer, then summed over the
  // four lanes sharing the row
  float y[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll 1
  for (int mt = 0; mt < 2; mt++) {
    uint32_t a1[2][4];
#pragma unroll
    for (int kc = 0; kc < 2; kc++) {
      const __nv_bfloat16* r0 = xt + (mt * 16 + g) * SEED_IN + kc * 16 + 2 * t;
      a1[kc][0]               = ld32(r0);
      a1[kc][1]               = ld32(r0 + 8 * SEED_IN);
      a1[kc][2]               = ld32(r0 + 8);
      a1[kc][3]               = ld32(r0 + 8 * SEED_IN + 8);
    }
    float    c[8][4];
    uint32_t a[4][4];
    denseRegs<SEED_IN>(a1, w.w1, w.b1, c, lane);
    reluToA(c, a);
    denseRegs<SEED_WIDTH>(a, w.w2, w.b2, c, lane);
    reluToA(c, a);
    denseRegs<SEED_WIDTH>(a, w.w3, w.b3, c, lane);
    float y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const float w0 = __bfloat162float(w.w4[nt * 8 + 2 * t]), w1 = __bfloat162float(w.w4[nt * 8 + 2 * t + 1]);
      y0 = fmaf(bf16r(fmaxf(c[nt][0], 0.f)), w0, fmaf(bf16r(fmaxf(c[nt][1], 0.f)), w1, y0));
      y1 = fmaf(bf16r(fmaxf(c[nt][2], 0.f)), w0, fmaf(bf16r(fmaxf(c[nt][3], 0.f)), w1, y1));
    }
    if (mt == 0) {
      y[0][0] = y0;
      y[0][1] = y1;
    }
    else {
      y[1][0] = y0;
      y[1][1] = y1;
    }
  }
#pragma unroll
  for (int mt = 0; mt < 2; mt++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      y[mt][h] += __shfl_xor_sync(FULL, y[mt][h], 1);
      y[mt][h] += __shfl_xor_sync(FULL, y[mt][h], 2);
    }
  }
  // row q = 16 mt + 8 h + g' lives on lane 4 g'; lane q takes its own row
  const int   srcLane = (lane & 7) * 4;
  const float r00 = __shfl_sync(FULL, y[0][0], srcLane), r01 = __shfl_sync(FULL, y[0][1], srcLane);
  const float r10 = __shfl_sync(FULL, y[1][0], srcLane), r11 = __shfl_sync(FULL, y[1][1], srcLane);
  const int   mtq = lane >> 4, hq = (lane >> 3) & 1;
  return w.b4 + (mtq == 0 ? (hq == 0 ? r00 : r01) : (hq == 0 ? r10 : r11));
}

// One prediction per point: lane q of a warp encodes point 32 * tile + q (clamped to n - 1), the
// warp runs the network on the 32 encodings.
__global__ void __launch_bounds__(PK_WARPS * 32, 2) kSeedPredict(const SeedView v, const float* __restrict__ pts,
                                                              int64_t n, float* __restrict__ out)
{
  extern __shared__ __align__(16) unsigned char smraw[];
  PredSmem&      S    = *reinterpret_cast<PredSmem*>(smraw);
  const int      lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  stageWeights(v.params, S.w);
  __syncthreads();
  __nv_bfloat16* xt    = S.x[wid];
  const int64_t  tiles = (n + 31) / 32;
  for (int64_t tile = int64_t(blockIdx.x) * PK_WARPS + wid; tile < tiles; tile += int64_t(gridDim.x) * PK_WARPS) {
    const int64_t i  = tile * 32 + lane;
    const int64_t ii = i < n ? i : n - 1;
    float         feat[SEED_IN];
    encode(v, __ldg(pts + 3 * ii), __ldg(pts + 3 * ii + 1), __ldg(pts + 3 * ii + 2), feat);
#pragma unroll
    for (int k = 0; k < SEED_IN; k += 2) {
      *reinterpret_cast<uint32_t*>(xt + lane * SEED_IN + k) = pack2(feat[k], feat[k + 1]);
    }
    __syncwarp();
    const float y = mlpRegs(S.w, xt, lane);
    if (i < n) {
      out[i] = y;
    }
    __syncwarp();
  }
}

__global__ void kAdam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                      int64_t n, float lr, float b1, float b2, float eps, float c1, float c2,
                      __nv_bfloat16* __restrict__ shadow)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i]           = mi;
    v[i]           = vi;
    const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    p[i]           = pi;
    g[i]           = 0.f;
    if (shadow) {
      shadow[i] = __float2bfloat16_rn(pi);
    }
  }
}

__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ float u01(uint64_t seed, uint64_t i, uint32_t k)
{
  return float(mix64(seed ^ mix64(i * 8 + k)) >> 40) * (1.f / 16777216.f);
}

__global__ void kInitUniform(float* p, int64_t n, float lo, float hi, uint64_t seed)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    p[i] = lo + (hi - lo) * u01(seed, uint64_t(i), 0);
  }
}

__global__ void kToBf16(const float* s, __nv_bfloat16* d, int64_t n)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    d[i] = __float2bfloat16_rn(s[i]);
  }
}

__global__ void kSampleUniform(float* out, int64_t n, float lx, float ly, float lz, float hx, float hy, float hz,
                               uint64_t seed, int stride)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    float* o = out + 3 * i * stride;
    o[0]     = lx + (hx - lx) * u01(seed, uint64_t(i), 0);
    o[1]     = ly + (hy - ly) * u01(seed, uint64_t(i), 1);
    o[2]     = lz + (hz - lz) * u01(seed, uint64_t(i), 2);
  }
}

__global__ void kSampleBand(float* out, int64_t n, const double* __restrict__ cdf, int64_t nt,
                            const double* __restrict__ tri, float width, uint64_t seed, int stride)
{
  const double total = cdf[nt - 1];
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const double u  = double(u01(seed, uint64_t(i), 0)) * total;
    int64_t      lo = 0, hi = nt - 1;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (cdf[mid] <= u) {
        lo = mid + 1;
      }
      else {
        hi = mid;
      }
    }
    const double* t  = tri + 30 * size_t(lo);
    const double  r1 = sqrt(double(u01(seed, uint64_t(i), 1))), r2 = double(u01(seed, uint64_t(i), 2));
    const double  a = 1.0 - r1, b = r1 * (1.0 - r2), c = r1 * r2;
    const double  off = (2.0 * double(u01(seed, uint64_t(i), 3)) - 1.0) * double(width);
    for (int k = 0; k < 3; k++) {
      out[3 * i * stride + k] = float(a * t[k] + b * t[3 + k] + c * t[6 + k] + off * t[9 + k]);
    }
  }
}

template <class S>
cudaError_t setSmem(const void* fn)
{
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(S)));
}

} // namespace

void seedLevels(int baseRes, int maxRes, uint32_t log2T, SeedView& v)
{
  const double b = std::exp((std::log(double(maxRes)) - std::log(double(baseRes))) / double(SEED_LEVELS - 1));
  const double T = double(1u << log2T);
  for (int l = 0; l < SEED_LEVELS; l++) {
    v.res[l]   = int(std::floor(double(baseRes) * std::pow(b, double(l)) + 1e-9));
    v.dense[l] = std::pow(double(v.res[l] + 1), 3.0) <= T ? 1 : 0;
  }
  v.log2T = log2T;
}

cudaError_t launchSeedTrainStep(const SeedTrainArgs& a, int numSms, cudaStream_t s)
{
  // the dynamic shared-memory opt-in is per device, so it is set on every launch (cheap)
  const cudaError_t e = setSmem<TrainSmem>(reinterpret_cast<const void*>(kSeedTrain));
  if (e != cudaSuccess) {
    return e;
  }
  const int tiles  = (a.batch + 31) / 32;
  int       blocks = (tiles + WARPS - 1) / WARPS;
  blocks           = blocks < numSms ? blocks : numSms;
  kSeedTrain<<<blocks, WARPS * 32, sizeof(TrainSmem), s>>>(a);
  return cudaGetLastError();
}

cudaError_t launchSeedPredict(const SeedView& v, const float* pts, int64_t n, float* out, int numSms, cudaStream_t s)
{
  // the dynamic shared-memory opt-in is per device, so it is set on every launch (cheap)
  const cudaError_t e = setSmem<PredSmem>(reinterpret_cast<const void*>(kSeedPredict));
  if (e != cudaSuccess) {
    return e;
  }
  const int64_t tiles  = (n + 31) / 32;
  int64_t       blocks = (tiles + PK_WARPS - 1) / PK_WARPS;
  blocks               = blocks < int64_t(numSms) * 2 ? blocks : int64_t(numSms) * 2;
  blocks               = blocks < 1 ? 1 : blocks;
  kSeedPredict<<<unsigned(blocks), PK_WARPS * 32, sizeof(PredSmem), s>>>(v, pts, n, out);
  return cudaGetLastError();
}

cudaError_t launchAdam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                       int step, __nv_bfloat16* shadow, cudaStream_t s)
{
  const float c1 = 1.f / (1.f - std::pow(b1, float(step)));
  const float c2 = 1.f / (1.f - std::pow(b2, float(step)));
  kAdam<<<2048, 256, 0, s>>>(p, const_cast<float*>(g), m, v, n, lr, b1, b2, eps, c1, c2, shadow);
  return cudaGetLastError();
}

cudaError_t launchInitUniform(float* p, int64_t n, float lo, float hi, uint64_t seed, cudaStream_t s)
{
  kInitUniform<<<1024, 256, 0, s>>>(p, n, lo, hi, seed);
  return cudaGetLastError();
}

cudaError_t launchToBf16(const float* src, __nv_bfloat16* dst, int64_t n, cudaStream_t s)
{
  kToBf16<<<1024, 256, 0, s>>>(src, dst, n);
  return cudaGetLastError();
}

cudaError_t launchSampleUniform(float* out, int64_t n, const float* lo, const float* hi, uint64_t seed, int stride,
                                cudaStream_t s)
{
  kSampleUniform<<<2048, 256, 0, s>>>(out, n, lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], seed, stride);
  return cudaGetLastError();
}

cudaError_t launchSampleBand(float* out, int64_t n, const double* cdf, int64_t nt, const double* tri64, float width,
                             uint64_t seed, int stride, cudaStream_t s)
{
  kSampleBand<<<2048, 256, 0, s>>>(out, n, cdf, nt, tri64, width, seed, stride);
  return cudaGetLastError();
}

} // namespace ebg
