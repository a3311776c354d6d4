// Learned pruning-radius model (no counterpart in the reference): a multiresolution hash-grid
// encoding (16 levels x 2 BF16 features, 2^log2T entries per level) feeding a 32-64-64-64-1 ReLU
// MLP.  The exact mesh SDF path generates the training labels.
//
// A training step is three kernels: kSeedEncode writes the batch's encodings (BF16); kSeedTrainTc
// runs the MLP's forward and backward on the fifth-generation tensor cores (tiles of 128 samples,
// BF16 operands in shared memory, FP32 products in tensor memory through tcgen05.mma, the weight
// gradients accumulated there over all of a CTA's tiles) and writes each sample's input gradient;
// kSeedEncodeBackward scatters those to the FP32 table gradient with vector atomics (several
// samples touch one entry).  Adam then updates the FP32 master copies and refreshes the BF16 table.
//
// Inference (kSeedPredict: the attach's one prediction per cell, and the far-field surrogate)
// keeps a warp's 32 activations in registers between layers on m16n8k16 warp MMAs.
#include <cfloat>
#include <cmath>
#include <cstdint>

#include "ebg_device.cuh"
#include "seed_kernels.h"
#include "tc_sm100.cuh"

namespace ebg {

namespace {

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ uint32_t pack2(float lo, float hi)
{
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
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

// x rounded to BF16 (round to nearest even), as a float
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

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

// ---- training on the fifth-generation tensor cores (tcgen05) ----------------------------------
//
// One CTA of 128 threads works on tiles of 128 samples: thread t owns sample t of the tile, which
// is also row t of every MMA and lane t of tensor memory.  Per tile (all products BF16 x BF16 ->
// FP32 in TMEM, issued by thread 0, completion through one mbarrier):
//   forward   D = X W1^T -> H1 = relu(D + b1); D = H1 W2^T -> H2; D = H2 W3^T -> H3; y = H3 . w4 + b4
//   backward  dH3 = dy w4 [H3 > 0]; D = dH3 W3 -> dH2 (.) [H2 > 0]; D = dH2 W2 -> dH1 (.) [H1 > 0];
//             D = dH1 W1 -> dX (written out for kSeedEncodeBackward)
// The weight gradients accumulate over all of the CTA's tiles in TMEM, as two M = 128 products over
// the tile's 128 samples (K):
//   Gw32 += [dH3^T; dH2^T] [H2^T; H1^T; 1]^T   rows 0-63: dW3 | db3, rows 64-127: dW2 | db2
//   Gw1  += [H3^T; dH1^T] [X^T; 1; dy]^T       rows 0-63: dW4 (column dy), rows 64-127: dW1 | db1
// (a row of ones gives the bias gradients as sums over the samples; the off-diagonal blocks are
// not used).  The transposed activations are written by each thread as its own column.

namespace tcs {

constexpr int      TILE = 128;
constexpr uint32_t LBO  = 128;     // K-adjacent core matrices are contiguous
constexpr uint32_t SBO32  = 4 * 128;  // R-adjacent core matrices of a K = 32 tile
constexpr uint32_t SBO64  = 8 * 128;  // K = 64
// Tiles whose K is the tile's 128 samples are written a column (one sample) per thread; their
// K-adjacent core matrices sit 144 bytes apart, so that the 2-byte stores of a warp's 32 samples
// fall in distinct shared-memory banks.
constexpr uint32_t LBO_S = 144;
constexpr uint32_t SBO_S = 16 * LBO_S;
constexpr uint32_t N_W32 = 144;       // H2^T (64) + H1^T (64) + ones + 15 zero rows
constexpr uint32_t N_W1  = 48;        // X^T (32) + ones + dy + 14 zero rows
// TMEM columns (256 allocated): the two gradient accumulators and the per-layer product
constexpr uint32_t TM_W32 = 0, TM_W1 = 144, TM_D = 192, TM_COLS = 256;
constexpr uint32_t WAIT_POLLS = 1u << 22; // polls of one wait (64 ns sleeps): under half a second

struct alignas(128) Smem
{
  unsigned char w1[64 * 32 * 2], w2[64 * 64 * 2], w3[64 * 64 * 2];     // B of the forward products
  unsigned char w1t[32 * 64 * 2], w2t[64 * 64 * 2], w3t[64 * 64 * 2];  // B of the input gradients
  unsigned char x[TILE * 32 * 2];                                       // A of layer 1
  unsigned char ha[TILE * 64 * 2];                                      // H1, then dH2
  unsigned char hb[TILE * 64 * 2];                                      // H2, then dH3, then dH1
  unsigned char t[256 / 8 * SBO_S];     // dH3^T, dH2^T, H3^T, dH1^T (rows), samples along K
  unsigned char bw32[N_W32 / 8 * SBO_S]; // H2^T, H1^T, ones, zeros
  unsigned char bw1[N_W1 / 8 * SBO_S];   // X^T, ones, dy, zeros
  float         b1[64], b2[64], b3[64], w4[64];
  float         b4;
  uint32_t      tmemSlot;
  uint64_t      bar;
};

__device__ __forceinline__ void st16(unsigned char* base, uint32_t off, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
  *reinterpret_cast<uint4*>(base + off) = make_uint4(a, b, c, d);
}

__device__ __forceinline__ void stb(unsigned char* base, uint32_t off, float v)
{
  *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

// Row r of an R x K tile (K-major) from 8 consecutive values per 16-byte chunk, rounded to BF16.
template <int K>
__device__ __forceinline__ void storeRow(unsigned char* tile, uint32_t sbo, int r, const float* v)
{
#pragma unroll
  for (int c = 0; c < K / 8; c++) {
    st16(tile, tc::kmajorOffset(uint32_t(r), uint32_t(8 * c), LBO, sbo), pack2(v[8 * c], v[8 * c + 1]),
         pack2(v[8 * c + 2], v[8 * c + 3]), pack2(v[8 * c + 4], v[8 * c + 5]), pack2(v[8 * c + 6], v[8 * c + 7]));
  }
}

// Column s (a sample) of rows r0 .. r0 + n - 1 of a tile whose K is the tile's samples.
__device__ __forceinline__ void storeCol(unsigned char* tile, int r0, int n, int s, const float* v)
{
  for (int i = 0; i < n; i++) {
    stb(tile, tc::kmajorOffset(uint32_t(r0 + i), uint32_t(s), LBO_S, SBO_S), v[i]);
  }
}

// W [R][K] (FP32, row-major) -> BF16 K-major tile; transposed: W^T [K][R].
__device__ void stageMatrix(const float* __restrict__ W, int R, int K, unsigned char* tile, unsigned char* tileT)
{
  for (int i = threadIdx.x; i < R * K; i += blockDim.x) {
    const int r = i / K, k = i - r * K;
    stb(tile, tc::kmajorOffset(uint32_t(r), uint32_t(k), LBO, uint32_t(K / 8) * 128u), W[i]);
    stb(tileT, tc::kmajorOffset(uint32_t(k), uint32_t(r), LBO, uint32_t(R / 8) * 128u), W[i]);
  }
}

// The per-layer product of this stage: operands written by every thread are made visible to the
// tensor cores, thread 0 issues `steps` K-steps of D = A B^T into TMEM column `dcol` (K = 16 each,
// the A and B tiles advancing 2 * LBO bytes per step), commits them, and every thread waits for
// them.  `extra` issues further products before the commit (they complete with it).  Returns
// false if the wait gave up.
template <class Extra>
__device__ __forceinline__ bool stage(uint32_t tmem, uint32_t dcol, uint32_t aAddr, uint32_t aSbo, uint32_t bAddr,
                                     uint32_t bSbo, uint32_t n, int steps, uint32_t bar, uint32_t& phase,
                                     Extra extra)
{
  tc::fenceProxyAsync();
  tc::fenceBeforeSync();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::fenceAfterSync();
    extra();
    for (int k = 0; k < steps; k++) {
      tc::mma(tmem + dcol, tc::smemDesc(aAddr + uint32_t(k) * 2u * LBO, LBO, aSbo),
              tc::smemDesc(bAddr + uint32_t(k) * 2u * LBO, LBO, bSbo), tc::idescBf16(n), k > 0 ? 1u : 0u);
    }
    tc::commit(bar);
  }
  const bool ok = tc::mbarWait(bar, phase, WAIT_POLLS);
  phase ^= 1u;
  tc::fenceAfterSync();
  return __syncthreads_and(ok) != 0;
}

struct NoExtra
{
  __device__ void operator()() const {}
};

// This thread's TMEM lane, columns [col, col + N) (N a multiple of 16).
template <int N>
__device__ __forceinline__ void loadRow(uint32_t tmem, uint32_t col, float* v)
{
  const uint32_t lane = (threadIdx.x & ~31u) << 16;
#pragma unroll
  for (int c = 0; c < N; c += 16) {
    float r[16];
    tc::ld16(tmem + lane + col + uint32_t(c), r);
#pragma unroll
    for (int i = 0; i < 16; i++) {
      v[c + i] = r[i];
    }
  }
}

__global__ void __launch_bounds__(TILE, 1) kSeedTrainTc(const SeedTrainArgs a)
{
  extern __shared__ __align__(128) unsigned char smraw[];
  Smem&     S = *reinterpret_cast<Smem*>(smraw);
  const int t = threadIdx.x;

  // weights (BF16, as the forward and backward products read them) and the constant rows
  stageMatrix(a.net.params + SEED_W1, 64, 32, S.w1, S.w1t);
  stageMatrix(a.net.params + SEED_W2, 64, 64, S.w2, S.w2t);
  stageMatrix(a.net.params + SEED_W3, 64, 64, S.w3, S.w3t);
  if (t < 64) {
    S.b1[t] = a.net.params[SEED_B1 + t];
    S.b2[t] = a.net.params[SEED_B2 + t];
    S.b3[t] = a.net.params[SEED_B3 + t];
    S.w4[t] = bf16r(a.net.params[SEED_W4 + t]);
  }
  if (t == 0) {
    S.b4 = a.net.params[SEED_B4];
  }
  for (int r = 128; r < int(N_W32); r++) {
    stb(S.bw32, tc::kmajorOffset(uint32_t(r), uint32_t(t), LBO_S, SBO_S), r == 128 ? 1.f : 0.f);
  }
  for (int r = 32; r < int(N_W1); r++) {
    stb(S.bw1, tc::kmajorOffset(uint32_t(r), uint32_t(t), LBO_S, SBO_S), r == 32 ? 1.f : 0.f);
  }
  const uint32_t bar = tc::smemAddr(&S.bar);
  if (t < 32) {
    tc::tmemAlloc(tc::smemAddr(&S.tmemSlot), TM_COLS);
  }
  if (t == 0) {
    tc::mbarInit(bar, 1);
  }
  tc::fenceBeforeSync();
  __syncthreads();
  tc::fenceAfterSync();
  const uint32_t tmem  = S.tmemSlot;
  uint32_t       phase = 0;
  bool           ok    = true;

  const uint32_t aX = tc::smemAddr(S.x), aHA = tc::smemAddr(S.ha), aHB = tc::smemAddr(S.hb);
  const uint32_t aT = tc::smemAddr(S.t), aW32 = tc::smemAddr(S.bw32), aW1 = tc::smemAddr(S.bw1);
  const int      tiles   = (a.batch + TILE - 1) / TILE;
  float          lossAcc = 0.f, dyAcc = 0.f;
  bool           first   = true;

  for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const int     m      = tile * TILE + t;
    const bool    valid  = m < a.batch;
    const int64_t si     = (a.offset + (valid ? m : 0)) % a.poolSize;
    const float   target = a.target[si];
    float         v[64]; // one row of a layer (registers: only constant indices reach it)

    // forward: the sample's encoding (BF16, from kSeedEncode; zeros past the batch), then three layers
    {
      uint4 xr[4] = {make_uint4(0u, 0u, 0u, 0u), make_uint4(0u, 0u, 0u, 0u), make_uint4(0u, 0u, 0u, 0u),
                     make_uint4(0u, 0u, 0u, 0u)};
      if (valid) {
        const uint4* src = reinterpret_cast<const uint4*>(a.feat + size_t(m) * SEED_IN);
#pragma unroll
        for (int c = 0; c < 4; c++) {
          xr[c] = __ldg(src + c);
        }
      }
#pragma unroll
      for (int c = 0; c < 4; c++) {
        *reinterpret_cast<uint4*>(S.x + tc::kmajorOffset(uint32_t(t), uint32_t(8 * c), LBO, SBO32)) = xr[c];
        const uint32_t w[4] = {xr[c].x, xr[c].y, xr[c].z, xr[c].w};
#pragma unroll
        for (int h = 0; h < 8; h++) {
          const unsigned short b = (unsigned short)(h & 1 ? (w[h >> 1] >> 16) : (w[h >> 1] & 0xffffu));
          *reinterpret_cast<unsigned short*>(S.bw1 + tc::kmajorOffset(uint32_t(8 * c + h), uint32_t(t), LBO_S, SBO_S)) = b;
        }
      }
    }
    ok = stage(tmem, TM_D, aX, SBO32, tc::smemAddr(S.w1), SBO32, 64, 2, bar, phase, NoExtra{});
    if (!ok) {
      break;
    }
    uint32_t mask1[2] = {0u, 0u}, mask2[2] = {0u, 0u};
    loadRow<64>(tmem, TM_D, v);
#pragma unroll
    for (int n = 0; n < 64; n++) {
      v[n] = bf16r(fmaxf(v[n] + S.b1[n], 0.f));
      mask1[n >> 5] |= (v[n] > 0.f ? 1u : 0u) << (n & 31);
    }
    storeRow<64>(S.ha, SBO64, t, v);
    storeCol(S.bw32, 64, 64, t, v);
    ok = stage(tmem, TM_D, aHA, SBO64, tc::smemAddr(S.w2), SBO64, 64, 4, bar, phase, NoExtra{});
    if (!ok) {
      break;
    }
    loadRow<64>(tmem, TM_D, v);
#pragma unroll
    for (int n = 0; n < 64; n++) {
      v[n] = bf16r(fmaxf(v[n] + S.b2[n], 0.f));
      mask2[n >> 5] |= (v[n] > 0.f ? 1u : 0u) << (n & 31);
    }
    storeRow<64>(S.hb, SBO64, t, v);
    storeCol(S.bw32, 0, 64, t, v);
    ok = stage(tmem, TM_D, aHB, SBO64, tc::smemAddr(S.w3), SBO64, 64, 4, bar, phase, NoExtra{});
    if (!ok) {
      break;
    }
    loadRow<64>(tmem, TM_D, v);
    float y = S.b4;
#pragma unroll
    for (int n = 0; n < 64; n++) {
      v[n] = bf16r(fmaxf(v[n] + S.b3[n], 0.f));
      y    = fmaf(v[n], S.w4[n], y);
    }
    storeCol(S.t, 128, 64, t, v); // H3^T

    // loss = mean w (y - d)^2, w = 1 / (|d| + eps)^2 (relative error away from the surface)
    const float wgt  = 1.f / ((fabsf(target) + a.eps) * (fabsf(target) + a.eps));
    const float diff = y - target;
    const float dy   = valid ? 2.f * wgt * diff / float(a.batch) : 0.f;
    lossAcc += valid ? wgt * diff * diff : 0.f;
    dyAcc += dy;
    stb(S.bw1, tc::kmajorOffset(33u, uint32_t(t), LBO_S, SBO_S), dy);

    // backward: dH3 = dy w4 [H3 > 0]
#pragma unroll
    for (int n = 0; n < 64; n++) {
      v[n] = v[n] > 0.f ? dy * S.w4[n] : 0.f;
    }
    storeRow<64>(S.hb, SBO64, t, v);
    storeCol(S.t, 0, 64, t, v); // dH3^T
    ok = stage(tmem, TM_D, aHB, SBO64, tc::smemAddr(S.w3t), SBO64, 64, 4, bar, phase, NoExtra{});
    if (!ok) {
      break;
    }
    loadRow<64>(tmem, TM_D, v);
#pragma unroll
    for (int n = 0; n < 64; n++) {
      v[n] = (mask2[n >> 5] >> (n & 31)) & 1u ? v[n] : 0.f;
    }
    storeRow<64>(S.ha, SBO64, t, v);
    storeCol(S.t, 64, 64, t, v); // dH2^T
    // with dH2 = dD W2: the layer-3 and layer-2 weight gradients accumulate first
    const uint32_t acc = first ? 0u : 1u;
    ok = stage(tmem, TM_D, aHA, SBO64, tc::smemAddr(S.w2t), SBO64, 64, 4, bar, phase, [&] {
      for (int k = 0; k < TILE / 16; k++) {
        tc::mma(tmem + TM_W32, tc::smemDesc(aT + uint32_t(k) * 2u * LBO_S, LBO_S, SBO_S),
                tc::smemDesc(aW32 + uint32_t(k) * 2u * LBO_S, LBO_S, SBO_S), tc::idescBf16(N_W32),
                (k > 0 || acc) ? 1u : 0u);
      }
    });
    if (!ok) {
      break;
    }
    loadRow<64>(tmem, TM_D, v);
#pragma unroll
    for (int n = 0; n < 64; n++) {
      v[n] = (mask1[n >> 5] >> (n & 31)) & 1u ? v[n] : 0.f;
    }
    storeRow<64>(S.hb, SBO64, t, v);
    storeCol(S.t, 192, 64, t, v); // dH1^T
    // dX = dH1 W1, after the layer-1 and output-layer weight gradients
    ok = stage(tmem, TM_D, aHB, SBO64, tc::smemAddr(S.w1t), SBO64, 32, 4, bar, phase, [&] {
      const uint32_t a1 = aT + 16u * SBO_S; // rows 128-255 of T: H3^T, dH1^T
      for (int k = 0; k < TILE / 16; k++) {
        tc::mma(tmem + TM_W1, tc::smemDesc(a1 + uint32_t(k) * 2u * LBO_S, LBO_S, SBO_S),
                tc::smemDesc(aW1 + uint32_t(k) * 2u * LBO_S, LBO_S, SBO_S), tc::idescBf16(N_W1),
                (k > 0 || acc) ? 1u : 0u);
      }
    });
    if (!ok) {
      break;
    }
    first = false;
    // dX, which kSeedEncodeBackward scatters to the hash tables' gradient
    loadRow<32>(tmem, TM_D, v);
    if (valid) {
      float4* dst = reinterpret_cast<float4*>(a.dfeat + size_t(m) * SEED_IN);
#pragma unroll
      for (int c = 0; c < SEED_IN / 4; c++) {
        dst[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
      }
    }
  }

  if (!ok) {
    if (t == 0) {
      atomicOr(a.status, ST_COPY);
    }
    // the products may still be running: wait once more (bounded) before the memory goes away
    tc::mbarWait(bar, phase ^ 1u, WAIT_POLLS);
  }
  else if (!first) {
    // this CTA's weight gradients, from the accumulators in TMEM
    const int o = t & 63;
    float     g[64];
    if (t < 64) {
      loadRow<64>(tmem, TM_W32, g); // dW3 row o
      for (int k = 0; k < 64; k++) {
        atomicAdd(a.gradParams + SEED_W3 + o * 64 + k, g[k]);
      }
    }
    else {
      loadRow<64>(tmem, TM_W32 + 64, g); // dW2 row o
      for (int k = 0; k < 64; k++) {
        atomicAdd(a.gradParams + SEED_W2 + o * 64 + k, g[k]);
      }
    }
    loadRow<16>(tmem, TM_W32 + 128, g); // column 128: the bias gradient of the row's layer
    atomicAdd(a.gradParams + (t < 64 ? SEED_B3 : SEED_B2) + o, g[0]);
    loadRow<48>(tmem, TM_W1, g);
    if (t < 64) {
      atomicAdd(a.gradParams + SEED_W4 + o, g[33]);
    }
    else {
      for (int k = 0; k < 32; k++) {
        atomicAdd(a.gradParams + SEED_W1 + o * 32 + k, g[k]);
      }
      atomicAdd(a.gradParams + SEED_B1 + o, g[32]);
    }
    const float sdy = warpSum(dyAcc);
    if ((t & 31) == 0 && sdy != 0.f) {
      atomicAdd(a.gradParams + SEED_B4, sdy);
    }
  }
  lossAcc = warpSum(lossAcc);
  if ((t & 31) == 0 && lossAcc != 0.f) {
    atomicAdd(a.lossSum, lossAcc);
  }
  tc::fenceBeforeSync();
  __syncthreads();
  if (t < 32) {
    tc::fenceAfterSync();
    tc::tmemDealloc(tmem, TM_COLS);
  }
}

// The encodings of a training step's samples (BF16 rows of 32, the MLP's input as the training
// kernel reads it), one sample per thread at full occupancy: its 16 x 8 table reads are the step's
// latency-bound part.
__global__ void __launch_bounds__(256) kSeedEncode(const SeedTrainArgs a)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.batch; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t si = (a.offset + i) % a.poolSize;
    float         feat[SEED_IN];
    encode(a.net, a.points[3 * si], a.points[3 * si + 1], a.points[3 * si + 2], feat);
    uint4* dst = reinterpret_cast<uint4*>(a.feat + size_t(i) * SEED_IN);
#pragma unroll
    for (int c = 0; c < 4; c++) {
      dst[c] = make_uint4(pack2(feat[8 * c], feat[8 * c + 1]), pack2(feat[8 * c + 2], feat[8 * c + 3]),
                          pack2(feat[8 * c + 4], feat[8 * c + 5]), pack2(feat[8 * c + 6], feat[8 * c + 7]));
    }
  }
}

// The encoding's gradient: each sample's dX (from the training kernel) scattered to the FP32
// table gradient through its 16 x 8 corners, one sample per thread at full occupancy.
__global__ void __launch_bounds__(256) kSeedEncodeBackward(const SeedTrainArgs a)
{
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.batch; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t si = (a.offset + i) % a.poolSize;
    float         dx[SEED_IN];
    const float4* src = reinterpret_cast<const float4*>(a.dfeat + size_t(i) * SEED_IN);
#pragma unroll
    for (int c = 0; c < SEED_IN / 4; c++) {
      const float4 q = __ldg(src + c);
      dx[4 * c]      = q.x;
      dx[4 * c + 1]  = q.y;
      dx[4 * c + 2]  = q.z;
      dx[4 * c + 3]  = q.w;
    }
    encodeBackward(a.net, a.points[3 * si], a.points[3 * si + 1], a.points[3 * si + 2], dx, a.gradTable);
  }
}

} // namespace tcs

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
  const cudaError_t e = setSmem<tcs::Smem>(reinterpret_cast<const void*>(tcs::kSeedTrainTc));
  if (e != cudaSuccess) {
    return e;
  }
  // the encodings, then the MLP's forward and backward on the tensor cores (one CTA per SM at
  // most: its shared memory allows no second one, so its TMEM allocation never waits for another
  // CTA's), then the encodings' gradient
  const int64_t nb   = (int64_t(a.batch) + 255) / 256;
  const int     gEnc = int(nb < int64_t(numSms) * 8 ? nb : int64_t(numSms) * 8);
  tcs::kSeedEncode<<<gEnc > 0 ? gEnc : 1, 256, 0, s>>>(a);
  const int tiles  = (a.batch + tcs::TILE - 1) / tcs::TILE;
  const int blocks = tiles < numSms ? tiles : numSms;
  tcs::kSeedTrainTc<<<blocks, tcs::TILE, sizeof(tcs::Smem), s>>>(a);
  tcs::kSeedEncodeBackward<<<gEnc > 0 ? gEnc : 1, 256, 0, s>>>(a);
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
