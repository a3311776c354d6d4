// Learned pruning-radius model: multiresolution hash-grid encoding + BF16 MLP (sm_100a).
#ifndef EBG_SEED_KERNELS_H
#define EBG_SEED_KERNELS_H

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace ebg {

constexpr int SEED_LEVELS   = 16;  // hash-grid levels
constexpr int SEED_FEATS    = 2;   // features per level
constexpr int SEED_IN       = SEED_LEVELS * SEED_FEATS;  // 32 MLP inputs
constexpr int SEED_WIDTH    = 64;  // hidden width (3 hidden layers)
// flat FP32 parameter layout of the MLP (master copy, gradients and Adam moments share it)
constexpr int SEED_W1 = 0;                                 // [64][32]  (out, in)
constexpr int SEED_B1 = SEED_W1 + SEED_WIDTH * SEED_IN;    // [64]
constexpr int SEED_W2 = SEED_B1 + SEED_WIDTH;              // [64][64]
constexpr int SEED_B2 = SEED_W2 + SEED_WIDTH * SEED_WIDTH; // [64]
constexpr int SEED_W3 = SEED_B2 + SEED_WIDTH;              // [64][64]
constexpr int SEED_B3 = SEED_W3 + SEED_WIDTH * SEED_WIDTH; // [64]
constexpr int SEED_W4 = SEED_B3 + SEED_WIDTH;              // [64]
constexpr int SEED_B4 = SEED_W4 + SEED_WIDTH;              // [1]
constexpr int SEED_NPARAM = SEED_B4 + 1;                   // 10,497

// Device view of the model.  The hash tables are level-major: entry e of level l holds features
// table[(l * T + e) * 2 + f].
struct SeedView
{
  const __nv_bfloat16* table;  // BF16 features (forward)
  const float*         params; // FP32 MLP parameters (converted to BF16 when staged into shared memory)
  uint32_t             log2T;
  int                  res[SEED_LEVELS];   // grid resolution per level
  int                  dense[SEED_LEVELS]; // 1: (res+1)^3 <= T, direct indexing; 0: spatial hash
  float                lo[3], scale[3];    // u = (p - lo) * scale maps the domain to [0,1]^3
  float                alpha, beta;        // radius = (1 + alpha) |prediction| + beta
};

struct SeedTrainArgs
{
  SeedView      net;
  const float*  points;   // samples (xyz)
  const float*  target;   // exact signed distances
  int64_t       offset;   // first sample of this step in the (cyclic) pool
  int64_t       poolSize;
  int           batch;
  float*        gradTable; // FP32 [L][T][2]
  float*        gradParams; // FP32 [NPARAM]
  float*        lossSum;    // accumulated loss (diagnostics)
  float         eps;        // loss weight floor: w = 1 / (|d| + eps)^2
  int*          status;     // device status word: ST_COPY when a wait for the tensor cores gave up
  __nv_bfloat16* feat;      // workspace: the batch's encodings, [batch][32]
  float*         dfeat;     // workspace: their gradients, [batch][32]
};

void        seedLevels(int baseRes, int maxRes, uint32_t log2T, SeedView& v);
cudaError_t launchSeedTrainStep(const SeedTrainArgs& a, int numSms, cudaStream_t s);
cudaError_t launchSeedPredict(const SeedView& v, const float* pts, int64_t n, float* out, int numSms, cudaStream_t s);
cudaError_t launchAdam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                       int step, __nv_bfloat16* shadow, cudaStream_t s);
cudaError_t launchInitUniform(float* p, int64_t n, float lo, float hi, uint64_t seed, cudaStream_t s);
cudaError_t launchToBf16(const float* src, __nv_bfloat16* dst, int64_t n, cudaStream_t s);
// Training samples: n uniform points in [lo, hi] and n points within +-width of the surface
// (triangle by area through the cumulative-area table, uniform barycentric, offset along the
// face normal), from the FP64 leaf-order triangle records (30 doubles each).
// Point i is written at out + 3 * i * stride.
cudaError_t launchSampleUniform(float* out, int64_t n, const float* lo, const float* hi, uint64_t seed, int stride,
                                cudaStream_t s);
cudaError_t launchSampleBand(float* out, int64_t n, const double* cdf, int64_t nt, const double* tri64, float width,
                             uint64_t seed, int stride, cudaStream_t s);

} // namespace ebg

#endif
