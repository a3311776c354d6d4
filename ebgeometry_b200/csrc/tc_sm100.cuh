// Fifth-generation tensor-core helpers for sm_100a: tensor-memory (TMEM) allocation, tcgen05.mma
// with BF16 operands in shared memory and an FP32 accumulator in TMEM, completion through an
// mbarrier, and TMEM loads.  Written from the PTX ISA's descriptions of these instructions.
//
// Operand layout (both A and B, "K-major, no swizzle"): an R x K BF16 tile (R rows along M or N,
// K the reduction dimension) is made of core matrices of 8 rows x 8 elements (16 bytes per row,
// 128 bytes per core matrix, rows 16 bytes apart).  Core matrix (r / 8, k / 8) starts at
//   (r / 8) * sbo + (k / 8) * lbo
// bytes from the tile's start: `lbo` is the distance between core matrices adjacent along K,
// `sbo` between core matrices adjacent along R.  One kind::f16 MMA consumes K = 16 (two core
// matrices along K); the next K step starts 2 * lbo bytes further.
#ifndef EBG_TC_SM100_CUH
#define EBG_TC_SM100_CUH

#include <cstdint>

namespace ebg {
namespace tc {

// Byte offset of element (r, k) in a K-major tile with strides lbo (along K) and sbo (along R).
__host__ __device__ constexpr uint32_t kmajorOffset(uint32_t r, uint32_t k, uint32_t lbo, uint32_t sbo)
{
  return (r >> 3) * sbo + (k >> 3) * lbo + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor: start address, leading (K) and stride (R) byte offsets, all
// in 16-byte units; descriptor version 1 (bits 46-47); no swizzle (layout type 0, bits 61-63).
__device__ __forceinline__ uint64_t smemDesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  return uint64_t((saddr & 0x3FFFFu) >> 4) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 accumulator, both operands K-major,
// M = 128 and the given N (a multiple of 16, at most 256).
__host__ __device__ constexpr uint32_t idescBf16(uint32_t n)
{
  return (1u << 4)              // D format: F32
         | (1u << 7)            // A format: BF16
         | (1u << 10)           // B format: BF16
         | ((n >> 3) << 17)     // N / 8
         | ((128u >> 4) << 24); // M / 16
}

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// TMEM allocation of `cols` columns (a power of two, 32..512) by one whole warp; the base address
// is written to the shared-memory word at `slot`.
__device__ __forceinline__ void tmemAlloc(uint32_t slot, uint32_t cols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(cols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmemDealloc(uint32_t taddr, uint32_t cols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// D (TMEM) = A * B^T (+ D when `accumulate`), one K = 16 step; issued by a single thread.
__device__ __forceinline__ void mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
               " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(dtmem),
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
               : "memory");
}

// The mbarrier at `bar` gets one arrival when every tcgen05 operation this thread issued before
// has completed.
__device__ __forceinline__ void commit(uint32_t bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Orders this thread's generic-proxy shared-memory writes before later async-proxy reads (the MMA's).
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane (shape 32x32b: thread i of the warp reads
// lane (warp % 4) * 32 + i); `taddr` carries the warp's lane base in bits 16-31.
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16])
{
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
               "%14, %15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) {
    v[i] = __uint_as_float(r[i]);
  }
}

__device__ __forceinline__ void mbarInit(uint32_t bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbarTest(uint32_t bar, uint32_t phase)
{
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok)
               : "r"(bar), "r"(phase)
               : "memory");
  return ok != 0;
}

// Waits until the mbarrier completed the phase of parity `phase`: at most `polls` tests, sleeping
// about 64 ns between tests after the first 32.  Returns false if it gave up.
__device__ __forceinline__ bool mbarWait(uint32_t bar, uint32_t phase, uint32_t polls)
{
  bool done = mbarTest(bar, phase);
  for (uint32_t t = 1; t < polls && !done; t++) {
    if (t >= 32) {
      __nanosleep(64);
    }
    done = mbarTest(bar, phase);
  }
  return done;
}

} // namespace tc
} // namespace ebg

#endif
