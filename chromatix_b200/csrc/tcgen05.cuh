// Blackwell (sm_100a) tensor-core primitives in inline PTX: tensor-memory
// allocation, shared-memory matrix descriptors, tcgen05.mma of kind f16 with
// FP32 accumulation in tensor memory, completion through an mbarrier, and
// tensor-memory loads.  Used by the split-precision DFT stages (a complex
// DFT as a real GEMM whose FP16 operands carry an FP32 value as hi + lo).
//
// Conventions (one CTA, cta_group::1):
//  * operands are in shared memory in the canonical "no swizzle" layouts:
//    core matrices of 8 rows x 16 bytes (8 fp16), 128 contiguous bytes each;
//      K-major:  element (r, k) at ((k/8) * (R/8) + r/8) * 128 + (r%8) * 16 + (k%8) * 2
//      MN-major: element (r, k) at ((k/8) * (R/8) + r/8) * 128 + (k%8) * 16 + (r%8) * 2
//    so the offset between 8-row groups (SBO) is 128 B and between 8-column
//    groups of K (LBO) is (R/8) * 128 B, R = rows of the operand tile;
//  * D (M x N, FP32) lives in tensor memory: row m in lane m, column j in
//    column j of the allocation;
//  * every wait on an mbarrier is bounded: past the limit the caller records
//    an error and skips the work instead of spinning forever.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

#include "common.cuh"

namespace cx {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// ---------------------------------------------------------------------------
// tensor memory (allocated and freed by one whole warp)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// ordering of tcgen05 operations around thread synchronisation
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// mbarrier
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

// wait until the phase with parity `phase` has completed; false after
// `max_polls` unsuccessful polls (each poll may suspend the thread briefly)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int max_polls) {
  const uint32_t a = smem_u32(bar);
  for (int i = 0; i < max_polls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// descriptors
// ---------------------------------------------------------------------------
// shared-memory matrix descriptor, no swizzle: start address, LBO (offset
// between 8-column K groups), SBO (offset between 8-row groups), version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16 with F16 A and B, F32 accumulation;
// a_mn / b_mn: 1 = MN-major operand, 0 = K-major
__host__ __device__ constexpr uint32_t idesc_f16_f32(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// D (tmem) = A * B (+ D when accumulate != 0), issued by one thread
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive on `bar` once every tcgen05.mma issued so far by this thread has completed
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// ---------------------------------------------------------------------------
// tensor memory -> registers: 32 lanes (this warp's quarter) x 16 columns
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// FP32 -> FP16 hi + lo (x ~= hi + lo to ~22 bits for |x| in the normal FP16
// range): pack two values per 32-bit word
// ---------------------------------------------------------------------------
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __half2 h = __floats2half2_rn(a, b);
  const float2 hf = __half22float2(h);
  const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// byte offset of element (r, k) of an R-row operand tile in the canonical layouts
__host__ __device__ constexpr uint32_t off_kmajor(int R, int r, int k) {
  return (uint32_t)((((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}
__host__ __device__ constexpr uint32_t off_mnmajor(int R, int r, int k) {
  return (uint32_t)((((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((k & 7) << 4) + ((r & 7) << 1));
}

}  // namespace tc
}  // namespace cx
