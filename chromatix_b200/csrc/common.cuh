// Common device helpers for the chromatix_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cx_b200.h"

namespace cx {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
__device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }

// (n + s) mod m for 0 <= n < m and 0 <= s < m, without an integer division
__host__ __device__ __forceinline__ int add_mod(int n, int s, int m) {
  const int t = n + s;
  return t >= m ? t - m : t;
}

// fftfreq numerator of FFT bin k for length n (numpy/jax convention).
__host__ __device__ __forceinline__ int freq_index(int k, int n) { return k < (n + 1) / 2 ? k : k - n; }

// Reduce an FP64 phase to [-pi, pi] before the FP32 sin/cos.
__device__ __forceinline__ float reduce_phase(double ph) {
  const double inv2pi = 0.15915494309189533576888376337251;
  const double twopi = 6.283185307179586476925286766559;
  return (float)(ph - twopi * rint(ph * inv2pi));
}

// exp(i ph) for an FP64 phase: exact reduction to [-pi, pi] in FP64, then the
// hardware sin/cos, whose absolute error on [-pi, pi] is at most 2^-21.41
// (< 4e-7) -- far inside the 1e-5 relative-L2 budget of the accurate mode.
__device__ __forceinline__ float2 expi_reduced(double ph) {
  float s, c;
  __sincosf(reduce_phase(ph), &s, &c);
  return make_float2(c, s);
}

// exp(i ph) with FP64 sin/cos, rounded once to float: for values that are
// evaluated once and reused (tables, per-row factors)
__device__ __forceinline__ float2 expi_precise(double ph) {
  double s, c;
  sincos(ph, &s, &c);
  return make_float2((float)c, (float)s);
}

// Asynchronous 16-byte global -> shared copies (cp.async): the copy proceeds
// while the thread goes on computing; cp_async_wait_all() waits for this
// thread's copies, a barrier then publishes them to the other threads.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// wait until at most N of this thread's committed copy groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Bulk (TMA) copies global -> shared completing on an mbarrier: one thread
// arms the barrier with the byte count of the copies it then issues; the
// barrier's phase completes when every byte has landed.  Source, destination
// and size must be multiples of 16 bytes.
__device__ __forceinline__ void bulk_mbar_init(uint64_t* bar) {
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b) : "memory");
}
__device__ __forceinline__ void bulk_expect(uint64_t* bar, unsigned bytes) {
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* smem, const void* gmem, unsigned bytes, uint64_t* bar) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(s),
               "l"(gmem), "r"(bytes), "r"(b)
               : "memory");
}
// L2 policy for data read or written once per pass (slice rows, records):
// evicted first, so that the state that every pass reuses stays in L2
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
// bulk copy global -> shared with an L2 cache policy
__device__ __forceinline__ void bulk_copy_g2s_hint(void* smem, const void* gmem, unsigned bytes, uint64_t* bar,
                                                   uint64_t policy) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;\n" ::"r"(s),
      "l"(gmem), "r"(bytes), "r"(b), "l"(policy)
      : "memory");
}
// 8-byte global store with an L2 cache policy
__device__ __forceinline__ void st_hint(float2* p, float2 v, uint64_t policy) {
  asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;\n" ::"l"(p), "f"(v.x), "f"(v.y), "l"(policy)
               : "memory");
}
// hint: start bringing [gmem, gmem + bytes) into L2 (bulk prefetch; the
// address and the size must be multiples of 16 bytes; no completion to wait on)
__device__ __forceinline__ void bulk_prefetch_l2(const void* gmem, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(gmem), "r"(bytes) : "memory");
}
// shared-memory reads by the generic proxy are ordered before later bulk writes
__device__ __forceinline__ void bulk_fence() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// bounded wait for the phase with parity `phase`; false after `polls` polls
__device__ __forceinline__ bool bulk_wait(uint64_t* bar, unsigned phase, int polls) {
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  for (int i = 0; i < polls; ++i) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(b), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Cast helpers that block FMA contraction, for the float32 reference-order
// evaluation mode.
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }

}  // namespace cx
