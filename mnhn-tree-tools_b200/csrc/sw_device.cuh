// Device-side building blocks for the Smith-Waterman kernels (sm_100a).
//
// Packed 16x2 arithmetic uses the DPX integer min/max intrinsics; the
// substitution score of a DP cell is looked up with one byte permute (PRMT)
// from an 8-entry per-column table.  Bulk copies into shared memory use the
// TMA bulk-copy engine (cp.async.bulk) completed on an mbarrier; every wait on
// that barrier is bounded and reports a timeout through the kernel's status
// word instead of spinning forever.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace swgpu {

// Status bits a kernel may raise in its status word.
enum : unsigned {
  KST_TIMEOUT = 1u,        // a bounded wait gave up
  KST_RERUN_OVERFLOW = 2u, // the 32-bit rerun queue was full
  KST_BAD_TILE = 4u,       // a tile descriptor failed validation
  KST_REPLAY_OVERFLOW = 8u, // a device DBSCAN replay's frontier outgrew its set
};

// Symbol codes shared by host and device.  Codes 0..6 are the fast alphabet;
// code 7 is never given to a symbol and pads the row side of the 16x2 kernel.
enum : int {
  CODE_A = 0, CODE_C = 1, CODE_G = 2, CODE_T = 3, CODE_N = 4, CODE_NUL = 5,
  CODE_EXTRA = 6, CODE_ROWPAD = 7, FAST_CODES = 7,
};

// Row selector for a pair of row symbols (ca in the low half, cb in the high
// half): PRMT nibbles {ca, ca|8, cb, cb|8} copy the table byte and then
// sign-extend it into the upper byte of each 16-bit lane.
__host__ __device__ __forceinline__ uint16_t make_sel(int ca, int cb) {
  return (uint16_t)(ca | ((ca | 8) << 4) | (cb << 8) | ((cb | 8) << 12));
}
constexpr uint16_t SEL_PAD = (uint16_t)(7 | (15 << 4) | (7 << 8) | (15 << 12));

__device__ __forceinline__ uint32_t prmt(uint32_t lo, uint32_t hi, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(lo), "r"(hi), "r"(sel));
  return d;
}

// Per-halfword max(a, b, 0).
__device__ __forceinline__ uint32_t vmax0(uint32_t a, uint32_t b) { return __vimax_s16x2_relu(a, b); }
// Per-halfword max(a + b, c).
__device__ __forceinline__ uint32_t vaddmax(uint32_t a, uint32_t b, uint32_t c) {
  return __viaddmax_s16x2(a, b, c);
}
// Per-halfword max(a + b, c, 0).
__device__ __forceinline__ uint32_t vaddmax0(uint32_t a, uint32_t b, uint32_t c) {
  return __viaddmax_s16x2_relu(a, b, c);
}
// Per-halfword max(a, b, c, 0).
__device__ __forceinline__ uint32_t vmax3_0(uint32_t a, uint32_t b, uint32_t c) {
  return __vimax3_s16x2_relu(a, b, c);
}
// Per-halfword max(a, b, c).
__device__ __forceinline__ uint32_t vmax3(uint32_t a, uint32_t b, uint32_t c) {
  return __vimax3_s16x2(a, b, c);
}
// Per-halfword wrapping add.  Measured on B200 this issues on the FMA pipe,
// leaving the ALU pipe (PRMT and the packed maxima) free.
__device__ __forceinline__ uint32_t vadd(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("add.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}

// ---------------------------------------------------------------------------
// mbarrier + bulk copy (TMA engine, non-tensor form)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// One attempt; returns true once the phase with the given parity completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after max_iter attempts and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t max_iter) {
  for (uint32_t it = 0; it < max_iter; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it > 64) __nanosleep(128);
  }
  return false;
}

// Global -> shared bulk copy of `bytes` (multiple of 16, both addresses
// 16-byte aligned) that completes on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace swgpu
