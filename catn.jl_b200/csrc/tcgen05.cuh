// Blackwell (sm_100a) tensor-core primitives for the split-precision mode:
// tcgen05.mma of kind::tf32 on shared-memory operands with the accumulator
// in tensor memory (TMEM), issued by one thread, completion signalled to an
// mbarrier by tcgen05.commit, results read back with tcgen05.ld.
//
// 3xTF32: an FP32 value x is split into hi = x rounded to TF32 (10 explicit
// mantissa bits) and lo = x - hi rounded to TF32, so x = hi + lo to about
// 2^-22; a product is accumulated as hi_a hi_b + hi_a lo_b + lo_a hi_b in
// FP32, which keeps about 21 bits of each product (measured: errors about
// 3.5e-7 of |A| |B|).  Operands arrive here in FP64 and are rounded to FP32
// first.
//
// Operand layout in shared memory: K-major, no swizzle ("interleave"), the
// canonical layout whose core matrix is 8 rows x 16 bytes (4 TF32 values of
// K) stored contiguously (128 bytes).  For a tile of R rows and KC values of
// K, element (r, k) lives at byte
//     (r / 8) * SBO + (k / 4) * LBO + (r % 8) * 16 + (k % 4) * 4
// with LBO = 128 (core matrices adjacent in K) and SBO = KC / 4 * 128.  One
// MMA consumes K = 8 (two core matrices along K), so the descriptor of k-step
// s starts 2 * LBO * s bytes further.
//
// Every wait on an mbarrier is bounded; a wait that runs out reports failure
// to the caller, which then records an error status and stops issuing work.
#pragma once
#include <stdint.h>

namespace catn {
namespace tc {

constexpr uint32_t kLBO = 128;

#if defined(__CUDACC__)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor (K-major, no swizzle): start address,
// leading (K) and stride (8-row group) byte offsets, all in 16-byte units;
// bits 46-47 hold the descriptor version 1 of sm_100; layout type 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::tf32 with FP32 accumulation, both
// operands K-major, dense: D format F32 (bits 4-5 = 1), A and B format TF32
// (bits 7-9 and 10-12 = 2), N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// TMEM allocation of `ncols` columns (a power of two >= 32) by one whole
// warp; the base address is written to *slot (shared memory).
//
// A translation unit that defines CATN_NO_TCGEN05 before including this file
// compiles no tcgen05 instruction: there tc_setup leaves the staging area
// unset (tc_ready is false) and no tensor-core routine is reached.
#if !defined(CATN_NO_TCGEN05)
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
#else
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t) { *slot = 0; }
__device__ __forceinline__ void tmem_dealloc(uint32_t, uint32_t) {}
__device__ __forceinline__ void fence_before_sync() {}
__device__ __forceinline__ void fence_after_sync() {}
#endif
// Make this thread's generic-proxy shared-memory writes visible to the
// tensor core (async proxy); followed by a barrier before the MMA issue.
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Bounded wait for the phase with parity `parity` of *bar to complete.
// Returns false when `limit` polls passed without it.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit) {
  const uint32_t a = smem_u32(bar);
  for (long long i = 0; i < limit; ++i) {
    uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

#if !defined(CATN_NO_TCGEN05)
// D[tmem] (+)= A[smem] * B[smem], one instruction (issued by one thread).
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// Arrive on *bar once every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// 32 consecutive TMEM columns of the warp's 32 lanes: lane l of the warp
// receives row (lane base + l), columns col .. col + 31, as FP32 bits.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
#else
__device__ __forceinline__ void mma_tf32(uint32_t, uint64_t, uint64_t, uint32_t, uint32_t) {}
__device__ __forceinline__ void mma_commit(uint64_t*) {}
__device__ __forceinline__ void tmem_ld32(uint32_t, float* v) {
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = 0.f;
}
#endif

// x rounded to TF32: nearest on the dropped 13 mantissa bits, ties away
// from zero (a carry into the exponent is the correct rounding).
__device__ __forceinline__ float round_tf32(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
// hi = TF32(x), lo = TF32(x - hi) for x = FP32(xd); x - hi is exact in FP32.
__device__ __forceinline__ void split_tf32(double xd, float* hi, float* lo) {
  const float x = (float)xd;
  const float h = round_tf32(x);
  *hi = h;
  *lo = round_tf32(x - h);
}

// Byte offset of element (r, k) in a K-major no-swizzle tile of kc values
// of K per row.
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int kc) {
  return (uint32_t)((r >> 3) * (kc / 4) * 128 + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

#endif  // __CUDACC__

}  // namespace tc
}  // namespace catn
