// tcgen05 (5th-generation tensor core) helpers shared by the float32 factor
// and solve kernels: shared-memory matrix descriptors for K-major operands
// without swizzle, TF32 rounding, TMEM allocation, MMA issue and a bounded
// mbarrier wait.
//
// Operand layout (K-major, no swizzle): core matrices of 8 rows x 16 bytes
// (4 float values); element (m, k) lives at byte
// (m / 8) * SBO + (k / 4) * LBO + (m % 8) * 16 + (k % 4) * 4, with the
// strides chosen by each kernel.  One tcgen05.mma of kind::tf32 consumes
// K = 8, i.e. two core matrices along K, so successive K steps start 2 * LBO
// bytes further.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace dct {

constexpr int kTcM = 128;                 // MMA M (rows of the A operand)
constexpr int kTcN = 128;                 // MMA N of the trailing update
constexpr int kTcThreads = 512;
constexpr uint32_t kTcWaitLimit = 1u << 20;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: start address and core-matrix strides
// (bytes, multiples of 16)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t((saddr >> 4) & 0x3FFF)) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

// instruction descriptor: D float32, A and B tf32, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(N >> 3) << 17) |
         (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(1u));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// warp-wide: allocate `ncols` TMEM columns (power of two >= 32); the address
// is written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
               "r"(ncols));
}

// generic-proxy shared stores -> tensor cores, then a CTA barrier
__device__ __forceinline__ void tc_publish_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t da, uint64_t db,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
          tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// try_wait that may suspend the thread for up to kTcSuspendNs while the phase
// is incomplete (it returns as soon as the phase completes); 0 = the form
// without a time hint (a system-dependent bound)
#ifndef DCT_TC_SUSPEND_NS
#define DCT_TC_SUSPEND_NS 2000
#endif
constexpr uint32_t kTcSuspendNs = DCT_TC_SUSPEND_NS;
__device__ __forceinline__ bool mbar_try_wait_sleep(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  if constexpr (kTcSuspendNs > 0) {
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(kTcSuspendNs)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
  }
  return ok != 0;
}

// All threads: bounded wait for phase `parity` of the mbarrier; the result is
// the same in every thread of the CTA.  Only warp 0 polls (the other warps
// wait at the CTA barrier and issue nothing); at most `limit` polls
// (kTcWaitLimit unless given) of at most kTcSuspendNs each.  On timeout the
// first error is flagged.
__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity, int* status,
                                        int code, int s, int b,
                                        uint32_t limit = kTcWaitLimit) {
  bool done = true;
  if (threadIdx.x < 32) {
    done = false;
    for (uint32_t it = 0; it < limit && !done; ++it)
      done = mbar_try_wait_sleep(smem_u32(bar), parity);
  }
  done = __syncthreads_and(done) != 0;
  if (!done && threadIdx.x == 0) {
    if (atomicCAS(&status[0], 0, code) == 0) {
      status[1] = s;
      status[2] = b;
    }
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return done;
}

// 32 consecutive TMEM columns of this warp's 32 lanes (one row per thread)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
        "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
        "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Store value v (float) of operand element (m, k) into the hi/lo operands:
// hi = v rounded to TF32, lo = v - hi (exact in float; the tensor core reads
// its leading 19 bits, so the part of v below both is dropped, ~2^-22 |v|).
__device__ __forceinline__ void tc_store_split(unsigned char* hi, unsigned char* lo,
                                               uint32_t off, float v) {
  const uint32_t h = tf32_rna(v);
  *reinterpret_cast<uint32_t*>(hi + off) = h;
  *reinterpret_cast<float*>(lo + off) = v - __uint_as_float(h);
}

}  // namespace dct
