// Blackwell 5th-generation tensor-core helpers (tcgen05, sm_100a): shared-
// memory matrix descriptors, the instruction descriptor of a BF16 x BF16 ->
// FP32 product, tensor-memory (TMEM) allocation, the MMA issue, its commit to
// an mbarrier and the 32-lane TMEM loads of the epilogue.
//
// Operand layout (K-major, no swizzle): an R x K bf16 operand is stored as
// 8-row x 16-byte core matrices (8 rows x 8 elements, 128 contiguous bytes);
// core matrices adjacent along K are kTcLBO bytes apart, 8-row groups are
// SBO = (K / 8) * 128 bytes apart.  One MMA consumes K = 16 elements, i.e.
// two core matrices along K, so successive K steps start 256 bytes apart.
#pragma once

#include <cuda_bf16.h>

#include "jfb_common.cuh"

namespace jfb {

constexpr uint32_t kTcLBO = 128;  // bytes between K-adjacent core matrices

// Byte offset of element (r, k) of a K-major no-swizzle bf16 operand with K
// columns (K a multiple of 16).
__host__ __device__ inline uint32_t tc_offset(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K / 8) * 128 + (k >> 3) * (int)kTcLBO + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (sm_100 layout: start >> 4 in bits 0-13,
// leading byte offset >> 4 in 16-29, stride byte offset >> 4 in 32-45,
// version 1 in 46-47, base offset 0, no swizzle in 61-63).
__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t saddr, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((kTcLBO >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16 with BF16 A and B (K-major both) and
// an FP32 accumulator, M x N (M = 128, N a multiple of 16 up to 256).
__host__ __device__ constexpr uint32_t tc_idesc_bf16(int M, int N) {
  return (1u << 4)                        // D format: F32
         | (1u << 7)                      // A format: BF16
         | (1u << 10)                     // B format: BF16
         | ((uint32_t)(N >> 3) << 17)     // N / 8
         | ((uint32_t)(M >> 4) << 24);    // M / 16
}

// Allocate `ncols` TMEM columns (a power of two >= 32); one whole warp calls
// it; the TMEM address is written to *slot (shared memory).
__device__ __forceinline__ void tc_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy shared-memory writes become visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one thread issues it.
__device__ __forceinline__ void tc_mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, bool accumulate) {
  const uint32_t acc = accumulate ? 1u : 0u, z = 0u;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}
// Arrive (once) on an mbarrier when every MMA issued so far by this thread
// has completed.
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(bar))
               : "memory");
}

// 32 consecutive FP32 columns of this warp's 32 TMEM lanes (lane i of the
// warp gets row 32 (warp % 4) + i); taddr carries the lane base in bits 16-31.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Three-way BF16 split v = b0 + b1 + b2 (each part rounded to nearest), so
// that products of split operands carry about 24 significant bits.
__device__ __forceinline__ void bf16_split3(double v, __nv_bfloat16 (&b)[3]) {
  b[0] = __float2bfloat16_rn((float)v);
  double r = v - (double)__bfloat162float(b[0]);
  b[1] = __float2bfloat16_rn((float)r);
  r -= (double)__bfloat162float(b[1]);
  b[2] = __float2bfloat16_rn((float)r);
}

}  // namespace jfb
