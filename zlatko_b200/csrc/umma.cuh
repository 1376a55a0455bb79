// Blackwell fifth-generation tensor-core building blocks (sm_100a): TMEM allocation, shared-memory matrix
// descriptors for the canonical K-major layout without swizzle, the BF16 x BF16 -> FP32 MMA issued by one
// thread, its completion through an mbarrier, and TMEM -> register loads.
//
// Canonical K-major layout (no swizzle) of an R x K bf16 operand tile as used here: the tile is cut into
// core matrices of 8 rows x 8 elements (16 bytes per row, 128 contiguous bytes per core matrix); core
// matrix (row group g, k group kg) starts at byte g * 128 + kg * (R / 8) * 128.  In descriptor terms the
// stride byte offset (between 8-row groups) is 128 and the leading byte offset (between adjacent k groups)
// is R * 16.  One MMA of K = 16 reads two k groups, so the MMA for k groups [2i, 2i + 2) starts at
// byte 2 i R 16.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

#include "zk_device.cuh"

namespace zk {
namespace umma {

__device__ __forceinline__ uint32_t smem(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Byte offset of element (row r, k) in the canonical K-major tile with R rows.
__device__ __forceinline__ uint32_t kMajorOffset(uint32_t r, uint32_t k, uint32_t R) {
  return (r & 7u) * 16u + (r >> 3) * 128u + (k >> 3) * (R * 16u) + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor: start address, leading byte offset, stride byte offset (all >> 4),
// version 1 (Blackwell), base offset 0, no swizzle.
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1u) << 46;  // version
  return d;                               // layout type 0: no swizzle
}

// Instruction descriptor of kind::f16: BF16 A and B (both K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t idescBf16(uint32_t M, uint32_t N) {
  return (1u << 4)            // D format F32
         | (1u << 7)          // A format BF16
         | (1u << 10)         // B format BF16
         | ((N >> 3) << 17)   // N / 8
         | ((M >> 4) << 24);  // M / 16
}

// Instruction descriptor of kind::f16 with FP16 A and B (both K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t idescF16(uint32_t M, uint32_t N) {
  return (1u << 4)            // D format F32
         | ((N >> 3) << 17)   // N / 8; A and B format 0: F16
         | ((M >> 4) << 24);  // M / 16
}

// D[tmem] (+)= A[desc] * B[desc]^T, issued by the calling thread.
__device__ __forceinline__ void mma(uint32_t tmemD, uint64_t da, uint64_t db, uint32_t idesc, bool accumulate) {
  const uint32_t acc = accumulate ? 1u : 0u, z = 0u;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
      :
      : "r"(tmemD), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z)
      : "memory");
}

// The mbarrier arrives once every tcgen05 operation this thread issued before has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem(bar)) : "memory");
}

__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
// Generic-proxy writes to shared memory (st.shared, cp.async) made visible to the tensor core's async proxy.
__device__ __forceinline__ void fenceAsyncShared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Warp-wide TMEM allocation of `cols` columns (a power of two >= 32); the address lands in *slot.
__device__ __forceinline__ void alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem(slot)), "r"(cols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp w of the CTA reads lanes 32 (w % 4) ..).
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive 32-bit columns of this thread's TMEM lane, one wait for all of them.
__device__ __forceinline__ void ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Four runs of 8 consecutive 32-bit columns of this thread's TMEM lane (at a0..a3) and the wait for them, in one
// statement, so that no use of the registers can be scheduled before the wait.
__device__ __forceinline__ void ld8x4(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%32];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8, %9, %10, %11, %12, %13, %14, %15}, [%33];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%16, %17, %18, %19, %20, %21, %22, %23}, [%34];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%24, %25, %26, %27, %28, %29, %30, %31}, [%35];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3)
      : "memory");
}
// Three runs of 8 consecutive 32-bit columns of this thread's TMEM lane (at a0..a2) and the wait for them.
__device__ __forceinline__ void ld8x3(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t (&r)[24]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%24];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%8, %9, %10, %11, %12, %13, %14, %15}, [%25];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%16, %17, %18, %19, %20, %21, %22, %23}, [%26];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23])
      : "r"(a0), "r"(a1), "r"(a2)
      : "memory");
}
// 8 consecutive 32-bit columns of this thread's TMEM lane from registers (the registers are read at issue;
// waitSt completes the stores before the columns are read back or handed to another thread).
__device__ __forceinline__ void st8(uint32_t a, const uint32_t (&r)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(a), "r"(r[0]),
               "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
               : "memory");
}
__device__ __forceinline__ void waitSt() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// Three runs of 8 consecutive 32-bit columns of this thread's TMEM lane (at a0..a2) from registers, and the wait
// for the stores, in one statement (the registers may be reused as soon as it returns).
__device__ __forceinline__ void st8x3(uint32_t a0, uint32_t a1, uint32_t a2, const uint32_t (&r)[24]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%3, %4, %5, %6, %7, %8, %9, %10};\n\t"
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%1], {%11, %12, %13, %14, %15, %16, %17, %18};\n\t"
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%2], {%19, %20, %21, %22, %23, %24, %25, %26};\n\t"
      "tcgen05.wait::st.sync.aligned;" ::"r"(a0),
      "r"(a1), "r"(a2), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
      "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]),
      "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23])
      : "memory");
}

// 16-byte asynchronous global -> shared copy (LDGSTS) and its completion.
__device__ __forceinline__ void cpAsync16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

// SiLU of two activations for inference, in packed bf16 arithmetic, from h = z / 2 (the caller folds the 1/2
// into its bias add): sigmoid(z) = (1 + tanh(z / 2)) / 2, so silu(z) = h (1 + tanh h) = fma(h, tanh h, h).  One
// tanh.approx.bf16x2 (a single special-function op for both) and one bf16x2 FMA; h0 lands in the low half (the
// first of the two in memory).  h is rounded to bf16 on the integer pipe -- half a bf16 unit added to the bit
// pattern, the upper halves of both words kept by one byte permute: round half away from zero, which differs
// from round-to-nearest-even only on exact ties -- so the special-function pipe only sees the tanh.  Against silu
// rounded once to bf16 the result carries the rounding of h and the approximate tanh, about one bf16 unit in the
// last place more.
__device__ __forceinline__ uint32_t siluHalfBf16x2(float h0, float h1) {
  uint32_t p, t, s;
  asm("prmt.b32 %0, %1, %2, 0x7632;" : "=r"(p) : "r"(__float_as_uint(h0) + 0x8000u), "r"(__float_as_uint(h1) + 0x8000u));
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(p));
  asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(s) : "r"(p), "r"(t));
  return s;
}
// d/dz silu(z) = s (1 + z (1 - s)), s = sigmoid(z)
__device__ __forceinline__ float siluGrad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

}  // namespace umma
}  // namespace zk
