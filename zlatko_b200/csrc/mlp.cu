// The surrogate's tensor-core kernels: a BF16 GEMM with FP32 accumulation in TMEM (tcgen05.mma, operands
// staged in shared memory in the canonical K-major layout, one elected thread issuing the MMAs), with the
// epilogues a multilayer perceptron needs (bias, SiLU, BF16 activations row-major and transposed, the
// pre-activations, FP32 output or accumulation).  Forward and backward passes of the MLP are chains of it:
//
//   forward   Z = H W^T + b, H' = silu(Z)                       A = H [batch][in],  B = W [out][in]
//   backward  dH = dZ W                                          A = dZ [batch][out], B = W^T [in][out]
//             dW = dZ^T H                                        A = dZ^T [out][batch], B = H^T [in][batch]
//
// so every product is "A B^T" with both operands K-major, and the epilogue writes the transposed copies the
// next product reads.
#include <cuda_bf16.h>

#include "umma.cuh"
#include "zk_kernels.h"

namespace zk {

namespace {

constexpr int kGemmThreads = 128;
constexpr uint32_t kGemmBK = 64;
constexpr uint32_t kWaitLimit = 1u << 26;  // polls of an MMA-completion barrier before the kernel gives up

template <int BN>
__global__ void __launch_bounds__(kGemmThreads) gemmKernel(const GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* sA = sm;                       // 128 x 64 bf16, canonical K-major
  unsigned char* sB = sm + 128 * kGemmBK * 2;   // BN x 64 bf16
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const uint32_t m0 = blockIdx.x * 128u, n0 = blockIdx.y * BN, K = g.K;
  if (warp == 0) umma::alloc(&tslot, 128);
  if (tid == 0) mbarInit(&bar, 1);
  umma::fenceBeforeSync();
  __syncthreads();
  umma::fenceAfterSync();
  const uint32_t tmem = tslot;
  constexpr uint32_t idesc = umma::idescBf16(128, BN);
  uint32_t phase = 0;
  bool ok = true, pending = false;
  for (uint32_t k0 = 0; k0 < K && ok; k0 += kGemmBK) {
    const uint32_t kw = min(kGemmBK, K - k0), groups = kw >> 3;
    for (uint32_t v = tid; v < 128u * groups; v += kGemmThreads) {
      const uint32_t r = v / groups, kg = v % groups;
      umma::cpAsync16(sA + umma::kMajorOffset(r, kg * 8, 128), g.A + static_cast<size_t>(m0 + r) * K + k0 + kg * 8);
    }
    for (uint32_t v = tid; v < BN * groups; v += kGemmThreads) {
      const uint32_t r = v / groups, kg = v % groups;
      umma::cpAsync16(sB + umma::kMajorOffset(r, kg * 8, BN), g.B + static_cast<size_t>(n0 + r) * K + k0 + kg * 8);
    }
    umma::cpAsyncCommit();
    umma::cpAsyncWaitAll();
    umma::fenceAsyncShared();
    __syncthreads();
    if (tid == 0) {
      umma::fenceAfterSync();
      for (uint32_t i = 0; i < kw / 16; ++i) {
        const uint64_t da = umma::desc(umma::smem(sA) + i * 2 * 128 * 16, 128 * 16, 128);
        const uint64_t db = umma::desc(umma::smem(sB) + i * 2 * BN * 16, BN * 16, 128);
        umma::mma(tmem, da, db, idesc, k0 > 0 || i > 0);
      }
      umma::commit(&bar);
    }
    // The MMAs read sA / sB: the next chunk may overwrite them only once they have completed.  The vote keeps
    // every thread on the same path if one poll gives up.
    const bool done = mbarWait(&bar, phase, kWaitLimit);
    ok = __syncthreads_and(done) != 0;
    pending = !ok;
    phase ^= 1u;
  }
  if (!ok) {
    if (tid == 0) atomicExch(g.err, kDevTimeout);
    if (pending) mbarWait(&bar, phase ^ 1u, kWaitLimit);  // the MMAs in flight, before the TMEM goes away
  } else {
    umma::fenceAfterSync();
    const uint32_t row = m0 + warp * 32 + lane;
    const uint32_t taddr = tmem + ((warp * 32u) << 16);
    float head = 0.0f;
#pragma unroll 1
    for (uint32_t c = 0; c < BN; c += 16) {
      float v[16];
      umma::ld16(taddr + c, v);
      // A thread holds 16 adjacent columns of its row: the bf16 outputs leave as two 16-byte stores each.
      __align__(16) __nv_bfloat16 zb[16], hb[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const uint32_t n = n0 + c + j;
        const size_t at = static_cast<size_t>(row) * g.N + n;
        float z = v[j] + (g.bias ? g.bias[n] : 0.0f);
        if (g.gradOf) z *= umma::siluGrad(__bfloat162float(g.gradOf[at]));
        if (g.C) g.C[at] = g.accumulate ? g.C[at] + z : z;
        const float h = g.act ? umma::silu(z) : z;
        zb[j] = __float2bfloat16_rn(z);
        hb[j] = __float2bfloat16_rn(h);
        if (g.HT) g.HT[static_cast<size_t>(n) * g.M + row] = hb[j];
        if (g.headOut) head += __bfloat162float(hb[j]) * g.headW[n];
      }
      const size_t at0 = static_cast<size_t>(row) * g.N + n0 + c;  // 32-byte aligned: N and n0 + c are multiples of 16
      if (g.Z) {
        reinterpret_cast<uint4*>(g.Z + at0)[0] = reinterpret_cast<const uint4*>(zb)[0];
        reinterpret_cast<uint4*>(g.Z + at0)[1] = reinterpret_cast<const uint4*>(zb)[1];
      }
      if (g.H) {
        reinterpret_cast<uint4*>(g.H + at0)[0] = reinterpret_cast<const uint4*>(hb)[0];
        reinterpret_cast<uint4*>(g.H + at0)[1] = reinterpret_cast<const uint4*>(hb)[1];
      }
    }
    if (g.headOut) g.headOut[row] = head + g.headB[0];
  }
  umma::fenceBeforeSync();
  __syncthreads();
  if (warp == 0) umma::dealloc(tmem, 128);
}

template <int BN>
cudaError_t launchGemmBN(const GemmArgs& g, cudaStream_t s) {
  const size_t smemBytes = (128 + BN) * kGemmBK * 2;
  // At least 55 KB per CTA (56 KB with the 1 KB the SM reserves per CTA) keeps at most four CTAs on an SM,
  // 4 x 128 TMEM columns, so an allocation never waits on another CTA; 58 KB allowed only three.
  const size_t dyn = smemBytes < 55 * 1024 ? 55 * 1024 : smemBytes;
  cudaError_t e = cudaFuncSetAttribute(gemmKernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dyn));
  if (e != cudaSuccess) return e;
  gemmKernel<BN><<<dim3(g.M / 128, g.N / BN), kGemmThreads, dyn, s>>>(g);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launchGemm(const GemmArgs& g, cudaStream_t s) {
  if (g.M == 0 || g.N == 0 || g.K == 0) return cudaSuccess;
  if (g.M % 128 || g.N % 16 || g.K % 16) return cudaErrorInvalidValue;
  if (g.headOut && g.N != 128) return cudaErrorInvalidValue;  // the head needs a row's columns in one tile
  if (g.N % 128 == 0) return launchGemmBN<128>(g, s);
  if (g.N % 64 == 0) return launchGemmBN<64>(g, s);
  if (g.N % 32 == 0) return launchGemmBN<32>(g, s);
  return launchGemmBN<16>(g, s);
}

}  // namespace zk
