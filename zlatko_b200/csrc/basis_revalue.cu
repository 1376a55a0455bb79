// basisRevalueKernel: the revaluation, netting, cash collateral and statistics of up to 128 netting sets on a tile
// of 128 paths, with the linear revaluation of all of them as one tensor-core product per date.
//
// The plans' semantics are those of revalueKernel (the reference's fused kernel, src/gpu/fused_kernels.cpp:224-530,
// for plans whose terms are bonds, floating coupons with their fixings, FX forwards and Black options, under no CSA
// or a cash CSA whose margin call looks back at most one date).  The work is organised for a B200 instead of term
// by term:
//
//   1. Basis (CUDA cores).  Four threads per path evaluate the date's basis functions Phi[path][k] (each distinct
//      bond exponential, fixing x bond, foreign bond x FX rate, FX rate and option price of the group once, however
//      many netting sets hold it), split each into FP16 hi + lo (lo = the rounding residue of hi), and write them
//      into shared memory in the K-major layout of the tensor core's B operand, 64 columns per chunk.
//   2. Product (tensor core).  One thread issues, per chunk, tcgen05.mma kind::f16 C_hi Phi_hi + C_hi Phi_lo +
//      C_lo Phi_hi into an FP32 accumulator in TMEM: lane = netting set, column = path.  The coefficient chunk
//      C (128 netting sets x 64 columns, hi and lo) arrives by a bulk copy issued a chunk ahead; the next chunk's
//      basis is evaluated while the tensor core multiplies this one.
//   3. Netting set epilogue (CUDA cores).  Thread (netting set r, path block b) takes its 32 paths in order: the
//      netted value (accumulator x the date's power-of-two scale), the margin call and the collateral, the
//      exposure row, the CVA increment and the date's 8 statistics summed over the 32 paths -- the partial of the
//      32-path unit, no shuffles.  The per-(netting set, path) state -- collateral held, the previous value, the
//      previous discounted positive exposure -- lives in TMEM beside the accumulator (columns 128..511).
//
// Every wait is bounded: an MMA-completion or bulk-copy barrier that does not complete sets kDevTimeout, every
// thread leaves at the next barrier, and the TMEM is freed after the work in flight settles.
#include <cuda_fp16.h>

#include "basis.cuh"
#include "umma.cuh"

namespace zk {
namespace {

constexpr uint32_t kThreads = 512;
constexpr uint32_t kWaitLimit = 1u << 26;               // polls of a barrier before the kernel gives up
constexpr uint32_t kPhiImage = kBasisPaths * 64 * 2;     // one FP16 image of a basis chunk: 16 KB
constexpr uint32_t kCoefImage = kBasisRows * 64 * 2;     // one FP16 image of a coefficient chunk: 16 KB
constexpr uint32_t kOffPhi = 0;                          // [2 buffers][hi, lo]
constexpr uint32_t kOffCoef = kOffPhi + 4 * kPhiImage;   // [2 buffers][hi, lo]
constexpr uint32_t kOffFix = kOffCoef + 4 * kCoefImage;  // fixings x 64: [slot][path]
constexpr uint32_t kOffStage = kOffFix + kBasisMaxFix * kBasisPaths * 4;  // D, Q0, Q1, dQ0, dQ1 per path
constexpr uint32_t kSmem = kOffStage + 5 * kBasisPaths * 4;
// TMEM columns: the accumulator [0, 128), then per netting set and path the collateral held, the previous value
// and the previous discounted positive exposure.
constexpr uint32_t kColHeld = 128, kColPrev = 256, kColDE = 384;

struct Factors {
  float x, D, S[4], Q[2], xf[2];
};

__device__ __forceinline__ float pick(const float (&a)[4], uint32_t i) {
  return i == 0 ? a[0] : i == 1 ? a[1] : i == 2 ? a[2] : a[3];
}

// The unscaled Black price of an option record (revalueKernel's kOption / kForeignOption).
__device__ __forceinline__ float optionPrice(const float* rec, bool foreign, const Factors& f) {
  const float4 r0 = __ldg(reinterpret_cast<const float4*>(rec)), r1 = __ldg(reinterpret_cast<const float4*>(rec) + 1);
  const float b0 = r0.w * fastExp(-r1.x * f.x);
  float F;
  if (!foreign) {
    F = pick(f.S, static_cast<uint32_t>(r0.y) & 3u) * r1.y / b0;
  } else {
    const uint32_t a = min(static_cast<uint32_t>(r0.x) >> 12u, 1u);
    F = pick(f.S, a) * (r1.y * fastExp(-r0.y * (a == 0 ? f.xf[0] : f.xf[1]))) / b0;
  }
  return black(F, r1.z, fabsf(r1.w), b0, r1.w > 0.0f);
}

// One k-group of the basis for this thread's path: 8 values of one column type, as FP16 hi and lo.
__device__ __forceinline__ void basisGroup(const BasisKg* kg, const float* options, const Factors& f, const float* fixS,
                                           uint32_t row, uint4& hi, uint4& lo) {
  const float4 b0 = __ldg(reinterpret_cast<const float4*>(kg)), b1 = __ldg(reinterpret_cast<const float4*>(kg) + 1);
  const uint4 sw = __ldg(reinterpret_cast<const uint4*>(kg) + 2);
  const uint4 tm = __ldg(reinterpret_cast<const uint4*>(kg) + 3);
  const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
  const uint32_t sel[8] = {sw.x & 0xFFFFu, sw.x >> 16, sw.y & 0xFFFFu, sw.y >> 16,
                           sw.z & 0xFFFFu, sw.z >> 16, sw.w & 0xFFFFu, sw.w >> 16};
  const uint32_t type = tm.x;
  const float mult = __uint_as_float(tm.y);
  float phi[8];
  switch (type) {
    case kColBond:
#pragma unroll
      for (int e = 0; e < 8; ++e) phi[e] = ex2(b[e] * f.x);
      break;
    case kColCoupon:
#pragma unroll
      for (int e = 0; e < 8; ++e) phi[e] = fixS[sel[e] * kBasisPaths + row] * ex2(b[e] * f.x);
      break;
    case kColForeign:
#pragma unroll
      for (int e = 0; e < 8; ++e) phi[e] = pick(f.S, sel[e]) * ex2(b[e] * (sel[e] == 0 ? f.xf[0] : f.xf[1]));
      break;
    case kColSpot:
#pragma unroll
      for (int e = 0; e < 8; ++e) phi[e] = pick(f.S, sel[e]);
      break;
    default:  // options, one record per column
#pragma unroll
      for (int e = 0; e < 8; ++e) phi[e] = mult * optionPrice(options + 8 * sel[e], type == kColForeignOption, f);
  }
  uint32_t h[4], l[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const __half2 hh = __floats2half2_rn(phi[2 * k], phi[2 * k + 1]);
    const float2 back = __half22float2(hh);
    const __half2 ll = __floats2half2_rn(phi[2 * k] - back.x, phi[2 * k + 1] - back.y);
    h[k] = *reinterpret_cast<const uint32_t*>(&hh);
    l[k] = *reinterpret_cast<const uint32_t*>(&ll);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

__global__ void __launch_bounds__(kThreads, 1) basisRevalueKernel(const BasisArgs* __restrict__ groups, uint32_t* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ BasisArgs G;
  __shared__ __align__(8) uint64_t mmaBar[2], loadBar[2];
  __shared__ uint32_t tslot;
  const uint32_t tid = threadIdx.x, warp = tid >> 5, wg = warp >> 2, row = tid & 127u;
  if (warp == 0) umma::alloc(&tslot, 512);  // one CTA per SM (its shared memory): the whole TMEM is free
  if (tid == 0) {
    G = groups[blockIdx.y];
    mbarInit(&mmaBar[0], 1), mbarInit(&mmaBar[1], 1), mbarInit(&loadBar[0], 1), mbarInit(&loadBar[1], 1);
  }
  umma::fenceBeforeSync();
  __syncthreads();
  umma::fenceAfterSync();
  const uint32_t nP = G.nP, nT = G.nT, tile = blockIdx.x;
  float* fixS = reinterpret_cast<float*>(sm + kOffFix);
  float* stage = reinterpret_cast<float*>(sm + kOffStage);  // [D | Q0 | Q1 | dQ0 | dQ1][128]

  // ---- the basis side: this thread's path (row) ----
  const uint32_t path = tile * kBasisPaths + row, pp = path < nP ? path : nP - 1;
  const size_t fs = static_cast<size_t>(nT) * nP;
  const float* cubeP = G.cube + pp;
  auto loadFactors = [&](uint32_t j, Factors& f) {
    const float* c = cubeP + static_cast<size_t>(j) * nP;
    f.x = __ldg(c), f.D = __ldg(c + fs);
#pragma unroll
    for (uint32_t a = 0; a < 4; ++a) f.S[a] = a < G.nA ? __ldg(c + (G.fS + a) * fs) : 0.0f;
#pragma unroll
    for (uint32_t q = 0; q < 2; ++q) f.Q[q] = q < G.nC ? __ldg(c + (G.fQ + q) * fs) : 1.0f;
#pragma unroll
    for (uint32_t a = 0; a < 2; ++a) f.xf[a] = a < G.nF ? __ldg(c + (G.fXf + a) * fs) : 0.0f;
  };
  float prevQ[2] = {1.0f, 1.0f};

  // ---- the netting-set side: TMEM lane = netting set `row`, paths [32 wg, 32 wg + 32) of the tile ----
  const uint32_t nsRow = row, pb = wg;
  const bool nsLive = nsRow < G.numNs;
  const uint32_t taddr = tslot + ((32u * (warp & 3u)) << 16) + pb * 32u;
  uint32_t hasCsa = 0, cpty = 0xFFFFFFFFu;
  float hc = 0.0f, hb = 0.0f, mta = 0.0f, ia = 0.0f;
  float* rowEP = nullptr;
  float* partials = nullptr;
  if (nsLive) {
    const NsArgs<float>& A = G.ns[nsRow];
    hasCsa = A.hasCsa, cpty = A.cpty, hc = A.hc, hb = A.hb, mta = A.mta, ia = A.ia;
    rowEP = A.expo + static_cast<size_t>(A.rowEP) * nP;
    partials = A.partials;
  }
  __syncwarp();  // the TMEM accesses below are warp-collective
  {
    uint32_t z[24];
#pragma unroll
    for (int i = 0; i < 24; ++i) z[i] = 0u;
#pragma unroll
    for (uint32_t q = 0; q < 32; q += 8) umma::st8x3(taddr + kColHeld + q, taddr + kColPrev + q, taddr + kColDE + q, z);
  }
  const uint32_t blockFirst = tile * kBasisPaths + pb * 32u;
  const uint32_t blockPaths = blockFirst < nP ? min(32u, nP - blockFirst) : 0u;
  const uint32_t unit = tile * 4u + pb;
  const bool vecRows = nP % 4u == 0u;

  constexpr uint32_t idesc = umma::idescF16(kBasisRows, kBasisPaths);
  uint32_t g = 0;              // chunks started (all dates)
  int issued = -1, loaded = -1, consumed = -1;  // thread 0: the last chunk whose MMAs / bulk copy were issued / waited
  bool ok = true;
  if (tid == 0 && G.numChunks > 0) {
    const uint32_t bytes = G.chunks[1] * 8192u;
    mbarExpectTx(&loadBar[0], bytes);
    bulkLoad(sm + kOffCoef, G.blob + G.chunks[0], bytes, &loadBar[0]);
    loaded = 0;
  }
  Factors nf;
  loadFactors(0, nf);
  umma::fenceBeforeSync();
  __syncthreads();

  for (uint32_t j = 0; j < nT && ok; ++j) {
    const uint32_t* dj = G.dates + static_cast<size_t>(j) * kBasisDateWords;
    const uint4 d0 = __ldg(reinterpret_cast<const uint4*>(dj)), d1 = __ldg(reinterpret_cast<const uint4*>(dj) + 1);
    const uint32_t firstChunk = d0.x, numChunks = d0.y, firstKg = d0.z;
    const uint32_t fixBegin = d1.x, fixEnd = d1.y, optBegin = d1.z, callJ = d1.w, rs = __ldg(dj + bdRep);
    const Factors f = nf;
    if (j + 1 < nT) loadFactors(j + 1, nf);
    if (wg == 0) {  // the path's discount factor and survivals for the epilogue threads
      stage[row] = f.D;
#pragma unroll
      for (uint32_t q = 0; q < 2; ++q) {
        stage[(1 + q) * kBasisPaths + row] = f.Q[q];
        stage[(3 + q) * kBasisPaths + row] = j > 0 && rs > 0 ? prevQ[q] - f.Q[q] : 0.0f;
        if (rs > 0) prevQ[q] = f.Q[q];
      }
    }
    // ---- basis chunks and their products ----
    for (uint32_t c = 0; c < numChunks; ++c, ++g) {
      const uint32_t buf = g & 1u;
      if (g >= 2) ok = mbarWait(&mmaBar[buf], ((g - 2) >> 1) & 1u, kWaitLimit) && ok;  // chunk g - 2 released both buffers
      const uint32_t kgs = 2u * __ldg(G.chunks + 2 * (firstChunk + c) + 1);
      unsigned char* phiHi = sm + kOffPhi + buf * 2 * kPhiImage;
#pragma unroll
      for (uint32_t q = 0; q < 2; ++q) {
        const uint32_t kgl = 2u * wg + q;
        if (kgl < kgs) {
          uint4 hi, lo;
          basisGroup(G.kgs + firstKg + c * kBasisChunkKg + kgl, G.options + 8 * static_cast<size_t>(optBegin), f, fixS, row,
                     hi, lo);
          const uint32_t off = umma::kMajorOffset(row, kgl * 8u, kBasisPaths);
          *reinterpret_cast<uint4*>(phiHi + off) = hi;
          *reinterpret_cast<uint4*>(phiHi + kPhiImage + off) = lo;
        }
      }
      umma::fenceAsyncShared();
      ok = __syncthreads_and(ok) != 0;
      if (!ok) break;
      if (tid == 0) {
        bool t0 = mbarWait(&loadBar[buf], (g >> 1) & 1u, kWaitLimit);
        if (t0) {
          consumed = static_cast<int>(g);
          umma::fenceAfterSync();
          const uint32_t steps = kgs / 2u;
          const uint32_t aHi = umma::smem(sm + kOffCoef + buf * 2 * kCoefImage), aLo = aHi + steps * 4096u;
          const uint32_t bHi = umma::smem(phiHi), bLo = bHi + kPhiImage;
          for (uint32_t i = 0; i < steps; ++i) {
            const uint64_t dAh = umma::desc(aHi + i * 4096u, 2048u, 128u), dAl = umma::desc(aLo + i * 4096u, 2048u, 128u);
            const uint64_t dBh = umma::desc(bHi + i * 4096u, 2048u, 128u), dBl = umma::desc(bLo + i * 4096u, 2048u, 128u);
            umma::mma(tslot, dAh, dBh, idesc, c > 0 || i > 0);
            umma::mma(tslot, dAh, dBl, idesc, true);
            umma::mma(tslot, dAl, dBh, idesc, true);
          }
          umma::commit(&mmaBar[buf]);
          issued = static_cast<int>(g);
          // the next chunk's coefficients into the other buffer, once chunk g - 1's MMAs have read it
          if (g + 1 < G.numChunks) {
            if (g >= 1) t0 = mbarWait(&mmaBar[buf ^ 1u], ((g - 1) >> 1) & 1u, kWaitLimit);
            if (t0) {
              const uint32_t bytes = __ldg(G.chunks + 2 * (g + 1) + 1) * 8192u;
              mbarExpectTx(&loadBar[buf ^ 1u], bytes);
              bulkLoad(sm + kOffCoef + (buf ^ 1u) * 2 * kCoefImage, G.blob + __ldg(G.chunks + 2 * (g + 1)), bytes,
                       &loadBar[buf ^ 1u]);
              loaded = static_cast<int>(g + 1);
            }
          }
        }
        ok = t0;
      }
    }
    ok = __syncthreads_and(ok) != 0;  // thread 0's last issue; the staging above, when the date has no chunk
    if (!ok) break;
    // ---- the date's fixings (read from the next date on) ----
    for (uint32_t q = fixBegin + wg; q < fixEnd; q += 4) {
      const float4 r = __ldg(G.fixings + q);
      fixS[static_cast<uint32_t>(r.w) * kBasisPaths + row] = (r.x * ex2(r.y * f.x) - 1.0f) * r.z * kCouponScale;
    }
    if (numChunks > 0) ok = mbarWait(&mmaBar[(g - 1) & 1u], ((g - 1) >> 1) & 1u, kWaitLimit);
    umma::fenceAfterSync();
    // ---- netting-set epilogue (warp-uniform: the TMEM accesses are warp-collective; lanes past the group's netting
    // sets compute on zeros and store nothing) ----
    if (blockPaths > 0 && ok) {
      __syncwarp();
      const float sc = __ldg(G.scale + static_cast<size_t>(j) * kBasisRows + nsRow);
      const bool hasQ = cpty < 2u;
      float s8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
      for (uint32_t q8 = 0; q8 < 32; q8 += 8) {
        uint32_t r[32];
        umma::ld8x4(taddr + q8, taddr + kColHeld + q8, taddr + kColPrev + q8, taddr + kColDE + q8, r);
        uint32_t st[24];
        float ep8[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const uint32_t p = pb * 32u + q8 + i;  // path within the tile
          const float v = numChunks > 0 ? __uint_as_float(r[i]) * sc : 0.0f;
          float held = __uint_as_float(r[8 + i]), vPrev = __uint_as_float(r[16 + i]), prevDE = __uint_as_float(r[24 + i]);
          float collateral = 0.0f;
          if (hasCsa) {  // cash, the margin call at t - MPR, at most one date back (collateral.cpp:10-47)
            const float vc = callJ != j ? vPrev : v;
            float required = 0.0f;
            if (vc > hc) required += vc - hc;
            if (hb >= 0.0f && -vc > hb) required -= -vc - hb;
            if (j == 0 || fabsf(required - held) >= mta) held = required;
            collateral = held + ia;
          }
          vPrev = v;
          const float e = v - collateral, ep = fmaxf(e, 0.0f), en = fminf(e, 0.0f);
          const float D = stage[p], Q = hasQ ? stage[(1 + cpty) * kBasisPaths + p] : 1.0f;
          const float de = D * ep;
          float cva = 0.0f;
          if (rs > 0) {
            if (hasQ) cva = 0.5f * (prevDE + de) * stage[(3 + cpty) * kBasisPaths + p];
            prevDE = de;
          }
          ep8[i] = ep;
          if (q8 + i < blockPaths) {
            s8[0] += e, s8[1] += ep, s8[2] += en, s8[3] += de, s8[4] += D * en, s8[5] += cva, s8[6] += Q, s8[7] += D;
          }
          st[i] = __float_as_uint(held), st[8 + i] = __float_as_uint(vPrev), st[16 + i] = __float_as_uint(prevDE);
        }
        umma::st8x3(taddr + kColHeld + q8, taddr + kColPrev + q8, taddr + kColDE + q8, st);
        if (rs > 0 && nsLive) {
          float* dst = rowEP + static_cast<size_t>(rs - 1) * nP + blockFirst + q8;
          if (vecRows && q8 + 8 <= blockPaths) {
            reinterpret_cast<float4*>(dst)[0] = make_float4(ep8[0], ep8[1], ep8[2], ep8[3]);
            reinterpret_cast<float4*>(dst)[1] = make_float4(ep8[4], ep8[5], ep8[6], ep8[7]);
          } else {
#pragma unroll
            for (uint32_t i = 0; i < 8; ++i)
              if (q8 + i < blockPaths) dst[i] = ep8[i];
          }
        }
      }
      if (nsLive) {
        float4* pt = reinterpret_cast<float4*>(partials + (static_cast<size_t>(unit) * nT + j) * kStatsPerDate);
        pt[0] = make_float4(s8[0], s8[1], s8[2], s8[3]);
        pt[1] = make_float4(s8[4], s8[5], s8[6], s8[7]);
      }
    }
    umma::fenceBeforeSync();
    ok = __syncthreads_and(ok) != 0;  // the accumulator is free for the next date's products
  }
  if (!ok && tid == 0) {
    atomicExch(err, kDevTimeout);
    // the work in flight settles before the TMEM and the shared memory go away
    if (issued >= 0) mbarWait(&mmaBar[issued & 1], (static_cast<uint32_t>(issued) >> 1) & 1u, kWaitLimit);
    if (loaded > consumed) mbarWait(&loadBar[loaded & 1], (static_cast<uint32_t>(loaded) >> 1) & 1u, kWaitLimit);
  }
  umma::fenceBeforeSync();
  __syncthreads();
  __syncwarp();
  if (warp == 0) umma::dealloc(tslot, 512);
}

}  // namespace

cudaError_t launchBasisRevalue(const BasisArgs* groups, uint32_t numGroups, uint32_t nP, uint32_t* err, cudaStream_t stream) {
  if (numGroups == 0 || nP == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(basisRevalueKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSmem));
  if (e != cudaSuccess) return e;
  const dim3 grid((nP + kBasisPaths - 1) / kBasisPaths, numGroups);
  basisRevalueKernel<<<grid, kThreads, kSmem, stream>>>(groups, err);
  return cudaGetLastError();
}

}  // namespace zk
