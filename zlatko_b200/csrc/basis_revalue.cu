// basisRevalueKernel: the revaluation, netting, cash collateral and statistics of up to 128 netting sets on a tile
// of 128 paths, with the linear revaluation of all of them as one tensor-core product per date.
//
// The plans' semantics are those of revalueKernel (the reference's fused kernel, src/gpu/fused_kernels.cpp:224-530,
// for plans whose terms are bonds, floating coupons with their fixings, FX forwards and Black options, under no CSA
// or a cash CSA whose margin call looks back at most one date).  The work is organised for a B200 instead of term
// by term, as a pipeline of two warp-specialised halves of the CTA:
//
//   Producers (warps 0-7, two threads per path).  Date by date: the path's factors, staged for the consumers
//   (discount factor, survivals and their CVA differences, and per 32-path unit their sums); the date's basis
//   functions Phi[path][k] -- each distinct bond exponential, fixing x bond, foreign bond x FX rate, FX rate and
//   option price of the group once, however many netting sets hold it -- split into FP16 hi + lo (lo = the
//   rounding residue of hi) in the K-major layout of the tensor core's B operand, 64 columns per chunk.  One
//   thread issues per chunk tcgen05.mma kind::f16 C_hi Phi_hi + C_hi Phi_lo + C_lo Phi_hi into the date's FP32
//   accumulator in TMEM (lane = netting set, column = path); the coefficient chunk C (128 netting sets x 64
//   columns, hi and lo) arrives by a bulk copy issued a chunk ahead.  Then the fixings the date sets.
//   Consumers (warps 8-15).  Warp (lane quarter q, path half h) takes netting sets 32 q + lane over paths
//   [64 h, 64 h + 64) in order: the netted value (the accumulator x the date's power-of-two scale), the margin call
//   on the previous date's value (the previous accumulator, kept: three accumulators rotate) and the collateral
//   held (TMEM columns 384..511), the exposure row and the date's 8 statistics summed over its 64 paths in order --
//   the partial of the 64 paths, no shuffles.  The CVA increment 0.5 (DE' + DE)(Q' - Q) between reporting dates is summed as
//   0.5 DE (Q - Q_next) on the earlier date (the next survival staged by the producers) plus 0.5 DE (Q' - Q) on
//   the later one, so no per-path state carries the previous DE.
//
// The producers work on date j + 1 while the consumers finish date j.  mbarriers order the halves: a date's
// staging (stageFull) and products (accFull) before its epilogue; an epilogue (epiDone) before the producers
// reuse its staging buffer three dates later and its accumulator for the products two dates later.  Every wait
// is bounded: one that does not complete sets kDevTimeout, the threads leave their loops (each further wait on
// the other half is bounded too), and the TMEM is freed after the work in flight settles.
#include <cuda_fp16.h>

#include "basis.cuh"
#include "umma.cuh"

namespace zk {
namespace {

constexpr uint32_t kThreads = 512, kProducers = 256;
constexpr uint32_t kPhiImage = kBasisPaths * 64 * 2;     // one FP16 image of a basis chunk: 16 KB
constexpr uint32_t kCoefImage = kBasisRows * 64 * 2;     // one FP16 image of a coefficient chunk: 16 KB
constexpr uint32_t kOffPhi = 0;                          // [2 buffers][hi, lo]
constexpr uint32_t kOffCoef = kOffPhi + 4 * kPhiImage;   // [2 buffers][hi, lo]
// A date's staging, per credit c (2: none) and path a float4 {D, (Q' - Q) / 2 since the previous reporting date,
// (Q - Q at the next reporting date) / 2, Q} -- the no-credit record {D, 0, 0, 1} -- then per 32-path unit the sums
// of D, Q0, Q1 and the count of live paths.
constexpr uint32_t kStageFloats = kBasisStageBytes / 4;
constexpr uint32_t kOffStage = kOffCoef + 4 * kCoefImage;     // [3 buffers]
constexpr uint32_t kOffDesc = kOffStage + 3 * kBasisStageBytes;  // [2 buffers of descBytes] k-groups, then options;
                                                                  // then the fixings x 64, [slot][path]
static_assert(kOffDesc == kBasisFixedSmem, "the layout of basisSmemBytes");
// TMEM columns: the accumulators of three consecutive dates [0, 128), [128, 256), [256, 384); the collateral held
// per netting set and path [384, 512).
constexpr uint32_t kColHeld = 384;

struct Factors {
  float x, D, S[4], Q[2], xf[2];
};

__device__ __forceinline__ float pick(const float (&a)[4], uint32_t i) {
  return i == 0 ? a[0] : i == 1 ? a[1] : i == 2 ? a[2] : a[3];
}

// The unscaled Black price of an option (a basis option record in shared memory: A, B, P_f, B_f, K, 1 / K, 1 / sd,
// sd / 2, sd, flags): revalueKernel's kOption / kForeignOption with the reference's guards and A&S normal CDF
// (fused_kernels.cpp:201-215), the divisions by K and sd replaced by the record's reciprocals.
__device__ __forceinline__ float optionPrice(const float* rec, bool foreign, const Factors& f) {
  const float4 r0 = reinterpret_cast<const float4*>(rec)[0], r1 = reinterpret_cast<const float4*>(rec)[1];
  const float4 r2 = reinterpret_cast<const float4*>(rec)[2];
  const uint32_t flags = static_cast<uint32_t>(r2.y), a = flags & 3u;
  const float b0 = r0.x * fastExp(-r0.y * f.x);
  const float q = foreign ? r0.z * fastExp(-r0.w * (a == 0 ? f.xf[0] : f.xf[1])) : r0.z;
  const float F = __fdividef(pick(f.S, a) * q, b0), K = r1.x;
  const float s = (flags & 4u) ? 1.0f : -1.0f;
  if (r1.z == 0.0f || F <= 0.0f) return b0 * fmaxf(s * (F - K), 0.0f);
  const float d1 = __logf(F * r1.y) * r1.z + r1.w, d2 = d1 - r2.x;
  return b0 * s * (F * ncdf(s * d1) - K * ncdf(s * d2));
}

// One k-group of the basis for this thread's path: 8 values of one column type, as FP16 hi and lo (the k-group and
// the option records in shared memory).
__device__ __forceinline__ void basisGroup(const BasisKg* kg, const float* options, const Factors& f, const float* fixS,
                                           uint32_t row, uint4& hi, uint4& lo) {
  const float4 b0 = reinterpret_cast<const float4*>(kg)[0], b1 = reinterpret_cast<const float4*>(kg)[1];
  const uint4 sw = reinterpret_cast<const uint4*>(kg)[2];
  const uint4 tm = reinterpret_cast<const uint4*>(kg)[3];
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
    case kColForeign: {  // one asset per k-group
      const float S = pick(f.S, sel[0]), xf = sel[0] == 0 ? f.xf[0] : f.xf[1];
#pragma unroll
      for (int e = 0; e < 8; ++e) phi[e] = S * ex2(b[e] * xf);
      break;
    }
    case kColSpot: {
      const float S = pick(f.S, sel[0]);
#pragma unroll
      for (int e = 0; e < 8; ++e) phi[e] = S;
      break;
    }
    default:  // options, one record per column
#pragma unroll
      for (int e = 0; e < 8; ++e)
        phi[e] = mult * optionPrice(options + kBasisOptWords * sel[e], type == kColForeignOption, f);
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

// A bounded mbarrier wait whose polls suspend the warp (up to kSuspendNs each) instead of spinning, so waiting warps
// leave the issue slots to the working ones.
constexpr uint32_t kSuspendNs = 1000, kSleepLimit = 1u << 22;  // at most about 4 s
__device__ __forceinline__ bool waitSleep(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < kSleepLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smemAddr(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Producers' barrier (named barrier 1, the 256 producer threads), and-reducing a predicate.
__device__ __forceinline__ bool producersAnd(bool v) {
  uint32_t r;
  asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, 1, 256, p;\n selp.u32 %0, 1, 0, q;\n}\n"
               : "=r"(r)
               : "r"(v ? 1u : 0u)
               : "memory");
  return r != 0;
}

__global__ void __launch_bounds__(kThreads, 1) basisRevalueKernel(const BasisArgs* __restrict__ groups, uint32_t descBytes,
                                                                  uint32_t* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ BasisArgs G;
  __shared__ __align__(8) uint64_t loadBar[2], mmaBar[2], descBar[2], accFull[3], stageFull[3], epiDone[3];
  __shared__ uint32_t tslot;
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  if (warp == 0) umma::alloc(&tslot, 512);  // one CTA per SM (its shared memory): the whole TMEM is free
  if (tid == 0) {
    G = groups[blockIdx.y];
    for (int b = 0; b < 2; ++b) mbarInit(&loadBar[b], 1), mbarInit(&mmaBar[b], 1), mbarInit(&descBar[b], 1);
    for (int b = 0; b < 3; ++b) mbarInit(&accFull[b], 1), mbarInit(&stageFull[b], 1), mbarInit(&epiDone[b], 8);
  }
  umma::fenceBeforeSync();
  __syncthreads();
  umma::fenceAfterSync();
  if (tid >= kProducers) {  // the three accumulators and the collateral held start at zero (finite) for every lane
    const uint32_t cw = warp - kProducers / 32, base = tslot + ((32u * (cw & 3u)) << 16) + (cw >> 2) * 64u;
    const uint32_t z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
    for (uint32_t c = 0; c < 512; c += 128)
#pragma unroll
      for (uint32_t q8 = 0; q8 < 64; q8 += 8) umma::st8(base + c + q8, z);
    umma::waitSt();
  }
  umma::fenceBeforeSync();
  __syncthreads();  // before any product writes an accumulator
  umma::fenceAfterSync();
  const uint32_t nP = G.nP, nT = G.nT, tile = blockIdx.x;
  float* fixS = reinterpret_cast<float*>(sm + kOffDesc + 2 * descBytes);
  float* stageAll = reinterpret_cast<float*>(sm + kOffStage);
  const size_t fs = static_cast<size_t>(nT) * nP;
  bool ok = true;

  if (tid < kProducers) {
    // ================================ producers ================================
    const uint32_t row = tid & 127u, half = tid >> 7;
    const uint32_t path = tile * kBasisPaths + row, pp = path < nP ? path : nP - 1;
    const bool live = path < nP;
    const float* cubeP = G.cube + pp;
    // A date's record: (firstChunk, numChunks, firstKg, numKg), (fixBegin, fixEnd, optBegin, callIndex),
    // (reportingSlot, nextReporting, prevChunks, numOptions).
    auto loadDate = [&](uint32_t j, uint4 (&d)[3]) {
      const uint4* dj = reinterpret_cast<const uint4*>(G.dates + static_cast<size_t>(j) * kBasisDateWords);
      d[0] = __ldg(dj), d[1] = __ldg(dj + 1), d[2] = __ldg(dj + 2);
    };
    // The factors of date j, and on a reporting date the survivals at the next reporting date.
    auto loadFactors = [&](uint32_t j, const uint4 (&d)[3], Factors& f, float (&qn)[2]) {
      const float* c = cubeP + static_cast<size_t>(j) * nP;
      f.x = __ldg(c), f.D = __ldg(c + fs);
#pragma unroll
      for (uint32_t a = 0; a < 4; ++a) f.S[a] = a < G.nA ? __ldg(c + (G.fS + a) * fs) : 0.0f;
#pragma unroll
      for (uint32_t q = 0; q < 2; ++q) f.Q[q] = q < G.nC ? __ldg(c + (G.fQ + q) * fs) : 1.0f;
#pragma unroll
      for (uint32_t a = 0; a < 2; ++a) f.xf[a] = a < G.nF ? __ldg(c + (G.fXf + a) * fs) : 0.0f;
      const uint32_t rs = d[2].x, nextRep = d[2].y;
#pragma unroll
      for (uint32_t q = 0; q < 2; ++q)
        qn[q] = rs > 0 && nextRep < nT && q < G.nC ? __ldg(cubeP + (G.fQ + q) * fs + static_cast<size_t>(nextRep) * nP)
                                                   : f.Q[q];
    };
    // Thread 0: the k-groups and option records of date j into descriptor buffer j % 2 (issued a date ahead).
    auto loadDesc = [&](const uint4 (&d)[3], uint32_t j) {
      const uint32_t kgBytes = d[0].w * static_cast<uint32_t>(sizeof(BasisKg)), optBytes = d[2].w * 4u * kBasisOptWords;
      unsigned char* dst = sm + kOffDesc + (j & 1u) * descBytes;
      if (kgBytes + optBytes == 0) {
        mbarArrive(&descBar[j & 1u]);
        return;
      }
      mbarExpectTx(&descBar[j & 1u], kgBytes + optBytes);
      if (kgBytes) bulkLoad(dst, G.kgs + d[0].z, kgBytes, &descBar[j & 1u]);
      if (optBytes) bulkLoad(dst + kgBytes, G.options + kBasisOptWords * static_cast<size_t>(d[1].z), optBytes, &descBar[j & 1u]);
    };
    float prevQ[2] = {1.0f, 1.0f};
    uint32_t g = 0;                               // chunks started (all dates)
    int issued = -1, loaded = -1, consumed = -1;  // thread 0: the last chunk whose MMAs / copy were issued / waited
    int descIssued = -1;                          // thread 0: the last date whose descriptors were requested
    uint4 nd[3];
    loadDate(0, nd);
    Factors nf;
    float nqn[2];
    loadFactors(0, nd, nf, nqn);
    if (tid == 0) loadDesc(nd, 0), descIssued = 0;
    for (uint32_t j = 0; j < nT; ++j) {
      const uint4 d0 = nd[0], d1 = nd[1], d2 = nd[2];
      const uint32_t numChunks = d0.y, numKg = d0.w;
      const uint32_t fixBegin = d1.x, fixEnd = d1.y, rs = d2.x;
      const Factors f = nf;
      const float qn[2] = {nqn[0], nqn[1]};
      if (j + 1 < nT) {
        loadDate(j + 1, nd);
        loadFactors(j + 1, nd, nf, nqn);
        // descriptor buffer (j + 1) % 2 held date j - 1's, which every producer finished (the last barrier)
        if (tid == 0) loadDesc(nd, j + 1), descIssued = static_cast<int>(j + 1);
      }
      // the staging buffer of date j was last read by the epilogue of date j - 3
      if (j >= 3) ok = waitSleep(&epiDone[j % 3], ((j - 3) / 3) & 1u) && ok;
      if (half == 0) {
        float* st = stageAll + (j % 3) * kStageFloats;
        float4* cs = reinterpret_cast<float4*>(st);
#pragma unroll
        for (uint32_t q = 0; q < 2; ++q) {
          cs[q * kBasisPaths + row] = make_float4(f.D, j > 0 && rs > 0 ? 0.5f * (prevQ[q] - f.Q[q]) : 0.0f,
                                                  rs > 0 ? 0.5f * (f.Q[q] - qn[q]) : 0.0f, f.Q[q]);
          if (rs > 0) prevQ[q] = f.Q[q];
        }
        cs[2 * kBasisPaths + row] = make_float4(f.D, 0.0f, 0.0f, 1.0f);
        float u[4] = {live ? f.D : 0.0f, live ? f.Q[0] : 0.0f, live ? f.Q[1] : 0.0f, live ? 1.0f : 0.0f};
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
          for (uint32_t o = 16; o > 0; o >>= 1) u[k] += __shfl_xor_sync(0xFFFFFFFFu, u[k], o);
        if (lane == 0) {
          float* us = st + 12 * kBasisPaths + (row >> 5) * 4;
          us[0] = u[0], us[1] = u[1], us[2] = u[2], us[3] = u[3];
        }
      }
      const unsigned char* desc = sm + kOffDesc + (j & 1u) * descBytes;
      const BasisKg* kgS = reinterpret_cast<const BasisKg*>(desc);
      const float* optS = reinterpret_cast<const float*>(desc + numKg * sizeof(BasisKg));
      ok = waitSleep(&descBar[j & 1u], (j >> 1) & 1u) && ok;
      // ---- basis chunks and their products ----
      for (uint32_t c = 0; c < numChunks; ++c, ++g) {
        const uint32_t buf = g & 1u;
        if (g >= 2) ok = waitSleep(&mmaBar[buf], ((g - 2) >> 1) & 1u) && ok;  // chunk g - 2 freed both buffers
        const uint32_t kgs = 2u * __ldg(G.chunks + 2 * g + 1);
        if (tid == 0 && ok) {  // this chunk's coefficients, landing while the basis below is evaluated
          const uint32_t bytes = kgs * 4096u;
          mbarExpectTx(&loadBar[buf], bytes);
          bulkLoad(sm + kOffCoef + buf * 2 * kCoefImage, G.blob + __ldg(G.chunks + 2 * g), bytes, &loadBar[buf]);
          loaded = static_cast<int>(g);
        }
        unsigned char* phiHi = sm + kOffPhi + buf * 2 * kPhiImage;
        for (uint32_t kgl = half; kgl < kgs; kgl += 2) {
          uint4 hi, lo;
          basisGroup(kgS + c * kBasisChunkKg + kgl, optS, f, fixS, row, hi, lo);
          const uint32_t off = umma::kMajorOffset(row, kgl * 8u, kBasisPaths);
          *reinterpret_cast<uint4*>(phiHi + off) = hi;
          *reinterpret_cast<uint4*>(phiHi + kPhiImage + off) = lo;
        }
        umma::fenceAsyncShared();
        ok = producersAnd(ok);
        if (!ok) break;
        if (tid == 0) {
          bool t0 = waitSleep(&loadBar[buf], (g >> 1) & 1u);
          if (t0) consumed = static_cast<int>(g);
          // the date's accumulator held date j - 3, read last (as the previous value) by the epilogue of date j - 2
          if (t0 && c == 0 && j >= 2) t0 = waitSleep(&epiDone[(j - 2) % 3], ((j - 2) / 3) & 1u);
          if (t0) {
            umma::fenceAfterSync();
            const uint32_t steps = kgs / 2u, acc = tslot + (j % 3) * 128u;
            const uint32_t aHi = umma::smem(sm + kOffCoef + buf * 2 * kCoefImage), aLo = aHi + steps * 4096u;
            const uint32_t bHi = umma::smem(phiHi), bLo = bHi + kPhiImage;
            constexpr uint32_t idesc = umma::idescF16(kBasisRows, kBasisPaths);
            for (uint32_t i = 0; i < steps; ++i) {
              const uint64_t dAh = umma::desc(aHi + i * 4096u, 2048u, 128u), dAl = umma::desc(aLo + i * 4096u, 2048u, 128u);
              const uint64_t dBh = umma::desc(bHi + i * 4096u, 2048u, 128u), dBl = umma::desc(bLo + i * 4096u, 2048u, 128u);
              umma::mma(acc, dAh, dBh, idesc, c > 0 || i > 0);
              umma::mma(acc, dAh, dBl, idesc, true);
              umma::mma(acc, dAl, dBh, idesc, true);
            }
            umma::commit(&mmaBar[buf]);
            if (c + 1 == numChunks) umma::commit(&accFull[j % 3]);
            issued = static_cast<int>(g);
          }
          ok = t0;
        }
      }
      ok = producersAnd(ok);  // the staging written, thread 0's last issue known
      if (!ok) break;
      if (tid == 0) {
        mbarArrive(&stageFull[j % 3]);
        if (numChunks == 0) mbarArrive(&accFull[j % 3]);  // no products: the epilogue takes the value as 0
      }
      // ---- the date's fixings, read from the next date on ----
      for (uint32_t q = fixBegin + half; q < fixEnd; q += 2) {
        const float4 r = __ldg(G.fixings + q);
        fixS[static_cast<uint32_t>(r.w) * kBasisPaths + row] = (r.x * ex2(r.y * f.x) - 1.0f) * r.z * kCouponScale;
      }
      ok = producersAnd(ok);
      if (!ok) break;
    }
    if (tid == 0) {
      if (!ok) atomicExch(err, kDevTimeout);
      // the work in flight settles before the TMEM and the shared memory go away
      if (!ok && issued >= 0) waitSleep(&mmaBar[issued & 1], (static_cast<uint32_t>(issued) >> 1) & 1u);
      if (loaded > consumed) waitSleep(&loadBar[loaded & 1], (static_cast<uint32_t>(loaded) >> 1) & 1u);
      // a date's descriptors requested and never waited for (the last date's, or after a failure)
      for (int d = descIssued; d >= 0 && d + 2 > descIssued; --d)
        waitSleep(&descBar[d & 1], (static_cast<uint32_t>(d) >> 1) & 1u);
    }
  } else {
    // ================================ consumers ================================
    const uint32_t cw = warp - kProducers / 32, qtr = cw & 3u, half = cw >> 2;
    const uint32_t nsRow = 32u * qtr + lane;
    const bool nsLive = nsRow < G.numNs;
    const uint32_t tl = tslot + ((32u * qtr) << 16);  // this warp's TMEM lanes
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
    const bool hasQ = cpty < 2u;
    const uint32_t qc = hasQ ? cpty : 2u;  // the staging record of the counterparty's survival (2: none)
    // the call rule (collateral.cpp:10-47) branch-free: required = max(vc - hc, 0) + min(vc + hb, 0), the second
    // term absent for a one-way CSA (hb < 0); one of the two is always zero, so the sum is exact
    const float hbEff = hb >= 0.0f ? hb : __int_as_float(0x7F800000);
    const bool vecRows = nP % 4u == 0u;
    float fwd[2] = {0.0f, 0.0f};  // 0.5 sum DE (Q - Q_next) of the last reporting date, per unit
    // the date's record words and scale, loaded a date ahead
    auto loadDate = [&](uint32_t j, uint4& w, float& scale) {
      const uint32_t* dj = G.dates + static_cast<size_t>(j) * kBasisDateWords;
      w = make_uint4(__ldg(dj + bdChunks), __ldg(dj + bdCall), __ldg(dj + bdRep), __ldg(dj + bdPrevChunks));
      scale = __ldg(G.scale + static_cast<size_t>(j) * kBasisRows + nsRow);
    };
    uint4 nw;
    float nsc, sc = 0.0f;
    loadDate(0, nw, nsc);
    for (uint32_t j = 0; j < nT; ++j) {
      const uint32_t numChunks = nw.x, callJ = nw.y, rs = nw.z, prevChunks = nw.w;
      const float scPrev = sc;
      sc = nsc;
      if (j + 1 < nT) loadDate(j + 1, nw, nsc);
      bool w = waitSleep(&stageFull[j % 3], (j / 3) & 1u);
      w = w && waitSleep(&accFull[j % 3], (j / 3) & 1u);
      if (!__all_sync(0xFFFFFFFFu, w)) {
        ok = false;
        break;
      }
      umma::fenceAfterSync();
      const float* st = stageAll + (j % 3) * kStageFloats;
      const float4* cs = reinterpret_cast<const float4*>(st) + qc * kBasisPaths;
      const float scJ = numChunks > 0 ? sc : 0.0f, scP = prevChunks > 0 ? scPrev : 0.0f;  // no products: value 0
      const uint32_t accCol = (j % 3) * 128u, prevCol = ((j + 2) % 3) * 128u;
      const float mtaJ = j == 0 ? -1.0f : mta;  // date 0 always calls
      float* const rowJ = rs > 0 && nsLive ? rowEP + static_cast<size_t>(rs - 1) * nP + tile * kBasisPaths : nullptr;
#pragma unroll 1
      float h8[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};  // the warp's 64 paths: its two units in order
      for (uint32_t u = 0; u < 2; ++u) {
        const uint32_t p00 = half * 64u + u * 32u;  // the unit's first path in the tile
        const uint32_t first = tile * kBasisPaths + p00;
        const uint32_t paths = first < nP ? min(32u, nP - first) : 0u;
        if (paths == 0) continue;
        float s[7] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};  // e, ep, en, D ep, D en, CVA, next CVA part
#pragma unroll 1
        for (uint32_t q8 = 0; q8 < 32; q8 += 8) {
          const uint32_t p0 = p00 + q8;
          uint32_t r[24];
          umma::ld8x3(tl + accCol + p0, tl + prevCol + p0, tl + kColHeld + p0, r);
          uint32_t hs[8];
          float ep8[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const uint32_t p = p0 + i;
            const float v = __uint_as_float(r[i]) * scJ, vPrev = __uint_as_float(r[8 + i]) * scP;
            // cash, the margin call at t - MPR, at most one date back; without a CSA the state runs and is not used
            float held = __uint_as_float(r[16 + i]);
            const float vc = callJ != j ? vPrev : v;
            const float required = fmaxf(vc - hc, 0.0f) + fminf(vc + hbEff, 0.0f);
            held = fabsf(required - held) >= mtaJ ? required : held;
            const float collateral = hasCsa ? held + ia : 0.0f;
            hs[i] = __float_as_uint(held);
            const float e = v - collateral, ep = fmaxf(e, 0.0f), en = fminf(e, 0.0f);
            const float4 z = cs[p];  // D, the CVA survival differences (zero without a counterparty), Q
            const float de = z.x * ep;
            ep8[i] = ep;
            if (q8 + i < paths) {
              s[0] += e, s[1] += ep, s[2] += en, s[3] += de, s[4] = fmaf(z.x, en, s[4]);
              if (rs > 0) s[5] = fmaf(de, z.y, s[5]), s[6] = fmaf(de, z.z, s[6]);
            }
          }
          umma::st8(tl + kColHeld + p0, hs);
          if (rowJ) {
            float* dst = rowJ + p0;
            if (vecRows && q8 + 8 <= paths) {
              reinterpret_cast<float4*>(dst)[0] = make_float4(ep8[0], ep8[1], ep8[2], ep8[3]);
              reinterpret_cast<float4*>(dst)[1] = make_float4(ep8[4], ep8[5], ep8[6], ep8[7]);
            } else {
#pragma unroll
              for (uint32_t i = 0; i < 8; ++i)
                if (q8 + i < paths) dst[i] = ep8[i];
            }
          }
        }
        umma::waitSt();  // the unit's collateral held, in TMEM before the next date reads it
        const float cva = rs > 0 ? s[5] + fwd[u] : 0.0f;
        if (rs > 0) fwd[u] = s[6];
        const float* us = st + 12 * kBasisPaths + (p00 >> 5) * 4;
        h8[0] += s[0], h8[1] += s[1], h8[2] += s[2], h8[3] += s[3], h8[4] += s[4], h8[5] += cva;
        h8[6] += us[hasQ ? 1 + qc : 3], h8[7] += us[0];
      }
      // one partial per 64 paths (the reduce kernel's two-paths-per-lane layout): written when its first path is live
      if (nsLive && tile * kBasisPaths + half * 64u < nP) {
        const uint32_t unit = tile * 2u + half;
        float4* pt = reinterpret_cast<float4*>(partials + (static_cast<size_t>(unit) * nT + j) * kStatsPerDate);
        pt[0] = make_float4(h8[0], h8[1], h8[2], h8[3]);
        pt[1] = make_float4(h8[4], h8[5], h8[6], h8[7]);
      }
      __syncwarp();
      umma::fenceBeforeSync();
      if (lane == 0) mbarArrive(&epiDone[j % 3]);
    }
    if (!ok && lane == 0) atomicExch(err, kDevTimeout);
  }
  umma::fenceBeforeSync();
  __syncthreads();
  __syncwarp();
  if (warp == 0) umma::dealloc(tslot, 512);
}

}  // namespace

cudaError_t launchBasisRevalue(const BasisArgs* groups, uint32_t numGroups, uint32_t nP, uint32_t descBytes, uint32_t fixSlots,
                               uint32_t* err, cudaStream_t stream) {
  if (numGroups == 0 || nP == 0) return cudaSuccess;
  const uint32_t smem = basisSmemBytes(descBytes, fixSlots);
  if (smem > kBasisMaxSmem) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(basisRevalueKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  const dim3 grid((nP + kBasisPaths - 1) / kBasisPaths, numGroups);
  basisRevalueKernel<<<grid, kThreads, smem, stream>>>(groups, descBytes, err);
  return cudaGetLastError();
}

}  // namespace zk
