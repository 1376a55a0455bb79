// Device-side constants, plan views and math shared by the kernels of zlatko_b200.
//
// The plan layout is the reference's (include/ccr/gpu/fused_exposure.hpp:35-151): a 32-word
// header, index table, 84 parameters, 24 step coefficients per date and 8-word valuation terms.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace zk {

constexpr int kTile = 128;             // threads per CTA of the revalue kernel
constexpr int kWarps = kTile / 32;
constexpr int kHeaderWords = 32;
constexpr int kStepStride = 24;
constexpr int kTermStride = 8;
constexpr int kRequestStride = 8;
constexpr int kChol = 8;               // padded Cholesky row length
constexpr int kParamCount = 16 + kChol * kChol + 4;
constexpr int kStatsPerDate = 8;
constexpr int kTradeStats = 5;
constexpr int kMaxAssets = 4;
constexpr int kMaxCredits = 2;
constexpr int kMaxSwapSlots = 32;
constexpr int kMaxNormals = 64;
constexpr int kMaxBermudans = 4;          // Bermudans of a plan in the reference's layout (exercise state in registers)
constexpr int kMaxBermudansPerPlan = 256;  // beyond 4: exercise state in shared memory, the index's high bits in the code
constexpr int kMaxTradeGroups = 16;
constexpr int kMaxRing = 32;           // look-back depth (dates) of the CSA margin call kept on chip
constexpr int kMaxInnerPaths = 1024;    // inner paths of the nested initial margin per outer path and date
constexpr int kTermChunk = 128;        // terms staged in shared memory at a time
constexpr uint32_t kNoRow = 0xFFFFFFFFu;

enum TermKind : uint32_t {
  kBond = 0, kFixedFloat = 1, kAsset = 2, kSetFixing = 3, kOption = 4,
  kBermExercise = 5, kBermDecide = 6, kBermContinue = 7, kBermBond = 8, kBermFloat = 9, kProbe = 10,
  // Terms on an asset whose foreign short rate is stochastic (an extension of the reference's kinds; the asset is
  // the code's extra field, rec[1] the foreign bond's B_f): a forward's c S P_f(t, T | x_f) and a Black option on
  // the forward S P_f(t, T | x_f) / P(t, T | x).
  kForeignForward = 11, kForeignOption = 12,
  // A Bermudan's two-regressor basis (an extension): before its policy or continuation record the co-terminal swap's
  // annuity terms (tau, A, B) and float-leg terms (+-1, A, B), each c A e^{-B x}; after it two records of its
  // coefficients.  The record (center_x, 1 / scale_x, center_s, 1 / scale_s, c0, c1) and the extensions (c2..c8),
  // (c9) give sum_k c_k m_k(z, w) over the graded monomials 1, z, w, z^2, z w, w^2, z^3, z^2 w, z w^2, w^3 of
  // z = (x - center_x) / scale_x and w = (s - center_s) / scale_s, s = float leg / annuity.
  kBermAnnuity = 13, kBermCoterm = 14, kBermExt = 15,
};

// Header words (fused_kernels.cpp:32-41).
enum HeaderWord : int {
  hP = 0, hT = 1, hA = 2, hC = 3, hSub = 4, hNormals = 5, hSeed = 6, hAnti = 7, hCsa = 8, hCpty = 9,
  hStepVec = 10, hCorr = 11, hOffCall = 12, hOffRep = 13, hQuantile = 14, hNumWG = 15, hS = 16, hR = 17,
  hTr = 18, hRowDV = 19, hRowE = 20, hRowV = 21, hRowC = 22, hRowGross = 23, hRowTrades = 24, hRowEx = 25,
  hReq = 26, hBerm = 27, hRowEP = 28, hRowIm = 29, hInner = 30, hImLevel = 31,
};

// Error word written by kernels (checked by the host after each launch sequence).
enum DeviceError : uint32_t { kDevOk = 0, kDevTimeout = 1, kDevBadTerm = 2 };

// ---- the scenario: everything the risk-factor simulation needs (shared by a batch of plans) ----
template <typename R>
struct ScenarioArgs {
  uint32_t nP, nT, nA, nC, substeps, nNormals, nCorr, seed, antithetic, nStreams;
  uint32_t nF, stepStride;  // stochastic foreign rates (of assets 0 .. nF - 1) and the step row length (24 + 8 nF)
  const R* steps;     // [nT][24]; columns 0..21 are shared by every plan of the batch
  const R* normals;   // injected normals [step][normal][stream], or nullptr (counter-based generator)
  // Path p of the launch simulates path pathMap[p] of the plan (its normals and antithetic sign; null: p itself):
  // the re-run of chosen paths by the exact-decision check.
  const uint32_t* pathMap;
  R cir[8];           // (kappa, theta, xi, y0) per credit
  R spots[4];
  R chol[kChol * kChol];
};

// ---- the simulated risk factors, path-major: data[(field * nT + date) * nP + path] ----
// fields: 0 x, 1 D, fS + a the asset levels, fQ + c the survival of credit c, and when probes read
// them fLnS + a the log asset returns and fY + c the CIR states.
template <typename R>
struct CubeArgs {
  R* data;
  uint32_t nP, nT, nA, nC;
  uint32_t fS, fQ, fLnS, fY;
  uint32_t probes, pad;
  uint32_t fXf, nF;  // the foreign short-rate states x_f of assets 0 .. nF - 1 (fields fXf + f)
};

// ---- one netting set (one plan) inside a launch ----
template <typename R>
struct NsArgs {
  // The plan's term table lowered at upload (lowerTerms in capi.cu): per date a descriptor
  // {floatBegin, bondBegin, assetBegin, genericBegin, fixingBegin, end, callIndex, reportingSlot} into a
  // table of 4-value records holding the date's floating coupons, bond pairs, asset forwards, generic
  // 8-word terms and fixings.
  const uint32_t* dates;   // [nT][8]
  const R* table;          // [*][4]
  const R* steps;          // this plan's step table (columns 22, 23: collateral bond A, B)
  R* expo;                 // [rowsTotal][nP] rows of the path views
  R* partials;             // [numTiles][nT][nS]
  R hc, hb, mta, ia, keepHaircut;
  uint32_t hasCsa, ctype, casset, cpty, nS, nTr, nBerm, nR;
  uint32_t rowEP, rowDV, rowE, rowV, rowC, rowGross, rowTrades, rowEx;
  uint32_t offCall, offRep, nSlots, ring;
  uint32_t usesAssets;     // some term reads an asset level
  uint32_t usesForeign;    // some term reads a foreign short-rate state
  uint32_t manyBerm;       // more than 4 Bermudans: exercise indices in shared memory, bytes [nBerm][PPT][kTile]
  uint32_t stepStride;     // values per row of `steps`
  uint32_t pad0;
  // AMC state pass (zk_amc_states, zk_fit_amc): x / deflator [date][path] and exercise values [row][path].
  R* sinkX;
  R* sinkD;
  R* sinkEx;
  const uint32_t* sinkRowOfBermudan;  // first exercise row of each Bermudan
  // Nested initial margin: on each reporting date the outer state the inner paths start from, written to
  // imState[(slot * imWords + w) * nP + path] with w = 0 the netted value, 1..4 the Bermudans' exercise
  // indices, 5.. the fixings (imWords = 5 + nSlots; imState null without the nested margin).
  R* imState;
  uint32_t imWords, pad1;
  // Exact decisions (zk_context_set_exact_decisions): a path with a margin call or an exercise decision whose margin
  // lies within guard[date] of the rule's boundary sets its bit in flags[path / 32]; the host re-runs those paths in
  // double precision.  flags null: off.
  uint32_t* flags;
  const R* guard;
};

// Marks path p for the double-precision re-check (a rare event: one atomic per flagged decision).
__device__ __forceinline__ void flagPath(uint32_t* flags, uint32_t p) { atomicOr(flags + (p >> 5), 1u << (p & 31u)); }

// ---- counter-based normals: PCG hash + Box-Muller, keyed by (seed, path stream, date, pair) ----
// The hash and the key mixing follow the reference kernel (fused_kernels.cpp:185-199,
// fused_reference.cpp:19-34) so that both draw the same normals for the same plan.
__device__ __forceinline__ uint32_t pcg(uint32_t v) {
  const uint32_t state = v * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

__device__ __forceinline__ void gauss2(uint32_t stream, uint32_t j, uint32_t k, float& z0, float& z1) {
  const uint32_t h1 = pcg(stream ^ pcg(j * 131u + k));
  const uint32_t h2 = pcg(h1 ^ 0x68E31DA4u);
  const float u1 = (static_cast<float>(h1 >> 8u) + 0.5f) * (1.0f / 16777216.0f);
  const float u2 = (static_cast<float>(h2 >> 8u) + 0.5f) * (1.0f / 16777216.0f);
  const float r = sqrtf(-2.0f * logf(u1)), a = 6.2831853f * u2;
  float s, c;
  sincosf(a, &s, &c);
  z0 = r * c;
  z1 = r * s;
}

__device__ __forceinline__ void gauss2(uint32_t stream, uint32_t j, uint32_t k, double& z0, double& z1) {
  const uint32_t h1 = pcg(stream ^ pcg(j * 131u + k));
  const uint32_t h2 = pcg(h1 ^ 0x68E31DA4u);
  const double u1 = (static_cast<double>(h1 >> 8u) + 0.5) / 16777216.0;
  const double u2 = (static_cast<double>(h2 >> 8u) + 0.5) / 16777216.0;
  const double r = sqrt(-2.0 * log(u1)), a = 6.283185307179586 * u2;
  double s, c;
  sincos(a, &s, &c);
  z0 = r * c;
  z1 = r * s;
}

// 2^x on the special-function unit (ex2.approx.ftz: relative error about 2^-22).
__device__ __forceinline__ float ex2(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Exponentials of the hot term loop.  In single precision the special-function unit evaluates
// 2^(x log2 e) (relative error about 2^-22 for the small arguments of bond terms); double precision
// uses the library exp (within 1 ulp).
__device__ __forceinline__ float fastExp(float x) { return ex2(x * 1.4426950408889634f); }
__device__ __forceinline__ double fastExp(double x) { return exp(x); }

__device__ __forceinline__ float rexp(float x) { return expf(x); }
__device__ __forceinline__ double rexp(double x) { return exp(x); }
__device__ __forceinline__ float rlog(float x) { return logf(x); }
__device__ __forceinline__ double rlog(double x) { return log(x); }
__device__ __forceinline__ float rsqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double rsqrt_(double x) { return sqrt(x); }

// Normal CDF.  Single precision uses the Abramowitz-Stegun 7.1.26 erf approximation, the form the
// reference kernel prices options with (fused_kernels.cpp:201-207); double precision uses the exact
// 0.5 erfc(-x / sqrt 2) of the FP64 engine (include/ccr/core/math.hpp:15), its oracle.
__device__ __forceinline__ float ncdf(float x) {
  const float z = fabsf(x) * 0.70710678f;
  const float t = __fdividef(1.0f, 1.0f + 0.3275911f * z);
  const float poly = ((((1.061405429f * t - 1.453152027f) * t + 1.421413741f) * t - 0.284496736f) * t + 0.254829592f) * t;
  const float erf = 1.0f - poly * fastExp(-z * z);
  return x >= 0.0f ? 0.5f * (1.0f + erf) : 0.5f * (1.0f - erf);
}
__device__ __forceinline__ double ncdf(double x) { return 0.5 * erfc(-x / 1.4142135623730951); }

// df * Black(F, K, sd), call or put: the reference kernel's guards in single precision
// (fused_kernels.cpp:209-215; log, divisions and the erf exponential on the special-function unit),
// the FP64 engine's in double (math.hpp:24-31).
__device__ __forceinline__ float black(float F, float K, float sd, float df, bool isCall) {
  const float s = isCall ? 1.0f : -1.0f;
  if (sd <= 1e-7f || F <= 0.0f) return df * fmaxf(s * (F - K), 0.0f);
  const float d1 = __fdividef(__logf(__fdividef(F, K)), sd) + 0.5f * sd;
  const float d2 = d1 - sd;
  return df * s * (F * ncdf(s * d1) - K * ncdf(s * d2));
}
__device__ __forceinline__ double black(double F, double K, double sd, double df, bool isCall) {
  const double s = isCall ? 1.0 : -1.0;
  if (sd <= 1e-14 || F <= 0.0 || K <= 0.0) return df * fmax(s * (F - K), 0.0);
  const double d1 = log(F / K) / sd + 0.5 * sd;
  const double d2 = d1 - sd;
  return df * s * (F * ncdf(s * d1) - K * ncdf(s * d2));
}

// Per-trade statistic m of trade value vi in netting-set value v (fused_kernels.cpp:174-183).
template <typename R>
__device__ __forceinline__ R tradeStat(uint32_t m, R vi, R v, R D) {
  const R pos = v > R(0) ? R(1) : R(0);
  switch (m) {
    case 0: return D * vi * pos;
    case 1: return vi * pos;
    case 2: return D * (fmax(v, R(0)) - fmax(v - vi, R(0)));
    case 3: return D * fmax(vi, R(0));
    default: return fmax(vi, R(0));
  }
}

// AMC regression z = (x - c) * A, B + p1 z + p2 z^2 + p3 z^3 (fused_kernels.cpp:78-81).
template <typename R>
__device__ __forceinline__ R amcPoly(const R* rec, R x) {
  const R z = (x - rec[2]) * rec[3];
  return ((rec[7] * z + rec[6]) * z + rec[5]) * z + rec[4];
}

// The two-regressor continuation (see kBermAnnuity) at (x, s): rec the policy / continuation record, e1 and e2 its
// extension records.
template <typename R>
__device__ __forceinline__ R amcPoly2(const R* rec, const R* e1, const R* e2, R x, R s) {
  const R z = (x - rec[2]) * rec[3], w = (s - rec[4]) * rec[5];
  const R zz = z * z, zw = z * w, ww = w * w;
  return rec[6] + rec[7] * z + e1[1] * w + e1[2] * zz + e1[3] * zw + e1[4] * ww + e1[5] * zz * z + e1[6] * zz * w +
         e1[7] * zw * w + e2[1] * ww * w;
}

// The Bermudan of an AMC term's code: bits 8-11, and with more than 4 Bermudans in the plan bits 4-7 above them
// (the trade-group field, which such plans leave to the Bermudan index).
__host__ __device__ __forceinline__ uint32_t bermudanOf(uint32_t code, bool many) {
  return many ? (((code >> 8u) & 15u) | (((code >> 4u) & 15u) << 4u)) : ((code >> 8u) & 15u) < 3u ? ((code >> 8u) & 15u) : 3u;
}

// Order-preserving float <-> uint32 keys (for min / max / radix selection of signed values).
__device__ __forceinline__ uint32_t floatKey(float v) {
  const uint32_t b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float keyFloat(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}
__device__ __forceinline__ unsigned long long doubleKey(double v) {
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(v));
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double keyDouble(unsigned long long k) {
  return __longlong_as_double(static_cast<long long>((k & 0x8000000000000000ull) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k));
}

// ---- bounded mbarrier waits (the kernel never spins forever) ----
__device__ __forceinline__ uint32_t smemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbarInit(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbarExpectTx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}

// One-dimensional bulk copy global -> shared completing on `bar` (TMA, untiled).  Source, destination
// and size must be multiples of 16 bytes.
__device__ __forceinline__ void bulkLoad(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smemAddr(dst)),
      "l"(src), "r"(bytes), "r"(smemAddr(bar))
      : "memory");
}

// One arrival on `bar` (release semantics: the thread's earlier writes are visible to a waiter that sees the phase
// complete).
__device__ __forceinline__ void mbarArrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}

// Waits for phase `parity` of `bar` to complete; gives up after `limit` polls and returns false.
__device__ __forceinline__ bool mbarWait(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace zk
