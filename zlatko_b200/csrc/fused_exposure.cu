// The exposure kernels: risk-factor simulation, then revalue -> net -> collateralise -> reduce.
//
// They execute the reference's plan semantics (the fused-exposure WGSL kernel,
// src/gpu/fused_kernels.cpp:224-530, and its CPU mirror simulatePath,
// src/gpu/fused_reference.cpp:198-422), organised for a B200 and for books of many netting sets:
//
//   simulateKernel   one thread per path draws the counter-based normals, correlates them and steps
//                    Hull-White, the lognormal assets and the CIR++ intensities once per date, writing
//                    the factor state (x, D, S, Q; lnS and y when probes read them) path-major to HBM.
//                    Every netting set of the launch reuses it: the reference re-simulates per plan.
//                    Only factors are stored, never the paths x dates x trades value cube.
//   revalueKernel    one CTA per (tile of kTile paths, netting set).  CTA ids run tile-major, so the
//                    netting sets of one tile execute together and its factor slice stays in L2.
//                    Each thread revalues its path date by date from the netting set's merged term
//                    table (warp-uniform loads, served to all 32 lanes by one L1 broadcast), applies
//                    the CSA with the margin-call look-back kept in a shared-memory ring, writes the
//                    reporting-date rows and reduces the 8 (+5 per trade) statistics of the date with a
//                    warp reduce-scatter (9 shuffles) and one cross-warp pass per 128-path group into
//                    per-group partials, which the reduce kernel sums in path order: the results are
//                    deterministic and the same for every tile shape.
#include "zk_device.cuh"
#include "zk_kernels.h"

namespace zk {

namespace {

// Lane l ends with the warp sum of statistic statSlotOfLane(l).  The lanes are combined as a binary tree over
// neighbours (xor 1, then 2, 4, 8, 16: the first three halve the 8 values, the last two complete the sums), so
// a statistic's sum over the warp's paths has the same tree whether a lane holds one path or the in-thread sum
// of 2 or 4 adjacent paths: the partials do not depend on the tile shape.
template <typename R>
__device__ __forceinline__ R warpReduceScatter8(const R (&v)[8], uint32_t lane) {
  const bool b0 = lane & 1u, b1 = lane & 2u, b2 = lane & 4u;
  R a[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const R send = b0 ? v[i] : v[i + 4];
    const R keep = b0 ? v[i + 4] : v[i];
    a[i] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, 1);
  }
  R b[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const R send = b1 ? a[i] : a[i + 2];
    const R keep = b1 ? a[i + 2] : a[i];
    b[i] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, 2);
  }
  R c = (b2 ? b[1] : b[0]) + __shfl_xor_sync(0xFFFFFFFFu, b2 ? b[0] : b[1], 4);
  c += __shfl_xor_sync(0xFFFFFFFFu, c, 8);
  c += __shfl_xor_sync(0xFFFFFFFFu, c, 16);
  return c;
}

__device__ __forceinline__ uint32_t statSlotOfLane(uint32_t lane) {
  return (lane & 1u) * 4u + ((lane >> 1) & 1u) * 2u + ((lane >> 2) & 1u);
}

template <typename R>
__device__ __forceinline__ R sel4(const R (&a)[4], uint32_t i) {
  return i == 0 ? a[0] : i == 1 ? a[1] : i == 2 ? a[2] : a[3];
}

template <typename R>
__device__ __forceinline__ void add4(R (&a)[4], uint32_t i, R v) {
  if (i == 0) a[0] += v;
  else if (i == 1) a[1] += v;
  else if (i == 2) a[2] += v;
  else a[3] += v;
}

template <typename R>
__device__ __forceinline__ void set4(R (&a)[4], uint32_t i, R v) {
  if (i == 0) a[0] = v;
  else if (i == 1) a[1] = v;
  else if (i == 2) a[2] = v;
  else a[3] = v;
}

// One term record (8 values) with warp-uniform vector loads through the read-only path.
__device__ __forceinline__ void loadTerm(const float* t, float (&r)[8]) {
  const float4 a = __ldg(reinterpret_cast<const float4*>(t));
  const float4 b = __ldg(reinterpret_cast<const float4*>(t) + 1);
  r[0] = a.x, r[1] = a.y, r[2] = a.z, r[3] = a.w, r[4] = b.x, r[5] = b.y, r[6] = b.z, r[7] = b.w;
}
__device__ __forceinline__ void loadTerm(const double* t, double (&r)[8]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(t) + k);
    r[2 * k] = v.x, r[2 * k + 1] = v.y;
  }
}

// Whether the record at lowered unit u (of a run ending at `end`) is a two-regressor policy / continuation record:
// the next record an extension (kBermExt); then its two extension records into e1, e2.
template <typename R>
__device__ __forceinline__ bool twoRegressors(const R* table, uint32_t u, uint32_t end, R (&e1)[8], R (&e2)[8]) {
  if (u + 2 >= end || (static_cast<uint32_t>(table[4 * (u + 2)]) & 15u) != kBermExt) return false;
  loadTerm(table + 4 * (u + 2), e1);
  loadTerm(table + 4 * (u + 4), e2);
  return true;
}

// The co-terminal swap rate from its float leg and annuity (0 without an annuity).
template <typename R>
__device__ __forceinline__ R swapRate(R flt, R ann) {
  return ann != R(0) ? flt / ann : R(0);
}

constexpr int kSimThreads = 256;  // threads per CTA of the simulate kernel (one path each)

// The normals of one date: every Box-Muller pair drawn up front (independent of one another, so they overlap),
// or the injected normals, into this thread's column of shared memory, normal m at col[m * kSimThreads].
template <typename R>
__device__ __forceinline__ void drawDate(uint32_t stream, uint32_t j, R sign, const R* injected, uint32_t nStreams,
                                         uint32_t injectedStream, uint32_t nNormals, R* col) {
  if (injected) {
    for (uint32_t m = 0; m < nNormals; ++m)
      col[m * kSimThreads] = sign * injected[(static_cast<size_t>(j - 1) * nNormals + m) * nStreams + injectedStream];
    return;
  }
#pragma unroll 4
  for (uint32_t q = 0; 2 * q < nNormals; ++q) {
    R z0, z1;
    gauss2(stream, j, q, z0, z1);
    col[2 * q * kSimThreads] = sign * z0;
    if (2 * q + 1 < nNormals) col[(2 * q + 1) * kSimThreads] = sign * z1;
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Risk factors of every path and date (the transitions of the reference's ScenarioGenerator:
// hull_white.cpp:40-68, lognormal_asset.cpp:17-22, cir_intensity.cpp:49-66, in the statement order
// of the reference kernel).
template <typename R>
__global__ void __launch_bounds__(kSimThreads) simulateKernel(const ScenarioArgs<R> sc, CubeArgs<R> cb, bool bridgeTable) {
  extern __shared__ __align__(16) unsigned char simRaw[];
  R* col = reinterpret_cast<R*>(simRaw) + threadIdx.x;  // this thread's normals of the current date
  // The Brownian-bridge coefficients of the CIR sub-steps are the same for every path: with bridgeTable the
  // CTA computes them once, [date][sub-step][a, b] after the normals, by the very operations of the loop below.
  const uint32_t nB = sc.substeps - 1;
  R* bridge = reinterpret_cast<R*>(simRaw) + static_cast<size_t>(sc.nNormals) * kSimThreads;
  if (bridgeTable) {
    for (uint32_t jj = threadIdx.x + 1; jj < sc.nT; jj += blockDim.x) {
      const R dt = sc.steps[static_cast<size_t>(jj) * sc.stepStride + 6], h = dt / static_cast<R>(sc.substeps);
      R remT = dt;
      for (uint32_t q = 0; q < nB; ++q) {
        bridge[(static_cast<size_t>(jj) * nB + q) * 2] = h / remT;
        bridge[(static_cast<size_t>(jj) * nB + q) * 2 + 1] = rsqrt_(fmax(h * (remT - h) / remT, R(0)));
        remT -= h;
      }
    }
    __syncthreads();
  }
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= sc.nP) return;
  const uint32_t nP = sc.nP, nT = sc.nT;
  const uint32_t po = sc.pathMap ? sc.pathMap[p] : p;  // the plan's path this thread simulates
  R sign = R(1);
  uint32_t pathStream = po;
  if (sc.antithetic) {
    pathStream = po >> 1u;
    if (po & 1u) sign = R(-1);
  }
  const uint32_t injectedStream = sc.nStreams > 0 ? min(pathStream, sc.nStreams - 1) : 0u;
  const uint32_t stream = pcg(pcg(sc.seed) ^ pcg(pathStream + 0x9E3779B9u));
  auto normal = [&](uint32_t m) { return col[m * kSimThreads]; };
  // The deflator's exponent -sum of the integrated short rate accumulates in double precision in both modes (the
  // reference's kernel sums it in single precision, fused_kernels.cpp:250-253); D = exp(lnD) is then taken in R.
  R x = R(0), D = R(1);
  double lnD = 0.0;
  R S[4], lnS[4] = {R(0), R(0), R(0), R(0)}, y[2], Y[2] = {R(0), R(0)};
  R xf[2] = {R(0), R(0)};  // stochastic foreign short-rate states of assets 0 and 1
#pragma unroll
  for (int a = 0; a < 4; ++a) S[a] = sc.spots[a];
#pragma unroll
  for (int c = 0; c < 2; ++c) y[c] = sc.cir[4 * c + 3];
  auto put = [&](uint32_t field, uint32_t j, R v) { cb.data[(static_cast<size_t>(field) * nT + j) * nP + p] = v; };

  for (uint32_t j = 0; j < nT; ++j) {
    R Qc[2] = {R(1), R(1)};
    if (j > 0) {
      const R* step = sc.steps + static_cast<size_t>(j) * sc.stepStride;
      drawDate<R>(stream, j, sign, sc.normals, sc.nStreams, injectedStream, sc.nNormals, col);
      // Correlated drivers: each padded Cholesky row as two 4-term dot products (as the reference).
      R z[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) z[k] = static_cast<uint32_t>(k) < sc.nCorr ? normal(k) : R(0);
      R w[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const R* row = sc.chol + i * kChol;
        const R d0 = row[0] * z[0] + row[1] * z[1] + row[2] * z[2] + row[3] * z[3];
        const R d1 = row[4] * z[4] + row[5] * z[5] + row[6] * z[6] + row[7] * z[7];
        w[i] = d0 + d1;
      }
      const R zI = normal(sc.nCorr);
      const R integratedRate = x * step[5] + step[2] * w[0] + step[3] * zI + step[4];
      x = x * step[0] + step[1] * w[0];
      lnD -= static_cast<double>(integratedRate);
      D = rexp(static_cast<R>(lnD));
      // Stochastic foreign rates: the exact Hull-White step of x_f (with its quanto drift) and of its integral, on
      // driver 1 + nA + nC + f and the independent normal nCorr + 1 + f; the asset's carry is then the simulated
      // integral of r_f instead of the deterministic one.
      R carry[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) carry[a] = step[8 + a];
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        if (static_cast<uint32_t>(f) < sc.nF) {
          const R* fs = step + kStepStride + 8 * f;
          const uint32_t wi = 1 + sc.nA + sc.nC + f;
          R wf = w[7];
#pragma unroll
          for (int i = 6; i >= 0; --i)
            if (wi == static_cast<uint32_t>(i)) wf = w[i];
          const R zf = normal(sc.nCorr + 1 + f);
          carry[f] = xf[f] * fs[5] + fs[2] * wf + fs[3] * zf + fs[4] + fs[7];
          xf[f] = xf[f] * fs[0] + fs[1] * wf + fs[6];
        }
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        if (static_cast<uint32_t>(a) < sc.nA) {
          lnS[a] = lnS[a] + (integratedRate - carry[a] - step[16 + a] + step[12 + a] * w[1 + a]);
          S[a] = sc.spots[a] * rexp(lnS[a]);
        }
      }
      const R dt = step[6];
      uint32_t off = sc.nCorr + 1 + sc.nF;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        if (static_cast<uint32_t>(c) < sc.nC) {
          const R kappa = sc.cir[4 * c], theta = sc.cir[4 * c + 1], xi = sc.cir[4 * c + 2];
          const R h = dt / static_cast<R>(sc.substeps);
          const uint32_t wi = 1 + sc.nA + c;
          R wc = w[7];
#pragma unroll
          for (int i = 6; i >= 0; --i)
            if (wi == static_cast<uint32_t>(i)) wc = w[i];
          R rem = rsqrt_(dt) * wc, remT = dt, yy = y[c], YY = Y[c];
          const R* bj = bridge + static_cast<size_t>(j) * nB * 2;
          for (uint32_t s = 0; s < sc.substeps; ++s) {
            R dW = rem;
            if (s + 1 < sc.substeps) {
              const R a = bridgeTable ? bj[2 * s] : h / remT;
              const R b = bridgeTable ? bj[2 * s + 1] : rsqrt_(fmax(h * (remT - h) / remT, R(0)));
              dW = a * rem + b * normal(off + s);
            }
            rem -= dW;
            remT -= h;
            const R yp = fmax(yy, R(0));
            const R yn = yy + kappa * (theta - yp) * h + xi * rsqrt_(yp) * dW;
            YY += R(0.5) * (yp + fmax(yn, R(0))) * h;
            yy = yn;
          }
          y[c] = yy;
          Y[c] = YY;
          off += sc.substeps - 1;
          Qc[c] = rexp(-Y[c] - step[20 + c]);
        }
      }
    }
    put(0, j, x);
    put(1, j, D);
    for (uint32_t a = 0; a < sc.nA; ++a) put(cb.fS + a, j, sel4(S, a));
    for (uint32_t c = 0; c < sc.nC; ++c) put(cb.fQ + c, j, c == 0 ? Qc[0] : Qc[1]);
    for (uint32_t f = 0; f < sc.nF; ++f) put(cb.fXf + f, j, f == 0 ? xf[0] : xf[1]);
    if (cb.probes) {
      for (uint32_t a = 0; a < sc.nA; ++a) put(cb.fLnS + a, j, sel4(lnS, a));
      for (uint32_t c = 0; c < sc.nC; ++c) put(cb.fY + c, j, c == 0 ? y[0] : y[1]);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// The exponential of a lowered term: 2^(b x) with b = -B log2 e in single precision, e^(b x) with b = -B
// in double (lowerTerms, capi.cu).
__device__ __forceinline__ float termExp(float b, float x) { return ex2(b * x); }
__device__ __forceinline__ double termExp(double b, double x) { return exp(b * x); }

template <typename R> struct Vec4;
template <> struct Vec4<float> { using T = float4; };
template <> struct Vec4<double> { using T = double4; };
__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ double4 ld4(const double* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// Prefetches into L1 the 128-byte lines of one date's lowered terms, one line per thread of the CTA:
// the next date's block arrives while the current date computes.
__device__ __forceinline__ void prefetchL1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(__cvta_generic_to_global(p)));
}
template <typename R>
__device__ __forceinline__ void prefetchDate(uint32_t begin, uint32_t end, const R* table, uint32_t tid) {
  const size_t b = static_cast<size_t>(begin) * 4 * sizeof(R), e = static_cast<size_t>(end) * 4 * sizeof(R);
  const uint32_t lines = e > b ? static_cast<uint32_t>((e - 1) / 128 - b / 128 + 1) : 0u;
  if (tid < lines) prefetchL1(reinterpret_cast<const char*>(table) + (b / 128 + tid) * 128);
}

// A thread's PPT adjacent paths in one 8- or 16-byte access (p aligned to PPT values).
template <typename R, int PPT>
__device__ __forceinline__ void ldPaths(const R* p, R (&v)[PPT]) {
  if constexpr (PPT == 1) {
    v[0] = __ldg(p);
  } else if constexpr (sizeof(R) == 4 && PPT == 2) {
    const float2 t = __ldg(reinterpret_cast<const float2*>(p));
    v[0] = t.x, v[1] = t.y;
  } else if constexpr (sizeof(R) == 4 && PPT == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
  } else {
#pragma unroll
    for (int q = 0; q < PPT; q += 2) {
      const double2 t = __ldg(reinterpret_cast<const double2*>(p) + q / 2);
      v[q] = t.x, v[q + 1] = t.y;
    }
  }
}
template <typename R, int PPT>
__device__ __forceinline__ void stPaths(R* p, const R (&v)[PPT]) {
  if constexpr (PPT == 1) {
    p[0] = v[0];
  } else if constexpr (sizeof(R) == 4 && PPT == 2) {
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  } else if constexpr (sizeof(R) == 4 && PPT == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
#pragma unroll
    for (int q = 0; q < PPT; q += 2) reinterpret_cast<double2*>(p)[q / 2] = make_double2(v[q], v[q + 1]);
  }
}

template <typename R, int PPT>
__device__ __forceinline__ R pick4(const R (&a)[4][PPT], uint32_t k, int i) {
  return k == 0 ? a[0][i] : k == 1 ? a[1][i] : k == 2 ? a[2][i] : a[3][i];
}

// Resident CTAs per SM the lean variants are compiled for (register budget 65536 / (128 x blocks)).  The
// shared-memory state of a netting set with many swap slots allows 6 CTAs of 2-path threads; netting sets
// with little state (kSmallState: at most kSmallStateWords words per path) fit 8, and their variant is
// compiled for 8 (64 registers).
template <int PPT, bool kLean, bool kSmallState = false>
constexpr int revalueMinBlocks() {
  return !kLean ? 1 : PPT == 1 ? 8 : PPT == 2 ? (kSmallState ? 8 : 6) : (kSmallState ? 4 : 3);
}

// Each thread owns PPT paths (p, p + kTile, ...): every term record, kind decode, date descriptor and
// statistics reduction is shared by PPT paths, and their independent exponentials keep the SFU busy.
// kCash: every netting set of the launch has a cash CSA whose margin calls look back at most one date and writes
// none of the optional value, exposure, collateral or change rows, so the collateral code is that case alone (no
// securities price, no shared-memory ring) and the optional rows are compiled out.
template <typename R, int PPT, bool kPerTrade, bool kSink, bool kLean, bool kSmallState = false, bool kCash = false>
__global__ void __launch_bounds__(kTile, (revalueMinBlocks<PPT, kLean, kSmallState>())) revalueKernel(const CubeArgs<R> cb, const NsArgs<R>* __restrict__ nsArgs,
                                                        uint32_t numNs) {
  extern __shared__ __align__(16) unsigned char smemRaw[];
  __shared__ NsArgs<R> sA;
  R* vtBuf = reinterpret_cast<R*>(smemRaw);                        // [16][PPT][kTile] per-trade values
  R* state = vtBuf + (kPerTrade ? kMaxTradeGroups * PPT * kTile : 0);  // fixings [nSlots][PPT][kTile] | ring

  const uint32_t n = blockIdx.x % numNs, tile = blockIdx.x / numNs;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  if (tid == 0) sA = nsArgs[n];
  __syncthreads();
  const NsArgs<R>& A = sA;  // read from shared memory: no global reloads after the stores below
  const uint4* __restrict__ dates = reinterpret_cast<const uint4*>(A.dates);
  const R* __restrict__ table = A.table;
  R* __restrict__ expo = A.expo;
  const uint32_t nP = cb.nP, nT = cb.nT;
  // Lean launches hold only plans with the netting set's 8 statistics per date (no per-trade ones).
  const uint32_t nSlots = A.nSlots, ringLen = kCash ? 2u : A.ring, nS = kLean ? static_cast<uint32_t>(kStatsPerDate) : A.nS;
  const uint32_t ctype = kCash ? 0u : A.ctype;
  const bool hasCsa = kCash || A.hasCsa != 0, usesAssets = A.usesAssets != 0;
  R* __restrict__ const rowEP = expo + static_cast<size_t>(A.rowEP) * nP;
  const bool moreRows = !kCash && (A.rowDV != kNoRow || A.rowE != kNoRow || A.rowV != kNoRow || A.rowC != kNoRow);
  uint32_t pth[PPT], pp[PPT];
  bool act[PPT];
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    pth[i] = tile * (kTile * PPT) + tid * PPT + i;  // a thread's paths are adjacent
    act[i] = pth[i] < nP;
    // Threads past the last path read valid paths and contribute nothing: the last PPT paths when nP is a
    // multiple of PPT (an aligned group, read as one vector), else the last path.
    pp[i] = act[i] ? pth[i] : nP % PPT == 0 ? nP - PPT + i : nP - 1;
  }
  auto fix = [&](uint32_t slot, int i) -> R& { return state[(slot * PPT + i) * kTile + tid]; };
  auto ring = [&](uint32_t r, int i) -> R& { return state[((nSlots + r) * PPT + i) * kTile + tid]; };
  // More than 4 Bermudans (non-lean launches only): each path's exercise index of Bermudan b is a byte of shared
  // memory after the fixings and the margin ring, [b][PPT][kTile], -1 while not exercised.
  const bool manyBerm = !kLean && A.manyBerm != 0;
  signed char* exS = reinterpret_cast<signed char*>(
      state + static_cast<size_t>(nSlots + (hasCsa ? ringLen * (ctype != 0 ? 2u : 1u) : 0u)) * PPT * kTile);
  if (manyBerm)
    for (uint32_t b = 0; b < A.nBerm; ++b)
#pragma unroll
      for (int i = 0; i < PPT; ++i) exS[(b * PPT + i) * kTile + tid] = -1;
  auto vt = [&](uint32_t g, int i) -> R& { return vtBuf[(g * PPT + i) * kTile + tid]; };
  for (uint32_t s = 0; s < nSlots; ++s)
#pragma unroll
    for (int i = 0; i < PPT; ++i) fix(s, i) = R(0);
  const uint32_t nTr = kPerTrade ? min(A.nTr, static_cast<uint32_t>(kMaxTradeGroups)) : 0u;
  const uint32_t fQ = A.cpty < cb.nC ? cb.fQ + A.cpty : 0xFFFFFFFFu;
  // Factor loads: per path a base pointer, per date an offset j * nP, per field a stride nT * nP.
  const size_t fieldStride = static_cast<size_t>(nT) * nP;
  const R* cubeP[PPT];
#pragma unroll
  for (int i = 0; i < PPT; ++i) cubeP[i] = cb.data + pp[i];
  auto cube = [&](uint32_t field, uint32_t j, int i) { return cubeP[i][field * fieldStride + static_cast<size_t>(j) * nP]; };

  R held[PPT], prevDE[PPT], prevQ[PPT], prevRV[PPT], ex[4][PPT];
  // The exercise index (-1: not exercised) of Bermudan b on the thread's path i.
  auto exOf = [&](uint32_t b, int i) -> R {
    return manyBerm ? static_cast<R>(exS[(b * PPT + i) * kTile + tid]) : pick4<R, PPT>(ex, b, i);
  };
  // Look-back of at most one date (the margin-call dates t - MPR sit on the grid): the previous date's value
  // and collateral price in registers instead of the shared-memory ring.
  const bool shortLook = kCash || ringLen <= 2;
  R vPrev[PPT], pPrev[PPT];
#pragma unroll
  for (int i = 0; i < PPT; ++i) vPrev[i] = R(0), pPrev[i] = R(1);
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    held[i] = R(0), prevDE[i] = R(0), prevQ[i] = R(1), prevRV[i] = R(0);
#pragma unroll
    for (int b = 0; b < 4; ++b) ex[b][i] = R(-1);  // exercise index of each Bermudan, -1 if not exercised
  }
  uint32_t ringPos = 0;

  // Software pipeline: the factors and the date descriptor of date j + 1 load while date j computes.
  R nx[PPT], nD[PPT], nQ[PPT], nS4[4][PPT];
  const size_t qOff = fQ != 0xFFFFFFFFu ? fQ * fieldStride : 0, sOff = static_cast<size_t>(cb.fS) * fieldStride;
  // With nP a multiple of PPT a thread's paths are all live or all past the end, and their factors are one
  // vector access per field (past the end: the last PPT paths).
  const bool vecPaths = PPT > 1 && nP % PPT == 0;
  auto loadFactors = [&](uint32_t j) {
    const size_t off = static_cast<size_t>(j) * nP;
    if (vecPaths) {
      const R* c = cubeP[0] + off;
      ldPaths<R, PPT>(c, nx);
      ldPaths<R, PPT>(c + fieldStride, nD);
      if (fQ != 0xFFFFFFFFu) {
        ldPaths<R, PPT>(c + qOff, nQ);
      } else {
#pragma unroll
        for (int i = 0; i < PPT; ++i) nQ[i] = R(1);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        if (usesAssets && static_cast<uint32_t>(a) < cb.nA) {
          ldPaths<R, PPT>(c + sOff + a * fieldStride, nS4[a]);
        } else {
#pragma unroll
          for (int i = 0; i < PPT; ++i) nS4[a][i] = R(0);
        }
      }
      return;
    }
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      const R* c = cubeP[i] + off;
      nx[i] = __ldg(c), nD[i] = __ldg(c + fieldStride), nQ[i] = fQ != 0xFFFFFFFFu ? __ldg(c + qOff) : R(1);
#pragma unroll
      for (int a = 0; a < 4; ++a)
        nS4[a][i] = usesAssets && static_cast<uint32_t>(a) < cb.nA ? __ldg(c + sOff + a * fieldStride) : R(0);
    }
  };
  loadFactors(0);
  uint4 nd0 = __ldg(dates), nd1 = __ldg(dates + 1);
  // The block of the date after next is prefetched one date ahead of use.
  uint32_t fBeg = nT > 1 ? __ldg(A.dates + 8) : 0u, fEnd = nT > 1 ? __ldg(A.dates + 13) : 0u;
  prefetchDate<R>(nd0.x, nd1.y, table, tid);

  for (uint32_t j = 0; j < nT; ++j) {
    R x[PPT], D[PPT], Q[PPT], S[4][PPT];
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      x[i] = nx[i], D[i] = nD[i], Q[i] = nQ[i];
#pragma unroll
      for (int a = 0; a < 4; ++a) S[a][i] = nS4[a][i];
    }
    const uint4 d0 = nd0, d1 = nd1;
    const R guardJ = A.flags ? A.guard[j] : R(-1);  // < 0: no check
    if (j + 1 < nT) {
      loadFactors(j + 1);
      nd0 = __ldg(dates + 2 * (j + 1)), nd1 = __ldg(dates + 2 * (j + 1) + 1);
      prefetchDate<R>(fBeg, fEnd, table, tid);
      if (j + 2 < nT) {
        fBeg = __ldg(A.dates + 8 * (j + 2)), fEnd = __ldg(A.dates + 8 * (j + 2) + 5);
      }
    }
    if (kSink && n == 0)
#pragma unroll
      for (int i = 0; i < PPT; ++i)
        if (act[i]) {
          A.sinkX[static_cast<size_t>(j) * nP + pth[i]] = x[i];
          A.sinkD[static_cast<size_t>(j) * nP + pth[i]] = D[i];
        }

    R value[PPT], ev[4][PPT];
    R annS[PPT], fltS[PPT];  // the co-terminal swap of the next two-regressor record: annuity, float leg
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      value[i] = R(0), annS[i] = R(0), fltS[i] = R(0);
#pragma unroll
      for (int b = 0; b < 4; ++b) ev[b][i] = R(0);
    }
    using R4 = typename Vec4<R>::T;
    for (uint32_t u = d0.x; u < d0.y; ++u) {  // running floating coupons
      const R4 r = ld4(table + 4 * u);
      const uint32_t slot = static_cast<uint32_t>(r.w);
#pragma unroll
      for (int i = 0; i < PPT; ++i) value[i] += (r.x * fix(slot, i) + r.y) * termExp(r.z, x[i]);
    }
#pragma unroll 2
    for (uint32_t u = d0.y; u < d0.z; ++u) {  // bonds, two per record
      const R4 r = ld4(table + 4 * u);
#pragma unroll
      for (int i = 0; i < PPT; ++i) value[i] += r.x * termExp(r.y, x[i]) + r.z * termExp(r.w, x[i]);
    }
    for (uint32_t u = d0.z; u < d0.w; ++u) {  // asset forwards: (c, A, asset)
      const R4 r = ld4(table + 4 * u);
      const uint32_t a = static_cast<uint32_t>(r.z) & 3u;
#pragma unroll
      for (int i = 0; i < PPT; ++i) value[i] += r.x * pick4<R, PPT>(S, a, i) * r.y;
    }
    if (kPerTrade && A.nTr > 0)
      for (uint32_t g = 0; g < kMaxTradeGroups; ++g)
#pragma unroll
        for (int i = 0; i < PPT; ++i) vt(g, i) = R(0);
    for (uint32_t u = d0.w; u < d1.x; u += 2) {  // generic terms: the reference's records
      R rec[8];
      loadTerm(table + 4 * u, rec);
      const uint32_t code = static_cast<uint32_t>(rec[0]);
      const uint32_t kind = code & 15u, bm = bermudanOf(code, manyBerm), extra = code >> 12u;
      const uint32_t grp = min((code >> 4u) & 15u, 15u);
      if (!kLean && kind == kBermBond && rec[1] < R(0)) {
        // A block of nb bonds of Bermudan bm (the lowering's run of its kBermBond records): each counts on a path
        // that exercised at or before the bond's exercise index; a warp with no such path skips the block.
        const uint32_t nb = static_cast<uint32_t>(-rec[1]);
        R exi[PPT];
        bool live = false;
#pragma unroll
        for (int i = 0; i < PPT; ++i) exi[i] = exOf(bm, i), live = live || (exi[i] >= R(0) && exi[i] <= rec[2]);
        if (__any_sync(0xFFFFFFFFu, live))
          for (uint32_t q = 0; q < nb; ++q) {
            const R4 b = ld4(table + 4 * (u + 2 + q));
            const R nBq = -b.z;
#pragma unroll
            for (int i = 0; i < PPT; ++i) {
              R term = R(0);
              if (exi[i] >= R(0) && exi[i] <= b.w) term = b.x * (b.y * fastExp(nBq * x[i]));
              if (kPerTrade && A.nTr > 0) vt(grp, i) += term;
              else value[i] += term;
            }
          }
        u += 2 * ((nb + 1) / 2);
        continue;
      }
      const uint32_t slot = static_cast<uint32_t>(rec[1]);
      const R c = rec[2], nB = -rec[4];
      R term[PPT];
#pragma unroll
      for (int i = 0; i < PPT; ++i) term[i] = R(0);
      switch (kind) {
        case kBond:
#pragma unroll
          for (int i = 0; i < PPT; ++i) term[i] = c * (rec[3] * fastExp(nB * x[i]));
          break;
        case kFixedFloat:
#pragma unroll
          for (int i = 0; i < PPT; ++i) term[i] = (c * fix(slot, i) + rec[5]) * (rec[3] * fastExp(nB * x[i]));
          break;
        case kAsset:
#pragma unroll
          for (int i = 0; i < PPT; ++i) term[i] = c * pick4<R, PPT>(S, slot & 3u, i) * rec[3];
          break;
        case kSetFixing:
#pragma unroll
          for (int i = 0; i < PPT; ++i) fix(slot, i) = (rec[3] * fastExp(nB * x[i]) - R(1)) / c;
          break;
        case kOption: {
          const R p3 = rec[7];
#pragma unroll
          for (int i = 0; i < PPT; ++i) {
            const R b0 = rec[3] * fastExp(nB * x[i]);
            term[i] = c * black(pick4<R, PPT>(S, slot & 3u, i) * rec[5] / b0, rec[6], fabs(p3), b0, p3 > R(0));
          }
          break;
        }
        case kForeignForward: {  // c S P_f(t, T | x_f), P_f = A_f e^{-B_f x_f}: the foreign bond of the asset's currency
          const uint32_t a = min(extra, 1u);
#pragma unroll
          for (int i = 0; i < PPT; ++i) term[i] = c * pick4<R, PPT>(S, a, i) * (rec[3] * fastExp(-rec[1] * cube(cb.fXf + a, j, i)));
          break;
        }
        case kForeignOption: {  // Black on S P_f(t, T | x_f) / P(t, T | x)
          const uint32_t a = min(extra, 1u);
          const R p3 = rec[7];
#pragma unroll
          for (int i = 0; i < PPT; ++i) {
            const R b0 = rec[3] * fastExp(nB * x[i]);
            const R q = rec[5] * fastExp(-rec[1] * cube(cb.fXf + a, j, i));
            term[i] = c * black(pick4<R, PPT>(S, a, i) * q / b0, rec[6], fabs(p3), b0, p3 > R(0));
          }
          break;
        }
        default:
          if constexpr (!kLean) switch (kind) {  // the AMC and probe terms (absent from lean launches)
          case kBermExercise:
  #pragma unroll
            for (int i = 0; i < PPT; ++i) {
              const R v = c * (rec[3] * fastExp(nB * x[i]));
              if (manyBerm || bm == 0) ev[0][i] += v;  // with many Bermudans, one running value: its policy follows
              else if (bm == 1) ev[1][i] += v;
              else if (bm == 2) ev[2][i] += v;
              else ev[3][i] += v;
            }
            break;
          case kBermAnnuity:
  #pragma unroll
            for (int i = 0; i < PPT; ++i) annS[i] += c * (rec[3] * fastExp(nB * x[i]));
            break;
          case kBermCoterm:
  #pragma unroll
            for (int i = 0; i < PPT; ++i) fltS[i] += c * (rec[3] * fastExp(nB * x[i]));
            break;
          case kBermExt:
            break;  // read with its policy or continuation record
          case kBermDecide: {
            R e1[8], e2[8];
            const bool twoD = twoRegressors(table, u, d1.x, e1, e2);
  #pragma unroll
            for (int i = 0; i < PPT; ++i) {
              const R e = manyBerm ? ev[0][i] : pick4<R, PPT>(ev, bm, i);
              if (manyBerm) ev[0][i] = R(0);
              const R cont = twoD ? amcPoly2(rec, e1, e2, x[i], swapRate(fltS[i], annS[i])) : amcPoly(rec, x[i]);
              annS[i] = R(0), fltS[i] = R(0);
              if (kSink) {
                if (act[i]) A.sinkEx[static_cast<size_t>(A.sinkRowOfBermudan[bm] + extra) * nP + pth[i]] = e;
              } else if (exOf(bm, i) < R(0)) {
                // the exact-decision check: the rule's margins are e (against 0) and e - cont
                if (act[i] && (fabs(e) <= guardJ || fabs(e - cont) <= guardJ)) flagPath(A.flags, pth[i]);
                if (e > R(0) && e > cont) {
                  const R v = static_cast<R>(extra);
                  if (manyBerm) exS[(bm * PPT + i) * kTile + tid] = static_cast<signed char>(extra);
                  else if (bm == 0) ex[0][i] = v;
                  else if (bm == 1) ex[1][i] = v;
                  else if (bm == 2) ex[2][i] = v;
                  else ex[3][i] = v;
                }
              }
            }
            break;
          }
          case kBermContinue: {
            R e1[8], e2[8];
            const bool twoD = twoRegressors(table, u, d1.x, e1, e2);
  #pragma unroll
            for (int i = 0; i < PPT; ++i) {
              const R cont = twoD ? amcPoly2(rec, e1, e2, x[i], swapRate(fltS[i], annS[i])) : amcPoly(rec, x[i]);
              annS[i] = R(0), fltS[i] = R(0);
              if (exOf(bm, i) < R(0)) term[i] = rec[1] * fmax(cont, R(0));
            }
            break;
          }
          case kBermBond:
  #pragma unroll
            for (int i = 0; i < PPT; ++i) {
              const R e = exOf(bm, i);
              if (e >= R(0) && e <= static_cast<R>(extra)) term[i] = c * (rec[3] * fastExp(nB * x[i]));
            }
            break;
          case kProbe: {
            const uint32_t what = slot & 15u, ix = min(slot >> 4u, 3u), ic = min(ix, 1u);
  #pragma unroll
            for (int i = 0; i < PPT; ++i) {
              R q;
              switch (what) {
                case 0: q = x[i]; break;
                case 1: q = D[i]; break;
                case 2: q = pick4<R, PPT>(S, ix, i); break;
                case 3: q = ix < cb.nA ? cube(cb.fLnS + ix, j, i) : R(0); break;
                case 4: q = ic < cb.nC ? cube(cb.fY + ic, j, i) : R(0); break;
                case 5: q = ic < cb.nC ? cube(cb.fQ + ic, j, i) : R(1); break;
                case 6: q = D[i] * pick4<R, PPT>(S, ix, i); break;
                default: q = D[i] * (rec[3] * fastExp(nB * x[i]));
              }
              if (!kSink && act[i]) expo[static_cast<size_t>(static_cast<uint32_t>(rec[5])) * nP + pth[i]] = q + c;
            }
            break;
          }
          default:  // kBermFloat
  #pragma unroll
            for (int i = 0; i < PPT; ++i) {
              const R e = exOf(bm, i);
              if (e >= R(0) && e <= static_cast<R>(extra)) term[i] = (c * fix(slot, i) + rec[5]) * (rec[3] * fastExp(nB * x[i]));
            }
          }
      }
      if (kPerTrade && A.nTr > 0) {
#pragma unroll
        for (int i = 0; i < PPT; ++i) vt(grp, i) += term[i];
      } else {
#pragma unroll
        for (int i = 0; i < PPT; ++i) value[i] += term[i];
      }
    }
    for (uint32_t u = d1.x; u < d1.y; ++u) {  // fixings, after every use of the previous fixing
      const R4 r = ld4(table + 4 * u);
      const uint32_t slot = static_cast<uint32_t>(r.w);
#pragma unroll
      for (int i = 0; i < PPT; ++i) fix(slot, i) = (r.x * termExp(r.y, x[i]) - R(1)) * r.z;
    }
    for (uint32_t g = 0; g < nTr; ++g)
#pragma unroll
      for (int i = 0; i < PPT; ++i) value[i] += vt(g, i);
    if (kSink) continue;

    // ---- CSA: collateral called on the value at t - MPR (collateral.cpp:10-47) ----
    R e[PPT], ep[PPT], en[PPT];
    const uint32_t callJ = d1.z, rs = d1.w;
    // Ring slots without a modulo: ringPos = j mod ringLen, advanced by one per date; the margin-call date
    // lies j - callJ < ringLen dates back.
    const uint32_t lag = j - callJ, callPos = ringPos >= lag ? ringPos - lag : ringPos + ringLen - lag;
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      R collateral = R(0);
      if (hasCsa) {
        R price = R(1);
        if (ctype == 1) price = A.steps[static_cast<size_t>(j) * A.stepStride + 22] * rexp(-A.steps[static_cast<size_t>(j) * A.stepStride + 23] * x[i]);
        else if (ctype == 2) price = pick4<R, PPT>(S, min(A.casset, 3u), i);
        R vc, pc = price;
        if (shortLook) {
          vc = callJ != j ? vPrev[i] : value[i];
          if (callJ != j) pc = pPrev[i];
          vPrev[i] = value[i], pPrev[i] = price;
        } else {
          ring(ringPos, i) = value[i];
          if (ctype != 0) ring(ringLen + ringPos, i) = price;
          vc = callJ != j ? ring(callPos, i) : value[i];
          if (ctype != 0 && callJ != j) pc = ring(ringLen + callPos, i);
        }
        R required = R(0);
        if (vc > A.hc) required += vc - A.hc;
        if (A.hb >= R(0) && -vc > A.hb) required -= -vc - A.hb;
        // The call rule |required - held| >= MTA; the exact-decision check flags the path when its margin
        // | |required - held| - MTA | is within the date's guard.
        if (ctype == 0) {  // cash: one unit is worth one, no division
          const R gap = fabs(required - held[i]);
          if (j > 0 && act[i] && fabs(gap - A.mta) <= guardJ) flagPath(A.flags, pth[i]);
          if (j == 0 || gap >= A.mta) held[i] = required;
          collateral = held[i] + A.ia;
        } else {
          const R keep = A.keepHaircut;
          const R gap = fabs(required - held[i] * keep * pc);
          if (j > 0 && act[i] && fabs(gap - A.mta) <= guardJ) flagPath(A.flags, pth[i]);
          if (j == 0 || gap >= A.mta) held[i] = required / (keep * pc);
          collateral = held[i] * price + A.ia;
        }
      }
      e[i] = value[i] - collateral, ep[i] = fmax(e[i], R(0)), en[i] = fmin(e[i], R(0));
      if (act[i] && rs > 0) {
        const size_t k = rs - 1, pi = pth[i], at = k * nP + pi;
        if (!vecPaths) rowEP[at] = ep[i];
        if (moreRows) {
          if (A.rowDV != kNoRow) expo[(A.rowDV + k) * nP + pi] = rs == 1 ? R(0) : fabs(value[i] - prevRV[i]);
          if (A.rowE != kNoRow) expo[(A.rowE + k) * nP + pi] = e[i];
          if (A.rowV != kNoRow) expo[(A.rowV + k) * nP + pi] = value[i];
          if (A.rowC != kNoRow) expo[(A.rowC + k) * nP + pi] = collateral;
        }
        if (!kLean && A.rowGross != kNoRow) {
          R gross = R(0);
          for (uint32_t g = 0; g < nTr; ++g) gross += fmax(vt(g, i), R(0));
          expo[(A.rowGross + k) * nP + pi] = gross;
        }
        if (!kLean && A.rowTrades != kNoRow)
          for (uint32_t g = 0; g < nTr; ++g) expo[(A.rowTrades + g * A.nR + k) * nP + pi] = vt(g, i);
      }
      if (!kLean && !kSink && rs > 0 && A.imState && act[i]) {  // the start of this path's inner paths
        R* st = A.imState + static_cast<size_t>(rs - 1) * A.imWords * nP + pth[i];
        st[0] = value[i];
#pragma unroll
        for (int b = 0; b < 4; ++b) st[static_cast<size_t>(1 + b) * nP] = pick4<R, PPT>(ex, b, i);
        for (uint32_t q = 0; q < nSlots; ++q) st[static_cast<size_t>(5 + q) * nP] = fix(q, i);
      }
      if (!kLean && act[i] && A.rowEx != kNoRow)
        for (uint32_t b = 0; b < (manyBerm ? A.nBerm : min(A.nBerm, 4u)); ++b) {
          const R v = exOf(b, i);
          expo[(A.rowEx + b) * static_cast<size_t>(nP) + pth[i]] = v < R(0) ? R(-1) : v;
        }
    }
    if (vecPaths && act[0] && rs > 0) stPaths<R, PPT>(rowEP + static_cast<size_t>(rs - 1) * nP + pth[0], ep);
    R cvaInc[PPT];
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      cvaInc[i] = R(0);
      if (rs > 0) {
        prevRV[i] = value[i];
        const R de = D[i] * ep[i];
        if (j > 0) cvaInc[i] = R(0.5) * (prevDE[i] + de) * (prevQ[i] - Q[i]);
        prevDE[i] = de;
        prevQ[i] = Q[i];
      }
    }

    // ---- statistics of this date: the netting set's 8, then kTradeStats per trade, summed per warp over its
    // 32 PPT adjacent paths as a binary tree (a thread's adjacent paths first, then the lanes) into one partial
    // per warp: no block barrier.  The reduce kernel completes each 128-path group's tree from 4, 2 or 1 warp
    // partials, so the group sums and their bits do not depend on the tile shape ----
    const uint32_t unit = tile * kWarps + warp;
    const bool unitLive = unit * (32u * PPT) < nP;
    for (uint32_t q = 0; q < nS; q += 8) {
      R w8[PPT][8];
#pragma unroll
      for (int i = 0; i < PPT; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) w8[i][c] = R(0);
        if (act[i]) {
          if (q == 0) {
            w8[i][0] = e[i], w8[i][1] = ep[i], w8[i][2] = en[i], w8[i][3] = D[i] * ep[i], w8[i][4] = D[i] * en[i];
            w8[i][5] = cvaInc[i], w8[i][6] = Q[i], w8[i][7] = D[i];
          } else {
#pragma unroll
            for (int c = 0; c < 8; ++c) {
              const uint32_t k = q + c - kStatsPerDate, g = k / kTradeStats;
              if (q + c < nS && g < nTr) w8[i][c] = tradeStat<R>(k % kTradeStats, vt(g, i), value[i], D[i]);
            }
          }
        }
      }
      R v8[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if constexpr (PPT == 1) v8[c] = w8[0][c];
        else if constexpr (PPT == 2) v8[c] = w8[0][c] + w8[1][c];
        else v8[c] = (w8[0][c] + w8[1][c]) + (w8[2][c] + w8[3][c]);
      }
      const R s = warpReduceScatter8(v8, lane);
      const uint32_t c = statSlotOfLane(lane);
      if (lane < 8u && unitLive && q + c < nS) A.partials[(static_cast<size_t>(unit) * nT + j) * nS + q + c] = s;
    }
    ringPos = ringPos + 1 == ringLen ? 0u : ringPos + 1;
  }
}

// ---------------------------------------------------------------------------------------------
// Nested Monte Carlo for the conditional initial margin (the reference's innerStep / innerValue and the
// inner loop of simulatePath: fused_reference.cpp:108-196, 356-393).  The reference runs the nInner inner
// paths of an outer path one after the other inside the path's thread; here one warp takes one
// (reporting slot, outer path) and its lanes run inner paths lane, lane + 32, ... side by side: every lane of
// the warp steps the same dates, so the date's records are warp-uniform broadcasts, and the grid holds
// nR x nP warps instead of nP threads.

// One inner path's exact step to date jj on its own stream: the outer step's short rate and asset levels
// with the inner normals (the intensity enters no value and is not stepped).  Pairs past the normals the
// Cholesky rows and the integrated rate read stay zero; the Cholesky factor is zero there.
template <typename R>
__device__ __forceinline__ void innerStep(const ImArgs<R>& M, uint32_t jj, uint32_t stream, R sign, R& x, R (&lnS)[4],
                                          R (&S)[4]) {
  R z[8];
  const uint32_t pairs = M.nCorr / 2 + 1;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    z[2 * k] = z[2 * k + 1] = R(0);
    if (static_cast<uint32_t>(k) < pairs) {
      gauss2(stream, jj, static_cast<uint32_t>(k), z[2 * k], z[2 * k + 1]);
      z[2 * k] *= sign, z[2 * k + 1] *= sign;
    }
  }
  R w[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const R* row = M.model + 4 + i * kChol;
    const R d0 = __ldg(row) * z[0] + __ldg(row + 1) * z[1] + __ldg(row + 2) * z[2] + __ldg(row + 3) * z[3];
    const R d1 = __ldg(row + 4) * z[4] + __ldg(row + 5) * z[5] + __ldg(row + 6) * z[6] + __ldg(row + 7) * z[7];
    w[i] = d0 + d1;
  }
  R zc = R(0);  // the independent normal of the integrated rate, z[nCorr]
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (static_cast<uint32_t>(k) == M.nCorr) zc = z[k];
  const R* st = M.steps + static_cast<size_t>(jj) * kStepStride;
  const R integrated = x * __ldg(st + 5) + __ldg(st + 2) * w[0] + __ldg(st + 3) * zc + __ldg(st + 4);
  x = x * __ldg(st) + __ldg(st + 1) * w[0];
#pragma unroll
  for (int a = 0; a < 4; ++a)
    if (static_cast<uint32_t>(a) < M.nA) {
      lnS[a] = lnS[a] + (integrated - __ldg(st + 8 + a) - __ldg(st + 16 + a) + __ldg(st + 12 + a) * w[1 + a]);
      S[a] = __ldg(M.model + a) * rexp(lnS[a]);
    }
}

// The netting set's value on date jj of one inner path, from the date's lowered runs (the outer kernel's
// order: floating coupons, bonds, asset forwards, generic records, fixings); no trade groups, no probes.
// fix points at the lane's fixings, fixing s at fix[s * 32].
template <typename R>
__device__ R innerDateValue(const ImArgs<R>& M, uint32_t jj, R x, const R (&S)[4], R* fix, R (&ex)[4]) {
  using R4 = typename Vec4<R>::T;
  const uint4* dates = reinterpret_cast<const uint4*>(M.dates);
  const uint4 d0 = __ldg(dates + 2 * jj), d1 = __ldg(dates + 2 * jj + 1);
  const R* table = M.table;
  R value = R(0), ev[4] = {R(0), R(0), R(0), R(0)};
  for (uint32_t u = d0.x; u < d0.y; ++u) {
    const R4 r = ld4(table + 4 * u);
    value += (r.x * fix[static_cast<uint32_t>(r.w) * 32u] + r.y) * termExp(r.z, x);
  }
  for (uint32_t u = d0.y; u < d0.z; ++u) {
    const R4 r = ld4(table + 4 * u);
    value += r.x * termExp(r.y, x) + r.z * termExp(r.w, x);
  }
  for (uint32_t u = d0.z; u < d0.w; ++u) {
    const R4 r = ld4(table + 4 * u);
    value += r.x * sel4(S, static_cast<uint32_t>(r.z) & 3u) * r.y;
  }
  for (uint32_t u = d0.w; u < d1.x; u += 2) {
    R rec[8];
    loadTerm(table + 4 * u, rec);
    const uint32_t code = static_cast<uint32_t>(rec[0]);
    const uint32_t kind = code & 15u, bm = min((code >> 8u) & 15u, 3u), extra = code >> 12u;
    if (kind == kBermBond && rec[1] < R(0)) {  // a block of the Bermudan's bonds (see the outer kernel)
      const uint32_t nb = static_cast<uint32_t>(-rec[1]);
      const R e = sel4(ex, bm);
      if (e >= R(0) && e <= rec[2])
        for (uint32_t q = 0; q < nb; ++q) {
          const R4 b = ld4(table + 4 * (u + 2 + q));
          if (e <= b.w) value += b.x * (b.y * fastExp(-b.z * x));
        }
      u += 2 * ((nb + 1) / 2);
      continue;
    }
    const uint32_t slot = static_cast<uint32_t>(rec[1]);
    const R c = rec[2];
    switch (kind) {
      case kBond: value += c * (rec[3] * fastExp(-rec[4] * x)); break;
      case kFixedFloat: value += (c * fix[slot * 32u] + rec[5]) * (rec[3] * fastExp(-rec[4] * x)); break;
      case kAsset: value += c * sel4(S, slot & 3u) * rec[3]; break;
      case kSetFixing: fix[slot * 32u] = (rec[3] * fastExp(-rec[4] * x) - R(1)) / c; break;
      case kOption: {
        const R b0 = rec[3] * fastExp(-rec[4] * x);
        value += c * black(sel4(S, slot & 3u) * rec[5] / b0, rec[6], fabs(rec[7]), b0, rec[7] > R(0));
        break;
      }
      case kBermExercise: add4(ev, bm, c * (rec[3] * fastExp(-rec[4] * x))); break;
      case kBermDecide:
        if (sel4(ex, bm) < R(0) && sel4(ev, bm) > R(0) && sel4(ev, bm) > amcPoly(rec, x)) set4(ex, bm, static_cast<R>(extra));
        break;
      case kBermContinue:
        if (sel4(ex, bm) < R(0)) value += rec[1] * fmax(amcPoly(rec, x), R(0));
        break;
      case kBermBond: {
        const R e = sel4(ex, bm);
        if (e >= R(0) && e <= static_cast<R>(extra)) value += c * (rec[3] * fastExp(-rec[4] * x));
        break;
      }
      case kBermFloat: {
        const R e = sel4(ex, bm);
        if (e >= R(0) && e <= static_cast<R>(extra)) value += (c * fix[slot * 32u] + rec[5]) * (rec[3] * fastExp(-rec[4] * x));
        break;
      }
      default: break;  // probes write rows of the outer path only
    }
  }
  for (uint32_t u = d1.x; u < d1.y; ++u) {
    const R4 r = ld4(table + 4 * u);
    fix[static_cast<uint32_t>(r.w) * 32u] = (r.x * termExp(r.y, x) - R(1)) * r.z;
  }
  return value;
}

constexpr int kImWarps = 4;

// One warp per (reporting slot r, outer path p), item r * nP + p.  Each lane keeps the 16 largest of its
// samples |V_inner(target) - V| in descending order (the reference's insertion, which never admits a NaN);
// 16 rounds of a warp maximum over the lanes' heads then give the 16 largest of all nInner samples, the
// same multiset as the reference's single list, and the quantile interpolates between two of them.
template <typename R>
__global__ void __launch_bounds__(kImWarps * 32) nestedImKernel(const ImArgs<R> M) {
  extern __shared__ __align__(16) unsigned char smemRaw[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  R* fixIn = reinterpret_cast<R*>(smemRaw) + static_cast<size_t>(warp) * M.nSlots * 33u;  // [nSlots][32] inner
  R* fixOut = fixIn + M.nSlots * 32u;                                                     // [nSlots] outer
  const uint64_t item = static_cast<uint64_t>(blockIdx.x) * kImWarps + warp;
  if (item >= static_cast<uint64_t>(M.nR) * M.nP) return;  // warp-uniform; no block barrier below
  const uint32_t r = static_cast<uint32_t>(item / M.nP), p = static_cast<uint32_t>(item % M.nP);
  const uint32_t j = __ldg(M.slots + 2 * r), target = __ldg(M.slots + 2 * r + 1);
  if (j == kNoRow) return;  // a reporting slot on no date: the outer kernel writes no row for it either
  R* out = M.expo + static_cast<size_t>(M.rowIm + r) * M.nP + p;
  if (target == kNoRow) {
    if (lane == 0) *out = R(0);
    return;
  }
  const size_t nP = M.nP, fs = static_cast<size_t>(M.nT) * nP;
  const R* os = M.state + static_cast<size_t>(r) * (5 + M.nSlots) * nP + p;
  const R value = os[0];
  R ex0[4];
#pragma unroll
  for (int b = 0; b < 4; ++b) ex0[b] = os[(1 + b) * nP];
  for (uint32_t q = lane; q < M.nSlots; q += 32) fixOut[q] = os[(5 + q) * nP];
  __syncwarp();
  const R x0 = M.cube[static_cast<size_t>(j) * nP + p];
  R lnS0[4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
    lnS0[a] = static_cast<uint32_t>(a) < M.nA ? M.cube[(M.fLnS + a) * fs + static_cast<size_t>(j) * nP + p] : R(0);
  const uint32_t pathStream = M.anti ? p >> 1u : p;
  const uint32_t stream = pcg(pcg(M.seed) ^ pcg(pathStream + 0x9E3779B9u));

  R top[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) top[k] = R(0);
  for (uint32_t i = lane; i < M.nInner; i += 32) {
    R x = x0, lnS[4], S[4], ex[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) lnS[a] = lnS0[a], S[a] = R(0), ex[a] = ex0[a];
    for (uint32_t q = 0; q < M.nSlots; ++q) fixIn[q * 32u + lane] = fixOut[q];
    const uint32_t istream = pcg(stream ^ pcg(0x85EBCA6Bu + (i >> 1u) * 0x9E3779B9u + j));
    const R isign = (i & 1u) ? R(-1) : R(1);
    R vi = value;
    for (uint32_t jj = j + 1; jj <= target; ++jj) {
      innerStep(M, jj, istream, isign, x, lnS, S);
      vi = innerDateValue(M, jj, x, S, fixIn + lane, ex);
    }
    R cur = fabs(vi - value);
#pragma unroll
    for (int k = 0; k < 16; ++k)
      if (cur > top[k]) {
        const R t = top[k];
        top[k] = cur, cur = t;
      }
  }
  const R rank = M.level * static_cast<R>(M.nInner - 1);
  const uint32_t k = static_cast<uint32_t>(floor(rank));
  const uint32_t hi = min(M.nInner - 1 - k, 15u);
  R ok = R(0), ok1 = R(0);
  for (uint32_t round = 0; round <= hi; ++round) {
    R m = top[0];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) m = fmax(m, __shfl_xor_sync(0xFFFFFFFFu, m, d));
    if (round + 1 == hi) ok1 = m;
    if (round == hi) ok = m;
    const uint32_t owner = __ffs(__ballot_sync(0xFFFFFFFFu, top[0] == m)) - 1;
    if (lane == owner) {
#pragma unroll
      for (int q = 0; q < 15; ++q) top[q] = top[q + 1];
      top[15] = R(0);
    }
  }
  if (hi == 0) ok1 = ok;
  if (lane == 0) *out = ok + (rank - static_cast<R>(k)) * (ok1 - ok);
}

template <typename R>
cudaError_t launchNestedIm(const ImArgs<R>& M, cudaStream_t stream) {
  const uint64_t items = static_cast<uint64_t>(M.nR) * M.nP;
  if (items == 0 || M.nInner == 0) return cudaSuccess;
  const uint64_t blocks = (items + kImWarps - 1) / kImWarps;
  if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
  const size_t smem = static_cast<size_t>(kImWarps) * M.nSlots * 33u * sizeof(R);
  nestedImKernel<R><<<static_cast<uint32_t>(blocks), kImWarps * 32, smem, stream>>>(M);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
template <typename R>
cudaError_t launchSimulate(const ScenarioArgs<R>& sc, const CubeArgs<R>& cb, cudaStream_t stream) {
  const uint32_t blocks = (sc.nP + kSimThreads - 1) / kSimThreads;
  const size_t normals = static_cast<size_t>(sc.nNormals) * kSimThreads * sizeof(R);
  const size_t table = static_cast<size_t>(sc.nT) * (sc.substeps - 1) * 2 * sizeof(R);
  const bool bridgeTable = sc.nC > 0 && sc.substeps > 1 && normals + table <= 64 * 1024;
  const size_t smem = normals + (bridgeTable ? table : 0);
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(simulateKernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
  }
  simulateKernel<R><<<blocks, kSimThreads, smem, stream>>>(sc, cb, bridgeTable);
  return cudaGetLastError();
}

size_t revalueSmemBytes(size_t stateWordsMax, bool perTrade, bool f64, int ppt) {
  const size_t r = f64 ? 8 : 4;
  return ((perTrade ? kMaxTradeGroups * ppt * kTile : 0) + stateWordsMax * ppt * kTile) * r;
}

namespace {
template <typename R, int PPT>
cudaError_t launchRevaluePPT(const CubeArgs<R>& cb, const NsArgs<R>* nsArgs, uint32_t numNs, uint32_t numTiles, size_t stateWordsMax,
                             bool perTrade, bool sink, bool lean, bool smallState, bool cash, cudaStream_t stream) {
  const size_t smem = revalueSmemBytes(stateWordsMax, perTrade, sizeof(R) == 8, PPT);
  const uint64_t blocks = static_cast<uint64_t>(numTiles) * numNs;
  if (blocks == 0) return cudaSuccess;
  if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
  auto go = [&](auto kernel) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    kernel<<<static_cast<uint32_t>(blocks), kTile, smem, stream>>>(cb, nsArgs, numNs);
    return cudaGetLastError();
  };
  if (sink) return go(revalueKernel<R, PPT, false, true, false>);
  if (perTrade) return go(revalueKernel<R, PPT, true, false, false>);
  if (lean && smallState && stateWordsMax <= static_cast<size_t>(kSmallStateWords) && sizeof(R) == 4 && PPT > 1)
    return cash ? go(revalueKernel<R, PPT, false, false, true, true, true>) : go(revalueKernel<R, PPT, false, false, true, true>);
  if (lean) return cash ? go(revalueKernel<R, PPT, false, false, true, false, true>) : go(revalueKernel<R, PPT, false, false, true>);
  return go(revalueKernel<R, PPT, false, false, false>);
}
}  // namespace

template <typename R>
cudaError_t launchRevalue(const CubeArgs<R>& cb, const NsArgs<R>* nsArgs, uint32_t numNs, uint32_t numTiles, size_t stateWordsMax,
                          bool perTrade, bool sink, bool lean, int ppt, cudaStream_t stream, bool smallState, bool cash) {
  switch (ppt) {
    case 1: return launchRevaluePPT<R, 1>(cb, nsArgs, numNs, numTiles, stateWordsMax, perTrade, sink, lean, smallState, cash, stream);
    case 2: return launchRevaluePPT<R, 2>(cb, nsArgs, numNs, numTiles, stateWordsMax, perTrade, sink, lean, smallState, cash, stream);
    case 4:
      if (sizeof(R) == 4) return launchRevaluePPT<R, 4>(cb, nsArgs, numNs, numTiles, stateWordsMax, perTrade, sink, lean, smallState, cash, stream);
      return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}

template cudaError_t launchNestedIm<float>(const ImArgs<float>&, cudaStream_t);
template cudaError_t launchNestedIm<double>(const ImArgs<double>&, cudaStream_t);
template cudaError_t launchSimulate<float>(const ScenarioArgs<float>&, const CubeArgs<float>&, cudaStream_t);
template cudaError_t launchSimulate<double>(const ScenarioArgs<double>&, const CubeArgs<double>&, cudaStream_t);
template cudaError_t launchRevalue<float>(const CubeArgs<float>&, const NsArgs<float>*, uint32_t, uint32_t, size_t, bool, bool, bool,
                                          int, cudaStream_t, bool, bool);
template cudaError_t launchRevalue<double>(const CubeArgs<double>&, const NsArgs<double>*, uint32_t, uint32_t, size_t, bool, bool, bool,
                                           int, cudaStream_t, bool, bool);

}  // namespace zk
