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
//                    warp reduce-scatter (9 shuffles) and one cross-warp pass into per-tile partials,
//                    which the reduce kernel sums in a fixed order (deterministic results).
#include "zk_device.cuh"
#include "zk_kernels.h"

namespace zk {

namespace {

// lane l ends with the warp sum of statistic statSlotOfLane(l).
template <typename R>
__device__ __forceinline__ R warpReduceScatter8(const R (&v)[8], uint32_t lane) {
  const bool b4 = lane & 16u, b3 = lane & 8u, b2 = lane & 4u;
  R a[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const R send = b4 ? v[i] : v[i + 4];
    const R keep = b4 ? v[i + 4] : v[i];
    a[i] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, 16);
  }
  R b[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const R send = b3 ? a[i] : a[i + 2];
    const R keep = b3 ? a[i + 2] : a[i];
    b[i] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, 8);
  }
  R c = (b2 ? b[1] : b[0]) + __shfl_xor_sync(0xFFFFFFFFu, b2 ? b[0] : b[1], 4);
  c += __shfl_xor_sync(0xFFFFFFFFu, c, 2);
  c += __shfl_xor_sync(0xFFFFFFFFu, c, 1);
  return c;
}

__device__ __forceinline__ uint32_t statSlotOfLane(uint32_t lane) {
  return ((lane >> 4) & 1u) * 4u + ((lane >> 3) & 1u) * 2u + ((lane >> 2) & 1u);
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

// Normal m of the current date, drawn on demand from a one-pair cache (normals are consumed in
// increasing order, so every Box-Muller pair is drawn once).
template <typename R>
struct NormalStream {
  uint32_t stream, j, pair;
  R z0, z1, sign;
  const R* injected;
  uint32_t nStreams, injectedStream, nNormals;
  __device__ __forceinline__ R get(uint32_t m) {
    if (injected) return sign * injected[(static_cast<size_t>(j - 1) * nNormals + m) * nStreams + injectedStream];
    if (m / 2 != pair) {
      pair = m / 2;
      gauss2(stream, j, pair, z0, z1);
    }
    return sign * ((m & 1u) ? z1 : z0);
  }
};

}  // namespace

// ---------------------------------------------------------------------------------------------
// Risk factors of every path and date (the transitions of the reference's ScenarioGenerator:
// hull_white.cpp:40-68, lognormal_asset.cpp:17-22, cir_intensity.cpp:49-66, in the statement order
// of the reference kernel).
template <typename R>
__global__ void __launch_bounds__(256) simulateKernel(const ScenarioArgs<R> sc, CubeArgs<R> cb) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= sc.nP) return;
  const uint32_t nP = sc.nP, nT = sc.nT;
  R sign = R(1);
  uint32_t pathStream = p;
  if (sc.antithetic) {
    pathStream = p >> 1u;
    if (p & 1u) sign = R(-1);
  }
  const uint32_t injectedStream = sc.nStreams > 0 ? min(pathStream, sc.nStreams - 1) : 0u;
  NormalStream<R> ns{pcg(pcg(sc.seed) ^ pcg(pathStream + 0x9E3779B9u)), 0, 0xFFFFFFFFu, R(0), R(0), sign, sc.normals,
                     sc.nStreams, injectedStream, sc.nNormals};
  R x = R(0), lnD = R(0), D = R(1);
  R S[4], lnS[4] = {R(0), R(0), R(0), R(0)}, y[2], Y[2] = {R(0), R(0)};
#pragma unroll
  for (int a = 0; a < 4; ++a) S[a] = sc.spots[a];
#pragma unroll
  for (int c = 0; c < 2; ++c) y[c] = sc.cir[4 * c + 3];
  auto put = [&](uint32_t field, uint32_t j, R v) { cb.data[(static_cast<size_t>(field) * nT + j) * nP + p] = v; };

  for (uint32_t j = 0; j < nT; ++j) {
    R Qc[2] = {R(1), R(1)};
    if (j > 0) {
      const R* step = sc.steps + static_cast<size_t>(j) * kStepStride;
      ns.j = j;
      ns.pair = 0xFFFFFFFFu;
      // Correlated drivers: each padded Cholesky row as two 4-term dot products (as the reference).
      R z[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) z[k] = static_cast<uint32_t>(k) < sc.nCorr ? ns.get(k) : R(0);
      R w[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const R* row = sc.chol + i * kChol;
        const R d0 = row[0] * z[0] + row[1] * z[1] + row[2] * z[2] + row[3] * z[3];
        const R d1 = row[4] * z[4] + row[5] * z[5] + row[6] * z[6] + row[7] * z[7];
        w[i] = d0 + d1;
      }
      const R zI = ns.get(sc.nCorr);
      const R integratedRate = x * step[5] + step[2] * w[0] + step[3] * zI + step[4];
      x = x * step[0] + step[1] * w[0];
      lnD = lnD - integratedRate;
      D = rexp(lnD);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        if (static_cast<uint32_t>(a) < sc.nA) {
          lnS[a] = lnS[a] + (integratedRate - step[8 + a] - step[16 + a] + step[12 + a] * w[1 + a]);
          S[a] = sc.spots[a] * rexp(lnS[a]);
        }
      }
      const R dt = step[6];
      uint32_t off = sc.nCorr + 1;
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
          for (uint32_t s = 0; s < sc.substeps; ++s) {
            R dW = rem;
            if (s + 1 < sc.substeps) dW = h / remT * rem + rsqrt_(fmax(h * (remT - h) / remT, R(0))) * ns.get(off + s);
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
    if (cb.probes) {
      for (uint32_t a = 0; a < sc.nA; ++a) put(cb.fLnS + a, j, sel4(lnS, a));
      for (uint32_t c = 0; c < sc.nC; ++c) put(cb.fY + c, j, c == 0 ? y[0] : y[1]);
    }
  }
}

// ---------------------------------------------------------------------------------------------
template <typename R, bool kPerTrade, bool kSink>
__global__ void __launch_bounds__(kTile) revalueKernel(const CubeArgs<R> cb, const NsArgs<R>* __restrict__ nsArgs,
                                                        uint32_t numNs) {
  extern __shared__ __align__(16) unsigned char smemRaw[];
  R* red = reinterpret_cast<R*>(smemRaw);               // [2][kWarps][8]
  R* vtBuf = red + 2 * kWarps * 8;                      // [16][kTile] per-trade values (per-trade mode)
  R* state = vtBuf + (kPerTrade ? kMaxTradeGroups * kTile : 0);  // fixings [nSlots][kTile] | ring [ring (x2)][kTile]

  const uint32_t n = blockIdx.x % numNs, tile = blockIdx.x / numNs;
  const NsArgs<R>& A = nsArgs[n];
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t nP = cb.nP, nT = cb.nT;
  const uint32_t p = tile * kTile + tid;
  const bool active = p < nP;
  const uint32_t pp = active ? p : nP - 1;  // threads past the last path read a valid path and contribute nothing
  R* fix = state + tid;
  R* ring = state + A.nSlots * kTile + tid;
  for (uint32_t s = 0; s < A.nSlots; ++s) fix[s * kTile] = R(0);
  const uint32_t nTr = kPerTrade ? min(A.nTr, static_cast<uint32_t>(kMaxTradeGroups)) : 0u;
  const uint32_t fQ = A.cpty < cb.nC ? cb.fQ + A.cpty : 0xFFFFFFFFu;

  R held = R(0), prevDE = R(0), prevQ = R(1), prevRV = R(0);
  R ex[4] = {R(-1), R(-1), R(-1), R(-1)};  // exercise index of each Bermudan, -1 if not exercised
  uint32_t redBuf = 0;
  auto cube = [&](uint32_t field, uint32_t j) { return cb.data[(static_cast<size_t>(field) * nT + j) * nP + pp]; };

  for (uint32_t j = 0; j < nT; ++j) {
    const R x = cube(0, j), D = cube(1, j);
    R S[4] = {R(0), R(0), R(0), R(0)};
    if (A.usesAssets)
#pragma unroll
      for (int a = 0; a < 4; ++a)
        if (static_cast<uint32_t>(a) < cb.nA) S[a] = cube(cb.fS + a, j);
    const R Q = fQ != 0xFFFFFFFFu ? cube(fQ, j) : R(1);
    if (kSink && n == 0 && active) {
      A.sinkX[static_cast<size_t>(j) * nP + p] = static_cast<float>(x);
      A.sinkD[static_cast<size_t>(j) * nP + p] = static_cast<float>(D);
    }

    R value = R(0);
    R ev[4] = {R(0), R(0), R(0), R(0)};
    if (kPerTrade && A.nTr > 0)
      for (uint32_t i = 0; i < kMaxTradeGroups; ++i) vtBuf[i * kTile + tid] = R(0);
    const uint32_t tBegin = __ldg(A.idx + j), tEnd = __ldg(A.idx + j + 1);
    for (uint32_t t = tBegin; t < tEnd; ++t) {
      R rec[8];
      loadTerm(A.terms + static_cast<size_t>(t) * kTermStride, rec);
      const uint32_t code = static_cast<uint32_t>(rec[0]);
      const uint32_t kind = code & 15u, bm = min((code >> 8u) & 15u, 3u), extra = code >> 12u;
      const uint32_t slot = static_cast<uint32_t>(rec[1]);
      const R c = rec[2];
      R term = R(0);
      switch (kind) {
        case kBond: term = c * (rec[3] * fastExp(-rec[4] * x)); break;
        case kFixedFloat: term = (c * fix[slot * kTile] + rec[5]) * (rec[3] * fastExp(-rec[4] * x)); break;
        case kAsset: term = c * sel4(S, slot & 3u) * rec[3]; break;
        case kSetFixing: fix[slot * kTile] = (rec[3] * fastExp(-rec[4] * x) - R(1)) / c; break;
        case kOption: {
          const R b0 = rec[3] * fastExp(-rec[4] * x), p3 = rec[7];
          term = c * black(sel4(S, slot & 3u) * rec[5] / b0, rec[6], fabs(p3), b0, p3 > R(0));
          break;
        }
        case kBermExercise: add4(ev, bm, c * (rec[3] * fastExp(-rec[4] * x))); break;
        case kBermDecide: {
          const R e = sel4(ev, bm);
          if (kSink) {
            if (active) A.sinkEx[static_cast<size_t>(A.sinkRowOfBermudan[bm] + extra) * nP + p] = static_cast<float>(e);
          } else if (sel4(ex, bm) < R(0) && e > R(0) && e > amcPoly(rec, x)) {
            set4(ex, bm, static_cast<R>(extra));
          }
          break;
        }
        case kBermContinue:
          if (sel4(ex, bm) < R(0)) term = rec[1] * fmax(amcPoly(rec, x), R(0));
          break;
        case kBermBond: {
          const R e = sel4(ex, bm);
          if (e >= R(0) && e <= static_cast<R>(extra)) term = c * (rec[3] * fastExp(-rec[4] * x));
          break;
        }
        case kProbe: {
          const uint32_t what = slot & 15u, ix = min(slot >> 4u, 3u), ic = min(ix, 1u);
          R q;
          switch (what) {
            case 0: q = x; break;
            case 1: q = D; break;
            case 2: q = sel4(S, ix); break;
            case 3: q = ix < cb.nA ? cube(cb.fLnS + ix, j) : R(0); break;
            case 4: q = ic < cb.nC ? cube(cb.fY + ic, j) : R(0); break;
            case 5: q = ic < cb.nC ? cube(cb.fQ + ic, j) : R(1); break;
            case 6: q = D * sel4(S, ix); break;
            default: q = D * (rec[3] * fastExp(-rec[4] * x));
          }
          if (!kSink && active) A.expo[static_cast<size_t>(static_cast<uint32_t>(rec[5])) * nP + p] = q + c;
          break;
        }
        default: {  // kBermFloat
          const R e = sel4(ex, bm);
          if (e >= R(0) && e <= static_cast<R>(extra)) term = (c * fix[slot * kTile] + rec[5]) * (rec[3] * fastExp(-rec[4] * x));
        }
      }
      if (kPerTrade && A.nTr > 0) vtBuf[min((code >> 4u) & 15u, 15u) * kTile + tid] += term;
      else value += term;
    }
    for (uint32_t i = 0; i < nTr; ++i) value += vtBuf[i * kTile + tid];
    if (kSink) continue;

    // ---- CSA: collateral called on the value at t - MPR (collateral.cpp:10-47) ----
    R collateral = R(0);
    if (A.hasCsa) {
      R price = R(1);
      if (A.ctype == 1) price = A.steps[static_cast<size_t>(j) * kStepStride + 22] * rexp(-A.steps[static_cast<size_t>(j) * kStepStride + 23] * x);
      else if (A.ctype == 2) price = sel4(S, min(A.casset, 3u));
      ring[(j % A.ring) * kTile] = value;
      if (A.ctype != 0) ring[(A.ring + j % A.ring) * kTile] = price;
      const uint32_t callJ = __ldg(A.idx + A.offCall + j);
      const R vc = callJ != j ? ring[(callJ % A.ring) * kTile] : value;
      const R pc = callJ != j && A.ctype != 0 ? ring[(A.ring + callJ % A.ring) * kTile] : price;
      const R keep = A.ctype != 0 ? A.keepHaircut : R(1);
      R required = R(0);
      if (vc > A.hc) required += vc - A.hc;
      if (A.hb >= R(0) && -vc > A.hb) required -= -vc - A.hb;
      if (j == 0 || fabs(required - held * keep * pc) >= A.mta) held = required / (keep * pc);
      collateral = held * price + A.ia;
    }
    const R e = value - collateral, ep = fmax(e, R(0)), en = fmin(e, R(0));
    const uint32_t rs = __ldg(A.idx + A.offRep + j);
    if (active && rs > 0) {
      const size_t k = rs - 1;
      R* E = A.expo;
      E[(A.rowEP + k) * nP + p] = ep;
      if (A.rowDV != kNoRow) E[(A.rowDV + k) * nP + p] = rs == 1 ? R(0) : fabs(value - prevRV);
      if (A.rowE != kNoRow) E[(A.rowE + k) * nP + p] = e;
      if (A.rowV != kNoRow) E[(A.rowV + k) * nP + p] = value;
      if (A.rowC != kNoRow) E[(A.rowC + k) * nP + p] = collateral;
      if (A.rowGross != kNoRow) {
        R gross = R(0);
        for (uint32_t i = 0; i < nTr; ++i) gross += fmax(vtBuf[i * kTile + tid], R(0));
        E[(A.rowGross + k) * nP + p] = gross;
      }
      if (A.rowTrades != kNoRow)
        for (uint32_t i = 0; i < nTr; ++i) E[(A.rowTrades + i * A.nR + k) * nP + p] = vtBuf[i * kTile + tid];
    }
    if (active && A.rowEx != kNoRow)
      for (uint32_t i = 0; i < min(A.nBerm, 4u); ++i) A.expo[(A.rowEx + i) * static_cast<size_t>(nP) + p] = sel4(ex, i) < R(0) ? R(-1) : sel4(ex, i);
    R cvaInc = R(0);
    if (rs > 0) {
      prevRV = value;
      const R de = D * ep;
      if (j > 0) cvaInc = R(0.5) * (prevDE + de) * (prevQ - Q);
      prevDE = de;
      prevQ = Q;
    }

    // ---- statistics of this date: the netting set's 8, then kTradeStats per trade ----
    for (uint32_t q = 0; q < A.nS; q += 8) {
      R v8[8];
      if (q == 0) {
        v8[0] = e, v8[1] = ep, v8[2] = en, v8[3] = D * ep, v8[4] = D * en, v8[5] = cvaInc, v8[6] = Q, v8[7] = D;
      } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const uint32_t k = q + c - kStatsPerDate, i = k / kTradeStats;
          v8[c] = (q + c < A.nS && i < nTr) ? tradeStat<R>(k % kTradeStats, vtBuf[i * kTile + tid], value, D) : R(0);
        }
      }
      if (!active) {
#pragma unroll
        for (int c = 0; c < 8; ++c) v8[c] = R(0);
      }
      const R s = warpReduceScatter8(v8, lane);
      R* rb = red + redBuf * kWarps * 8;
      if ((lane & 3u) == 0) rb[warp * 8 + statSlotOfLane(lane)] = s;
      __syncthreads();
      if (tid < 8 && q + tid < A.nS) {
        R sum = R(0);
#pragma unroll
        for (int w = 0; w < kWarps; ++w) sum += rb[w * 8 + tid];
        A.partials[(static_cast<size_t>(tile) * nT + j) * A.nS + q + tid] = sum;
      }
      redBuf ^= 1u;  // the other buffer next time: one barrier per block of statistics
    }
  }
}

// ---------------------------------------------------------------------------------------------
template <typename R>
cudaError_t launchSimulate(const ScenarioArgs<R>& sc, const CubeArgs<R>& cb, cudaStream_t stream) {
  const uint32_t blocks = (sc.nP + 255) / 256;
  simulateKernel<R><<<blocks, 256, 0, stream>>>(sc, cb);
  return cudaGetLastError();
}

size_t revalueSmemBytes(size_t stateWordsMax, bool perTrade, bool f64) {
  const size_t r = f64 ? 8 : 4;
  return (2 * kWarps * 8 + (perTrade ? kMaxTradeGroups * kTile : 0) + stateWordsMax * kTile) * r;
}

template <typename R>
cudaError_t launchRevalue(const CubeArgs<R>& cb, const NsArgs<R>* nsArgs, uint32_t numNs, uint32_t numTiles, size_t stateWordsMax,
                          bool perTrade, bool sink, cudaStream_t stream) {
  const size_t smem = revalueSmemBytes(stateWordsMax, perTrade, sizeof(R) == 8);
  const uint64_t blocks = static_cast<uint64_t>(numTiles) * numNs;
  if (blocks == 0) return cudaSuccess;
  if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
  auto go = [&](auto kernel) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    kernel<<<static_cast<uint32_t>(blocks), kTile, smem, stream>>>(cb, nsArgs, numNs);
    return cudaGetLastError();
  };
  if (sink) return go(revalueKernel<R, false, true>);
  if (perTrade) return go(revalueKernel<R, true, false>);
  return go(revalueKernel<R, false, false>);
}

template cudaError_t launchSimulate<float>(const ScenarioArgs<float>&, const CubeArgs<float>&, cudaStream_t);
template cudaError_t launchSimulate<double>(const ScenarioArgs<double>&, const CubeArgs<double>&, cudaStream_t);
template cudaError_t launchRevalue<float>(const CubeArgs<float>&, const NsArgs<float>*, uint32_t, uint32_t, size_t, bool, bool,
                                          cudaStream_t);
template cudaError_t launchRevalue<double>(const CubeArgs<double>&, const NsArgs<double>*, uint32_t, uint32_t, size_t, bool, bool,
                                           cudaStream_t);

}  // namespace zk
