// reduce-partials and row statistics (the reference's second and third kernels,
// src/gpu/fused_kernels.cpp:538-563 and :565-771; CPU mirror finishFused,
// src/gpu/fused_reference.cpp:468-607).
//
// reduce: one thread per (date, statistic) sums the per-tile partials in tile order with a
// compensated double-precision sum, so the result does not depend on scheduling.
//
// row statistics: one CTA per request.  Quantiles are the *exact* empirical quantile interpolated
// between order statistics k = floor(p (n - 1)) and k + 1, as ccr::quantile does
// (include/ccr/core/math.hpp:39-47), found without sorting the row: a min/max pass (on rows of 64K values or
// more, over a 1/16 sample: it only sets the first histogram's range), a 4096-bin
// histogram pass that locates the bins of ranks k and k + 1, then either one pass that reads the
// maximum of k's bin and the minimum of k+1's bin (different bins) or a gather of k's bin into
// shared memory and a bitonic sort there (same bin; narrowed again if the bin holds more than
// kCap values).  The reference's histogram kernel interpolates inside the final bin instead and
// agrees with the exact quantile to about 5e-8 (README.md:182).
#include <cfloat>

#include "zk_device.cuh"
#include "zk_kernels.h"

namespace zk {

namespace {

constexpr int kRowThreads = 256;
constexpr int kRowWarps = kRowThreads / 32;
constexpr int kBins = 4096;
constexpr int kCap = 4096;
constexpr int kMaxRounds = 16;
constexpr int kHistBins = 3072;  // the reference's histogram-request limit (kPfeBins)
constexpr int kGather = 4096;    // values of the first histogram pass kept from the bins the sample points at

template <typename R>
struct RowSmem {
  union {  // the histogram is read up to the choice of the bins; the candidates are gathered after it
    uint32_t hist[kBins];
    R cand[kCap];
  };
  R gath[kGather];
  uint32_t gathCount;
  double dsum[kRowWarps];
  R rmin[kRowWarps], rmax[kRowWarps];
  uint32_t candCount;
  uint32_t usum[kRowWarps];
  uint32_t pick[4];
  double flo[kMaxRounds], finvw[kMaxRounds];
  uint32_t fb0[kMaxRounds], fb1[kMaxRounds];
};

__device__ __forceinline__ double blockSum(double v, double* scratch) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kRowWarps; ++w) s += scratch[w];
  __syncthreads();
  return s;  // valid in thread 0
}

// Bin 0 holds the row's minimum, the dominant duplicate of exposure rows (exact zeros): instead of counting it value
// by value, its count is the values binned less the other bins' counts, summed here over the CTA.
__device__ __forceinline__ void fillBinZero(uint32_t* hist, uint32_t binned, uint32_t* scratch) {
  uint32_t v = 0;
  for (uint32_t b = threadIdx.x; b < static_cast<uint32_t>(kBins); b += kRowThreads)
    if (b != 0) v += hist[b];
  v = __reduce_add_sync(0xFFFFFFFFu, v);
  if ((threadIdx.x & 31u) == 0) scratch[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kRowWarps; ++w) t += scratch[w];
    hist[0] = binned - t;
  }
  __syncthreads();
}

template <typename R>
__device__ __forceinline__ void blockMinMax(R& lo, R& hi, R* smin, R* smax) {
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) smin[warp] = lo, smax[warp] = hi;
  __syncthreads();
  lo = smin[0], hi = smax[0];
  for (int w = 1; w < kRowWarps; ++w) lo = fmin(lo, smin[w]), hi = fmax(hi, smax[w]);
  __syncthreads();
}

// The bin of a value over a range starting at lo, `scale` bins per unit: any non-decreasing map of the values to the
// bins serves the rank search, as long as every pass of a round uses the same one.  Double rows: floor((v - lo)
// scale) in double.  Single-precision rows: (v - lo) scale in float, clamped, rounded to an integer by adding 2^23
// (an FMA-pipe add and an integer subtract instead of two conversions per value); scaleOf gives the float scale.
__device__ __forceinline__ uint32_t binOf(double v, double lo, double scale) {
  const double f = (v - lo) * scale;
  const uint32_t b = f <= 0.0 ? 0u : (f >= static_cast<double>(kBins) ? static_cast<uint32_t>(kBins) : static_cast<uint32_t>(f));
  return min(b, static_cast<uint32_t>(kBins - 1));
}
__device__ __forceinline__ uint32_t binOf(float v, double lo, double scale) {
  const float f = fminf(fmaxf((v - static_cast<float>(lo)) * static_cast<float>(scale), 0.0f), static_cast<float>(kBins - 1));
  return __float_as_uint(f + 8388608.0f) - 0x4B000000u;
}
template <typename R>
__device__ __forceinline__ double scaleOf(R lo, R hi) {
  const double sc = static_cast<double>(kBins) / (static_cast<double>(hi) - static_cast<double>(lo));
  return sizeof(R) == 4 ? static_cast<double>(static_cast<float>(sc)) : sc;
}

template <typename R>
__device__ __forceinline__ bool passes(const RowSmem<R>& s, int rounds, R v) {
  for (int r = 0; r < rounds; ++r) {
    const uint32_t b = binOf(v, s.flo[r], s.finvw[r]);
    if (b < s.fb0[r] || b > s.fb1[r]) return false;
  }
  return true;
}

// Calls f(v, valid) for every value of the row, through max(x, 0) when pos, in warp-uniform steps (every lane
// calls f the same number of times, so f may vote).  Rows that start on a 16-byte boundary with a length a
// multiple of 16 bytes are read 16 bytes per load.
template <typename R, typename F>
__device__ __forceinline__ void forEachValue(const R* X, uint32_t nP, bool pos, F&& f) {
  const uint32_t tid = threadIdx.x;
  auto fix = [&](R x) { return pos ? fmax(x, R(0)) : x; };
  constexpr uint32_t kVec = 16 / sizeof(R);
  if ((nP % kVec) == 0 && (reinterpret_cast<uintptr_t>(X) & 15u) == 0) {
    const uint32_t nv = nP / kVec;
#pragma unroll 2
    for (uint32_t base = 0; base < nv; base += kRowThreads) {
      const uint32_t i = base + tid;
      const bool ok = i < nv;
      if constexpr (sizeof(R) == 4) {
        const float4 q = ok ? __ldg(reinterpret_cast<const float4*>(X) + i) : make_float4(0.f, 0.f, 0.f, 0.f);
        f(fix(q.x), ok), f(fix(q.y), ok), f(fix(q.z), ok), f(fix(q.w), ok);
      } else {
        const double2 q = ok ? __ldg(reinterpret_cast<const double2*>(X) + i) : make_double2(0.0, 0.0);
        f(fix(q.x), ok), f(fix(q.y), ok);
      }
    }
  } else {
    for (uint32_t base = 0; base < nP; base += kRowThreads) {
      const uint32_t i = base + tid;
      const bool ok = i < nP;
      f(fix(ok ? X[i] : R(0)), ok);
    }
  }
}

// A quantile's histogram needs a range, not the row's exact extremes: values outside it fall into the end bins,
// and the ranks are still located exactly.  On long rows the range is the minimum and maximum of a sample,
// every 16th block of 32 vectors (512 bytes, one 16-byte load per lane of a warp), about 1/16 of the row.
constexpr uint32_t kSampleStride = 16;
constexpr uint32_t kSampleMinVectors = 16384;  // rows of 64K floats or 32K doubles and more

template <typename R>
__device__ __forceinline__ bool canSample(const R* X, uint32_t nP) {
  constexpr uint32_t kVec = 16 / sizeof(R);
  return (nP % kVec) == 0 && (reinterpret_cast<uintptr_t>(X) & 15u) == 0 && nP / kVec >= kSampleMinVectors;
}

template <typename R>
__device__ __forceinline__ void sampleMinMax(const R* X, uint32_t nP, bool pos, R& lo, R& hi) {
  constexpr uint32_t kVec = 16 / sizeof(R);
  const uint32_t nv = nP / kVec, blocks = nv / 32, lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  auto take = [&](R x) {
    x = pos ? fmax(x, R(0)) : x;
    lo = fmin(lo, x), hi = fmax(hi, x);
  };
  for (uint32_t b = warp * kSampleStride; b < blocks; b += kRowWarps * kSampleStride) {
    const uint32_t i = b * 32 + lane;
    if constexpr (sizeof(R) == 4) {
      const float4 q = __ldg(reinterpret_cast<const float4*>(X) + i);
      take(q.x), take(q.y), take(q.z), take(q.w);
    } else {
      const double2 q = __ldg(reinterpret_cast<const double2*>(X) + i);
      take(q.x), take(q.y);
    }
  }
}

// The histogram of the same sample as sampleMinMax over the bins of (dlo, invw), bin 0's votes per warp as in the
// full pass; returns the number of values sampled.
template <typename R>
__device__ __forceinline__ uint32_t sampleHistogram(const R* X, uint32_t nP, bool pos, double dlo, double invw, uint32_t* hist) {
  constexpr uint32_t kVec = 16 / sizeof(R);
  const uint32_t nv = nP / kVec, blocks = nv / 32, lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  auto put = [&](R x) {  // bin 0 is filled afterwards (fillBinZero)
    x = pos ? fmax(x, R(0)) : x;
    const uint32_t b = binOf(x, dlo, invw);
    if (b != 0) atomicAdd(&hist[b], 1u);
  };
  for (uint32_t b = warp * kSampleStride; b < blocks; b += kRowWarps * kSampleStride) {
    const uint32_t i = b * 32 + lane;
    if constexpr (sizeof(R) == 4) {
      const float4 q = __ldg(reinterpret_cast<const float4*>(X) + i);
      put(q.x), put(q.y), put(q.z), put(q.w);
    } else {
      const double2 q = __ldg(reinterpret_cast<const double2*>(X) + i);
      put(q.x), put(q.y);
    }
  }
  return (blocks + kSampleStride - 1) / kSampleStride * 32u * kVec;
}

// The bins of ranks k and k1 >= k among the candidates counted in s.hist, `below` values ranking under bin 0:
// pick = {bin of k, bin of k1, values under k's bin, count of k's bin}, as a walk over the bins in order would
// find them.  One warp: lane l owns bins [128 l, 128 l + 128) (read skewed by l, free of bank conflicts), a
// warp scan of the lanes' counts finds the lane holding each rank, and that lane walks its own bins.
template <typename R>
__device__ __forceinline__ void locateRanks(RowSmem<R>& s, uint32_t below, uint32_t k, uint32_t k1, uint32_t lane) {
  constexpr uint32_t kPer = kBins / 32;
  uint32_t own = 0;
  for (uint32_t j = 0; j < kPer; ++j) own += s.hist[lane * kPer + ((j + lane) & (kPer - 1))];
  uint32_t incl = own;
  for (uint32_t o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += v;
  }
  const uint32_t start = below + incl - own;  // values under this lane's first bin
  const uint32_t m0 = __ballot_sync(0xFFFFFFFFu, below + incl > k), m1 = __ballot_sync(0xFFFFFFFFu, below + incl > k1);
  const uint32_t l0 = m0 ? __ffs(m0) - 1 : 31u, l1 = m1 ? __ffs(m1) - 1 : 31u;
  auto walk = [&](uint32_t r, uint32_t& bin, uint32_t& under) {
    uint32_t cum = start;
    bin = lane * kPer + kPer - 1, under = cum;
    for (uint32_t b = lane * kPer; b < lane * kPer + kPer; ++b) {
      const uint32_t c = s.hist[b];
      if (cum + c > r) {
        bin = b, under = cum;
        return;
      }
      cum += c;
    }
  };
  if (lane == l0) {
    uint32_t b0, under0;
    walk(k, b0, under0);
    if (!m0) b0 = kBins - 1, under0 = below;  // no rank k among the candidates (cannot happen): the last bin
    s.pick[0] = b0, s.pick[2] = under0, s.pick[3] = s.hist[b0];
  }
  if (lane == l1) {
    uint32_t b1, under1;
    walk(k1, b1, under1);
    if (!m1) b1 = kBins - 1;
    s.pick[1] = b1;
  }
}

// Bitonic sort of n (<= kCap) values in shared memory, padded with +inf to a power of two.
template <typename R>
__device__ void bitonicSort(R* a, uint32_t n) {
  uint32_t m = 1;
  while (m < n) m <<= 1;
  for (uint32_t i = n + threadIdx.x; i < m; i += kRowThreads) a[i] = R(INFINITY);
  __syncthreads();
  for (uint32_t size = 2; size <= m; size <<= 1)
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < m; i += kRowThreads) {
        const uint32_t partner = i ^ stride;
        if (partner > i) {
          const bool up = (i & size) == 0;
          const R ai = a[i], ap = a[partner];
          if ((ai > ap) == up) a[i] = ap, a[partner] = ai;
        }
      }
      __syncthreads();
    }
}

template <typename R>
__global__ void __launch_bounds__(kRowThreads, 6) rowStatsKernel(const RowJob<R>* __restrict__ jobs, uint32_t* __restrict__ err,
                                                                 uint32_t maxRounds) {
  extern __shared__ __align__(16) unsigned char raw[];
  RowSmem<R>& s = *reinterpret_cast<RowSmem<R>*>(raw);
  const RowJob<R> J = jobs[blockIdx.x];
  const R* rq = J.request;
  const uint32_t op = static_cast<uint32_t>(rq[0]), row = static_cast<uint32_t>(rq[1]), row2 = static_cast<uint32_t>(rq[2]);
  const uint32_t count = static_cast<uint32_t>(rq[3]);
  const size_t outAt = static_cast<size_t>(rq[7]);
  const uint32_t nP = J.nP, tid = threadIdx.x;
  const R* X = J.expo + static_cast<size_t>(row) * nP;
  R* out = J.out + outAt;

  if (op == 4) {  // samples: the first `count` paths
    for (uint32_t i = tid; i < count && i < nP; i += kRowThreads) out[i] = X[i];
    return;
  }
  if (op != 0 && op != 5 && op != 7) {  // means, in double precision
    const R* Y = J.expo + static_cast<size_t>(row2) * nP;
    double acc = 0.0;
    if (op == 1 || op == 2 || op == 3) {
      forEachValue(X, nP, false, [&](R x, bool ok) {
        const R f = op == 2 ? fmax(x, R(0)) : op == 3 ? fmin(x, R(0)) : x;
        if (ok) acc += static_cast<double>(f);
      });
    } else {
      for (uint32_t i = tid; i < nP; i += kRowThreads) {
        const R x = X[i];
        R f = x;
        switch (op) {
          case 6: f = x * Y[i]; break;
          case 8: f = fmax(x, R(0)) * Y[i]; break;
          case 9: f = fmin(x, R(0)) * Y[i]; break;
          default: break;
        }
        acc += static_cast<double>(f);
      }
    }
    const double total = blockSum(acc, s.dsum);
    if (tid == 0) out[0] = static_cast<R>(total / static_cast<double>(nP));
    return;
  }

  const bool pos = op == 7;
  R lo = R(INFINITY), hi = R(-INFINITY);
  // Quantiles of long rows take their first histogram's range from a sample (the row is then read twice, not
  // three times); a histogram request reports its range, and a sample without spread proves nothing, so those
  // read the whole row for its exact minimum and maximum.
  bool sampled = false;
  if (op != 5 && canSample(X, nP)) {
    sampleMinMax(X, nP, pos, lo, hi);
    blockMinMax(lo, hi, s.rmin, s.rmax);
    sampled = lo < hi;
  }
  if (!sampled) {
    lo = R(INFINITY), hi = R(-INFINITY);
    forEachValue(X, nP, pos, [&](R v, bool ok) {
      if (ok) lo = fmin(lo, v), hi = fmax(hi, v);
    });
    blockMinMax(lo, hi, s.rmin, s.rmax);
  }

  if (op == 5) {  // histogram of `count` bins on [lo, hi] (the request's range unless lo == hi there)
    if (rq[5] != rq[6]) lo = rq[5], hi = rq[6];
    const R span = fmax(hi - lo, R(1e-30));
    const uint32_t nb = min(count, static_cast<uint32_t>(kHistBins));
    for (uint32_t b = tid; b < nb; b += kRowThreads) s.hist[b] = 0;
    __syncthreads();
    for (uint32_t i = tid; i < nP; i += kRowThreads) {
      const R f = fmax((X[i] - lo) / span, R(0)) * static_cast<R>(nb);
      const uint32_t b = min(f >= R(4294967295.0) ? 0xFFFFFFFFu : static_cast<uint32_t>(f), nb - 1);
      atomicAdd(&s.hist[b], 1u);
    }
    __syncthreads();
    for (uint32_t b = tid; b < nb; b += kRowThreads) out[b] = static_cast<R>(s.hist[b]);
    if (tid == 0) out[nb] = lo, out[nb + 1] = hi;
    return;
  }

  // Exact interpolated quantile (ccr::quantile): ranks k and k1 = min(k + 1, n - 1).
  const double h = static_cast<double>(rq[4]) * static_cast<double>(nP - 1);
  const uint32_t k = min(static_cast<uint32_t>(floor(h)), nP - 1), k1 = min(k + 1, nP - 1);
  const double frac = h - static_cast<double>(k);
  if (!(lo < hi)) {
    if (tid == 0) out[0] = lo;
    return;
  }
  uint32_t below = 0, binned = nP;  // the values each round bins: the row, then the previous round's bin
  int rounds = 0;
  R vk = lo, vk1 = lo;
  bool done = false;
  // On a sampled row the sample's own histogram (same bins as round 0's) says where ranks k, k1 lie to within the
  // sample's rank error: round 0 then keeps the row's values of the bins holding sample ranks k_s -+ (3 sd + 4) and,
  // when those hold every value of the bins of k and k1, the quantile is read from them without another pass.
  uint32_t winLo = 1, winHi = 0;
  if (sampled) {
    const double dlo0 = static_cast<double>(lo), invw0 = scaleOf(lo, hi);
    for (uint32_t b = tid; b < kBins; b += kRowThreads) s.hist[b] = 0;
    if (tid == 0) s.gathCount = 0;
    __syncthreads();
    const uint32_t ns = sampleHistogram(X, nP, pos, dlo0, invw0, s.hist);
    __syncthreads();
    fillBinZero(s.hist, ns, s.usum);
    const double q = static_cast<double>(k) / static_cast<double>(nP), ks = q * static_cast<double>(ns);
    const double sd = sqrt(static_cast<double>(ns) * q * (1.0 - q)) * 3.0 + 4.0;
    const uint32_t rlo = static_cast<uint32_t>(fmax(ks - sd, 0.0)), rhi = static_cast<uint32_t>(fmin(ks + sd + 1.0, ns - 1.0));
    if (tid < 32) locateRanks(s, 0u, rlo, rhi, tid);
    __syncthreads();
    winLo = s.pick[0], winHi = s.pick[1];
  }
  while (!done) {
    if (rounds >= static_cast<int>(maxRounds)) {
      if (tid == 0) atomicExch(err, kDevBadTerm), out[0] = R(NAN);
      return;
    }
    // Range of the current candidates (round 0: the whole row, already known).
    if (rounds > 0) {
      lo = R(INFINITY), hi = R(-INFINITY);
      forEachValue(X, nP, pos, [&](R v, bool ok) {
        if (ok && passes(s, rounds, v)) lo = fmin(lo, v), hi = fmax(hi, v);
      });
      blockMinMax(lo, hi, s.rmin, s.rmax);
      if (!(lo < hi)) {  // every candidate has the same value
        vk = lo, vk1 = lo;
        break;
      }
    }
    const double dlo = static_cast<double>(lo), invw = scaleOf(lo, hi);
    for (uint32_t b = tid; b < kBins; b += kRowThreads) s.hist[b] = 0;
    __syncthreads();
    const bool gather = rounds == 0 && winLo <= winHi;
    const uint32_t winSpan = winHi - winLo;
    forEachValue(X, nP, pos, [&](R x, bool ok) {
      const bool in = ok && passes(s, rounds, x);
      const uint32_t b = binOf(x, dlo, invw);
      if (in && b != 0) atomicAdd(&s.hist[b], 1u);  // bin 0 is filled afterwards (fillBinZero)
      if (gather && in && b - winLo <= winSpan) {
        const uint32_t at = atomicAdd(&s.gathCount, 1u);
        if (at < static_cast<uint32_t>(kGather)) s.gath[at] = x;
      }
    });
    __syncthreads();
    fillBinZero(s.hist, binned, s.usum);
    if (tid < 32) locateRanks(s, below, k, k1, tid);
    __syncthreads();
    const uint32_t b0 = s.pick[0], b1 = s.pick[1], below0 = s.pick[2], c0 = s.pick[3];
    if (gather && winLo <= b0 && b1 <= winHi && s.gathCount <= static_cast<uint32_t>(kGather)) {
      // Every value of bins b0..b1 was kept (no bin between them holds one): sort them, read ranks k and k1.
      if (tid == 0) s.candCount = 0;
      __syncthreads();
      const uint32_t ng = s.gathCount;
      for (uint32_t i = tid; i < ng; i += kRowThreads) {
        const R v = s.gath[i];
        const uint32_t b = binOf(v, dlo, invw);
        if (b >= b0 && b <= b1) {
          const uint32_t at = atomicAdd(&s.candCount, 1u);
          if (at < static_cast<uint32_t>(kCap)) s.cand[at] = v;
        }
      }
      __syncthreads();
      const uint32_t n = s.candCount;
      if (n <= static_cast<uint32_t>(kCap) && k1 - below0 < n) {
        bitonicSort(s.cand, n);
        vk = s.cand[k - below0];
        vk1 = s.cand[k1 - below0];
        done = true;
        continue;
      }
      // more than kCap values: the passes below
    }
    if (b0 != b1) {
      // k is the largest value of bin b0, k + 1 the smallest of bin b1.
      R mx = R(-INFINITY), mn = R(INFINITY);
      forEachValue(X, nP, pos, [&](R v, bool ok) {
        if (!ok || !passes(s, rounds, v)) return;
        const uint32_t b = binOf(v, dlo, invw);
        if (b == b0) mx = fmax(mx, v);
        if (b == b1) mn = fmin(mn, v);
      });
      blockMinMax(mn, mx, s.rmin, s.rmax);  // block minimum of mn, block maximum of mx
      vk = mx, vk1 = mn;
      done = true;
    } else if (c0 <= static_cast<uint32_t>(kCap)) {
      if (tid == 0) s.candCount = 0;
      __syncthreads();
      forEachValue(X, nP, pos, [&](R v, bool ok) {
        if (ok && passes(s, rounds, v) && binOf(v, dlo, invw) == b0) s.cand[atomicAdd(&s.candCount, 1u)] = v;
      });
      __syncthreads();
      const uint32_t n = s.candCount;
      bitonicSort(s.cand, n);
      vk = s.cand[k - below0];
      vk1 = s.cand[min(k1 - below0, n - 1)];
      done = true;
    } else {
      if (tid == 0) s.flo[rounds] = dlo, s.finvw[rounds] = invw, s.fb0[rounds] = b0, s.fb1[rounds] = b0;
      __syncthreads();
      below = below0, binned = c0;
      ++rounds;
    }
  }
  if (tid == 0) {
    const double a = static_cast<double>(vk), b = static_cast<double>(vk1);
    out[0] = static_cast<R>(a + frac * (b - a));
  }
}

// Partials come one per warp of the revalue kernel: the sum over its 32 ppt adjacent paths.  A 128-path group's
// sum completes the binary tree of the warp sums ((w0 + w1) + (w2 + w3) for one path per thread, w0 + w1 for
// two, w0 for four), absent warps past the last path counting as 0, so it has the same bits for every tile
// shape; the groups are then summed in path order with a compensated double sum.
template <typename R, int PPT>
__global__ void reduceKernel(const ReduceJob<R>* __restrict__ jobs) {
  const ReduceJob<R> J = jobs[blockIdx.y];
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= J.n) return;
  // A job with pad 1 or 2 has partials of 32 or 64 paths whatever the batch's shape (the basis kernel's: 64).
  const uint32_t ppt = J.pad == 1u || J.pad == 2u ? J.pad : static_cast<uint32_t>(PPT);
  const uint32_t kUnits = 4 / ppt, kUnitPaths = 32 * ppt;
  auto unit = [&](uint32_t u) { return u * kUnitPaths < J.nP ? J.partials[static_cast<size_t>(u) * J.n + i] : R(0); };
  double sum = 0.0, comp = 0.0;
  for (uint32_t t = 0; t < J.numTiles; ++t) {
    const uint32_t u0 = t * kUnits;
    R g;
    if (ppt == 1) g = (unit(u0) + unit(u0 + 1)) + (unit(u0 + 2) + unit(u0 + 3));
    else if (ppt == 2) g = unit(u0) + unit(u0 + 1);
    else g = unit(u0);
    const double yv = static_cast<double>(g) - comp;
    const double tv = sum + yv;
    comp = (tv - sum) - yv;
    sum = tv;
  }
  J.sums[i] = static_cast<R>(sum / static_cast<double>(J.nP));
}

}  // namespace

template <typename R>
cudaError_t launchReduce(const ReduceJob<R>* jobs, uint32_t numJobs, uint32_t maxN, int ppt, cudaStream_t stream) {
  if (numJobs == 0 || maxN == 0) return cudaSuccess;
  const dim3 grid((maxN + 255) / 256, numJobs);
  switch (ppt) {
    case 1: reduceKernel<R, 1><<<grid, 256, 0, stream>>>(jobs); break;
    case 2: reduceKernel<R, 2><<<grid, 256, 0, stream>>>(jobs); break;
    case 4: reduceKernel<R, 4><<<grid, 256, 0, stream>>>(jobs); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename R>
cudaError_t launchRowStats(const RowJob<R>* jobs, uint32_t numJobs, uint32_t* err, cudaStream_t stream, uint32_t maxRounds) {
  if (numJobs == 0) return cudaSuccess;
  maxRounds = maxRounds < static_cast<uint32_t>(kMaxRounds) ? maxRounds : static_cast<uint32_t>(kMaxRounds);
  const size_t smem = sizeof(RowSmem<R>);
  cudaError_t e = cudaFuncSetAttribute(rowStatsKernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  rowStatsKernel<R><<<numJobs, kRowThreads, smem, stream>>>(jobs, err, maxRounds);
  return cudaGetLastError();
}

// The exact-decision check's patch: dst[r][map[q]] = src[r][q] (rounded to single precision) for every row r and
// re-run path q.  One thread per element; map holds distinct paths below nP.
__global__ void scatterRowsKernel(const double* __restrict__ src, uint32_t m, const uint32_t* __restrict__ map, uint32_t rows,
                                  float* __restrict__ dst, uint32_t nP) {
  const uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= static_cast<uint64_t>(rows) * m) return;
  const uint32_t r = static_cast<uint32_t>(k / m), q = static_cast<uint32_t>(k % m);
  dst[static_cast<size_t>(r) * nP + map[q]] = static_cast<float>(src[static_cast<size_t>(r) * m + q]);
}

cudaError_t launchScatterRows(const double* src, uint32_t m, const uint32_t* map, uint32_t rows, float* dst, uint32_t nP,
                              cudaStream_t stream) {
  const uint64_t n = static_cast<uint64_t>(rows) * m;
  if (n == 0) return cudaSuccess;
  scatterRowsKernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(src, m, map, rows, dst, nP);
  return cudaGetLastError();
}

template cudaError_t launchReduce<float>(const ReduceJob<float>*, uint32_t, uint32_t, int, cudaStream_t);
template cudaError_t launchReduce<double>(const ReduceJob<double>*, uint32_t, uint32_t, int, cudaStream_t);
template cudaError_t launchRowStats<float>(const RowJob<float>*, uint32_t, uint32_t*, cudaStream_t, uint32_t);
template cudaError_t launchRowStats<double>(const RowJob<double>*, uint32_t, uint32_t*, cudaStream_t, uint32_t);

}  // namespace zk
