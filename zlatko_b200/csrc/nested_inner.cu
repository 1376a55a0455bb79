// Inner paths of the nested exposure (the reference's InnerSimulator of nestedExposure,
// src/nested/nested_exposure.cpp:211-244): from an outer path's state at date t, exact Hull-White and lognormal
// steps to each later event date of the netting set, coupons paid on their fixings, terminal flows paid on the
// spot, all discounted to t.  The reference runs one scenario's batch sequentially on one thread; here one thread
// runs one inner path of a round's jobs, whatever the scenario: the normals are counter-based (the reference's
// CounterNormals: SplitMix64 pairs and Box-Muller), so inner path q of a job starts at normal
// q x events x (nA + 2) of the job's stream without drawing the ones before it.  Double precision throughout.
#include "zk_kernels.h"

namespace zk {

namespace {

__device__ __forceinline__ unsigned long long splitMix(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Normals m0, m0 + 1, ..., m0 + n - 1 of CounterNormals(seed): pair k = m / 2 draws from state seed + (k + 1)
// golden ratios; the even normal is the cosine half.
__device__ void counterNormals(unsigned long long seed, unsigned long long m0, int n, double* z) {
  unsigned long long pair = ~0ull;
  double c = 0.0, s = 0.0;
  for (int i = 0; i < n; ++i) {
    const unsigned long long m = m0 + static_cast<unsigned long long>(i), k = m >> 1;
    if (k != pair) {
      pair = k;
      const unsigned long long h1 = splitMix(seed + (k + 1) * 0x9E3779B97F4A7C15ull);
      const unsigned long long h2 = splitMix(h1 ^ 0x68E31DA4B5297A4Dull);
      const double u1 = (static_cast<double>(h1 >> 11) + 0.5) * 0x1.0p-53;
      const double u2 = static_cast<double>(h2 >> 11) * 0x1.0p-53;
      const double r = sqrt(-2.0 * log(u1)), a = 6.283185307179586 * u2;
      sincos(a, &s, &c);
      c *= r, s *= r;
    }
    z[i] = (m & 1ull) ? s : c;
  }
}

__global__ void __launch_bounds__(128) nestInnerKernel(const NestArgs M) {
  const unsigned long long g = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (g >= M.totalPaths) return;
  // The job of this inner path: the last job starting at or before g.
  uint32_t lo = 0, hi = M.numJobs - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (M.jobStart[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  const uint32_t job = lo, p = static_cast<uint32_t>(M.jobScenario[job]);
  const unsigned long long seed = M.jobSeed[job], q = g - M.jobStart[job];
  const uint32_t nA = M.nA, per = nA + 2;
  double x = M.x0[p], lnD = 0.0, y = 0.0;
  double spot[kMaxAssets], fix[kMaxNestSlots], z[kMaxAssets + 2], w[kMaxAssets + 1];
  for (uint32_t a = 0; a < nA; ++a) spot[a] = M.spot0[static_cast<size_t>(p) * nA + a];
  for (uint32_t k = 0; k < M.numSlots; ++k) fix[k] = M.fix0[static_cast<size_t>(p) * M.numSlots + k];
  for (uint32_t k = 0; k < M.numFixToday; ++k) {  // coupons fixing at t itself, from x at t
    const double* r = M.periods + 8 * M.fixToday[k];
    const double bond = r[4] * exp(r[5] - r[6] * x);
    fix[static_cast<uint32_t>(r[3])] = (1.0 / bond - 1.0) / r[0];
  }
  const unsigned long long base = q * static_cast<unsigned long long>(M.numEvents) * per;
  for (uint32_t e = 0; e < M.numEvents; ++e) {
    counterNormals(seed, base + static_cast<unsigned long long>(e) * per, static_cast<int>(per), z);
    for (uint32_t i = 0; i <= nA; ++i) {
      double sum = 0.0;
      for (uint32_t j = 0; j <= i; ++j) sum += M.chol[i * (nA + 1) + j] * z[j];
      w[i] = sum;
    }
    const double* st = M.coef + static_cast<size_t>(e) * kStepStride;
    const double integratedX = x * (1.0 - st[0]) / st[7] + st[2] * w[0] + st[3] * z[nA + 1];  // hull_white.cpp:57
    x = x * st[0] + st[1] * w[0];
    const double integrated = integratedX + st[4];
    lnD -= integrated;
    for (uint32_t a = 0; a < nA; ++a) spot[a] = spot[a] * exp(integrated - st[8 + a] - st[16 + a] + st[12 + a] * w[1 + a]);
    const double D = exp(lnD);
    for (uint32_t o = M.opBegin[e]; o < M.opBegin[e + 1]; ++o) {
      const uint32_t op = M.ops[o], kind = op >> 28, idx = op & 0x0FFFFFFFu;
      if (kind == 0) {  // a coupon paid on its fixing
        const double* r = M.periods + 8 * idx;
        y += r[1] * (fix[static_cast<uint32_t>(r[3])] - r[2]) * r[0] * D;
      } else if (kind == 1) {  // a coupon fixed on the rate state
        const double* r = M.periods + 8 * idx;
        const double bond = r[4] * exp(r[5] - r[6] * x);
        fix[static_cast<uint32_t>(r[3])] = (1.0 / bond - 1.0) / r[0];
      } else {  // a forward or an option paid on the spot
        const double* r = M.terminals + 8 * idx;
        const double s = spot[static_cast<uint32_t>(r[0])], k = r[4];
        const double pay = r[1] != 0.0 ? fmax(r[2] != 0.0 ? s - k : k - s, 0.0) : s - k;
        y += r[3] * pay * D;
      }
    }
  }
  M.out[g] = y;
}

}  // namespace

cudaError_t launchNestInner(const NestArgs& M, cudaStream_t stream) {
  if (M.totalPaths == 0) return cudaSuccess;
  const unsigned long long blocks = (M.totalPaths + 127) / 128;
  if (blocks > 0x7FFFFFFFull || M.numJobs == 0) return cudaErrorInvalidConfiguration;
  nestInnerKernel<<<static_cast<uint32_t>(blocks), 128, 0, stream>>>(M);
  return cudaGetLastError();
}

}  // namespace zk
