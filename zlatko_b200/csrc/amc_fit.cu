// Longstaff-Schwartz fit of the Bermudans of a plan on the GPU: the policy (exercise decision) and the
// continuation regressions that the fused kernel's AMC terms evaluate.
//
// It follows the reference's compile-time fit (fitAmc, src/gpu/fused_exposure.cpp:103-156, with
// PolynomialRegression, src/core/regression.cpp:29-98): backwards over the exercise dates, a masked
// (in-the-money) regression of the deflated realised value on the standardised short-rate state, the
// exercise rule "exercise value > 0 and > regression", and on every date with an exercise ahead an
// unmasked regression of the value of the policy from the next exercise on.  The degree falls back as the
// reference's does (degenerate regressor, too few samples) and the ridge is 1e-12 n.
//
// B200 layout: one thread-block cluster per Bermudan.  Each CTA owns a fixed strided share of the paths
// and keeps the realised values of its paths in a global scratch row that only it touches; every pass
// (moments, Gram, exercise update) is a streaming read of the AMC pass's x, deflator and exercise values.
// The per-CTA sums are reduced through distributed shared memory on rank 0 in rank order, so the fit is
// deterministic.  Rank 0 solves the normal equations by an FP64 Cholesky factorisation and broadcasts the
// coefficients back through DSMEM.  The Gram of a one-dimensional monomial basis is a handful of power
// moments, an FP64 CUDA-core reduction: the work per path is ~30 flops against 12-20 bytes read.
#include <cooperative_groups.h>

#include "zk_device.cuh"
#include "zk_kernels.h"

namespace cg = cooperative_groups;

namespace zk {

namespace {

constexpr int kFitThreads = 512;
constexpr int kFitWarps = kFitThreads / 32;
constexpr int kMomentVals = 4;   // count, sum x, sum x^2, sum y
constexpr int kGramVals = 14;    // 10 Gram entries (lower triangle, degree 3) + 4 right-hand sides
// The two-regressor basis: its Gram entries are the mixed moments sum z^a w^b, a + b <= 6 (28 of them, where the
// lower triangle of 10 functions has 55 entries), plus the 10 right-hand sides: one pass of 38 sums.
constexpr int kMom2 = 28, kSums2 = kMom2 + 10;

struct FitSmem {
  double warpBuf[kFitWarps][kSums2];
  double part[kSums2];      // this CTA's sums
  double res[16];           // rank 0: 1D center, scale, degree, c0..c3, status; 2D cx, sx, cs, ss, c0..c9, degree
};

// Sums V values over the CTA: a fixed shuffle tree per warp, then the warps in order.
template <int V>
__device__ __forceinline__ void blockSum(double (&v)[V], FitSmem& s) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < V; ++i)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[i] += __shfl_xor_sync(0xFFFFFFFFu, v[i], off);
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < V; ++i) s.warpBuf[warp][i] = v[i];
  __syncthreads();
  if (threadIdx.x < V) {
    double t = 0.0;
    for (int w = 0; w < kFitWarps; ++w) t += s.warpBuf[w][threadIdx.x];
    s.part[threadIdx.x] = t;
  }
}

// Rank 0 sums the cluster's parts in rank order into `tot` (its own shared memory).
template <int V>
__device__ __forceinline__ void clusterSum(cg::cluster_group& cl, FitSmem& s, double* tot) {
  cl.sync();
  if (cl.block_rank() == 0 && threadIdx.x < V) {
    double t = 0.0;
    for (unsigned r = 0; r < cl.num_blocks(); ++r) t += cl.map_shared_rank(s.part, r)[threadIdx.x];
    tot[threadIdx.x] = t;
  }
  __syncthreads();
}

// z^0 .. z^d by repeated multiplication, as the reference's design rows.
__device__ __forceinline__ void powers(double z, int d, double (&pw)[4]) {
  pw[0] = 1.0;
#pragma unroll
  for (int i = 1; i < 4; ++i) pw[i] = i <= d ? pw[i - 1] * z : 0.0;
}

__device__ __forceinline__ double predict(const double* res, double x) {
  const double z = (x - res[0]) / res[1];
  const int d = static_cast<int>(res[2]);
  double v = 0.0;
  for (int i = d; i >= 0; --i) v = v * z + res[3 + i];
  return v;
}

// One regression of y = realised / D on x over the CTA's paths (masked by E > 0 when E is given); the
// result lands in every CTA's `res` copy and, from rank 0, in out[0..5] = center, scale, c0..c3.
template <typename R>
__device__ void fitOnce(cg::cluster_group& cl, FitSmem& s, double* res, const R* __restrict__ X, const R* __restrict__ Dj,
                        const R* __restrict__ Ek, const double* __restrict__ realised, uint32_t nP, int degree, uint32_t first,
                        uint32_t stride, double* out, uint32_t* err) {
  __shared__ double tot[kGramVals];
  // Pass 1: count, sum x, sum x^2, sum y.
  double m[kMomentVals] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t p = first; p < nP; p += stride) {
    if (Ek && !(Ek[p] > R(0))) continue;
    const double x = static_cast<double>(X[p]);
    m[0] += 1.0, m[1] += x, m[2] += x * x, m[3] += realised[p] / static_cast<double>(Dj[p]);
  }
  blockSum(m, s);
  clusterSum<kMomentVals>(cl, s, tot);
  if (cl.block_rank() == 0 && threadIdx.x == 0) {
    const double n = tot[0];
    double center = 0.0, scale = 1.0;
    int d = degree;
    for (int i = 0; i < 4; ++i) s.res[3 + i] = 0.0;
    if (n == 0.0) {
      d = -1;  // no sample: the regression predicts 0
    } else {
      center = tot[1] / n;
      const double var = tot[2] / n - center * center;
      scale = sqrt(var > 0.0 ? var : 0.0);
      if (scale < 1e-12 * fmax(1.0, fabs(center))) d = 0;
      if (n < 2.0 * (d + 1)) d = n >= 4.0 ? static_cast<int>(n) / 2 - 1 : 0;
      if (d == 0) scale = 1.0, s.res[3] = tot[3] / n;
    }
    s.res[0] = center, s.res[1] = scale, s.res[2] = d < 0 ? 0.0 : static_cast<double>(d), s.res[7] = static_cast<double>(d);
  }
  cl.sync();
  const double* r0 = cl.map_shared_rank(s.res, 0);
  if (threadIdx.x < 8) res[threadIdx.x] = r0[threadIdx.x];
  __syncthreads();
  const int d = static_cast<int>(res[7]);
  if (d > 0) {
    // Pass 2: Gram (lower triangle) and right-hand side of the standardised design.
    double g[kGramVals];
#pragma unroll
    for (int i = 0; i < kGramVals; ++i) g[i] = 0.0;
    const double c = res[0], sc = res[1];
    for (uint32_t p = first; p < nP; p += stride) {
      if (Ek && !(Ek[p] > R(0))) continue;
      double pw[4];
      powers((static_cast<double>(X[p]) - c) / sc, d, pw);
      const double y = realised[p] / static_cast<double>(Dj[p]);
      int k = 0;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
#pragma unroll
        for (int b = 0; b <= a; ++b) g[k++] += pw[a] * pw[b];
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) g[10 + a] += pw[a] * y;
    }
    blockSum(g, s);
    clusterSum<kGramVals>(cl, s, tot);
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
      // Normal equations with the ridge, by FP64 Cholesky: G = L L^T, L y = b, L^T c = y.
      const int k = d + 1;
      double A[4][4], L[4][4] = {}, b[4], yv[4];
      int q = 0;
      for (int a = 0; a < 4; ++a)
        for (int bb = 0; bb <= a; ++bb) A[a][bb] = A[bb][a] = tot[q++];
      const double ridge = 1e-12 * tot[0];
      for (int a = 0; a < k; ++a) A[a][a] += ridge, b[a] = tot[10 + a];
      bool ok = true;
      for (int i = 0; i < k; ++i)
        for (int j = 0; j <= i; ++j) {
          double v = A[i][j];
          for (int m2 = 0; m2 < j; ++m2) v -= L[i][m2] * L[j][m2];
          if (i == j) {
            if (!(v > 0.0)) ok = false, v = 1.0;
            L[i][i] = sqrt(v);
          } else {
            L[i][j] = v / L[j][j];
          }
        }
      for (int i = 0; i < k; ++i) {
        double v = b[i];
        for (int j = 0; j < i; ++j) v -= L[i][j] * yv[j];
        yv[i] = v / L[i][i];
      }
      for (int i = k - 1; i >= 0; --i) {
        double v = yv[i];
        for (int j = i + 1; j < k; ++j) v -= L[j][i] * s.res[3 + j];
        s.res[3 + i] = v / L[i][i];
      }
      if (!ok) atomicExch(err, kDevBadTerm);
    }
    cl.sync();
    if (threadIdx.x < 4) res[3 + threadIdx.x] = cl.map_shared_rank(s.res, 0)[3 + threadIdx.x];
    __syncthreads();
  }
  if (cl.block_rank() == 0 && threadIdx.x == 0) {
    out[0] = res[0], out[1] = res[1];
    for (int i = 0; i < 4; ++i) out[2 + i] = res[3 + i];
  }
  // No CTA may start the next pass (and overwrite its part) before rank 0 has read every part, nor may
  // rank 0 overwrite res before every CTA has copied it: the syncs of the next fit order both.
}

// ---- the two-regressor basis (this library's extension: the reference regresses on x alone) ----

// The co-terminal swap rate of a path from its short rate, over the slot's bonds in plan order (as the fused
// kernel forms it: annuity and float leg each summed term by term, then their ratio).
__device__ __forceinline__ double swapRateOf(const double4* __restrict__ b, uint2 range, double x) {
  double ann = 0.0, flt = 0.0;
  for (uint32_t i = 0; i < range.y; ++i) {
    const double4 q = b[range.x + i];
    const double v = q.y * (q.z * exp(-q.w * x));
    if (q.x == 13.0) ann += v;
    else flt += v;
  }
  return ann != 0.0 ? flt / ann : 0.0;
}

// The graded monomials 1, z, w, z^2, z w, w^2, z^3, z^2 w, z w^2, w^3: the exponents of z and w of function i.
__host__ __device__ constexpr int powZ(int i) { return i == 1 || i == 4 || i == 8 ? 1 : i == 3 || i == 7 ? 2 : i == 6 ? 3 : 0; }
__host__ __device__ constexpr int powW(int i) { return i == 2 || i == 4 || i == 7 ? 1 : i == 5 || i == 8 ? 2 : i == 9 ? 3 : 0; }
// Index of the moment sum z^a w^b (a + b <= 6) among the 28.
__host__ __device__ constexpr int moment2(int a, int b) { return a * 7 - a * (a - 1) / 2 + b; }

__device__ __forceinline__ int basisCount2(int d) { return d <= 0 ? 1 : d == 1 ? 3 : d == 2 ? 6 : 10; }

// res: cx, sx, cs, ss, c0..c9, degree (-1: no sample, predicts 0)
__device__ __forceinline__ double predict2(const double* res, double x, double s) {
  const int d = static_cast<int>(res[14]);
  if (d < 0) return 0.0;
  const double z = (x - res[0]) / res[1], w = (s - res[2]) / res[3];
  const double m[10] = {1.0, z, w, z * z, z * w, w * w, z * z * z, z * z * w, z * w * w, w * w * w};
  const int count = basisCount2(d);
  double v = 0.0;
#pragma unroll
  for (int i = 0; i < 10; ++i)
    if (i < count) v += res[4 + i] * m[i];
  return v;
}

// One regression of y = realised / D on (x, s) over the cluster's paths (masked by E > 0 when E is given):
// standardised regressors, degree 0 when either is degenerate, lower while the samples are fewer than twice the
// basis, ridge 1e-6 n, FP64 Cholesky.  The ridge is larger than the one-regressor fit's: in a one-factor model the
// swap rate is a smooth function of the short rate, the graded Gram's condition number reaches 1e17, and 1e-6 n keeps
// the predictions stable to the summation order (~1e-11) at a negligible bias where the data are well conditioned.
// The first pass forms each included path's swap rate once (its bonds' exponentials) into the CTA's scratch row `sw`,
// which the Gram pass and the caller's exercise update read.  Result in every CTA's `res` and, from rank 0,
// out[0..13] = cx, sx, cs, ss, c0..c9.
template <typename R>
__device__ void fitOnce2(cg::cluster_group& cl, FitSmem& s, double* res, const R* __restrict__ X, const R* __restrict__ Dj,
                         const R* __restrict__ Ek, const double* __restrict__ realised, const double4* bonds, uint2 range,
                         double* __restrict__ sw, uint32_t nP, int degree, uint32_t first, uint32_t stride, double* out,
                         uint32_t* err) {
  __shared__ double tot[kSums2];
  double m[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (uint32_t p = first; p < nP; p += stride) {  // count, sum x, sum x^2, sum s, sum s^2, sum y
    if (Ek && !(Ek[p] > R(0))) continue;
    const double x = static_cast<double>(X[p]), r = swapRateOf(bonds, range, x);
    sw[p] = r;
    m[0] += 1.0, m[1] += x, m[2] += x * x, m[3] += r, m[4] += r * r, m[5] += realised[p] / static_cast<double>(Dj[p]);
  }
  blockSum<6>(m, s);
  clusterSum<6>(cl, s, tot);
  if (cl.block_rank() == 0 && threadIdx.x == 0) {
    const double n = tot[0];
    double* r = s.res;
    for (int i = 0; i < 16; ++i) r[i] = 0.0;
    r[1] = r[3] = 1.0;
    if (n == 0.0) {
      r[14] = -1.0;
    } else {
      r[0] = tot[1] / n, r[2] = tot[3] / n;
      const double vx = tot[2] / n - r[0] * r[0], vs = tot[4] / n - r[2] * r[2];
      r[1] = sqrt(vx > 0.0 ? vx : 0.0), r[3] = sqrt(vs > 0.0 ? vs : 0.0);
      int d = degree;
      if (r[1] < 1e-12 * fmax(1.0, fabs(r[0])) || r[3] < 1e-12 * fmax(1.0, fabs(r[2]))) d = 0;
      while (d > 0 && n < 2.0 * basisCount2(d)) --d;
      if (d == 0) r[0] = r[2] = 0.0, r[1] = r[3] = 1.0, r[4] = tot[5] / n;
      r[14] = static_cast<double>(d);
    }
  }
  cl.sync();
  const double* r0 = cl.map_shared_rank(s.res, 0);
  if (threadIdx.x < 16) res[threadIdx.x] = r0[threadIdx.x];
  __syncthreads();
  const int d = static_cast<int>(res[14]);
  if (d > 0) {
    // The moments sum z^a w^b (a + b <= 6) and sum z^a w^b y over the basis' exponents, one pass.
    double g[kSums2];
#pragma unroll
    for (int i = 0; i < kSums2; ++i) g[i] = 0.0;
    for (uint32_t p = first; p < nP; p += stride) {
      if (Ek && !(Ek[p] > R(0))) continue;
      const double z = (static_cast<double>(X[p]) - res[0]) / res[1], w = (sw[p] - res[2]) / res[3];
      const double y = realised[p] / static_cast<double>(Dj[p]);
      double zp[7], wp[7];
      zp[0] = wp[0] = 1.0;
#pragma unroll
      for (int i = 1; i < 7; ++i) zp[i] = zp[i - 1] * z, wp[i] = wp[i - 1] * w;
#pragma unroll
      for (int a = 0; a <= 6; ++a)
#pragma unroll
        for (int b = 0; a + b <= 6; ++b) g[moment2(a, b)] += zp[a] * wp[b];
#pragma unroll
      for (int i = 0; i < 10; ++i) g[kMom2 + i] += zp[powZ(i)] * wp[powW(i)] * y;  // the right-hand sides
    }
    blockSum<kSums2>(g, s);
    clusterSum<kSums2>(cl, s, tot);
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
      const int count = basisCount2(d);
      double A[10][10], L[10][10] = {}, b[10], z[10], c[10] = {};
      for (int i = 0; i < 10; ++i) {
        for (int j = 0; j < 10; ++j) A[i][j] = tot[moment2(powZ(i) + powZ(j), powW(i) + powW(j))];
        b[i] = tot[kMom2 + i];
      }
      const double n = tot[0];  // sum z^0 w^0: the sample count
      for (int a = 0; a < count; ++a) A[a][a] += 1e-6 * n;
      bool ok = true;
      for (int i = 0; i < count; ++i)
        for (int j = 0; j <= i; ++j) {
          double v = A[i][j];
          for (int k = 0; k < j; ++k) v -= L[i][k] * L[j][k];
          if (i == j) {
            if (!(v > 0.0)) ok = false, v = 1.0;
            L[i][i] = sqrt(v);
          } else {
            L[i][j] = v / L[j][j];
          }
        }
      for (int i = 0; i < count; ++i) {
        double v = b[i];
        for (int j = 0; j < i; ++j) v -= L[i][j] * z[j];
        z[i] = v / L[i][i];
      }
      for (int i = count - 1; i >= 0; --i) {
        double v = z[i];
        for (int j = i + 1; j < count; ++j) v -= L[j][i] * c[j];
        c[i] = v / L[i][i];
      }
      for (int i = 0; i < 10; ++i) s.res[4 + i] = c[i];
      if (!ok) atomicExch(err, kDevBadTerm);
    }
    cl.sync();
    if (threadIdx.x < 10) res[4 + threadIdx.x] = cl.map_shared_rank(s.res, 0)[4 + threadIdx.x];
    __syncthreads();
  }
  if (cl.block_rank() == 0 && threadIdx.x == 0)
    for (int i = 0; i < 14; ++i) out[i] = res[i];
}

// TwoD: the launch has two-regressor jobs (its one-regressor jobs run the same code as without).
template <typename R, bool TwoD>
__global__ void __launch_bounds__(kFitThreads) amcFitKernel(const AmcFitJob* __restrict__ jobs, const R* __restrict__ x,
                                                             const R* __restrict__ D, const R* __restrict__ E,
                                                             const uint32_t* __restrict__ contDates, const double4* __restrict__ bonds,
                                                             const uint2* __restrict__ bondRange, double* __restrict__ realised,
                                                             double* __restrict__ swapScratch, double* __restrict__ out,
                                                             uint32_t* err) {
  cg::cluster_group cl = cg::this_cluster();
  __shared__ FitSmem s;
  __shared__ double res[16];
  const uint32_t job = blockIdx.x / cl.num_blocks();
  const AmcFitJob J = jobs[job];
  const uint32_t nP = J.nP, stride = cl.num_blocks() * kFitThreads, first = cl.block_rank() * kFitThreads + threadIdx.x;
  double* rz = realised + static_cast<size_t>(job) * nP;
  double* sw = TwoD ? swapScratch + static_cast<size_t>(job) * nP : nullptr;
  for (uint32_t p = first; p < nP; p += stride) rz[p] = 0.0;
  for (int k = static_cast<int>(J.nE) - 1; k >= 0; --k) {
    const size_t j = J.exDate[k];
    const R* Ek = E + static_cast<size_t>(J.eRow + k) * nP;
    const bool twoD = TwoD && J.twoD;
    const uint2 rk = twoD ? bondRange[J.slotBase + k] : make_uint2(0, 0);
    if (twoD)
      fitOnce2<R>(cl, s, res, x + j * nP, D + j * nP, Ek, rz, bonds, rk, sw, nP, static_cast<int>(J.degree), first, stride,
                  out + static_cast<size_t>(J.slotBase + k) * kFitOut, err);
    else
      fitOnce<R>(cl, s, res, x + j * nP, D + j * nP, Ek, rz, nP, static_cast<int>(J.degree), first, stride,
                 out + static_cast<size_t>(J.slotBase + k) * kFitOut, err);
    // Exercise where the exercise value is positive and beats the regression: realised = D e (the swap rate of a
    // path with E > 0 is in its scratch row from the fit).
    for (uint32_t p = first; p < nP; p += stride) {
      const double e = static_cast<double>(Ek[p]);
      if (!(e > 0.0)) continue;
      const double xp = static_cast<double>(x[j * nP + p]);
      const double c = twoD ? predict2(res, xp, sw[p]) : predict(res, xp);
      if (e > c) rz[p] = static_cast<double>(D[j * nP + p]) * e;
    }
    // Continuation on the dates whose next exercise is k: exDate[k - 1] <= date < exDate[k].
    const uint32_t lo = k > 0 ? J.exDate[k - 1] : 0u;
    for (uint32_t i = 0; i < J.contCount; ++i) {
      const uint32_t jc = contDates[J.contBegin + i];
      if (jc < lo || jc >= j) continue;
      double* oc = out + static_cast<size_t>(J.slotBase + J.nE + i) * kFitOut;
      if (twoD)
        fitOnce2<R>(cl, s, res, x + static_cast<size_t>(jc) * nP, D + static_cast<size_t>(jc) * nP, static_cast<const R*>(nullptr),
                    rz, bonds, bondRange[J.slotBase + J.nE + i], sw, nP, static_cast<int>(J.degree), first, stride, oc, err);
      else
        fitOnce<R>(cl, s, res, x + static_cast<size_t>(jc) * nP, D + static_cast<size_t>(jc) * nP, static_cast<const R*>(nullptr),
                   rz, nP, static_cast<int>(J.degree), first, stride, oc, err);
    }
  }
  cl.sync();  // rank 0's shared memory stays alive until every CTA of the cluster is done reading it
}

}  // namespace

template <typename R>
cudaError_t launchAmcFit(const AmcFitJob* jobs, uint32_t numJobs, const R* x, const R* D, const R* E, const uint32_t* contDates,
                         const double4* bonds, const uint2* bondRange, double* realised, double* swapScratch, double* out,
                         uint32_t* err, uint32_t clusterSize, cudaStream_t stream) {
  if (numJobs == 0) return cudaSuccess;
  if (clusterSize < 1 || clusterSize > 8) return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(numJobs * clusterSize);
  cfg.blockDim = dim3(kFitThreads);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = clusterSize, attr[0].val.clusterDim.y = 1, attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (bonds) {
    if (!swapScratch) return cudaErrorInvalidValue;
    return cudaLaunchKernelEx(&cfg, amcFitKernel<R, true>, jobs, x, D, E, contDates, bonds, bondRange, realised, swapScratch, out, err);
  }
  return cudaLaunchKernelEx(&cfg, amcFitKernel<R, false>, jobs, x, D, E, contDates, bonds, bondRange, realised, swapScratch, out, err);
}

template cudaError_t launchAmcFit<float>(const AmcFitJob*, uint32_t, const float*, const float*, const float*, const uint32_t*,
                                         const double4*, const uint2*, double*, double*, double*, uint32_t*, uint32_t, cudaStream_t);
template cudaError_t launchAmcFit<double>(const AmcFitJob*, uint32_t, const double*, const double*, const double*, const uint32_t*,
                                          const double4*, const uint2*, double*, double*, double*, uint32_t*, uint32_t, cudaStream_t);

}  // namespace zk
