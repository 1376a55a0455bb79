// Host-visible launchers of the zlatko_b200 kernels.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "zk_device.cuh"

namespace zk {

// Risk factors of every path and date into the factor cube.
template <typename R>
cudaError_t launchSimulate(const ScenarioArgs<R>& sc, const CubeArgs<R>& cb, cudaStream_t stream);

// Revalue / net / collateralise / reduce: one CTA per (path tile, netting set); each thread owns `ppt`
// paths (1, 2 or 4 in single precision, 1 or 2 in double), so a tile holds kTile * ppt paths.  `lean`: no
// netting set of the launch has AMC or probe terms (a variant without their state).  `smallState`: every
// netting set of the launch keeps at most kSmallStateWords shared-memory words per path, so a lean single-
// precision launch of 2 or 4 paths per thread may use the variant compiled for more resident CTAs.  `cash`:
// every netting set of a lean launch has a cash CSA with a margin-call look-back of at most one date and none of
// the optional value, exposure, collateral or change rows.
constexpr int kSmallStateWords = 26;
template <typename R>
cudaError_t launchRevalue(const CubeArgs<R>& cb, const NsArgs<R>* nsArgs, uint32_t numNs, uint32_t numTiles, size_t stateWordsMax,
                          bool perTrade, bool sink, bool lean, int ppt, cudaStream_t stream, bool smallState = false,
                          bool cash = false);
size_t revalueSmemBytes(size_t stateWordsMax, bool perTrade, bool f64, int ppt);

// The nested initial margin of one plan (fused_reference.cpp:356-393), after its revalue launch: one warp
// per (reporting slot, outer path), the lanes running the inner paths; the margin into rows rowIm + r.
template <typename R>
struct ImArgs {
  const R* cube;          // the launch's factor cube: x in field 0, ln S of asset a in field fLnS + a
  const uint32_t* dates;  // the plan's lowered date descriptors [nT][8] and records
  const R* table;
  const R* steps;         // [nT][24]
  const R* model;         // spots [4] | padded Cholesky factor [8][8]
  const uint32_t* slots;  // [nR][2]: the date of reporting slot r (kNoRow: none), its target date (kNoRow: none)
  const R* state;         // the outer state on the reporting dates (NsArgs::imState)
  R* expo;                // the plan's rows
  uint32_t nP, nT, nA, fLnS, nR, nSlots, nInner, rowIm, seed, anti, nCorr, pad;
  R level;                // the margin's quantile level
};
template <typename R>
cudaError_t launchNestedIm(const ImArgs<R>& M, cudaStream_t stream);

// Inner paths of the nested exposure (nested_inner.cu) for one reporting date: the program of events after the
// date (nestProgram in plan_compiler.cpp) and a round's jobs (scenario, seed, paths), one thread per inner path.
constexpr uint32_t kMaxNestSlots = 64;  // swaps whose running coupon an inner path tracks
struct NestArgs {
  const double* coef;                 // [events][24] step rows, column 7 = a
  const uint32_t* opBegin;            // [events + 1]
  const uint32_t* ops;                // kind << 28 | index
  const double* periods;              // [nPer][8]
  const double* terminals;            // [nTerm][8]
  const double* chol;                 // [(1 + nA)^2]
  const uint32_t* fixToday;           // periods fixing at the date itself
  const double* x0;                   // [scenarios] rate state at the date
  const double* spot0;                // [scenarios][nA]
  const double* fix0;                 // [scenarios][numSlots] fixings known at the date
  const unsigned long long* jobScenario;
  const unsigned long long* jobSeed;
  const unsigned long long* jobStart;  // first inner path of each job (ascending)
  double* out;                         // [totalPaths], job after job
  unsigned long long totalPaths;
  uint32_t numJobs, numEvents, nA, numSlots, numFixToday, pad;
};
cudaError_t launchNestInner(const NestArgs& M, cudaStream_t stream);

// One reduce job per plan: sums[i] = (sum over the 128-path groups of the group's partials) / nP for i < n, the
// partials [warp][i] being one per revalue warp of the tile shape ppt (32 ppt paths); numTiles counts the groups.
template <typename R>
struct ReduceJob {
  const R* partials;
  R* sums;
  uint32_t n, numTiles, nP;
  uint32_t pad;  // 1 / 2: partials of 32 / 64 paths (the basis kernel's: 64), whatever the launch's tile shape
};
template <typename R>
cudaError_t launchReduce(const ReduceJob<R>* jobs, uint32_t numJobs, uint32_t maxN, int ppt, cudaStream_t stream);

// One row-statistics job per request (fused_kernels.cpp:565-771): the request record, its plan's rows.
template <typename R>
struct RowJob {
  const R* expo;      // [rows][nP]
  const R* request;   // 8 words: (op, row, row2, count) (level, lo, hi, out)
  R* out;             // the plan's values
  uint32_t nP, pad;
};
template <typename R>
// maxRounds caps the quantile's narrowing rounds (at most 16, the default); a row that needs more sets
// kDevBadTerm in err and NaN as its value.
cudaError_t launchRowStats(const RowJob<R>* jobs, uint32_t numJobs, uint32_t* err, cudaStream_t stream, uint32_t maxRounds = 16);
// dst[r][map[q]] = float(src[r][q]) for r < rows, q < m (the exact-decision check's patch of re-run paths' rows;
// the map's paths distinct and below nP).
cudaError_t launchScatterRows(const double* src, uint32_t m, const uint32_t* map, uint32_t rows, float* dst, uint32_t nP,
                              cudaStream_t stream);

// One Bermudan of the AMC fit (zk_fit_amc): its exercise dates (grid indices, ascending), its first row of
// exercise values in the AMC pass, the slots of its fitted records (slotBase + k: policy of exercise k;
// slotBase + nE + i: continuation on date contDates[contBegin + i]) and its regression degree.
constexpr int kMaxExercises = 64;
struct AmcFitJob {
  uint32_t nP, nT, nE, degree, eRow, slotBase, contBegin, contCount;
  uint32_t twoD, pad;  // twoD: the Bermudan's records use the two-regressor basis
  uint32_t exDate[kMaxExercises];
};
// The two-regressor basis: per fit slot (exercise k at slotBase + k, continuation i at slotBase + nE + i) the range
// [bondRange.x, + bondRange.y) of its co-terminal swap's bonds {kind (annuity 13 / float leg 14), c, A, B}; the
// regressor s = sum_float c A e^{-B x} / sum_annuity c A e^{-B x}, as the fused kernel forms it.
constexpr int kFitOut = 16;  // doubles per fitted slot: 1D center, scale, c0..c3; 2D cx, sx, cs, ss, c0..c9
// One thread-block cluster of clusterSize CTAs per job; out[slot][kFitOut]; realised and, with bonds, swapScratch:
// [numJobs][nP] doubles of scratch.
template <typename R>
cudaError_t launchAmcFit(const AmcFitJob* jobs, uint32_t numJobs, const R* x, const R* D, const R* E, const uint32_t* contDates,
                         const double4* bonds, const uint2* bondRange, double* realised, double* swapScratch, double* out,
                         uint32_t* err, uint32_t clusterSize, cudaStream_t stream);

// C = A B^T with A [M][K], B [N][K] bf16 row-major (K contiguous) and FP32 accumulation on the tensor cores
// (mlp.cu); M % 128 == 0, N % 16 == 0, K % 16 == 0.  Epilogue: z = acc + bias[n], times silu'(gradOf[m][n])
// when gradOf is given (back-propagation through a SiLU); C (fp32, or C += z when accumulate), Z = bf16(z),
// H = bf16(act(z)) row-major, HT = bf16(act(z)) transposed [N][M]; any may be null.
struct GemmArgs {
  const __nv_bfloat16* A;
  const __nv_bfloat16* B;
  uint32_t M, N, K;
  const float* bias;
  float* C;
  __nv_bfloat16* Z;
  __nv_bfloat16* H;
  __nv_bfloat16* HT;
  const __nv_bfloat16* gradOf;  // [M][N] pre-activations of the SiLU being back-propagated, or null
  uint32_t act;         // 0 identity, 1 SiLU
  uint32_t accumulate;
  uint32_t* err;
  // Fused linear head (N = 128, one column tile): headOut[row] = sum_n bf16(h[row][n]) headW[n] + headB[0],
  // summed over n in order; or null.
  const float* headW;
  const float* headB;
  float* headOut;
};
cudaError_t launchGemm(const GemmArgs& g, cudaStream_t stream);

}  // namespace zk
