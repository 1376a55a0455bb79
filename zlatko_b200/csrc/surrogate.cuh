// Host-side state of the learned revaluation surrogate (surrogate.cu): the MLP's parameters, Adam moments,
// BF16 weight copies and the workspace of one batch, all on the device.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "zk_kernels.h"

namespace zk {

constexpr uint32_t kIn = 16, kHid = 128;
using bf16 = __nv_bfloat16;

// Parameter blocks (fp32 masters, Adam moments, bf16 copies) and the activations of one batch.
struct SurrogateState {
  static constexpr uint32_t kW1 = kHid * kIn, kW2 = kHid * kHid, kW3 = kHid * kHid;
  static constexpr uint32_t kParams = kW1 + kHid + kW2 + kHid + kW3 + kHid + kHid + 1;
  cudaStream_t stream = nullptr;
  uint32_t* err = nullptr;
  float* p = nullptr;       // W1 b1 W2 b2 W3 b3 w4 b4 (the flattened order of the ABI)
  float* grad = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  bf16* wb = nullptr;       // W1 W2 W3 bf16 [out][in]
  bf16* wbT = nullptr;      // W1^T W2^T W3^T bf16 [in][out]
  float* scale = nullptr;   // mean[16], 1 / sd[16]
  float yMean = 0.0f, yScale = 1.0f;
  bool scaled = false;
  uint64_t step = 0;
  // workspace of one batch
  uint32_t cap = 0;
  unsigned char* ws = nullptr;
  bf16 *X = nullptr, *XT = nullptr, *Z1 = nullptr, *H1 = nullptr, *H1T = nullptr, *Z2 = nullptr, *H2 = nullptr, *H2T = nullptr;
  bf16 *Z3 = nullptr, *H3 = nullptr, *dZ3 = nullptr, *dZ3T = nullptr, *dZ2 = nullptr, *dZ2T = nullptr, *dZ1 = nullptr, *dZ1T = nullptr;
  float *ys = nullptr, *pred = nullptr, *dOut = nullptr, *part = nullptr, *lossPart = nullptr;

  float* W1() const { return p; }
  float* b1() const { return p + kW1; }
  float* W2() const { return p + kW1 + kHid; }
  float* b2() const { return W2() + kW2; }
  float* W3() const { return b2() + kHid; }
  float* b3() const { return W3() + kW3; }
  float* w4() const { return b3() + kHid; }
  float* b4() const { return w4() + kHid; }
  size_t offOf(const float* q) const { return static_cast<size_t>(q - p); }
};

// A trade of a book revalued by the surrogate (mirrors zk_surrogate_trade of the C ABI).
struct SurrogateTrade {
  uint32_t nettingSet, kind, asset;
  int32_t sign;
  float notional, strike, maturity, pad;
};

cudaError_t surrogateCreate(SurrogateState& S, cudaStream_t stream, uint32_t* err, uint32_t seed);
void surrogateFree(SurrogateState& S);
// bf16 copies (row-major and transposed) of the matrices from the fp32 masters.
cudaError_t surrogateSync(SurrogateState& S);
// Standardisation from a host training set: hostScale receives mean[16], 1 / sd[16] (to upload).
void surrogateScaleFrom(SurrogateState& S, const float* x, const float* y, size_t n, float* hostScale);
// One pass over n device rows in batches: forward, loss, gradients, and Adam when `train`; the mean squared
// error (standardised units) into *loss.  With train == false and batch >= n, S.grad holds the gradient.
cudaError_t surrogateEpoch(SurrogateState& S, const float* dx, const float* dy, size_t n, uint32_t batch, float lr, float decay,
                           bool train, double* loss);
// Predictions in original units for n device rows.
cudaError_t surrogatePredict(SurrogateState& S, const float* dx, size_t n, float* dout);

// Features of rows [row0, row0 + n) in (trade, reporting date, path) order into X [n][16].
cudaError_t surrogateFeatures(const float* factors, uint32_t nA, uint32_t nR, uint32_t nP, const float* times,
                              const SurrogateTrade* trades, const int32_t* resets, const float* periods, const float* bonds,
                              uint64_t row0, uint64_t n, float* X, cudaStream_t s);
// Netted values [numNs][nR][nP] (accumulated into `netted`, zeroed by the caller) of a book, chunkTrades trades
// at a time through features, prediction and netting; X and pred hold chunkTrades * nR * nP rows.
cudaError_t surrogateBook(SurrogateState& S, const float* factors, uint32_t nA, uint32_t nR, uint32_t nP, const float* times,
                          const SurrogateTrade* trades, uint32_t nTr, const int32_t* resets, const float* periods, const float* bonds,
                          float* netted, float* X, float* pred, uint32_t chunkTrades);
// The cash CSA of every netting set applied in place: netted[ns][j][p] becomes V - collateral, the collateral called
// on the value at date call[j] <= j (at most 31 dates back); csa[ns] = (hc, ho (< 0: none), mta (< 0: no CSA), ia).
cudaError_t surrogateCollateral(float* netted, const float* csa, const uint32_t* call, uint32_t numNs, uint32_t nR, uint32_t nP,
                                cudaStream_t s);
// out[ns][r] = (EE, EE*) of the netted values with the deflator D [nR][nP].
cudaError_t surrogateExposure(const float* netted, const float* D, uint32_t numNs, uint32_t nR, uint32_t nP, double* out,
                              cudaStream_t s);

}  // namespace zk
