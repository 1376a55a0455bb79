// The learned revaluation surrogate: a 16 -> 128 -> 128 -> 128 -> 1 multilayer perceptron with SiLU
// activations, BF16 weights and activations and FP32 accumulation, trained and evaluated on the GPU by this
// library's own kernels (no counterpart in the reference: its AI chapter fits a small FP64 tanh network to
// XVA adjustments on the CPU, src/ai/surrogate.cpp).
//
// Every product of the forward and backward passes is one tensor-core GEMM of mlp.cu (tcgen05, FP32 in TMEM)
// whose epilogue applies the bias, the SiLU or the SiLU derivative and writes the BF16 activations in the
// layouts the next product reads.  The scalar head (128 -> 1), the loss, the bias gradients and Adam are
// CUDA-core kernels here.  Inputs and targets are standardised with the training set's moments.
#include <algorithm>
#include <cmath>
#include <vector>

#include "surrogate.cuh"
#include "umma.cuh"

namespace zk {

namespace {

// Row pass of the head: pred = h3 . w4 + b4 (standardised units); with targets, dOut = 2 (pred - y) / n and the
// block's sum of squared errors.  Rows >= n are padding and contribute nothing.
__global__ void headKernel(const bf16* __restrict__ H3, const float* __restrict__ w4, const float* __restrict__ b4,
                           const float* __restrict__ y, uint32_t n, float* __restrict__ pred, float* __restrict__ dOut,
                           float* __restrict__ lossPart) {
  __shared__ float red[128];
  const uint32_t r = blockIdx.x * 128 + threadIdx.x;
  const bf16* h = H3 + static_cast<size_t>(r) * kHid;
  float p = 0.0f, l = 0.0f;
  for (uint32_t j = 0; j < kHid; ++j) p += __bfloat162float(h[j]) * w4[j];
  p += b4[0];
  if (pred) pred[r] = p;
  if (dOut) {
    const float d = r < n ? p - y[r] : 0.0f;
    dOut[r] = 2.0f * d / static_cast<float>(n);
    l = d * d;
  }
  if (lossPart) {
    red[threadIdx.x] = l;
    __syncthreads();
    for (uint32_t s = 64; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) lossPart[blockIdx.x] = red[0];
  }
}

// Column pass of the head on a block of 128 rows: the block's partial dw4 and db4, and
// dZ3 = dOut w4 silu'(Z3) row-major and transposed.
__global__ void headBackKernel(const bf16* __restrict__ H3, const bf16* __restrict__ Z3, const float* __restrict__ w4,
                               const float* __restrict__ dOut, uint32_t rows, float* __restrict__ part,
                               bf16* __restrict__ dZ3, bf16* __restrict__ dZ3T) {
  __shared__ float d[128];
  const uint32_t r0 = blockIdx.x * 128, j = threadIdx.x;
  d[j] = dOut[r0 + j];
  __syncthreads();
  float gw = 0.0f, gb = 0.0f;
  for (uint32_t i = 0; i < 128; ++i) {
    const size_t at = static_cast<size_t>(r0 + i) * kHid + j;
    gw += d[i] * __bfloat162float(H3[at]);
    gb += d[i];
    const bf16 v = __float2bfloat16_rn(d[i] * w4[j] * umma::siluGrad(__bfloat162float(Z3[at])));
    dZ3[at] = v;
    dZ3T[static_cast<size_t>(j) * rows + r0 + i] = v;
  }
  part[static_cast<size_t>(blockIdx.x) * (kHid + 1) + j] = gw;
  if (j == 0) part[static_cast<size_t>(blockIdx.x) * (kHid + 1) + kHid] = gb;
}

// out[c] = sum over blocks b of part[b][c], in block order (deterministic).
__global__ void sumRowsKernel(const float* __restrict__ part, uint32_t blocks, uint32_t w, float* __restrict__ out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= w) return;
  float s = 0.0f;
  for (uint32_t b = 0; b < blocks; ++b) s += part[static_cast<size_t>(b) * w + c];
  out[c] = s;
}

// Column sums of a bf16 [rows][128] matrix (the bias gradients), in row order.
__global__ void colSumKernel(const bf16* __restrict__ M, uint32_t rows, float* __restrict__ out) {
  const uint32_t j = threadIdx.x;
  float s = 0.0f;
  for (uint32_t r = 0; r < rows; ++r) s += __bfloat162float(M[static_cast<size_t>(r) * kHid + j]);
  out[j] = s;
}

// Adam on one parameter block [outDim][inDim] (or a vector); refreshes the bf16 copies of matrices.
__global__ void adamKernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g,
                           uint32_t n, uint32_t outDim, uint32_t inDim, float lr, float b1, float b2, float c1, float c2,
                           float eps, float decay, bf16* __restrict__ wb, bf16* __restrict__ wbT) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] + decay * w[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi, v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
  if (wbT) wbT[static_cast<size_t>(i % inDim) * outDim + i / inDim] = __float2bfloat16_rn(wi);
}

__global__ void castKernel(const float* __restrict__ w, uint32_t n, uint32_t outDim, uint32_t inDim, bf16* __restrict__ wb,
                           bf16* __restrict__ wbT) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  wb[i] = __float2bfloat16_rn(w[i]);
  wbT[static_cast<size_t>(i % inDim) * outDim + i / inDim] = __float2bfloat16_rn(w[i]);
}

// Standardised bf16 inputs X [rows][16] (and XT [16][rows]), zero rows past n; standardised targets.
__global__ void prepareKernel(const float* __restrict__ x, const float* __restrict__ y, uint32_t n, uint32_t rows,
                              const float* __restrict__ mean, const float* __restrict__ inv, float yMean, float yInv,
                              bf16* __restrict__ X, bf16* __restrict__ XT, float* __restrict__ ys) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  // A row is 16 floats in (four 16-byte loads) and 16 bf16 out (two 16-byte stores).
  float xv[kIn];
  if (r < n) {
#pragma unroll
    for (int q = 0; q < kIn / 4; ++q) {
      const float4 v = reinterpret_cast<const float4*>(x + static_cast<size_t>(r) * kIn)[q];
      xv[4 * q] = v.x, xv[4 * q + 1] = v.y, xv[4 * q + 2] = v.z, xv[4 * q + 3] = v.w;
    }
  }
  __align__(16) bf16 out[kIn];
#pragma unroll
  for (uint32_t k = 0; k < kIn; ++k) {
    const float v = r < n ? (xv[k] - mean[k]) * inv[k] : 0.0f;
    out[k] = __float2bfloat16_rn(v);
    if (XT) XT[static_cast<size_t>(k) * rows + r] = out[k];
  }
  reinterpret_cast<uint4*>(X + static_cast<size_t>(r) * kIn)[0] = reinterpret_cast<const uint4*>(out)[0];
  reinterpret_cast<uint4*>(X + static_cast<size_t>(r) * kIn)[1] = reinterpret_cast<const uint4*>(out)[1];
  if (ys) ys[r] = r < n ? (y[r] - yMean) * yInv : 0.0f;
}

__global__ void unscaleKernel(const float* __restrict__ pred, uint32_t n, float yMean, float yScale, float* __restrict__ out) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) out[r] = pred[r] * yScale + yMean;
}

uint32_t blocksOf(uint64_t n, uint32_t t) { return static_cast<uint32_t>((n + t - 1) / t); }

#define SG_CUDA(x)                    \
  do {                                \
    cudaError_t e_ = (x);             \
    if (e_ != cudaSuccess) return e_; \
  } while (0)

cudaError_t ensureWorkspace(SurrogateState& S, uint32_t rows) {
  if (rows <= S.cap) return cudaSuccess;
  if (S.ws) cudaFree(S.ws);
  S.ws = nullptr;
  S.cap = 0;
  const size_t r = rows, bh = r * kHid * 2, bi = r * kIn * 2;
  const size_t sizes[] = {bi, bi, bh, bh, bh, bh, bh, bh, bh, bh, bh, bh, bh, bh, bh, bh,
                          r * 4, r * 4, r * 4, (r / 128 + 1) * (kHid + 1) * 4, (r / 128 + 1) * 4};
  constexpr size_t nb = sizeof(sizes) / sizeof(sizes[0]);
  size_t off[nb], total = 0;
  for (size_t i = 0; i < nb; ++i) off[i] = total, total += (sizes[i] + 255) / 256 * 256;
  SG_CUDA(cudaMalloc(&S.ws, total));
  bf16** bp[] = {&S.X, &S.XT, &S.Z1, &S.H1, &S.H1T, &S.Z2, &S.H2, &S.H2T, &S.Z3, &S.H3, &S.dZ3, &S.dZ3T, &S.dZ2, &S.dZ2T, &S.dZ1, &S.dZ1T};
  for (size_t i = 0; i < 16; ++i) *bp[i] = reinterpret_cast<bf16*>(S.ws + off[i]);
  float** fp[] = {&S.ys, &S.pred, &S.dOut, &S.part, &S.lossPart};
  for (size_t i = 0; i < 5; ++i) *fp[i] = reinterpret_cast<float*>(S.ws + off[16 + i]);
  S.cap = rows;
  return cudaSuccess;
}

GemmArgs gemm(const bf16* A, const bf16* B, uint32_t M, uint32_t N, uint32_t K, uint32_t* err) {
  GemmArgs g{};
  g.A = A, g.B = B, g.M = M, g.N = N, g.K = K, g.err = err;
  return g;
}

// Forward pass of `rows` (a multiple of 128) standardised rows in S.X: Z and H of the three hidden layers
// (and the transposed H1, H2 that the weight gradients read, when training).
// headOut (inference): the last layer's epilogue evaluates the linear head into it and H3 is not written.
cudaError_t forward(SurrogateState& S, uint32_t rows, bool training, float* headOut = nullptr) {
  const cudaStream_t s = S.stream;
  GemmArgs g = gemm(S.X, S.wb, rows, kHid, kIn, S.err);
  g.bias = S.b1(), g.act = 1, g.Z = training ? S.Z1 : nullptr, g.H = S.H1, g.HT = training ? S.H1T : nullptr;  // Z: backward only
  SG_CUDA(launchGemm(g, s));
  g = gemm(S.H1, S.wb + SurrogateState::kW1, rows, kHid, kHid, S.err);
  g.bias = S.b2(), g.act = 1, g.Z = training ? S.Z2 : nullptr, g.H = S.H2, g.HT = training ? S.H2T : nullptr;
  SG_CUDA(launchGemm(g, s));
  g = gemm(S.H2, S.wb + SurrogateState::kW1 + SurrogateState::kW2, rows, kHid, kHid, S.err);
  g.bias = S.b3(), g.act = 1, g.Z = training ? S.Z3 : nullptr, g.H = headOut ? nullptr : S.H3;
  if (headOut) g.headW = S.w4(), g.headB = S.b4(), g.headOut = headOut;
  SG_CUDA(launchGemm(g, s));
  return cudaSuccess;
}

// Loss and gradient of the batch (n real rows of `rows`) into S.grad; the squared errors into S.lossPart.
cudaError_t backward(SurrogateState& S, uint32_t n, uint32_t rows) {
  const cudaStream_t s = S.stream;
  const uint32_t blocks = rows / 128;
  headKernel<<<blocks, 128, 0, s>>>(S.H3, S.w4(), S.b4(), S.ys, n, S.pred, S.dOut, S.lossPart);
  headBackKernel<<<blocks, 128, 0, s>>>(S.H3, S.Z3, S.w4(), S.dOut, rows, S.part, S.dZ3, S.dZ3T);
  sumRowsKernel<<<2, 128, 0, s>>>(S.part, blocks, kHid + 1, S.grad + S.offOf(S.w4()));
  // dW3 = dZ3^T H2, db3, dZ2 = (dZ3 W3) silu'(Z2)
  GemmArgs g = gemm(S.dZ3T, S.H2T, kHid, kHid, rows, S.err);
  g.C = S.grad + S.offOf(S.W3());
  SG_CUDA(launchGemm(g, s));
  colSumKernel<<<1, kHid, 0, s>>>(S.dZ3, rows, S.grad + S.offOf(S.b3()));
  g = gemm(S.dZ3, S.wbT + SurrogateState::kW1 + SurrogateState::kW2, rows, kHid, kHid, S.err);
  g.gradOf = S.Z2, g.H = S.dZ2, g.HT = S.dZ2T;
  SG_CUDA(launchGemm(g, s));
  // dW2 = dZ2^T H1, db2, dZ1 = (dZ2 W2) silu'(Z1)
  g = gemm(S.dZ2T, S.H1T, kHid, kHid, rows, S.err);
  g.C = S.grad + S.offOf(S.W2());
  SG_CUDA(launchGemm(g, s));
  colSumKernel<<<1, kHid, 0, s>>>(S.dZ2, rows, S.grad + S.offOf(S.b2()));
  g = gemm(S.dZ2, S.wbT + SurrogateState::kW1, rows, kHid, kHid, S.err);
  g.gradOf = S.Z1, g.H = S.dZ1, g.HT = S.dZ1T;
  SG_CUDA(launchGemm(g, s));
  // dW1 = dZ1^T X, db1
  g = gemm(S.dZ1T, S.XT, kHid, kIn, rows, S.err);
  g.C = S.grad + S.offOf(S.W1());
  SG_CUDA(launchGemm(g, s));
  colSumKernel<<<1, kHid, 0, s>>>(S.dZ1, rows, S.grad + S.offOf(S.b1()));
  return cudaGetLastError();
}

cudaError_t adam(SurrogateState& S, float lr, float decay) {
  ++S.step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, static_cast<float>(S.step)), c2 = 1.0f - std::pow(b2, static_cast<float>(S.step));
  struct Blk {
    float* w;
    uint32_t n, out, in;
    size_t wb;
    bool mat;
  } blks[] = {{S.W1(), SurrogateState::kW1, kHid, kIn, 0, true},
              {S.b1(), kHid, 1, 1, 0, false},
              {S.W2(), SurrogateState::kW2, kHid, kHid, SurrogateState::kW1, true},
              {S.b2(), kHid, 1, 1, 0, false},
              {S.W3(), SurrogateState::kW3, kHid, kHid, SurrogateState::kW1 + SurrogateState::kW2, true},
              {S.b3(), kHid, 1, 1, 0, false},
              {S.w4(), kHid + 1, 1, 1, 0, false}};  // w4 and b4
  for (const auto& b : blks) {
    const size_t o = S.offOf(b.w);
    adamKernel<<<blocksOf(b.n, 256), 256, 0, S.stream>>>(b.w, S.m + o, S.v + o, S.grad + o, b.n, b.out, b.in, lr, b1, b2, c1,
                                                         c2, 1e-8f, b.mat ? decay : 0.0f, b.mat ? S.wb + b.wb : nullptr,
                                                         b.mat ? S.wbT + b.wb : nullptr);
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t surrogateSync(SurrogateState& S) {
  const size_t o2 = SurrogateState::kW1, o3 = SurrogateState::kW1 + SurrogateState::kW2;
  castKernel<<<blocksOf(SurrogateState::kW1, 256), 256, 0, S.stream>>>(S.W1(), SurrogateState::kW1, kHid, kIn, S.wb, S.wbT);
  castKernel<<<blocksOf(SurrogateState::kW2, 256), 256, 0, S.stream>>>(S.W2(), SurrogateState::kW2, kHid, kHid, S.wb + o2,
                                                                        S.wbT + o2);
  castKernel<<<blocksOf(SurrogateState::kW3, 256), 256, 0, S.stream>>>(S.W3(), SurrogateState::kW3, kHid, kHid, S.wb + o3,
                                                                        S.wbT + o3);
  return cudaGetLastError();
}

cudaError_t surrogateCreate(SurrogateState& S, cudaStream_t stream, uint32_t* err, uint32_t seed) {
  S.stream = stream, S.err = err;
  const size_t P = SurrogateState::kParams;
  const size_t wbN = SurrogateState::kW1 + SurrogateState::kW2 + SurrogateState::kW3;
  void* mem = nullptr;
  SG_CUDA(cudaMalloc(&mem, P * 4 * 4 + wbN * 2 * 2 + 32 * 4));
  S.p = static_cast<float*>(mem);
  S.grad = S.p + P, S.m = S.grad + P, S.v = S.m + P;
  S.wb = reinterpret_cast<bf16*>(S.v + P);
  S.wbT = S.wb + wbN;
  S.scale = reinterpret_cast<float*>(S.wbT + wbN);
  // He-uniform initialisation (fan-in) from a seeded 64-bit LCG on the host; zero biases.
  std::vector<float> h(P, 0.0f), sc(32);
  uint64_t st = 0x9E3779B97F4A7C15ull ^ seed;
  auto uni = [&] {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return static_cast<float>((st >> 40) & 0xFFFFFF) / 16777216.0f * 2.0f - 1.0f;
  };
  auto fill = [&](size_t off, size_t n, uint32_t fanIn) {
    const float a = std::sqrt(6.0f / static_cast<float>(fanIn));
    for (size_t i = 0; i < n; ++i) h[off + i] = a * uni();
  };
  fill(0, SurrogateState::kW1, kIn);
  fill(SurrogateState::kW1 + kHid, SurrogateState::kW2, kHid);
  fill(SurrogateState::kW1 + kHid + SurrogateState::kW2 + kHid, SurrogateState::kW3, kHid);
  fill(SurrogateState::kW1 + kHid + SurrogateState::kW2 + kHid + SurrogateState::kW3 + kHid, kHid, kHid);
  for (uint32_t k = 0; k < 16; ++k) sc[k] = 0.0f, sc[16 + k] = 1.0f;
  SG_CUDA(cudaMemcpyAsync(S.p, h.data(), P * 4, cudaMemcpyHostToDevice, stream));
  SG_CUDA(cudaMemsetAsync(S.grad, 0, P * 4 * 3, stream));
  SG_CUDA(cudaMemcpyAsync(S.scale, sc.data(), 32 * 4, cudaMemcpyHostToDevice, stream));
  SG_CUDA(surrogateSync(S));
  return cudaStreamSynchronize(stream);  // the host vectors above go out of scope
}

void surrogateFree(SurrogateState& S) {
  if (S.p) cudaFree(S.p);
  if (S.ws) cudaFree(S.ws);
  S.p = nullptr, S.ws = nullptr, S.cap = 0;
}

void surrogateScaleFrom(SurrogateState& S, const float* x, const float* y, size_t n, float* hostScale) {
  double mu[kIn] = {}, m2[kIn] = {}, ym = 0.0, y2 = 0.0;
  for (size_t i = 0; i < n; ++i) {
    for (uint32_t k = 0; k < kIn; ++k) {
      const double v = x[i * kIn + k];
      mu[k] += v, m2[k] += v * v;
    }
    ym += y[i], y2 += static_cast<double>(y[i]) * y[i];
  }
  const double dn = static_cast<double>(n > 0 ? n : 1);
  for (uint32_t k = 0; k < kIn; ++k) {
    const double mean = mu[k] / dn, var = m2[k] / dn - mean * mean;
    hostScale[k] = static_cast<float>(mean);
    hostScale[16 + k] = var > 1e-24 ? static_cast<float>(1.0 / std::sqrt(var)) : 1.0f;
  }
  S.yMean = static_cast<float>(ym / dn);
  const double yv = y2 / dn - (ym / dn) * (ym / dn);
  S.yScale = yv > 1e-24 ? static_cast<float>(std::sqrt(yv)) : 1.0f;
  S.scaled = true;
}

cudaError_t surrogateEpoch(SurrogateState& S, const float* dx, const float* dy, size_t n, uint32_t batch, float lr, float decay,
                           bool train, double* loss) {
  const uint32_t rowsCap = (batch + 127) / 128 * 128;
  SG_CUDA(ensureWorkspace(S, rowsCap));
  double total = 0.0;
  std::vector<float> lp(rowsCap / 128);
  for (size_t b0 = 0; b0 < n; b0 += batch) {
    const uint32_t nb = static_cast<uint32_t>(std::min<size_t>(batch, n - b0)), rows = (nb + 127) / 128 * 128;
    prepareKernel<<<blocksOf(rows, 128), 128, 0, S.stream>>>(dx + b0 * kIn, dy + b0, nb, rows, S.scale, S.scale + 16, S.yMean,
                                                              1.0f / S.yScale, S.X, S.XT, S.ys);
    SG_CUDA(forward(S, rows, true));
    SG_CUDA(backward(S, nb, rows));
    if (train) SG_CUDA(adam(S, lr, decay));
    SG_CUDA(cudaMemcpyAsync(lp.data(), S.lossPart, rows / 128 * 4, cudaMemcpyDeviceToHost, S.stream));
    SG_CUDA(cudaStreamSynchronize(S.stream));
    for (uint32_t i = 0; i < rows / 128; ++i) total += lp[i];
  }
  if (loss) *loss = total / static_cast<double>(n > 0 ? n : 1);
  return cudaSuccess;
}

// ---- inference: the whole network per 128-row tile in one kernel ----------------------------------------
namespace {

constexpr uint32_t kMlpGroups = 4;                    // warpgroups per CTA, each running its own tiles
constexpr uint32_t kMlpThreads = 128 * kMlpGroups;
constexpr uint32_t kMlpWaitLimit = 1u << 26;          // polls of an MMA-completion barrier before giving up
// Shared memory (canonical K-major tiles, no swizzle): W1 [128 x 16], W2 and W3 [128 x 128] as the B operands,
// shared by the warpgroups; then per warpgroup its tile's inputs [128 x 16] and hidden activations [128 x 128]
// as the A operands; then b1 | b2 | b3 | w4 | b4.
constexpr uint32_t kMlpW1 = 0, kMlpW2 = kMlpW1 + kHid * kIn * 2, kMlpW3 = kMlpW2 + kHid * kHid * 2;
constexpr uint32_t kMlpTiles = kMlpW3 + kHid * kHid * 2, kMlpTileBytes = 128 * kIn * 2 + 128 * kHid * 2;
constexpr uint32_t kMlpParams = kMlpTiles + kMlpGroups * kMlpTileBytes;
constexpr uint32_t kMlpSmem = kMlpParams + (4 * kHid + 4) * 4;

// Copies a row-major [rows][K] bf16 block into the canonical K-major layout, 16 bytes per cp.async, by the
// `threads` threads numbered from 0 by t.
__device__ __forceinline__ void stageKMajor(unsigned char* dst, const bf16* src, uint32_t rows, uint32_t K, uint32_t t,
                                            uint32_t threads) {
  const uint32_t groups = K / 8;
  for (uint32_t v = t; v < rows * groups; v += threads) {
    const uint32_t r = v / groups, kg = v % groups;
    umma::cpAsync16(dst + umma::kMajorOffset(r, kg * 8, rows), src + static_cast<size_t>(r) * K + kg * 8);
  }
}

// Barrier of one warpgroup (named barrier 1 + g, 128 threads), optionally and-reducing a predicate.
__device__ __forceinline__ void groupSync(uint32_t g) { asm volatile("bar.sync %0, 128;" ::"r"(1u + g) : "memory"); }
__device__ __forceinline__ bool groupAnd(bool v, uint32_t g) {
  uint32_t r;
  asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, %2, 128, p;\n selp.u32 %0, 1, 0, q;\n}\n"
               : "=r"(r)
               : "r"(v ? 1u : 0u), "r"(1u + g)
               : "memory");
  return r != 0;
}

// pred[row] for `rows` (a multiple of 128) standardised inputs X [rows][16].  One CTA per SM loads the weights
// once; each of its warpgroups runs tiles (blockIdx.x * 4 + g), stepping by 4 gridDim.x, with its own 128 TMEM
// columns, activation tile and mbarrier, so four tiles' epilogues keep the SM busy.  Per tile, layer l is one
// chain of K/16 MMAs (the same products, in the same order, as the layer-by-layer GEMMs), and its epilogue
// (bias, SiLU, BF16) writes the activations straight into the next layer's A tile in shared memory; the last
// epilogue evaluates the linear head as gemmKernel's fused head does.  The next tile's inputs load while the
// tile's layers run.
__global__ void __launch_bounds__(kMlpThreads, 1) mlpInferKernel(const bf16* __restrict__ X, const bf16* __restrict__ wb,
                                                                 const float* __restrict__ b1, const float* __restrict__ b2,
                                                                 const float* __restrict__ b3, const float* __restrict__ w4,
                                                                 const float* __restrict__ b4, uint32_t rows,
                                                                 float* __restrict__ pred, uint32_t* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t bars[kMlpGroups];
  __shared__ uint32_t tslot;
  const uint32_t tid = threadIdx.x, warp = tid >> 5, g = warp >> 2, gt = tid & 127u;
  const uint32_t tiles = rows / 128, stride = gridDim.x * kMlpGroups;
  unsigned char* xs = sm + kMlpTiles + g * kMlpTileBytes;
  unsigned char* hs = xs + 128 * kIn * 2;
  float* par = reinterpret_cast<float*>(sm + kMlpParams);  // b1 | b2 | b3 | w4 | b4
  uint64_t* bar = &bars[g];
  if (warp == 0) umma::alloc(&tslot, 128 * kMlpGroups);
  if (gt == 0) mbarInit(bar, 1);
  // The hidden layers' biases halved (exactly): the epilogue forms h = z / 2 = acc / 2 + b / 2 in one FMA.
  for (uint32_t k = tid; k < kHid; k += kMlpThreads)
    par[k] = 0.5f * b1[k], par[kHid + k] = 0.5f * b2[k], par[2 * kHid + k] = 0.5f * b3[k], par[3 * kHid + k] = w4[k];
  if (tid == 0) par[4 * kHid] = b4[0];
  stageKMajor(sm + kMlpW1, wb, kHid, kIn, tid, kMlpThreads);
  stageKMajor(sm + kMlpW2, wb + SurrogateState::kW1, kHid, kHid, tid, kMlpThreads);
  stageKMajor(sm + kMlpW3, wb + SurrogateState::kW1 + SurrogateState::kW2, kHid, kHid, tid, kMlpThreads);
  uint32_t t = blockIdx.x * kMlpGroups + g;
  if (t < tiles) stageKMajor(xs, X + static_cast<size_t>(t) * 128 * kIn, 128, kIn, gt, 128);
  umma::cpAsyncCommit();
  umma::cpAsyncWaitAll();  // the weights are read by every warpgroup: all of them land before anyone starts
  umma::fenceAsyncShared();
  umma::fenceBeforeSync();
  __syncthreads();
  umma::fenceAfterSync();
  const uint32_t tmem = tslot + g * 128u, taddr = tmem + (((warp & 3u) * 32u) << 16);
  constexpr uint32_t idesc = umma::idescBf16(128, kHid);
  uint32_t phase = 0;
  bool ok = true, pending = false;
  // One layer: the MMA chain A (K wide) x B into this warpgroup's TMEM columns, then the wait for it.
  auto layer = [&](const unsigned char* a, const unsigned char* b, uint32_t K) {
    if (gt == 0) {
      umma::fenceAfterSync();
      for (uint32_t i = 0; i < K / 16; ++i) {
        const uint64_t da = umma::desc(umma::smem(a) + i * 2 * 128 * 16, 128 * 16, 128);
        const uint64_t db = umma::desc(umma::smem(b) + i * 2 * kHid * 16, kHid * 16, 128);
        umma::mma(tmem, da, db, idesc, i > 0);
      }
      umma::commit(bar);
    }
    const bool done = mbarWait(bar, phase, kMlpWaitLimit);
    ok = groupAnd(done, g);
    pending = !ok;
    phase ^= 1u;
    umma::fenceAfterSync();
  };
  // Epilogue of a hidden layer into the A tile of the next one (or, with the head, into pred).
  auto epilogue = [&](const float* bias, bool head, uint32_t row) {
    float acc = 0.0f;
#pragma unroll 1
    for (uint32_t c = 0; c < kHid; c += 32) {  // 32 columns per TMEM load and wait
      float v[32];
      umma::ld32(taddr + c, v);
      uint32_t hb[16];  // 32 activations as bf16 pairs
#pragma unroll
      for (int j = 0; j < 32; j += 2) {
        hb[j / 2] = umma::siluHalfBf16x2(fmaf(v[j], 0.5f, bias[c + j]), fmaf(v[j + 1], 0.5f, bias[c + j + 1]));
        if (head) {
          acc += __uint_as_float(hb[j / 2] << 16) * par[3 * kHid + c + j];
          acc += __uint_as_float(hb[j / 2] & 0xFFFF0000u) * par[3 * kHid + c + j + 1];
        }
      }
      if (!head) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          *reinterpret_cast<uint4*>(hs + umma::kMajorOffset(gt, c + 8 * q, 128)) =
              make_uint4(hb[4 * q], hb[4 * q + 1], hb[4 * q + 2], hb[4 * q + 3]);
      }
    }
    if (head) pred[row] = acc + par[4 * kHid];
    umma::fenceAsyncShared();  // the activations, written through the generic proxy, for the next MMAs
    umma::fenceBeforeSync();
    groupSync(g);
  };
  for (; t < tiles && ok; t += stride) {
    umma::cpAsyncWaitAll();  // this tile's inputs
    umma::fenceAsyncShared();
    umma::fenceBeforeSync();
    groupSync(g);
    layer(xs, sm + kMlpW1, kIn);
    if (!ok) break;
    // The inputs were consumed: the next tile's load overlaps this tile's layers.
    if (t + stride < tiles) stageKMajor(xs, X + static_cast<size_t>(t + stride) * 128 * kIn, 128, kIn, gt, 128);
    umma::cpAsyncCommit();
    const uint32_t row = t * 128 + gt;  // TMEM lane = thread of the warpgroup = row of the tile
    epilogue(par, false, row);
    layer(hs, sm + kMlpW2, kHid);
    if (!ok) break;
    epilogue(par + kHid, false, row);
    layer(hs, sm + kMlpW3, kHid);
    if (!ok) break;
    epilogue(par + 2 * kHid, true, row);
  }
  umma::cpAsyncWaitAll();
  if (!ok) {
    if (gt == 0) atomicExch(err, kDevTimeout);
    if (pending) mbarWait(bar, phase ^ 1u, kMlpWaitLimit);  // the MMAs in flight, before the TMEM goes away
  }
  umma::fenceBeforeSync();
  __syncthreads();
  if (warp == 0) umma::dealloc(tslot, 128 * kMlpGroups);
}

}  // namespace

cudaError_t surrogatePredict(SurrogateState& S, const float* dx, size_t n, float* dout) {
  const uint32_t chunk = 1u << 18;  // rows per pass: a few hundred passes for a book, a 0.9 GB workspace
  SG_CUDA(ensureWorkspace(S, chunk));
  for (size_t b0 = 0; b0 < n; b0 += chunk) {
    const uint32_t nb = static_cast<uint32_t>(std::min<size_t>(chunk, n - b0)), rows = (nb + 127) / 128 * 128;
    prepareKernel<<<blocksOf(rows, 128), 128, 0, S.stream>>>(dx + b0 * kIn, nullptr, nb, rows, S.scale, S.scale + 16, 0.0f, 1.0f,
                                                              S.X, nullptr, nullptr);
    const uint32_t tiles = rows / 128, grid = std::min<uint32_t>((tiles + kMlpGroups - 1) / kMlpGroups, 148);
    SG_CUDA(cudaFuncSetAttribute(mlpInferKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kMlpSmem)));
    mlpInferKernel<<<grid, kMlpThreads, kMlpSmem, S.stream>>>(S.X, S.wb, S.b1(), S.b2(), S.b3(), S.w4(), S.b4(), rows, S.pred, S.err);
    SG_CUDA(cudaGetLastError());
    unscaleKernel<<<blocksOf(nb, 256), 256, 0, S.stream>>>(S.pred, nb, S.yMean, S.yScale, dout + b0);
  }
  return cudaGetLastError();
}


// ---- revaluation of a book by the surrogate -------------------------------------------------------------
namespace {

// Features of row (trade, reporting date r, path p), rows in [row0, row0 + n) of the trade-major order
// ((trade * nR + r) * nP + p).  factors = [D | x | ln S_0 .. ln S_{nA-1}][nR][nP].
__global__ void featureKernel(const float* __restrict__ factors, uint32_t nA, uint32_t nR, uint32_t nP,
                              const float* __restrict__ times, const SurrogateTrade* __restrict__ trades,
                              const int32_t* __restrict__ resets, const float* __restrict__ periods,
                              const float* __restrict__ bonds, uint64_t row0, uint64_t n, float* __restrict__ X) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t row = row0 + i;
  const uint32_t p = static_cast<uint32_t>(row % nP), r = static_cast<uint32_t>((row / nP) % nR);
  const uint32_t tr = static_cast<uint32_t>(row / (static_cast<uint64_t>(nP) * nR));
  const SurrogateTrade T = trades[tr];
  const size_t plane = static_cast<size_t>(nR) * nP, at = static_cast<size_t>(r) * nP + p;
  const float t = times[r];
  float f[16];
  f[0] = factors[plane + at];                                                   // x
  f[1] = T.kind != 0 && T.asset < nA ? factors[(2 + T.asset) * plane + at] : 0.0f;  // ln S of the trade's factor
  f[2] = t;
  f[3] = fmaxf(T.maturity - t, 0.0f);
  f[4] = T.kind == 0 ? 1.0f : 0.0f, f[5] = T.kind == 1 ? 1.0f : 0.0f, f[6] = T.kind == 2 ? 1.0f : 0.0f;
  f[7] = T.strike;
  f[8] = static_cast<float>(T.sign);
  const size_t tr_r = static_cast<size_t>(tr) * nR + r;
  const int32_t k = resets[tr_r];
  f[9] = k >= 0 ? factors[plane + static_cast<size_t>(k) * nP + p] : 0.0f;  // x at the current period's reset
  const float ts = periods[2 * tr_r], te = periods[2 * tr_r + 1];
  f[10] = k >= 0 ? t - ts : 0.0f;
  f[11] = k >= 0 ? te - t : 0.0f;
  f[12] = te - ts;
  f[13] = static_cast<float>(T.asset);
  f[14] = 0.0f, f[15] = 0.0f;
  if (bonds) {  // P(t, maturity | x) and P(t, end of the running period | x) = exp(ln A - B x)
    const float* q = bonds + 4 * tr_r;
    f[14] = __expf(q[0] - q[1] * f[0]);
    f[15] = __expf(q[2] - q[3] * f[0]);
  }
  float4* dst = reinterpret_cast<float4*>(X + i * kIn);
#pragma unroll
  for (int q = 0; q < 4; ++q) dst[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
}

// netted[ns][r][p] += notional * pred for the trades [tr0, tr1) in trade order (one thread per (r, p)), zero
// past maturity.
__global__ void netKernel(const float* __restrict__ pred, const SurrogateTrade* __restrict__ trades, uint32_t tr0, uint32_t tr1,
                          const float* __restrict__ times, uint32_t nR, uint32_t nP, float* __restrict__ netted) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t plane = static_cast<uint64_t>(nR) * nP;
  if (i >= plane) return;
  const uint32_t r = static_cast<uint32_t>(i / nP);
  for (uint32_t tr = tr0; tr < tr1; ++tr) {
    const SurrogateTrade T = trades[tr];
    if (times[r] >= T.maturity - 1e-6f) continue;
    netted[T.nettingSet * plane + i] += T.notional * pred[static_cast<size_t>(tr - tr0) * plane + i];
  }
}

// The cash CSA of each netting set on its netted values, in place: one thread per (netting set, path) walks the
// dates in order with the collateral rule of the fused kernel (collateral.cpp:10-47): the value at the margin-call
// date call[j] (a look-back of at most kSurrogateRing dates, kept in a ring of the thread's past values), two-way
// thresholds, the minimum transfer amount, the independent amount; netted[ns][j][p] becomes the exposure value
// V - collateral.  csa[ns] = (hc, ho (< 0: none), mta (< 0: no CSA), ia).
constexpr int kSurrogateRing = 32;
__global__ void collateralKernel(float* __restrict__ netted, const float* __restrict__ csa, const uint32_t* __restrict__ call,
                                 uint32_t numNs, uint32_t nR, uint32_t nP) {
  const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<uint64_t>(numNs) * nP) return;
  const uint32_t ns = static_cast<uint32_t>(i / nP), p = static_cast<uint32_t>(i % nP);
  const float hc = csa[4 * ns], ho = csa[4 * ns + 1], mta = csa[4 * ns + 2], ia = csa[4 * ns + 3];
  if (mta < 0.0f) return;
  float* v = netted + static_cast<size_t>(ns) * nR * nP + p;
  float ring[kSurrogateRing];
  float held = 0.0f;
  for (uint32_t j = 0; j < nR; ++j) {
    const float value = v[static_cast<size_t>(j) * nP];
    ring[j % kSurrogateRing] = value;
    const float vc = ring[call[j] % kSurrogateRing];
    float required = 0.0f;
    if (vc > hc) required += vc - hc;
    if (ho >= 0.0f && -vc > ho) required -= -vc - ho;
    if (j == 0 || fabsf(required - held) >= mta) held = required;
    v[static_cast<size_t>(j) * nP] = value - (held + ia);
  }
}

// Per (netting set, date): EE = mean max(V, 0) and EE* = mean D max(V, 0), each thread summing a strided
// share of the paths in double, then a fixed tree.
__global__ void exposureKernel(const float* __restrict__ netted, const float* __restrict__ D, uint32_t nR, uint32_t nP,
                               double* __restrict__ out) {
  __shared__ double a[256], b[256];
  const uint32_t ns = blockIdx.y, r = blockIdx.x;
  const float* v = netted + (static_cast<size_t>(ns) * nR + r) * nP;
  const float* d = D + static_cast<size_t>(r) * nP;
  double ee = 0.0, dee = 0.0;
  for (uint32_t p = threadIdx.x; p < nP; p += 256) {
    const double e = fmax(static_cast<double>(v[p]), 0.0);
    ee += e, dee += static_cast<double>(d[p]) * e;
  }
  a[threadIdx.x] = ee, b[threadIdx.x] = dee;
  __syncthreads();
  for (uint32_t s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) a[threadIdx.x] += a[threadIdx.x + s], b[threadIdx.x] += b[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[(static_cast<size_t>(ns) * nR + r) * 2] = a[0] / nP;
    out[(static_cast<size_t>(ns) * nR + r) * 2 + 1] = b[0] / nP;
  }
}

}  // namespace

cudaError_t surrogateFeatures(const float* factors, uint32_t nA, uint32_t nR, uint32_t nP, const float* times,
                              const SurrogateTrade* trades, const int32_t* resets, const float* periods, const float* bonds,
                              uint64_t row0, uint64_t n, float* X, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  featureKernel<<<static_cast<uint32_t>((n + 255) / 256), 256, 0, s>>>(factors, nA, nR, nP, times, trades, resets, periods, bonds,
                                                                      row0, n, X);
  return cudaGetLastError();
}

cudaError_t surrogateBook(SurrogateState& S, const float* factors, uint32_t nA, uint32_t nR, uint32_t nP, const float* times,
                          const SurrogateTrade* trades, uint32_t nTr, const int32_t* resets, const float* periods, const float* bonds,
                          float* netted, float* X, float* pred, uint32_t chunkTrades) {
  const uint64_t plane = static_cast<uint64_t>(nR) * nP;
  for (uint32_t t0 = 0; t0 < nTr; t0 += chunkTrades) {
    const uint32_t t1 = std::min(nTr, t0 + chunkTrades);
    const uint64_t rows = plane * (t1 - t0);
    SG_CUDA(surrogateFeatures(factors, nA, nR, nP, times, trades, resets, periods, bonds, plane * t0, rows, X, S.stream));
    SG_CUDA(surrogatePredict(S, X, rows, pred));
    netKernel<<<static_cast<uint32_t>((plane + 255) / 256), 256, 0, S.stream>>>(pred, trades, t0, t1, times, nR, nP, netted);
    SG_CUDA(cudaGetLastError());
  }
  return cudaSuccess;
}

cudaError_t surrogateExposure(const float* netted, const float* D, uint32_t numNs, uint32_t nR, uint32_t nP, double* out,
                              cudaStream_t s) {
  exposureKernel<<<dim3(nR, numNs), 256, 0, s>>>(netted, D, nR, nP, out);
  return cudaGetLastError();
}

cudaError_t surrogateCollateral(float* netted, const float* csa, const uint32_t* call, uint32_t numNs, uint32_t nR, uint32_t nP,
                                cudaStream_t s) {
  const uint64_t n = static_cast<uint64_t>(numNs) * nP;
  if (n == 0) return cudaSuccess;
  collateralKernel<<<static_cast<uint32_t>((n + 255) / 256), 256, 0, s>>>(netted, csa, call, numNs, nR, nP);
  return cudaGetLastError();
}

}  // namespace zk
