// The C ABI of zlatko_b200 (include/zlatko_b200.h): plan validation, batching, device memory and
// the launch sequence fused-exposure -> reduce -> row statistics.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <exception>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/zlatko_b200.h"
#include "basis.cuh"
#include "plan_compiler.h"
#include "surrogate.cuh"
#include "zk_kernels.h"

using namespace zk;

namespace zk {
namespace {

// A fixed set of host threads for the per-call parallel loops (validating and lowering a book's plans, filling
// its upload image): spawning and joining a dozen threads for each loop of each call costs about as much as
// the loops.  run(n, fn) calls fn(w) for every w in [0, n) on the pool's threads and the caller's, and returns
// when all are done.  Idle threads sleep on a condition variable.
class HostPool {
 public:
  explicit HostPool(size_t threads) {
    for (size_t t = 0; t < threads; ++t) threads_.emplace_back([this] { loop(); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
    }
    wake_.notify_all();
    for (auto& t : threads_) t.join();
  }
  size_t workers() const { return threads_.size() + 1; }
  void run(size_t n, const std::function<void(size_t)>& fn) {
    if (n <= 1 || threads_.empty()) {
      for (size_t w = 0; w < n; ++w) fn(w);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(m_);
      job_ = &fn, n_ = n, next_ = 0, pending_ = n, ++gen_;
    }
    wake_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  void work() {
    for (;;) {
      const std::function<void(size_t)>* f;
      size_t w;
      {
        std::lock_guard<std::mutex> lk(m_);
        if (!job_ || next_ >= n_) return;
        f = job_, w = next_++;
      }
      (*f)(w);
      std::lock_guard<std::mutex> lk(m_);
      if (--pending_ == 0) done_.notify_all();
    }
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(m_);
        wake_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      work();
    }
  }
  std::vector<std::thread> threads_;
  std::mutex m_;
  std::condition_variable wake_, done_;
  const std::function<void(size_t)>* job_ = nullptr;
  size_t n_ = 0, next_ = 0, pending_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

}  // namespace
}  // namespace zk

struct zk_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  std::string lastError;
  uint32_t* dErr = nullptr;
  void* arena = nullptr;  // reusable device memory of zk_run_plan*
  size_t arenaBytes = 0;
  // Reusable page-locked staging of zk_run_plan*: the host image of a call's inputs and its read-back.  A call
  // ends with the stream synchronised, so the next call may overwrite them.
  unsigned char* stageIn = nullptr;
  size_t stageInBytes = 0;
  unsigned char* stageOut = nullptr;
  size_t stageOutBytes = 0;
  // A second stream for the large-state revalue launch of a split batch, beside the small-state launch on the
  // context's stream (fork and join events order the two); created by the first eager execute that splits.
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // Worker streams of a re-run of chosen paths (the exact-decision check), whose plans are separate small launches
  // that run side by side; created on first need, with one join event each.
  std::vector<cudaStream_t> workers;
  std::vector<cudaEvent_t> workerJoin;
  std::unique_ptr<zk::HostPool> pool;  // created by the first call that validates more than a few plans
  // Device blocks of short-lived work (a nest lives for one reporting date, an AMC fit for one call), reused by
  // later work and freed with the context: freeing device memory synchronises the device and took tens of
  // milliseconds per nest.
  std::vector<std::pair<unsigned char*, size_t>> spareBlocks;
  // Failure injection for tests (zk_debug_inject): the kernel launch, counted from the injection over the
  // context's eager launches, that fails instead of launching (0: none); the row statistics' cap on the
  // quantile's narrowing rounds.
  uint64_t failAtLaunch = 0, launchCount = 0;
  uint32_t rowRounds = 16;
  // Device bytes a batch may give to per-path rows and warp partials at once (zk_context_set_row_budget); 0: all
  // of its netting sets at once while that takes under 70% of the free device memory, else waves in 60% of it.
  uint64_t rowBudget = 0;
  // Which netting sets run on the tensor-core basis kernel (zk_context_set_basis): 0 groups of at least
  // kBasisMinNs eligible netting sets, 1 none, 2 every eligible netting set.
  uint32_t basisMode = 0;
  // Exact decisions (zk_context_set_exact_decisions): the relative guard band (0: off) and the paths the last
  // calls re-ran in double precision out of the paths they ran.
  double exactGuard = 0.0;
  uint64_t exactFlagged = 0, exactPaths = 0;
  // Host wall time of the last zk_run_plans call by phase (zk_context_call_timings): validate and lower the plans
  // (basis groups included), fill and send the inputs, the device run up to its read-back, the exact-decision check
  // and the copy into the caller's buffers; milliseconds.
  double callMs[5] = {0, 0, 0, 0, 0};
  // zk_run_plans simulates the first plan's scenario before it lowers the plans on the host: the cube and the step
  // table it reads, grown as needed.
  void* cube = nullptr;
  size_t cubeBytes = 0;
  void* presimSteps = nullptr;
  size_t presimStepsBytes = 0;
};

namespace {

// The smallest spare block of at least `need` bytes, else a new one; `bytes` receives its size.
unsigned char* takeBlock(zk_context* ctx, size_t need, size_t& bytes) {
  size_t best = ctx->spareBlocks.size();
  for (size_t i = 0; i < ctx->spareBlocks.size(); ++i)
    if (ctx->spareBlocks[i].second >= need && (best == ctx->spareBlocks.size() || ctx->spareBlocks[i].second < ctx->spareBlocks[best].second))
      best = i;
  if (best < ctx->spareBlocks.size()) {
    const auto blk = ctx->spareBlocks[best];
    ctx->spareBlocks.erase(ctx->spareBlocks.begin() + static_cast<std::ptrdiff_t>(best));
    bytes = blk.second;
    return blk.first;
  }
  unsigned char* p = nullptr;
  if (cudaMalloc(reinterpret_cast<void**>(&p), need) != cudaSuccess) return nullptr;
  bytes = need;
  return p;
}

void giveBlock(zk_context* ctx, unsigned char* p, size_t bytes) {
  if (p) ctx->spareBlocks.emplace_back(p, bytes);
}

}  // namespace

namespace {

struct Failure {
  zk_status status;
  std::string message;
};

Failure fail(zk_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return {s, buf};
}

#define ZK_CUDA(call)                                                                        \
  do {                                                                                       \
    const cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                                 \
      if (e_ == cudaErrorMemoryAllocation) throw fail(ZK_ERR_OUT_OF_MEMORY, "%s: %s", #call, cudaGetErrorString(e_)); \
      throw fail(ZK_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));                       \
    }                                                                                        \
  } while (0)

zk_status record(zk_context* ctx, const Failure& f) {
  if (ctx) ctx->lastError = f.message;
  return f.status;
}

template <typename R>
struct View {
  const uint32_t* header;
  size_t header_len;
  const uint32_t* indices;
  size_t indices_len;
  const R* params;
  size_t params_len;
  const R* steps;
  size_t steps_len;
  const R* terms;
  size_t terms_len;
  const R* requests;
  size_t requests_len;
  uint32_t rows_total, num_outputs;
};

View<float> viewOf(const zk_plan_view& v) {
  return {v.header, v.header_len, v.indices, v.indices_len, v.params, v.params_len, v.steps, v.steps_len,
          v.terms, v.terms_len, v.requests, v.requests_len, v.rows_total, v.num_outputs};
}
View<double> viewOf(const zk_plan_view_f64& v) {
  return {v.header, v.header_len, v.indices, v.indices_len, v.params, v.params_len, v.steps, v.steps_len,
          v.terms, v.terms_len, v.requests, v.requests_len, v.rows_total, v.num_outputs};
}

// A plan after validation, with the quantities the launch needs.
template <typename R>
struct Plan {
  View<R> v;
  const uint32_t* H;
  uint32_t nP, nT, nA, nC, sub, nNormals, seed, anti, hasCsa, cpty, nCorr, offCall, offRep, nS, nR, nTr, nBerm;
  uint32_t rowDV, rowE, rowV, rowC, rowGross, rowTrades, rowEx, rowEP;
  size_t nTerms, nReq, nIdx;
  uint32_t nSlots = 0, ring = 1, ctype = 0, stateWords = 0;
  // Nested initial margin: inner paths per outer path and date, the quantile level, the row block; `im` when
  // the plan asks for the margin rows, with the (date, target date) of each reporting slot.
  uint32_t nInner = 0, rowIm = kNoRow;
  float imLevel = 0.0f;
  bool im = false;
  std::vector<uint32_t> imSlots;  // [nR][2]
  bool usesAssets = false, probes = false;
  // Stochastic foreign rates (an extension of the reference's plan): nF of them, one per leading asset; the step
  // rows hold stepStride = 24 + 8 nF values (header word 10 counts them in fours).
  uint32_t nF = 0, stepStride = kStepStride;
  bool usesForeign = false;
  bool amcOrProbe = false;  // some term is an AMC or probe term (the lean revalue variant cannot run the plan)
  // The term table lowered for the revalue kernel (lowerTerms).
  std::vector<uint32_t> dates;  // [nT][8]: floatBegin, bondBegin, assetBegin, genericBegin, fixingBegin, end, callIndex, reportingSlot
  std::vector<R> table;         // records of 4 values
  uint32_t exerciseRows = 0;
  std::vector<uint32_t> bermRows;  // exercise dates of each Bermudan
  bool manyBerm = false;           // more than 4 Bermudans: exercise state in shared memory (one byte per path)
  uint64_t termEvals = 0, expEvals = 0;
  // The exact-decision check: the guard band of each date's decisions (empty: no check) and, for a re-run of
  // chosen paths, the plan path of each of its paths (empty: every path in order).
  std::vector<R> guard;
  std::vector<uint32_t> pathMap;
};

template <typename R>
Plan<R> parse(const View<R>& v, size_t index) {
  Plan<R> p;
  p.v = v;
  auto bad = [&](const char* what) { return fail(ZK_ERR_INVALID_PLAN, "plan %zu: %s", index, what); };
  if (!v.header || v.header_len != static_cast<size_t>(kHeaderWords)) throw bad("malformed plan header (32 words expected)");
  const uint32_t* H = v.header;
  p.H = H;
  p.nP = H[hP], p.nT = H[hT], p.nA = H[hA], p.nC = H[hC], p.sub = H[hSub], p.nNormals = H[hNormals], p.seed = H[hSeed];
  p.anti = H[hAnti], p.hasCsa = H[hCsa], p.cpty = H[hCpty], p.nCorr = H[hCorr], p.offCall = H[hOffCall], p.offRep = H[hOffRep];
  p.nS = H[hS], p.nR = H[hR], p.nTr = H[hTr], p.nBerm = H[hBerm];
  p.rowDV = H[hRowDV], p.rowE = H[hRowE], p.rowV = H[hRowV], p.rowC = H[hRowC], p.rowGross = H[hRowGross];
  p.rowTrades = H[hRowTrades], p.rowEx = H[hRowEx], p.rowEP = H[hRowEP];
  if (p.nP == 0 || p.nT == 0) throw bad("empty plan");
  p.nInner = H[hInner], p.rowIm = H[hRowIm];
  std::memcpy(&p.imLevel, &H[hImLevel], sizeof(float));
  if (!v.params || v.params_len != static_cast<size_t>(kParamCount)) throw bad("params must hold 84 values");
  const uint32_t stepVec = H[hStepVec];
  if (stepVec != 6 && stepVec != 8 && stepVec != 10) throw bad("step rows must hold 24 values (28 or 40 with stochastic foreign rates)");
  p.nF = (stepVec - 6) / 2, p.stepStride = 4 * stepVec;
  if (!v.steps || v.steps_len != static_cast<size_t>(p.nT) * p.stepStride) throw bad("steps must hold nT * (step row) values");
  if (p.nA > kMaxAssets) throw fail(ZK_ERR_UNSUPPORTED, "plan %zu: at most 4 assets", index);
  if (p.nC > kMaxCredits) throw fail(ZK_ERR_UNSUPPORTED, "plan %zu: at most 2 credits", index);
  if (p.nF > p.nA) throw bad("more stochastic foreign rates than assets");
  if (p.nCorr != 1 + p.nA + p.nC + p.nF || p.nCorr > kChol)
    throw bad("number of correlated factors must be 1 + assets + credits + foreign rates");
  if (p.sub == 0) throw bad("CIR sub-steps must be positive");
  if (p.nNormals > kMaxNormals || p.nNormals < p.nCorr + 1 + p.nF + p.nC * (p.sub - 1)) throw bad("inconsistent number of normals per step");
  if (p.nF > 0 && p.nInner > 0) throw fail(ZK_ERR_UNSUPPORTED, "plan %zu: the nested initial margin with stochastic foreign rates", index);
  if (p.nC > 0 && p.cpty >= p.nC) throw bad("counterparty index out of range");
  if (p.offCall != p.nT + 1 || p.offRep != 2 * p.nT + 1) throw bad("index table offsets do not match the reference layout");
  if (!v.indices || v.indices_len < 3 * static_cast<size_t>(p.nT) + 1) throw bad("index table too short");
  if (v.terms_len % kTermStride) throw bad("term table length is not a multiple of 8");
  if (v.requests_len % kRequestStride) throw bad("request table length is not a multiple of 8");
  if (p.nS < kStatsPerDate) throw bad("statsPerDate below 8");
  p.nTerms = v.terms_len / kTermStride;
  p.nReq = v.requests_len / kRequestStride;
  p.nIdx = v.indices_len;
  if (p.nTerms > 0 && !v.terms) throw bad("null term table");
  if (p.nReq > 0 && !v.requests) throw bad("null request table");
  const uint32_t* I = v.indices;
  for (uint32_t j = 0; j < p.nT; ++j)
    if (I[j] > I[j + 1]) throw bad("term starts must not decrease");
  if (I[p.nT] > p.nTerms) throw bad("term starts beyond the term table");
  if (p.nInner > 0) {
    // The reference's inner Monte Carlo (fused_reference.cpp:356-393): targets after their date, at most
    // kMaxInnerPaths inner paths, a quantile level in [0, 1].
    if (p.nInner > static_cast<uint32_t>(kMaxInnerPaths)) throw bad("more than 1024 inner paths");
    if (!(p.imLevel >= 0.0f && p.imLevel <= 1.0f)) throw bad("initial-margin quantile level outside [0, 1]");
    if (v.indices_len < 4 * static_cast<size_t>(p.nT) + 1) throw bad("index table too short for the initial-margin targets");
    for (uint32_t j = 0; j < p.nT; ++j) {
      const uint32_t t = I[p.offRep + p.nT + j];
      if (t != kNoRow && (t <= j || t >= p.nT)) throw bad("initial-margin target date not after its date");
    }
  }
  const uint32_t rows = v.rows_total;
  uint32_t maxLag = 0, maxSlot = 0;
  bool anySlot = false;
  for (uint32_t j = 0; j < p.nT; ++j) {
    const uint32_t c = I[p.offCall + j];
    if (c > j) throw bad("margin call date after the valuation date");
    maxLag = std::max(maxLag, j - c);
    if (I[p.offRep + j] > p.nR) throw bad("reporting slot beyond the reporting dates");
  }
  auto rowBlock = [&](uint32_t base, uint64_t n, const char* what) {
    if (base != kNoRow && static_cast<uint64_t>(base) + n > rows) throw bad(what);
  };
  rowBlock(p.rowEP, p.nR, "exposure rows beyond rows_total");
  rowBlock(p.rowDV, p.nR, "margin rows beyond rows_total");
  rowBlock(p.rowE, p.nR, "exposure-value rows beyond rows_total");
  rowBlock(p.rowV, p.nR, "netted rows beyond rows_total");
  rowBlock(p.rowC, p.nR, "collateral rows beyond rows_total");
  rowBlock(p.rowGross, p.nR, "gross rows beyond rows_total");
  rowBlock(p.rowTrades, static_cast<uint64_t>(std::min<uint32_t>(p.nTr, kMaxTradeGroups)) * p.nR, "trade rows beyond rows_total");
  if (p.nBerm > static_cast<uint32_t>(kMaxBermudansPerPlan)) throw fail(ZK_ERR_UNSUPPORTED, "plan %zu: more than 256 Bermudans", index);
  p.manyBerm = p.nBerm > static_cast<uint32_t>(kMaxBermudans);
  if (p.manyBerm && p.nInner > 0) throw fail(ZK_ERR_UNSUPPORTED, "plan %zu: the nested initial margin of more than 4 Bermudans", index);
  if (p.manyBerm && p.nTr > 0 && p.nBerm > 16) throw fail(ZK_ERR_UNSUPPORTED, "plan %zu: per-trade views of more than 16 Bermudans", index);
  p.bermRows.assign(p.nBerm, 0u);
  rowBlock(p.rowEx, p.nBerm, "exercise rows beyond rows_total");
  if (p.nInner > 0) rowBlock(p.rowIm, p.nR, "initial-margin rows beyond rows_total");
  if (p.rowEP == kNoRow) throw bad("the exposure rows are required");
  for (size_t t = 0; t < p.nTerms; ++t) {
    const R* rec = v.terms + t * kTermStride;
    if (!(rec[0] >= R(0)) || rec[0] >= R(4294967296.0)) throw bad("invalid term code");
    const uint32_t code = static_cast<uint32_t>(rec[0]), kind = code & 15u;
    if (kind > kBermExt) throw bad("unknown term kind");
    if (kind == kForeignForward || kind == kForeignOption) {  // rec[1] is B_f; the asset sits in the code's extra field
      if ((code >> 12u) >= p.nF) throw bad("a foreign-rate term on an asset without a stochastic foreign rate");
      if (!(rec[1] >= R(0))) throw bad("invalid foreign bond coefficient");
      p.usesAssets = p.usesForeign = true;
      continue;
    }
    // rec[1] is an index (swap slot, asset, probe selector) except for continuation terms, where it holds
    // the Bermudan's position.
    if (kind != kBermContinue && kind != kBermExt && (!(rec[1] >= R(0)) || rec[1] >= R(4294967296.0))) throw bad("invalid term slot");
    const uint32_t slot = kind == kBermContinue ? 0u : static_cast<uint32_t>(rec[1]);
    if (kind == kAsset || kind == kOption) p.usesAssets = true;
    if ((kind > kOption && kind <= kProbe) || kind >= kBermAnnuity) p.amcOrProbe = true;
    if (kind == kProbe) {
      const uint32_t what = slot & 15u;
      if (what == 2 || what == 6) p.usesAssets = true;
      if (what == 3 || what == 4) p.probes = true;
    }
    if (kind == kFixedFloat || kind == kSetFixing || (kind > kProbe && kind < kBermAnnuity) || kind == kBermFloat) {
      if (slot >= static_cast<uint32_t>(kMaxSwapSlots)) throw bad("swap slot beyond 32");
      maxSlot = std::max(maxSlot, slot);
      anySlot = true;
    }
    if (kind == kProbe) {
      if (!(rec[5] >= R(0)) || static_cast<double>(rec[5]) >= static_cast<double>(rows)) throw bad("probe row beyond rows_total");
    }
    if ((kind >= kBermExercise && kind <= kBermFloat) || kind >= kBermAnnuity) {
      const uint32_t bm = bermudanOf(code, p.manyBerm), extra = code >> 12u;
      if (bm >= p.nBerm) throw bad("an AMC term of a Bermudan beyond the plan's count");
      if (kind == kBermDecide) {
        if (extra >= 64u) throw bad("exercise index beyond 64");
        p.bermRows[bm] = std::max(p.bermRows[bm], extra + 1);
      }
    }
  }
  for (uint32_t b = 0; b < p.nBerm; ++b) p.exerciseRows += p.bermRows[b];
  // The two-regressor basis: a policy or continuation record followed by exactly two extension records of its
  // date, and extension records nowhere else (the kernel reads them with the record).
  for (uint32_t j = 0; j < p.nT; ++j)
    for (uint32_t t = I[j]; t < I[j + 1]; ++t) {
      const auto kindAt = [&](uint32_t u) { return static_cast<uint32_t>(v.terms[static_cast<size_t>(u) * kTermStride]) & 15u; };
      const uint32_t kind = kindAt(t);
      if (kind == kBermExt) throw bad("a regression extension record without its policy or continuation record");
      if ((kind == kBermDecide || kind == kBermContinue) && t + 1 < I[j + 1] && kindAt(t + 1) == kBermExt) {
        if (t + 2 >= I[j + 1] || kindAt(t + 2) != kBermExt || (t + 3 < I[j + 1] && kindAt(t + 3) == kBermExt))
          throw bad("a two-regressor record needs exactly two extension records");
        t += 2;
      }
    }
  for (uint32_t j = 0; j < p.nT; ++j) {
    for (uint32_t t = I[j]; t < I[j + 1]; ++t) {
      const uint32_t kind = static_cast<uint32_t>(v.terms[static_cast<size_t>(t) * kTermStride]) & 15u;
      p.termEvals += 1;
      if (kind != kAsset && kind != kBermDecide && kind != kBermContinue) p.expEvals += kind == kForeignOption ? 2 : 1;
    }
  }
  for (size_t q = 0; q < p.nReq; ++q) {
    const R* rq = v.requests + q * kRequestStride;
    const uint32_t op = static_cast<uint32_t>(rq[0]), row = static_cast<uint32_t>(rq[1]), row2 = static_cast<uint32_t>(rq[2]);
    const uint64_t count = static_cast<uint64_t>(rq[3]), out = static_cast<uint64_t>(rq[7]);
    if (op > 9) throw bad("unknown row-statistics operation");
    if (row >= rows) throw bad("request row beyond rows_total");
    if ((op == 6 || op == 8 || op == 9) && row2 >= rows) throw bad("request row2 beyond rows_total");
    const uint64_t width = op == 4 ? count : op == 5 ? count + 2 : 1;
    if (op == 5 && (count == 0 || count > 3072)) throw bad("histogram bins must be 1..3072");
    if (out + width > std::max<uint32_t>(1, v.num_outputs)) throw bad("request output beyond numOutputs");
  }
  p.nSlots = anySlot ? maxSlot + 1 : 0;
  p.ctype = p.hasCsa ? static_cast<uint32_t>(v.params[16 + kChol * kChol]) : 0u;
  if (p.ctype > 2) throw bad("unknown collateral type");
  p.ring = maxLag + 1;
  if (p.hasCsa && p.ring > static_cast<uint32_t>(kMaxRing))
    throw fail(ZK_ERR_UNSUPPORTED, "plan %zu: the margin-call look-back spans %u dates (at most %d)", index, maxLag, kMaxRing - 1);
  if (p.ctype == 2) p.usesAssets = true;
  p.stateWords = p.nSlots + (p.hasCsa ? p.ring * (p.ctype != 0 ? 2 : 1) : 0) + (p.manyBerm ? (p.nBerm + 3) / 4 : 0);
  p.im = p.nInner > 0 && p.rowIm != kNoRow;
  if (p.im) {
    // The full revalue variant records the outer state on the reporting dates; the inner paths start from it
    // and from ln S in the factor cube.
    p.probes = true;
    p.amcOrProbe = true;
    p.imSlots.assign(2 * static_cast<size_t>(p.nR), kNoRow);
    for (uint32_t j = 0; j < p.nT; ++j) {
      const uint32_t rs = I[p.offRep + j];
      if (rs > 0) p.imSlots[2 * (rs - 1)] = j, p.imSlots[2 * (rs - 1) + 1] = I[p.offRep + p.nT + j];
    }
  }
  lowerTerms(p);
  return p;
}

// Lowers a validated plan's term table for the revalue kernel into typed runs of 4-value records, one
// contiguous block per date, in the order [floating coupons | bond pairs | asset forwards | generic | fixings]:
//   floating coupon (kFixedFloat):  (c A, p1 A, b, slot)         value += (c A fix[slot] + p1 A) E(b x)
//   two bonds (kBond):               (c A, b, c' A', b')          value += c A E(b x) + c' A' E(b' x)
//   asset forward (kAsset):          (c, A, asset, 0)             value += c S[asset] A
//   generic (any other kind):        the reference's 8-word record in two 4-value records
//   fixing (kSetFixing):             (A, b, 1 / c, slot)          fix[slot] = (A E(b x) - 1) / c
// with b = -B log2 e and E = 2^ in single precision, b = -B and E = exp in double.  Fixings stay last, so a
// running coupon still reads the previous fixing on its fixing date (the reference's merge order).  In
// per-trade mode every term keeps its trade group in the generic run.  The date descriptor also carries
// the margin-call index and the reporting slot: the kernel reads one 32-byte record per date.
template <typename R>
void lowerTerms(Plan<R>& p) {
  const uint32_t* I = p.v.indices;
  const bool typed = p.nTr == 0;
  const double bScale = sizeof(R) == 4 ? 1.4426950408889634 : 1.0;
  p.dates.assign(static_cast<size_t>(p.nT) * 8, 0u);
  p.table.clear();
  auto units = [&] { return static_cast<uint32_t>(p.table.size() / 4); };
  auto push4 = [&](double a, double b, double c, double d) {
    p.table.push_back(static_cast<R>(a)), p.table.push_back(static_cast<R>(b));
    p.table.push_back(static_cast<R>(c)), p.table.push_back(static_cast<R>(d));
  };
  for (uint32_t j = 0; j < p.nT; ++j) {
    uint32_t* d = &p.dates[static_cast<size_t>(j) * 8];
    const R* first = p.v.terms + static_cast<size_t>(I[j]) * kTermStride;
    const R* last = p.v.terms + static_cast<size_t>(I[j + 1]) * kTermStride;
    auto isFloat = [&](const R* r) { return typed && r[0] == R(kFixedFloat); };
    auto isBond = [&](const R* r) { return typed && r[0] == R(kBond); };
    auto isFixing = [&](const R* r) { return typed && r[0] == R(kSetFixing); };
    auto isAsset = [&](const R* r) { return typed && r[0] == R(kAsset); };
    d[0] = units();
    for (const R* r = first; r < last; r += kTermStride)
      if (isFloat(r)) {
        const double A = r[3];
        push4(static_cast<double>(r[2]) * A, static_cast<double>(r[5]) * A, -static_cast<double>(r[4]) * bScale, r[1]);
      }
    d[1] = units();
    double pending[2] = {0, 0};
    bool half = false;
    for (const R* r = first; r < last; r += kTermStride)
      if (isBond(r)) {
        const double cA = static_cast<double>(r[2]) * static_cast<double>(r[3]), b = -static_cast<double>(r[4]) * bScale;
        if (!half) pending[0] = cA, pending[1] = b, half = true;
        else push4(pending[0], pending[1], cA, b), half = false;
      }
    if (half) push4(pending[0], pending[1], 0.0, 0.0);  // the odd bond with a zero partner
    d[2] = units();
    for (const R* r = first; r < last; r += kTermStride)
      if (isAsset(r)) push4(r[2], r[3], r[1], 0.0);
    d[3] = units();
    // Generic records in plan order.  A run of two or more Bermudan bonds (kBermBond) of one Bermudan and trade group
    // becomes a block: a header record (the run's code with extra 0, -count, the largest exercise index) and two
    // bonds (c, A, B, exercise index) per record; the kernel skips the block in a warp none of whose paths has
    // exercised that Bermudan by then, and otherwise adds each bond as the record would.
    auto bermBond = [&](const R* r) { return (static_cast<uint32_t>(r[0]) & 15u) == static_cast<uint32_t>(kBermBond); };
    for (const R* r = first; r < last;) {
      if (isFloat(r) || isBond(r) || isFixing(r) || isAsset(r)) {
        r += kTermStride;
        continue;
      }
      const uint32_t low = static_cast<uint32_t>(r[0]) & 0xFFFu;
      const R* e = r;
      if (bermBond(r))
        while (e < last && bermBond(e) && (static_cast<uint32_t>(e[0]) & 0xFFFu) == low) e += kTermStride;
      const size_t n = static_cast<size_t>(e - r) / kTermStride;
      if (n < 2) {
        p.table.insert(p.table.end(), r, r + kTermStride);
        r += kTermStride;
        continue;
      }
      double maxEx = 0.0;
      for (const R* q = r; q < e; q += kTermStride) maxEx = std::max(maxEx, static_cast<double>(static_cast<uint32_t>(q[0]) >> 12u));
      push4(static_cast<double>(low), -static_cast<double>(n), maxEx, 0.0);
      push4(0.0, 0.0, 0.0, 0.0);
      for (size_t q = 0; q < n; ++q) {
        const R* b = r + q * kTermStride;
        p.table.push_back(b[2]), p.table.push_back(b[3]), p.table.push_back(b[4]);
        p.table.push_back(static_cast<R>(static_cast<uint32_t>(b[0]) >> 12u));
      }
      if (n % 2) push4(0.0, 0.0, 0.0, -1.0);
      r = e;
    }
    d[4] = units();
    for (const R* r = first; r < last; r += kTermStride)
      if (isFixing(r)) push4(r[3], -static_cast<double>(r[4]) * bScale, 1.0 / static_cast<double>(r[2]), r[1]);
    d[5] = units();
    d[6] = I[p.offCall + j];
    d[7] = I[p.offRep + j];
  }
  if (p.table.empty()) p.table.assign(4, R(0));
}

// The guard band of the exact-decision check on each date: rel times a bound on the gross value of the netting
// set's terms, |value| summed term by term with each term's largest factor taken at its deterministic part (bonds at
// A, coupons at a fixing of 10%, asset terms at the largest spot, options at their forward's bond, a regression at
// |z| = 3).  The single-precision value of a path differs from the double-precision one by a few units of rounding
// of that gross sum (the terms' exponentials, the simulated factors, the sum), so a decision whose margin in single
// precision lies outside the band is taken the same way in double precision.  A margin call compares the value of
// the call date with the collateral held, itself set from an earlier call: the band of a date adds the gross sums
// of the date and of its call date.
template <typename R>
std::vector<R> decisionGuard(const Plan<R>& P, double rel) {
  const uint32_t* I = P.v.indices;
  double spot = 1.0;
  for (uint32_t a = 0; a < std::min<uint32_t>(P.nA, 4); ++a) spot = std::max(spot, std::fabs(static_cast<double>(P.v.params[12 + a])));
  std::vector<double> gross(P.nT, 0.0);
  for (uint32_t j = 0; j < P.nT; ++j) {
    double g = 0.0;
    for (uint32_t t = I[j]; t < I[j + 1]; ++t) {
      const R* r = P.v.terms + static_cast<size_t>(t) * kTermStride;
      const uint32_t kind = static_cast<uint32_t>(r[0]) & 15u;
      const double c = std::fabs(static_cast<double>(r[2])), a = std::fabs(static_cast<double>(r[3]));
      auto poly = [&](const R* q, int from, int n) {
        double v = 0.0, w = 1.0;
        for (int k = 0; k < n; ++k, w *= 3.0) v += std::fabs(static_cast<double>(q[from + k])) * w;
        return v;
      };
      switch (kind) {
        case kBond: case kBermExercise: case kBermBond: g += c * a; break;
        case kFixedFloat: case kBermFloat: g += (c * 0.1 + std::fabs(static_cast<double>(r[5]))) * a; break;
        case kAsset: case kForeignForward: g += c * spot * a; break;
        case kOption: case kForeignOption: g += c * spot * std::fabs(static_cast<double>(r[5])); break;
        case kBermDecide: g += poly(r, 4, 4); break;
        case kBermContinue: g += std::fabs(static_cast<double>(r[1])) * poly(r, 4, 4); break;
        default: break;
      }
    }
    gross[j] = g;
  }
  std::vector<R> out(P.nT);
  for (uint32_t j = 0; j < P.nT; ++j) {
    const uint32_t cj = std::min(I[P.offCall + j], P.nT - 1);
    out[j] = static_cast<R>(rel * (gross[j] + gross[cj]));
  }
  return out;
}

// Plans share a scenario when every input of the risk-factor simulation is identical.
template <typename R>
bool sameScenario(const Plan<R>& a, const Plan<R>& b) {
  if (a.nP != b.nP || a.nT != b.nT || a.nA != b.nA || a.nC != b.nC || a.sub != b.sub || a.nNormals != b.nNormals ||
      a.seed != b.seed || a.anti != b.anti || a.nCorr != b.nCorr || a.nF != b.nF)
    return false;
  if (std::memcmp(a.v.params, b.v.params, 8 * sizeof(R)) || std::memcmp(a.v.params + 12, b.v.params + 12, (4 + 64) * sizeof(R)))
    return false;
  for (uint32_t j = 0; j < a.nT; ++j) {
    const R* ra = a.v.steps + static_cast<size_t>(j) * a.stepStride;
    const R* rb = b.v.steps + static_cast<size_t>(j) * b.stepStride;
    if (std::memcmp(ra, rb, 22 * sizeof(R)) || std::memcmp(ra + kStepStride, rb + kStepStride, (a.stepStride - kStepStride) * sizeof(R)))
      return false;
  }
  return true;
}

size_t alignUp(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

uint32_t numTilesOf(uint32_t nP, int ppt) {
  const uint32_t tp = static_cast<uint32_t>(kTile * ppt);
  return (nP + tp - 1) / tp;
}

// A set of plans laid out in one device arena, ready to execute.
template <typename R>
struct Batch {
  zk_context* ctx = nullptr;
  std::vector<Plan<R>> plans;
  struct Launch {
    ScenarioArgs<R> sc;
    CubeArgs<R> cb;
    std::vector<uint32_t> planIdx;
    uint32_t numFields = 0;
    size_t stateWordsMax = 0;
    // Netting sets in decreasing order of shared-memory state: [splitAt, n) keep at most kSmallStateWords words
    // per path (at most smallStateMax) and may run as a second launch with more resident CTAs.
    size_t splitAt = 0, smallStateMax = 0;
    // Every netting set of [0, splitAt) (cashBig), of [splitAt, n) (cashSmall), of the launch (cashAll) has a cash
    // CSA with a margin-call look-back of at most one date and none of the optional value / collateral rows.
    bool cashBig = true, cashSmall = true, cashAll = true;
    bool perTrade = false, probes = false, lean = true;
    size_t nsOff = 0, cubeOff = 0;  // device offsets of NsArgs[] and the factor cube
    R* presim = nullptr;            // the cube, simulated ahead in the context's cube buffer (not in the arena)
    // Memory-bounded batches: the launch's netting sets [first, first + count) of planIdx run as one wave whose
    // rows and partials reuse the same device region as every other wave; its reduce and row-statistics jobs are
    // [reduceFirst, + count) and [rowFirst, + rowCount) of the job arrays.
    struct Wave {
      size_t first = 0, count = 0, reduceFirst = 0, rowFirst = 0, rowCount = 0;
    };
    std::vector<Wave> waves;
    // Single precision: planIdx[0, basisCount) run on basisRevalueKernel in groups of at most 128 netting sets
    // (planIdx[first, first + count) each, its tables and arguments in the input region); the rest on
    // revalueKernel, in decreasing order of shared-memory state.
    struct Group {
      size_t first = 0, count = 0;
      BasisImage img;
      size_t dates = 0, kgs = 0, options = 0, fixings = 0, chunks = 0, blob = 0, scale = 0;
    };
    size_t basisCount = 0, groupArgs = 0;  // groupArgs: index of the first group's BasisArgs in the batch's array
    uint32_t descBytes = 0, fixSlots = 0;  // the basis kernel's shared memory: the largest over the groups
    std::vector<Group> groups;
  };
  std::vector<Launch> launches;
  // device offsets per plan
  struct Dev {
    size_t dates, table, steps, req, expo, partials, sums, values;
    size_t imSlots = 0, imModel = 0, imState = 0;  // nested initial margin: slots [nR][2], spots + Cholesky, outer state
    size_t guard = 0, flags = 0, pathMap = 0;      // the exact-decision check; a re-run's path map (0: none)
  };
  std::vector<Dev> dev;
  size_t reduceOff = 0, rowOff = 0, normalsOff = 0, sinkOff[3] = {0, 0, 0}, bermRowOff = 0;
  size_t basisArgsOff = 0, numGroups = 0;  // BasisArgs of every launch's groups
  std::vector<uint8_t> onBasis;          // per plan: runs on the basis kernel (its partials cover 64 paths each)
  size_t inputBytes = 0, totalBytes = 0, outBegin = 0, outBytes = 0;
  uint32_t numRowJobs = 0, maxReduceN = 0;
  int ppt = 2;                        // paths per revalue thread: the tile shape (autotuned by zk_batch_create)
  bool waved = false;                 // the netting sets run in waves (Launch::waves) within a row budget
  std::vector<uint32_t> jobOrder;     // plans in the order of the reduce and row-statistics job arrays
  std::vector<ReduceJob<R>> reduceJobs;  // host copy; numTiles follows ppt
  std::vector<ImArgs<R>> im;             // nested initial margin launches, after the revalue launches
  std::vector<unsigned char> image;  // host image of the input region
  unsigned char* base = nullptr;     // device arena
  bool ownsArena = false;
  bool sink = false;
  bool exact = false;                // the exact-decision check: guard bands and flags (Dev::guard, Dev::flags)
  size_t flagsOff = 0, flagsBytes = 0;
  uint32_t exerciseRows = 0;
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  float ms[4] = {0, 0, 0, 0};
  bool timed = false;

  size_t spareBytes = 0;              // the arena is a spare block of the context (upload with spare), returned here
  ~Batch() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (ownsArena && base) cudaFree(base);
    if (spareBytes && base) {  // nothing in flight may still use the block when the next work takes it
      cudaStreamSynchronize(ctx->stream);
      for (auto w : ctx->workers) cudaStreamSynchronize(w);
      ctx->spareBlocks.emplace_back(base, spareBytes);
    }
  }
};


// Validates and lowers the plans, on several host threads for a book of many plans; the first failure in plan
// order is the one reported.
// The context's host threads, created on first need (a call with several plans); null without a context.
HostPool* hostPool(zk_context* ctx, size_t plans) {
  if (!ctx || plans < 8) return ctx ? ctx->pool.get() : nullptr;
  if (!ctx->pool) {
    const size_t hw = std::max<size_t>(1, std::thread::hardware_concurrency());
    ctx->pool = std::make_unique<HostPool>(std::min<size_t>(hw, 16) - 1);
  }
  return ctx->pool.get();
}

template <typename R>
void parseAll(const std::vector<View<R>>& views, std::vector<Plan<R>>& plans, HostPool* pool) {
  const size_t n = views.size();
  plans.assign(n, Plan<R>());
  const size_t workers = n >= 8 && pool ? std::min<size_t>(pool->workers(), n / 4) : 1;
  std::vector<std::exception_ptr> errs(n);
  auto work = [&](size_t w) {
    for (size_t i = w; i < n; i += workers) {
      try {
        plans[i] = parse(views[i], i);
      } catch (...) {
        errs[i] = std::current_exception();
      }
    }
  };
  if (workers == 1) {
    work(0);
  } else {
    pool->run(workers, work);
  }
  for (const auto& e : errs)
    if (e) std::rethrow_exception(e);
}

// Netting sets in a group of fewer run faster term by term (the group's epilogue warps work on 128 lanes).
constexpr size_t kBasisMinNs = 24;

// A plan the basis kernel runs: single precision, the netting set's 8 statistics, the exposure rows only, no AMC,
// probes, per-trade views or nested margin, and no CSA or a cash CSA with a look-back of at most one date (term
// kinds are checked by buildBasis).
template <typename R>
bool basisEligible(const Plan<R>& P) {
  return sizeof(R) == 4 && P.nTr == 0 && !P.amcOrProbe && !P.im && P.nBerm == 0 && P.nS == static_cast<uint32_t>(kStatsPerDate) &&
         P.rowGross == kNoRow && P.rowTrades == kNoRow && P.rowDV == kNoRow && P.rowE == kNoRow && P.rowV == kNoRow &&
         P.rowC == kNoRow && (!P.hasCsa || (P.ctype == 0 && P.ring <= 2)) && P.nC <= 2 && P.nF <= 2;
}

// Reorders a launch's plans into [basis groups | the rest]: eligible netting sets with the same margin-call and
// reporting dates, in near-equal groups of at most 128 (mode 0: of at least kBasisMinNs), each lowered by
// buildBasis on the context's host threads; a group that does not lower joins the rest.
template <typename R>
void formGroups(Batch<R>& B, typename Batch<R>::Launch& L, uint32_t mode, HostPool* pool) {
  if constexpr (sizeof(R) == 4) {
    if (mode == 1 || B.sink) return;
    std::vector<uint32_t> E, O;
    for (uint32_t k : L.planIdx) (basisEligible(B.plans[k]) ? E : O).push_back(k);
    if (E.empty()) return;
    auto tables = [&](uint32_t k) {
      const auto& P = B.plans[k];
      return std::vector<uint32_t>(P.v.indices + P.offCall, P.v.indices + P.offCall + 2 * static_cast<size_t>(P.nT));
    };
    std::vector<std::vector<uint32_t>> key(B.plans.size());
    for (uint32_t k : E) key[k] = tables(k);
    std::stable_sort(E.begin(), E.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
    ParallelFor par = nullptr;
    if (pool && pool->workers() > 1)
      par = [pool](size_t n, const std::function<void(size_t)>& fn) {
        const size_t w = std::min(pool->workers(), n);
        pool->run(w, [&](size_t t) {
          for (size_t i = t; i < n; i += w) fn(i);
        });
      };
    std::vector<uint32_t> ordered;
    for (size_t i = 0; i < E.size();) {
      size_t e = i + 1;
      while (e < E.size() && key[E[e]] == key[E[i]]) ++e;
      const size_t run = e - i, parts = (run + kBasisRows - 1) / kBasisRows;
      for (size_t q = 0; q < parts; ++q) {
        const size_t a = i + run * q / parts, b = i + run * (q + 1) / parts;
        typename Batch<R>::Launch::Group G;
        std::string why;
        bool ok = mode == 2 || b - a >= kBasisMinNs;
        if (ok) {
          std::vector<BasisPlanIn> in;
          for (size_t k = a; k < b; ++k) {
            const auto& P = B.plans[E[k]];
            in.push_back({P.v.terms, P.v.indices, P.nT, static_cast<uint32_t>(P.nTerms), P.offCall, P.offRep});
          }
          ok = buildBasis(in, G.img, why, par);
        }
        if (!ok) {
          O.insert(O.end(), E.begin() + a, E.begin() + b);
          continue;
        }
        G.first = ordered.size(), G.count = b - a;
        ordered.insert(ordered.end(), E.begin() + a, E.begin() + b);
        L.groups.push_back(std::move(G));
      }
      i = e;
    }
    L.basisCount = ordered.size();
    for (const auto& G : L.groups)
      L.descBytes = std::max(L.descBytes, G.img.descBytes), L.fixSlots = std::max(L.fixSlots, G.img.numFixSlots);
    for (size_t k = 0; k < L.basisCount; ++k) B.onBasis[ordered[k]] = 1;
    ordered.insert(ordered.end(), O.begin(), O.end());
    L.planIdx = std::move(ordered);
  }
}

// The simulation arguments of a launch whose first plan is P0 (probes: the launch's plans read ln S and the CIR
// states); returns the cube's number of fields.
template <typename R>
uint32_t scenarioOf(const Plan<R>& P0, bool probes, size_t streams, ScenarioArgs<R>& sc, CubeArgs<R>& cb) {
  sc.nP = P0.nP, sc.nT = P0.nT, sc.nA = P0.nA, sc.nC = P0.nC, sc.substeps = P0.sub, sc.nNormals = P0.nNormals;
  sc.nCorr = P0.nCorr, sc.seed = P0.seed, sc.antithetic = P0.anti, sc.nStreams = static_cast<uint32_t>(streams);
  sc.nF = P0.nF, sc.stepStride = P0.stepStride;
  sc.steps = nullptr, sc.normals = nullptr, sc.pathMap = nullptr;
  for (int k = 0; k < 8; ++k) sc.cir[k] = P0.v.params[k];
  for (int k = 0; k < 4; ++k) sc.spots[k] = P0.v.params[12 + k];
  for (int k = 0; k < 64; ++k) sc.chol[k] = P0.v.params[16 + k];
  cb.data = nullptr;
  cb.nP = P0.nP, cb.nT = P0.nT, cb.nA = P0.nA, cb.nC = P0.nC;
  cb.fS = 2, cb.fQ = 2 + P0.nA, cb.fXf = 2 + P0.nA + P0.nC, cb.nF = P0.nF;
  cb.fLnS = cb.fXf + P0.nF, cb.fY = cb.fLnS + P0.nA;
  cb.probes = probes ? 1u : 0u;
  cb.pad = 0;
  return (probes ? 2 + 2 * P0.nA + 2 * P0.nC : 2 + P0.nA + P0.nC) + P0.nF;
}

// A simulation launched ahead of the batch's host work (zk_run_plans): the factor cube of the first plan's scenario,
// in the context's cube buffer, with or without the probe fields.
struct Presim {
  float* cube = nullptr;
  bool probes = false;
};

// Options of a batch beyond its plans: the exact-decision check (guard bands and flags; term-by-term revaluation),
// or the re-run of chosen paths (maps[i]: the paths of plan i, its header's path count their number; every plan its
// own launch; term by term).
struct BuildOpts {
  bool exact = false;
  const std::vector<std::vector<uint32_t>>* maps = nullptr;
  const Presim* presim = nullptr;  // the first plan's scenario already simulated (single precision, counter normals)
};

// parsed: the plans already validated and lowered (their views' tables stay the caller's), else parsed from views.
template <typename R>
std::unique_ptr<Batch<R>> build(zk_context* ctx, std::vector<View<R>> views, bool sink, const double* normals, size_t streams,
                                const BuildOpts& opts = BuildOpts(), std::vector<Plan<R>>* parsed = nullptr) {
  auto B = std::make_unique<Batch<R>>();
  B->ctx = ctx;
  B->sink = sink;
  if (parsed) B->plans = std::move(*parsed);
  else parseAll(views, B->plans, hostPool(ctx, views.size()));
  const size_t nPlans = B->plans.size();
  if (opts.maps) {
    for (size_t i = 0; i < nPlans; ++i) {
      const auto& m = (*opts.maps)[i];
      if (m.size() != B->plans[i].nP) throw fail(ZK_ERR_INVALID_ARGUMENT, "plan %zu: a path map of %zu paths for %u", i, m.size(), B->plans[i].nP);
      B->plans[i].pathMap = m;
    }
  }
  B->exact = opts.exact;
  if (opts.exact)
    for (auto& P : B->plans)
      if (!P.im) P.guard = decisionGuard(P, ctx->exactGuard);
  // ---- launch groups: plans sharing the scenario (a re-run of chosen paths: every plan alone) ----
  std::vector<int> launchOf(nPlans, -1);
  for (size_t i = 0; i < nPlans; ++i) {
    if (launchOf[i] >= 0) continue;
    typename Batch<R>::Launch L;
    for (size_t k = i; k < nPlans; ++k)
      if (launchOf[k] < 0 && (k == i || (!opts.maps && sameScenario(B->plans[i], B->plans[k])))) {
        launchOf[k] = static_cast<int>(B->launches.size());
        L.planIdx.push_back(static_cast<uint32_t>(k));
      }
    B->launches.push_back(std::move(L));
  }
  if (normals && B->launches.size() != 1) throw fail(ZK_ERR_INVALID_ARGUMENT, "injected normals need plans of one scenario");
  // ---- per launch: the factor cube shared by its netting sets, one CTA column per netting set ----
  B->onBasis.assign(nPlans, 0);
  for (auto& L : B->launches) {
    formGroups(*B, L, ctx && !opts.exact && !opts.maps ? ctx->basisMode : 1u, hostPool(ctx, views.size()));
    const size_t nb = L.basisCount;
    std::stable_sort(L.planIdx.begin() + static_cast<std::ptrdiff_t>(nb), L.planIdx.end(),
                     [&](uint32_t a, uint32_t b) { return B->plans[a].stateWords > B->plans[b].stateWords; });
    L.splitAt = L.planIdx.size();
    while (L.splitAt > nb && B->plans[L.planIdx[L.splitAt - 1]].stateWords <= static_cast<uint32_t>(kSmallStateWords)) --L.splitAt;
    if (L.splitAt < L.planIdx.size()) L.smallStateMax = B->plans[L.planIdx[L.splitAt]].stateWords;
    for (size_t k = nb; k < L.planIdx.size(); ++k) {
      const auto& P = B->plans[L.planIdx[k]];
      const bool cash = P.hasCsa && P.ctype == 0 && P.ring <= 2 && P.rowDV == kNoRow && P.rowE == kNoRow && P.rowV == kNoRow &&
                        P.rowC == kNoRow;
      (k < L.splitAt ? L.cashBig : L.cashSmall) = (k < L.splitAt ? L.cashBig : L.cashSmall) && cash;
      L.cashAll = L.cashAll && cash;
    }
    for (size_t q = 0; q < L.planIdx.size(); ++q) {
      const auto& P = B->plans[L.planIdx[q]];
      L.probes = L.probes || P.probes;
      if (q < nb) continue;  // the rest: the term-by-term kernel's variant and shared memory
      L.stateWordsMax = std::max<size_t>(L.stateWordsMax, P.stateWords);
      L.perTrade = L.perTrade || P.nTr > 0;
      L.probes = L.probes || P.probes;
      // Lean kernels know nS and write no gross or per-trade rows.
      L.lean = L.lean && !P.amcOrProbe && P.nS == static_cast<uint32_t>(kStatsPerDate) && P.rowGross == kNoRow &&
               P.rowTrades == kNoRow;
    }
    const Plan<R>& P0 = B->plans[L.planIdx.front()];
    L.numFields = scenarioOf(P0, L.probes, streams, L.sc, L.cb);
    if constexpr (sizeof(R) == 4)  // the launch of plan 0 finds its cube simulated when the probe fields agree
      if (opts.presim && !sink && !normals && !opts.maps && opts.presim->probes == L.probes &&
          std::find(L.planIdx.begin(), L.planIdx.end(), 0u) != L.planIdx.end())
        L.presim = opts.presim->cube;
    if (revalueSmemBytes(L.stateWordsMax, L.perTrade, sizeof(R) == 8, 1) > 200 * 1024)
      throw fail(ZK_ERR_UNSUPPORTED, "a netting set needs more shared memory than a CTA has");
  }
  if (normals) {
    const Plan<R>& P0 = B->plans[0];
    const size_t need = P0.anti ? (P0.nP + 1) / 2 : P0.nP;
    if (streams < need) throw fail(ZK_ERR_INVALID_ARGUMENT, "injected normals: %zu streams for %zu needed", streams, need);
  }
  // ---- arena layout: inputs first (one upload), then device-only scratch, outputs last ----
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off = alignUp(off + std::max<size_t>(bytes, 16)); return o; };
  B->dev.resize(nPlans);
  for (size_t i = 0; i < nPlans; ++i) {
    const auto& P = B->plans[i];
    auto& D = B->dev[i];
    D.dates = take(P.dates.size() * 4);
    D.table = take(P.table.size() * sizeof(R));
    D.steps = take(static_cast<size_t>(P.nT) * P.stepStride * sizeof(R));
    D.req = take(P.nReq * kRequestStride * sizeof(R));
    if (P.im) {
      D.imSlots = take(P.imSlots.size() * 4);
      D.imModel = take((4 + kChol * kChol) * sizeof(R));
    }
    if (!P.guard.empty()) D.guard = take(P.guard.size() * sizeof(R));
    if (!P.pathMap.empty()) D.pathMap = take(P.pathMap.size() * 4);
  }
  for (auto& L : B->launches) L.nsOff = take(L.planIdx.size() * sizeof(NsArgs<R>));
  for (auto& L : B->launches) {
    L.groupArgs = B->numGroups;
    B->numGroups += L.groups.size();
    for (auto& G : L.groups) {
      G.dates = take(G.img.dates.size() * 4);
      G.kgs = take(G.img.kgs.size() * sizeof(BasisKg));
      G.options = take(G.img.options.size() * 4);
      G.fixings = take(G.img.fixings.size() * 4);
      G.chunks = take(G.img.chunks.size() * 4);
      G.blob = take(G.img.blob.size() * 2);
      G.scale = take(G.img.scale.size() * 4);
    }
  }
  B->basisArgsOff = take(B->numGroups * sizeof(BasisArgs));
  B->reduceOff = take(nPlans * sizeof(ReduceJob<R>));
  for (const auto& P : B->plans) B->numRowJobs += static_cast<uint32_t>(P.nReq);
  B->rowOff = take(B->numRowJobs * sizeof(RowJob<R>));
  if (sink) {
    const auto& P = B->plans[0];
    B->exerciseRows = P.exerciseRows;
    B->bermRowOff = take(std::max<uint32_t>(P.nBerm, 1) * 4);
  }
  if (normals) {
    const auto& P = B->plans[0];
    B->normalsOff = take(static_cast<size_t>(P.nT - 1) * P.nNormals * streams * sizeof(R));
  }
  B->inputBytes = off;
  for (auto& L : B->launches)
    if (!L.presim) L.cubeOff = take(static_cast<size_t>(L.numFields) * L.sc.nT * L.sc.nP * sizeof(R));
  // Rows and warp partials: one region per plan, or -- when they exceed the row budget -- waves of netting sets
  // (in each launch's order) that reuse one region, sized by the largest wave.
  auto rowsBytes = [&](const Plan<R>& P) {
    const uint32_t warps = (P.nP + 31) / 32;  // the most revalue warps any tile shape uses: one partial each
    return alignUp(static_cast<size_t>(std::max<uint32_t>(P.v.rows_total, 1)) * P.nP * sizeof(R)) +
           alignUp(static_cast<size_t>(warps) * P.nT * P.nS * sizeof(R));
  };
  size_t allRows = 0;
  bool anyIm = false;
  for (const auto& P : B->plans) allRows += rowsBytes(P), anyIm = anyIm || P.im;
  uint64_t budget = ctx ? ctx->rowBudget : 0;
  if (ctx && budget == 0) {
    size_t freeB = 0, totalB = 0;
    if (cudaMemGetInfo(&freeB, &totalB) == cudaSuccess && allRows > freeB / 10 * 7) budget = freeB / 10 * 6;
    else cudaGetLastError();
  }
  B->waved = budget > 0 && allRows > budget && !sink && !anyIm && !normals;
  auto placeRows = [&](size_t i, auto&& takeFn) {
    const auto& P = B->plans[i];
    const uint32_t warps = (P.nP + 31) / 32;
    B->dev[i].expo = takeFn(static_cast<size_t>(std::max<uint32_t>(P.v.rows_total, 1)) * P.nP * sizeof(R));
    B->dev[i].partials = takeFn(static_cast<size_t>(warps) * P.nT * P.nS * sizeof(R));
  };
  if (!B->waved) {
    for (size_t i = 0; i < nPlans; ++i) {
      const auto& P = B->plans[i];
      placeRows(i, take);
      if (P.im && !sink) B->dev[i].imState = take(static_cast<size_t>(P.nR) * (5 + P.nSlots) * P.nP * sizeof(R));
    }
    B->jobOrder.resize(nPlans);
    for (size_t i = 0; i < nPlans; ++i) B->jobOrder[i] = static_cast<uint32_t>(i);
  } else {
    const size_t region = off;
    size_t regionBytes = 0, jobs = 0, rowJobs = 0;
    for (auto& L : B->launches) {
      size_t k = 0;
      size_t gi = 0;  // the next basis group: a group runs in one wave
      while (k < L.planIdx.size()) {
        typename Batch<R>::Launch::Wave w;
        w.first = k, w.reduceFirst = jobs, w.rowFirst = rowJobs;
        size_t used = 0;
        while (k < L.planIdx.size()) {
          const size_t end = k < L.basisCount ? L.groups[gi].first + L.groups[gi].count : k + 1;
          size_t unitBytes = 0;
          for (size_t q = k; q < end; ++q) unitBytes += rowsBytes(B->plans[L.planIdx[q]]);
          if (k != w.first && used + unitBytes > budget) break;
          for (; k < end; ++k) {
            const uint32_t i = L.planIdx[k];
            size_t at = region + used;
            placeRows(i, [&](size_t bytes) { const size_t o = at; at = alignUp(at + std::max<size_t>(bytes, 16)); return o; });
            used += rowsBytes(B->plans[i]);
            B->jobOrder.push_back(i);
            w.rowCount += B->plans[i].nReq, ++jobs;
          }
          if (end <= L.basisCount) ++gi;
        }
        w.count = k - w.first;
        rowJobs += w.rowCount;
        regionBytes = std::max(regionBytes, used);
        L.waves.push_back(w);
      }
    }
    off = alignUp(region + regionBytes);
  }
  if (sink) {
    const auto& P = B->plans[0];
    B->sinkOff[0] = take(static_cast<size_t>(P.nT) * P.nP * sizeof(R));
    B->sinkOff[1] = take(static_cast<size_t>(P.nT) * P.nP * sizeof(R));
    B->sinkOff[2] = take(static_cast<size_t>(std::max<uint32_t>(P.exerciseRows, 1)) * P.nP * sizeof(R));
  }
  // The exact-decision check's flags: a bit per path of every checked plan, cleared by each execute.
  if (opts.exact) {
    B->flagsOff = off;
    for (size_t i = 0; i < nPlans; ++i)
      if (!B->plans[i].guard.empty()) B->dev[i].flags = take(static_cast<size_t>((B->plans[i].nP + 31) / 32) * 4);
    B->flagsBytes = off - B->flagsOff;
  }
  B->outBegin = off;
  for (size_t i = 0; i < nPlans; ++i) {
    const auto& P = B->plans[i];
    B->dev[i].sums = take(static_cast<size_t>(P.nT) * P.nS * sizeof(R));
    B->dev[i].values = take(static_cast<size_t>(std::max<uint32_t>(P.v.num_outputs, 1)) * sizeof(R));
  }
  B->outBytes = off - B->outBegin;
  B->totalBytes = off;
  return B;
}

// Fills the host image of the input region, once the arena base is known.
// img: the host image to fill (B.inputBytes), B.image when null.
template <typename R>
void fillImage(Batch<R>& B, const double* normals, size_t streams, unsigned char* img = nullptr) {
  B.im.clear();
  if (!img) {
    B.image.resize(B.inputBytes);
    img = B.image.data();
  }
  // A book's tables are megabytes: the image is cleared and filled on the context's host threads.
  HostPool* pool = B.ctx ? B.ctx->pool.get() : nullptr;
  const size_t workers = pool ? std::min<size_t>(pool->workers(), std::max<size_t>(1, B.inputBytes >> 19)) : 1;
  auto onThreads = [&](size_t n, const std::function<void(size_t)>& fn) {
    if (pool) {
      pool->run(n, fn);
    } else {
      for (size_t w = 0; w < n; ++w) fn(w);
    }
  };
  onThreads(workers, [&](size_t w) {
    const size_t a = B.inputBytes * w / workers, b = B.inputBytes * (w + 1) / workers;
    std::memset(img + a, 0, b - a);
  });
  const uintptr_t base = reinterpret_cast<uintptr_t>(B.base);
  auto dptr = [&](size_t o) { return reinterpret_cast<void*>(base + o); };
  onThreads(std::min(workers, B.plans.size()), [&](size_t w) {
    for (size_t i = w; i < B.plans.size(); i += std::min(workers, B.plans.size())) {
      const auto& P = B.plans[i];
      const auto& D = B.dev[i];
      std::memcpy(img + D.dates, P.dates.data(), P.dates.size() * 4);
      std::memcpy(img + D.table, P.table.data(), P.table.size() * sizeof(R));
      std::memcpy(img + D.steps, P.v.steps, static_cast<size_t>(P.nT) * P.stepStride * sizeof(R));
      if (P.nReq) std::memcpy(img + D.req, P.v.requests, P.nReq * kRequestStride * sizeof(R));
      if (P.im) {
        std::memcpy(img + D.imSlots, P.imSlots.data(), P.imSlots.size() * 4);
        std::memcpy(img + D.imModel, P.v.params + 12, (4 + kChol * kChol) * sizeof(R));
      }
      if (!P.guard.empty()) std::memcpy(img + D.guard, P.guard.data(), P.guard.size() * sizeof(R));
      if (!P.pathMap.empty()) std::memcpy(img + D.pathMap, P.pathMap.data(), P.pathMap.size() * 4);
    }
  });
  for (auto& L : B.launches) {
    std::vector<NsArgs<R>> args(L.planIdx.size());
    for (size_t k = 0; k < L.planIdx.size(); ++k) {
      const auto& P = B.plans[L.planIdx[k]];
      const auto& D = B.dev[L.planIdx[k]];
      NsArgs<R>& A = args[k];
      std::memset(&A, 0, sizeof A);
      A.dates = static_cast<const uint32_t*>(dptr(D.dates));
      A.table = static_cast<const R*>(dptr(D.table));
      A.steps = static_cast<const R*>(dptr(D.steps));
      A.expo = static_cast<R*>(dptr(D.expo));
      A.partials = static_cast<R*>(dptr(D.partials));
      const R* prm = P.v.params;
      A.hc = prm[8], A.hb = prm[9], A.mta = prm[10], A.ia = prm[11];
      A.keepHaircut = R(1) - prm[16 + kChol * kChol + 2];
      A.hasCsa = P.hasCsa, A.ctype = P.ctype, A.casset = static_cast<uint32_t>(prm[16 + kChol * kChol + 1]);
      A.cpty = P.nC > 0 ? P.cpty : 0xFFFFFFFFu;
      A.nS = P.nS, A.nTr = P.nTr, A.nBerm = P.nBerm, A.nR = P.nR;
      A.rowEP = P.rowEP, A.rowDV = P.rowDV, A.rowE = P.rowE, A.rowV = P.rowV, A.rowC = P.rowC, A.rowGross = P.rowGross;
      A.rowTrades = P.rowTrades, A.rowEx = P.rowEx;
      A.offCall = P.offCall, A.offRep = P.offRep, A.nSlots = P.nSlots, A.ring = P.ring;
      A.usesAssets = P.usesAssets ? 1u : 0u;
      A.usesForeign = P.usesForeign ? 1u : 0u;
      A.stepStride = P.stepStride;
      A.manyBerm = P.manyBerm ? 1u : 0u;
      if (!P.guard.empty()) {
        A.flags = static_cast<uint32_t*>(dptr(D.flags));
        A.guard = static_cast<const R*>(dptr(D.guard));
      }
      if (P.im && !B.sink) {
        A.imState = static_cast<R*>(dptr(D.imState));
        A.imWords = 5 + P.nSlots;
        ImArgs<R> M{};
        M.cube = L.presim ? L.presim : static_cast<const R*>(dptr(L.cubeOff));
        M.dates = A.dates, M.table = A.table, M.steps = A.steps;
        M.model = static_cast<const R*>(dptr(D.imModel));
        M.slots = static_cast<const uint32_t*>(dptr(D.imSlots));
        M.state = A.imState, M.expo = A.expo;
        M.nP = P.nP, M.nT = P.nT, M.nA = P.nA, M.fLnS = L.cb.fLnS, M.nR = P.nR, M.nSlots = P.nSlots, M.nInner = P.nInner;
        M.rowIm = P.rowIm, M.seed = P.seed, M.anti = P.anti, M.nCorr = P.nCorr, M.level = static_cast<R>(P.imLevel);
        B.im.push_back(M);
      }
      if (B.sink) {
        A.sinkX = static_cast<R*>(dptr(B.sinkOff[0]));
        A.sinkD = static_cast<R*>(dptr(B.sinkOff[1]));
        A.sinkEx = static_cast<R*>(dptr(B.sinkOff[2]));
        A.sinkRowOfBermudan = static_cast<const uint32_t*>(dptr(B.bermRowOff));
      }
    }
    std::memcpy(img + L.nsOff, args.data(), args.size() * sizeof(NsArgs<R>));
    if constexpr (sizeof(R) == 4) {
      for (size_t q = 0; q < L.groups.size(); ++q) {
        const auto& G = L.groups[q];
        const BasisImage& I = G.img;
        std::memcpy(img + G.dates, I.dates.data(), I.dates.size() * 4);
        std::memcpy(img + G.kgs, I.kgs.data(), I.kgs.size() * sizeof(BasisKg));
        if (!I.options.empty()) std::memcpy(img + G.options, I.options.data(), I.options.size() * 4);
        if (!I.fixings.empty()) std::memcpy(img + G.fixings, I.fixings.data(), I.fixings.size() * 4);
        if (!I.chunks.empty()) std::memcpy(img + G.chunks, I.chunks.data(), I.chunks.size() * 4);
        if (!I.blob.empty()) std::memcpy(img + G.blob, I.blob.data(), I.blob.size() * 2);
        std::memcpy(img + G.scale, I.scale.data(), I.scale.size() * 4);
        BasisArgs a{};
        a.cube = L.presim ? reinterpret_cast<const float*>(L.presim) : static_cast<const float*>(dptr(L.cubeOff));
        a.nP = L.sc.nP, a.nT = L.sc.nT, a.nA = L.cb.nA, a.nC = L.cb.nC, a.nF = L.cb.nF;
        a.fS = L.cb.fS, a.fQ = L.cb.fQ, a.fXf = L.cb.fXf;
        a.dates = static_cast<const uint32_t*>(dptr(G.dates));
        a.kgs = static_cast<const BasisKg*>(dptr(G.kgs));
        a.options = static_cast<const float*>(dptr(G.options));
        a.fixings = static_cast<const float4*>(dptr(G.fixings));
        a.chunks = static_cast<const uint32_t*>(dptr(G.chunks));
        a.blob = static_cast<const unsigned char*>(dptr(G.blob));
        a.scale = static_cast<const float*>(dptr(G.scale));
        a.ns = reinterpret_cast<const NsArgs<float>*>(dptr(L.nsOff)) + G.first;
        a.numNs = static_cast<uint32_t>(G.count), a.numFixSlots = I.numFixSlots, a.numChunks = I.numChunks;
        std::memcpy(img + B.basisArgsOff + (L.groupArgs + q) * sizeof(BasisArgs), &a, sizeof a);
      }
    }
    const auto& P0 = B.plans[L.planIdx.front()];
    L.sc.steps = static_cast<const R*>(dptr(B.dev[L.planIdx.front()].steps));
    L.sc.normals = normals ? static_cast<const R*>(dptr(B.normalsOff)) : nullptr;
    L.sc.pathMap = P0.pathMap.empty() ? nullptr : static_cast<const uint32_t*>(dptr(B.dev[L.planIdx.front()].pathMap));
    L.cb.data = L.presim ? L.presim : static_cast<R*>(dptr(L.cubeOff));
    (void)P0;
  }
  std::vector<ReduceJob<R>> red(B.plans.size());
  std::vector<RowJob<R>> rows;
  rows.reserve(B.numRowJobs);
  B.maxReduceN = 0;
  for (size_t o = 0; o < B.plans.size(); ++o) {
    const size_t i = B.jobOrder[o];  // plan order, or wave by wave when the batch runs in waves
    const auto& P = B.plans[i];
    const auto& D = B.dev[i];
    // pad: 2 for a basis plan (a partial per 64 paths), 0 for the batch's tile shape
    red[o] = {static_cast<const R*>(dptr(D.partials)), static_cast<R*>(dptr(D.sums)), P.nT * P.nS, numTilesOf(P.nP, 1), P.nP,
              B.onBasis[i] ? 2u : 0u};
    B.maxReduceN = std::max(B.maxReduceN, P.nT * P.nS);
    for (size_t q = 0; q < P.nReq; ++q)
      rows.push_back({static_cast<const R*>(dptr(D.expo)), static_cast<const R*>(dptr(D.req + q * kRequestStride * sizeof(R))),
                      static_cast<R*>(dptr(D.values)), P.nP, 0});
  }
  std::memcpy(img + B.reduceOff, red.data(), red.size() * sizeof(ReduceJob<R>));
  B.reduceJobs = red;
  if (!rows.empty()) std::memcpy(img + B.rowOff, rows.data(), rows.size() * sizeof(RowJob<R>));
  if (B.sink) {
    std::vector<uint32_t> offs(std::max<uint32_t>(B.plans[0].nBerm, 1), 0u);
    uint32_t acc = 0;
    for (uint32_t b = 0; b < B.plans[0].nBerm; ++b) offs[b] = acc, acc += B.plans[0].bermRows[b];
    std::memcpy(img + B.bermRowOff, offs.data(), offs.size() * 4);
  }
  if (normals) {
    const auto& P = B.plans[0];
    const size_t n = static_cast<size_t>(P.nT - 1) * P.nNormals * streams;
    R* dst = reinterpret_cast<R*>(img + B.normalsOff);
    for (size_t k = 0; k < n; ++k) dst[k] = static_cast<R>(normals[k]);
  }
}

void growStage(unsigned char*& stage, size_t& bytes, size_t need) {
  if (bytes >= need) return;
  if (stage) cudaFreeHost(stage);
  stage = nullptr, bytes = 0;
  ZK_CUDA(cudaMallocHost(reinterpret_cast<void**>(&stage), std::max<size_t>(need, 1)));
  bytes = need;
}

// The arena: the context's (useCtxArena), a spare block of the context (spare: short-lived batches), or its own.
template <typename R>
void upload(Batch<R>& B, zk_context* ctx, bool useCtxArena, const double* normals, size_t streams, bool spare = false) {
  if (!useCtxArena && spare) {
    size_t bytes = 0;
    B.base = takeBlock(ctx, B.totalBytes, bytes);
    if (!B.base) throw fail(ZK_ERR_OUT_OF_MEMORY, "%zu bytes of device memory", B.totalBytes);
    B.spareBytes = bytes;
  } else if (useCtxArena) {
    if (ctx->arenaBytes < B.totalBytes) {
      if (ctx->arena) cudaFree(ctx->arena);
      ctx->arena = nullptr;
      ctx->arenaBytes = 0;
      ZK_CUDA(cudaMalloc(&ctx->arena, B.totalBytes));
      ctx->arenaBytes = B.totalBytes;
    }
    B.base = static_cast<unsigned char*>(ctx->arena);
  } else {
    void* p = nullptr;
    ZK_CUDA(cudaMalloc(&p, B.totalBytes));
    B.base = static_cast<unsigned char*>(p);
    B.ownsArena = true;
  }
  if (useCtxArena) {
    // Calls on the context arena synchronise before they return, so the context's page-locked staging is free;
    // the waits below cover a previous call that failed with its copy, or a forked launch, in flight.
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->side) ZK_CUDA(cudaStreamSynchronize(ctx->side));
    growStage(ctx->stageIn, ctx->stageInBytes, B.inputBytes);
    fillImage(B, normals, streams, ctx->stageIn);
    ZK_CUDA(cudaMemcpyAsync(B.base, ctx->stageIn, B.inputBytes, cudaMemcpyHostToDevice, ctx->stream));
  } else {
    fillImage(B, normals, streams);
    ZK_CUDA(cudaMemcpyAsync(B.base, B.image.data(), B.inputBytes, cudaMemcpyHostToDevice, ctx->stream));
  }
}

// A point where zk_debug_inject may make a launch fail: the host-side failure of a kernel launch, which leaves
// the kernels launched before it in flight and the context usable.
void injectPoint(zk_context* ctx) {
  if (!ctx || ctx->failAtLaunch == 0) return;
  if (++ctx->launchCount < ctx->failAtLaunch) return;
  const unsigned long long k = ctx->launchCount;
  ctx->failAtLaunch = 0, ctx->launchCount = 0;
  throw fail(ZK_ERR_CUDA, "injected failure of kernel launch %llu", k);
}

// The revalue launches of one launch group on stream s.  Lean single-precision launches of 2 or 4 paths per
// thread run the netting sets with little state as their own launch, compiled for more resident CTAs than the
// shared memory of the largest allows.  The few large-state netting sets fill less than a wave of long CTAs:
// with a side stream (and its fork / join events) they run there while the small-state launch fills the rest
// of the GPU; without one, before it on s.  Either way the kernels and their output bits are the same.
// first / count select a wave of the launch's netting sets (all of them by default).
template <typename R>
void launchRevalues(const Batch<R>& B, const typename Batch<R>::Launch& L, uintptr_t base, cudaStream_t s, cudaStream_t side,
                    cudaEvent_t forkEv, cudaEvent_t joinEv, size_t first = 0, size_t count = SIZE_MAX) {
  count = std::min(count, L.planIdx.size() - first);
  if constexpr (sizeof(R) == 4) {
    // the basis groups of [first, first + count) (whole groups: waves never split one), as one launch
    if (first < L.basisCount && count > 0) {
      const size_t last = std::min(first + count, L.basisCount);
      size_t g0 = 0;
      while (g0 < L.groups.size() && L.groups[g0].first < first) ++g0;
      size_t g1 = g0;
      while (g1 < L.groups.size() && L.groups[g1].first + L.groups[g1].count <= last) ++g1;
      injectPoint(B.ctx);
      ZK_CUDA(launchBasisRevalue(reinterpret_cast<const BasisArgs*>(base + B.basisArgsOff) + L.groupArgs + g0,
                                 static_cast<uint32_t>(g1 - g0), L.sc.nP, L.descBytes, L.fixSlots, B.ctx->dErr, s));
      count -= last - first, first = last;
    }
  }
  if (count == 0) return;
  const auto* ns = reinterpret_cast<const NsArgs<R>*>(base + L.nsOff) + first;
  const uint32_t n = static_cast<uint32_t>(count), tiles = numTilesOf(L.sc.nP, B.ppt);
  const size_t splitAt = std::min(count, L.splitAt > first ? L.splitAt - first : 0);
  const bool split = L.lean && !L.perTrade && !B.sink && sizeof(R) == 4 && B.ppt > 1 && splitAt < n;
  if (!split) {
    injectPoint(B.ctx);
    ZK_CUDA(launchRevalue<R>(L.cb, ns, n, tiles, L.stateWordsMax, L.perTrade, B.sink, L.lean, B.ppt, s, false,
                             L.lean && !L.perTrade && !B.sink && L.cashAll));
    return;
  }
  const uint32_t big = static_cast<uint32_t>(splitAt);
  const bool fork = big > 0 && side;
  if (big > 0) injectPoint(B.ctx);
  if (fork) {
    ZK_CUDA(cudaEventRecord(forkEv, s));
    ZK_CUDA(cudaStreamWaitEvent(side, forkEv, 0));
    ZK_CUDA(launchRevalue<R>(L.cb, ns, big, tiles, L.stateWordsMax, false, false, true, B.ppt, side, false, L.cashBig));
  } else if (big > 0) {
    ZK_CUDA(launchRevalue<R>(L.cb, ns, big, tiles, L.stateWordsMax, false, false, true, B.ppt, s, false, L.cashBig));
  }
  if (fork) ZK_CUDA(cudaEventRecord(joinEv, side));  // joined before a failure below can leave the side stream behind
  injectPoint(B.ctx);
  ZK_CUDA(launchRevalue<R>(L.cb, ns + big, n - big, tiles, L.smallStateMax, false, false, true, B.ppt, s, true, L.cashSmall));
  if (fork) ZK_CUDA(cudaStreamWaitEvent(s, joinEv, 0));
}

cudaError_t recordEvent(cudaEvent_t e, cudaStream_t s, bool capturing) {
  return cudaEventRecordWithFlags(e, s, capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
}

// Inside a stream capture the timing events must be recorded as graph nodes (cudaEventRecordExternal); an
// ordinary record there only orders the capture.
template <typename R>
void execute(Batch<R>& B, bool capturing = false) {
  zk_context* ctx = B.ctx;
  cudaStream_t s = ctx->stream;
  if (!B.ev[0])
    for (auto& e : B.ev) ZK_CUDA(cudaEventCreate(&e));
  ZK_CUDA(cudaMemsetAsync(ctx->dErr, 0, 4, s));
  if (B.flagsBytes) ZK_CUDA(cudaMemsetAsync(B.base + B.flagsOff, 0, B.flagsBytes, s));
  ZK_CUDA(recordEvent(B.ev[0], s, capturing));
  const uintptr_t base = reinterpret_cast<uintptr_t>(B.base);
  // A re-run of chosen paths: every plan is a launch of a few paths; they run side by side on worker streams,
  // each its simulation then its revaluation, joined before the reduce.
  const bool fan = !capturing && !B.waved && B.launches.size() > 1 && !B.plans[B.launches[0].planIdx[0]].pathMap.empty();
  if (fan) {
    const size_t k = std::min<size_t>(B.launches.size(), 16);
    while (ctx->workers.size() < k) {
      cudaStream_t w = nullptr;
      cudaEvent_t e = nullptr;
      ZK_CUDA(cudaStreamCreateWithFlags(&w, cudaStreamNonBlocking));
      ctx->workers.push_back(w);
      ZK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ctx->workerJoin.push_back(e);
    }
    if (!ctx->fork) ZK_CUDA(cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming));
    ZK_CUDA(cudaEventRecord(ctx->fork, s));
    for (size_t q = 0; q < k; ++q) ZK_CUDA(cudaStreamWaitEvent(ctx->workers[q], ctx->fork, 0));
    for (size_t l = 0; l < B.launches.size(); ++l) {
      const auto& L = B.launches[l];
      cudaStream_t w = ctx->workers[l % k];
      injectPoint(ctx);
      ZK_CUDA(launchSimulate<R>(L.sc, L.cb, w));
      launchRevalues(B, L, base, w, nullptr, nullptr, nullptr);
    }
    for (size_t q = 0; q < k; ++q) {
      ZK_CUDA(cudaEventRecord(ctx->workerJoin[q], ctx->workers[q]));
      ZK_CUDA(cudaStreamWaitEvent(s, ctx->workerJoin[q], 0));
    }
    ZK_CUDA(recordEvent(B.ev[1], s, capturing));
  } else {
    for (auto& L : B.launches) {
      if (L.presim) continue;  // simulated ahead of the host work
      injectPoint(ctx);
      ZK_CUDA(launchSimulate<R>(L.sc, L.cb, s));
    }
    ZK_CUDA(recordEvent(B.ev[1], s, capturing));
  }
  for (auto& L : B.launches) {
    if (fan) break;  // revalued on the worker streams above
    const bool split = L.lean && !L.perTrade && !B.sink && sizeof(R) == 4 && B.ppt > 1 && L.splitAt < L.planIdx.size();
    if (split && L.splitAt > L.basisCount && !ctx->side && !capturing) {
      ZK_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
      ZK_CUDA(cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming));
      ZK_CUDA(cudaEventCreateWithFlags(&ctx->join, cudaEventDisableTiming));
    }
    if (!B.waved) {
      launchRevalues(B, L, base, s, ctx->side, ctx->fork, ctx->join);
      continue;
    }
    // Waves: a wave's rows and partials are reduced and read before the next wave overwrites them.  Its timings
    // count as revalue time ([1]); reduce and row statistics ([2], [3]) stay zero.
    for (const auto& w : L.waves) {
      injectPoint(ctx);
      launchRevalues(B, L, base, s, ctx->side, ctx->fork, ctx->join, w.first, w.count);
      ZK_CUDA(launchReduce<R>(reinterpret_cast<const ReduceJob<R>*>(base + B.reduceOff) + w.reduceFirst, static_cast<uint32_t>(w.count),
                              B.maxReduceN, B.ppt, s));
      ZK_CUDA(launchRowStats<R>(reinterpret_cast<const RowJob<R>*>(base + B.rowOff) + w.rowFirst, static_cast<uint32_t>(w.rowCount),
                                ctx->dErr, s, ctx->rowRounds));
    }
  }
  for (const auto& M : B.im) {
    injectPoint(ctx);
    ZK_CUDA(launchNestedIm<R>(M, s));
  }
  ZK_CUDA(recordEvent(B.ev[2], s, capturing));
  if (B.waved) {
    ZK_CUDA(recordEvent(B.ev[3], s, capturing));
  } else if (!B.sink) {
    injectPoint(ctx);
    ZK_CUDA(launchReduce<R>(reinterpret_cast<const ReduceJob<R>*>(base + B.reduceOff), static_cast<uint32_t>(B.plans.size()), B.maxReduceN,
                            B.ppt, s));
    ZK_CUDA(recordEvent(B.ev[3], s, capturing));
    injectPoint(ctx);
    ZK_CUDA(launchRowStats<R>(reinterpret_cast<const RowJob<R>*>(base + B.rowOff), B.numRowJobs, ctx->dErr, s, ctx->rowRounds));
  } else {
    ZK_CUDA(recordEvent(B.ev[3], s, capturing));
  }
  ZK_CUDA(recordEvent(B.ev[4], s, capturing));
  B.timed = true;
}

// The status of a kernel's error word (DeviceError), the same for every entry point.
void throwDeviceError(uint32_t err) {
  if (err == kDevOk) return;
  if (err == kDevTimeout) throw fail(ZK_ERR_DEVICE_TIMEOUT, "a bounded wait in a kernel gave up");
  if (err == kDevBadTerm)
    throw fail(ZK_ERR_CUDA, "a kernel met a case it does not handle (error %u: a quantile search that did not narrow to its ranks "
                            "within its rounds, or an AMC regression without a solution)", err);
  throw fail(ZK_ERR_CUDA, "a kernel reported error %u", err);
}

template <typename R>
void finish(Batch<R>& B) {
  zk_context* ctx = B.ctx;
  uint32_t err = 0;
  ZK_CUDA(cudaMemcpyAsync(&err, ctx->dErr, 4, cudaMemcpyDeviceToHost, ctx->stream));
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  if (B.timed) {
    for (int k = 0; k < 4; ++k) ZK_CUDA(cudaEventElapsedTime(&B.ms[k], B.ev[k], B.ev[k + 1]));
  }
  throwDeviceError(err);
}

template <typename R, typename Out>
void readOutputs(Batch<R>& B, Out* outs) {
  zk_context* ctx = B.ctx;
  growStage(ctx->stageOut, ctx->stageOutBytes, B.outBytes);
  unsigned char* host = ctx->stageOut;
  ZK_CUDA(cudaMemcpyAsync(host, B.base + B.outBegin, B.outBytes, cudaMemcpyDeviceToHost, ctx->stream));
  finish(B);
  for (size_t i = 0; i < B.plans.size(); ++i) {
    const auto& P = B.plans[i];
    const auto& D = B.dev[i];
    const R* sums = reinterpret_cast<const R*>(host + (D.sums - B.outBegin));
    const R* vals = reinterpret_cast<const R*>(host + (D.values - B.outBegin));
    const size_t nS = static_cast<size_t>(P.nT) * P.nS, nV = std::max<uint32_t>(P.v.num_outputs, 1);
    for (size_t k = 0; k < nS; ++k) outs[i].sums[k] = sums[k];
    for (size_t k = 0; k < nV; ++k) outs[i].values[k] = vals[k];
  }
}

// The exact-decision check, after an execute of a single-precision batch built with BuildOpts::exact.  The revalue
// kernel flagged every path with a margin call or exercise decision inside its guard band (decisionGuard): there the
// single-precision rule may decide otherwise than double precision would.  Those paths run again, alone, twice: in
// double precision (their decisions and values as the FP64 mode takes them on the same normals) and in single
// precision (what the batch summed for them).  Their rows are replaced by the double-precision rows and the plan's
// row statistics recomputed; the returned patches replace their share of the date statistics after readOutputs.
// Plans with the nested initial margin are not checked.  A batch in waves has no resident rows to patch.
struct SumPatch {
  size_t plan = 0;
  double share = 0.0;         // re-run paths / the plan's paths (the sums are means)
  std::vector<float> s32;     // the re-run paths' means in single precision
  std::vector<double> s64;    // and in double precision
};

std::vector<SumPatch> exactCheck(Batch<float>& B) {
  zk_context* ctx = B.ctx;
  std::vector<SumPatch> patches;
  if (!B.exact || B.flagsBytes == 0) return patches;
  if (B.waved)
    throw fail(ZK_ERR_UNSUPPORTED, "exact decisions: the batch runs in waves (its rows exceed the row budget), so its rows are not resident to patch");
  std::vector<uint32_t> bits(B.flagsBytes / 4);
  ZK_CUDA(cudaMemcpyAsync(bits.data(), B.base + B.flagsOff, B.flagsBytes, cudaMemcpyDeviceToHost, ctx->stream));
  finish(B);
  std::vector<size_t> which;
  std::vector<std::vector<uint32_t>> maps;
  for (size_t i = 0; i < B.plans.size(); ++i) {
    const auto& P = B.plans[i];
    if (P.guard.empty()) continue;
    const uint32_t* w = bits.data() + (B.dev[i].flags - B.flagsOff) / 4;
    std::vector<uint32_t> paths;
    for (uint32_t k = 0; k < (P.nP + 31) / 32; ++k)
      for (uint32_t m = w[k]; m; m &= m - 1) paths.push_back(32 * k + static_cast<uint32_t>(__builtin_ctz(m)));
    ctx->exactPaths += P.nP;
    ctx->exactFlagged += paths.size();
    if (paths.empty()) continue;
    which.push_back(i);
    maps.push_back(std::move(paths));
  }
  if (which.empty()) return patches;
  // The flagged paths of each plan as a plan of their own: its header counts them, the tables are the plan's
  // (converted to double for the double-precision run).
  const size_t n = which.size();
  std::vector<std::vector<uint32_t>> headers(n);
  std::vector<std::vector<double>> d64(4 * n);
  std::vector<View<float>> v32(n);
  std::vector<View<double>> v64(n);
  for (size_t k = 0; k < n; ++k) {
    const auto& P = B.plans[which[k]];
    headers[k].assign(P.v.header, P.v.header + P.v.header_len);
    headers[k][hP] = static_cast<uint32_t>(maps[k].size());
    v32[k] = P.v;
    v32[k].header = headers[k].data();
    auto widen = [&](std::vector<double>& dst, const float* src, size_t len) {
      dst.assign(src, src + len);
      return dst.empty() ? nullptr : dst.data();
    };
    View<double>& d = v64[k];
    d.header = headers[k].data(), d.header_len = P.v.header_len;
    d.indices = P.v.indices, d.indices_len = P.v.indices_len;
    d.params = widen(d64[4 * k], P.v.params, P.v.params_len), d.params_len = P.v.params_len;
    d.steps = widen(d64[4 * k + 1], P.v.steps, P.v.steps_len), d.steps_len = P.v.steps_len;
    d.terms = widen(d64[4 * k + 2], P.v.terms, P.v.terms_len), d.terms_len = P.v.terms_len;
    d.requests = widen(d64[4 * k + 3], P.v.requests, P.v.requests_len), d.requests_len = P.v.requests_len;
    d.rows_total = P.v.rows_total, d.num_outputs = P.v.num_outputs;
  }
  BuildOpts ro;
  ro.maps = &maps;
  // The single-precision re-run takes the batch's parsed and lowered plans, with the re-run's path count.
  std::vector<Plan<float>> p32(n);
  for (size_t k = 0; k < n; ++k) {
    p32[k] = B.plans[which[k]];
    p32[k].v = v32[k], p32[k].H = headers[k].data(), p32[k].nP = static_cast<uint32_t>(maps[k].size());
    p32[k].guard.clear(), p32[k].pathMap.clear();
  }
  auto B32 = build<float>(ctx, v32, false, nullptr, 0, ro, &p32);
  auto B64 = build<double>(ctx, v64, false, nullptr, 0, ro);
  for (size_t k = 0; k < n; ++k) {
    SumPatch sp;
    sp.plan = which[k];
    sp.share = static_cast<double>(maps[k].size()) / static_cast<double>(B.plans[which[k]].nP);
    patches.push_back(std::move(sp));
  }
  upload(*B32, ctx, false, nullptr, 0, true);
  execute(*B32);
  for (size_t k = 0; k < n; ++k) {
    const auto& P = B32->plans[k];
    patches[k].s32.resize(static_cast<size_t>(P.nT) * P.nS);
    ZK_CUDA(cudaMemcpyAsync(patches[k].s32.data(), B32->base + B32->dev[k].sums, patches[k].s32.size() * 4, cudaMemcpyDeviceToHost,
                            ctx->stream));
  }
  finish(*B32);
  upload(*B64, ctx, false, nullptr, 0, true);
  execute(*B64);
  for (size_t k = 0; k < n; ++k) {
    const auto& P = B64->plans[k];
    patches[k].s64.resize(static_cast<size_t>(P.nT) * P.nS);
    ZK_CUDA(cudaMemcpyAsync(patches[k].s64.data(), B64->base + B64->dev[k].sums, patches[k].s64.size() * 8, cudaMemcpyDeviceToHost,
                            ctx->stream));
  }
  finish(*B64);
  // The rows of the re-run paths from the double-precision run, then the plan's row statistics on the patched rows
  // (its jobs sit in plan order in the batch's job array).
  std::vector<size_t> jobFirst(B.plans.size() + 1, 0);
  for (size_t i = 0; i < B.plans.size(); ++i) jobFirst[i + 1] = jobFirst[i] + B.plans[i].nReq;
  for (size_t k = 0; k < n; ++k) {
    const size_t i = which[k];
    const auto& P = B.plans[i];
    ZK_CUDA(launchScatterRows(reinterpret_cast<const double*>(B64->base + B64->dev[k].expo), static_cast<uint32_t>(maps[k].size()),
                              reinterpret_cast<const uint32_t*>(B64->base + B64->dev[k].pathMap), P.v.rows_total,
                              reinterpret_cast<float*>(B.base + B.dev[i].expo), P.nP, ctx->stream));
    ZK_CUDA(launchRowStats<float>(reinterpret_cast<const RowJob<float>*>(B.base + B.rowOff) + jobFirst[i], static_cast<uint32_t>(P.nReq),
                                  ctx->dErr, ctx->stream, ctx->rowRounds));
  }
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));  // the sub-batches' arenas are freed with them
  return patches;
}

// The date statistics of the re-run paths: their single-precision share replaced by the double-precision one.
template <typename Out>
void applyPatches(const std::vector<SumPatch>& patches, Out* outs) {
  for (const auto& sp : patches)
    for (size_t k = 0; k < sp.s64.size(); ++k)
      outs[sp.plan].sums[k] = static_cast<float>(static_cast<double>(outs[sp.plan].sums[k]) +
                                                 sp.share * (sp.s64[k] - static_cast<double>(sp.s32[k])));
}

template <typename Out>
void checkOutput(const Out* o, size_t nSums, size_t nValues, size_t i) {
  if (!o || !o->sums || !o->values) throw fail(ZK_ERR_INVALID_ARGUMENT, "output %zu: null buffer", i);
  if (o->sums_len != nSums) throw fail(ZK_ERR_INVALID_ARGUMENT, "output %zu: sums must hold nT * statsPerDate = %zu values", i, nSums);
  if (o->values_len < nValues) throw fail(ZK_ERR_INVALID_ARGUMENT, "output %zu: values must hold max(1, numOutputs) = %zu values", i, nValues);
}

template <typename R>
void checkOutputs(const Batch<R>& B, const void* outs, bool f64) {
  for (size_t i = 0; i < B.plans.size(); ++i) {
    const auto& P = B.plans[i];
    const size_t nS = static_cast<size_t>(P.nT) * P.nS, nV = std::max<uint32_t>(P.v.num_outputs, 1);
    if (f64) checkOutput(static_cast<const zk_output_f64*>(outs) + i, nS, nV, i);
    else checkOutput(static_cast<const zk_output*>(outs) + i, nS, nV, i);
  }
}

// The tile shape: paths per revalue thread (kTile * ppt paths per CTA).  The reduce kernel completes the
// 128-path groups' sums from the warp partials of the shape, so the results do not change with it.
template <typename R>
void setTileShape(Batch<R>& B, int ppt) {
  B.ppt = ppt;
}

// Autotuner: times the revalue kernel of this batch once per candidate tile shape (after a warm-up
// run) with CUDA events and keeps the fastest.  Shapes whose shared memory does not fit are skipped.
template <typename R>
void autotune(Batch<R>& B) {
  const int candidates[3] = {1, 2, 4};
  const int count = sizeof(R) == 8 ? 2 : 3;
  float best = 0.0f;
  int bestPpt = B.ppt;
  for (int c = 0; c < count; ++c) {
    const int ppt = candidates[c];
    bool fits = true;
    for (const auto& L : B.launches)
      fits = fits && revalueSmemBytes(L.stateWordsMax, L.perTrade, sizeof(R) == 8, ppt) <= 200 * 1024;
    if (!fits) continue;
    setTileShape(B, ppt);
    execute(B);
    finish(B);
    execute(B);
    finish(B);
    if (bestPpt == B.ppt && best == 0.0f) best = B.ms[1], bestPpt = ppt;
    if (B.ms[1] < best) best = B.ms[1], bestPpt = ppt;
  }
  setTileShape(B, bestPpt);
}

void requireCtx(zk_context* ctx) {
  if (!ctx) throw fail(ZK_ERR_INVALID_ARGUMENT, "null context");
  ZK_CUDA(cudaSetDevice(ctx->device));
}

}  // namespace

namespace {
template <typename R, typename ViewT, typename OutT>
zk_status runInjected(zk_context* ctx, const ViewT* plan, const double* normals, size_t streams, OutT* out, R* rows) {
  try {
    requireCtx(ctx);
    if (!plan || !out) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    BuildOpts bo;
    bo.exact = sizeof(R) == 4 && !normals && ctx->exactGuard > 0.0;
    auto B = build<R>(ctx, {viewOf(*plan)}, false, normals, streams, bo);
    checkOutputs(*B, out, sizeof(R) == 8);
    upload(*B, ctx, true, normals, streams);
    execute(*B);
    std::vector<SumPatch> patches;
    if constexpr (sizeof(R) == 4) patches = exactCheck(*B);
    if (rows) {
      const auto& P = B->plans[0];
      ZK_CUDA(cudaMemcpyAsync(rows, B->base + B->dev[0].expo, static_cast<size_t>(P.v.rows_total) * P.nP * sizeof(R),
                              cudaMemcpyDeviceToHost, ctx->stream));
    }
    readOutputs(*B, out);
    if constexpr (sizeof(R) == 4) applyPatches(patches, out);
    return ZK_OK;
  } catch (const Failure& f) {
    return record(ctx, f);
  }
}

// The Longstaff-Schwartz fit of a plan's Bermudans (fitAmc, src/gpu/fused_exposure.cpp:103-156): the AMC
// state pass of the fused kernel (x, deflator, exercise values on the device), then one thread-block
// cluster per Bermudan fits the policy of every exercise and the continuation of every date, and the
// fitted records are written into a copy of the plan's term table.
template <typename R, typename ViewT>
zk_status fitAmc(zk_context* ctx, const ViewT* plan, const double* normals, size_t streams, const uint32_t* degrees,
                 size_t numBermudans, R* termsOut, size_t termsLen) {
  void* dmem = nullptr;
  size_t dmemBytes = 0;
  try {
    requireCtx(ctx);
    if (!plan || !termsOut || (numBermudans && !degrees)) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    if (termsLen != plan->terms_len) throw fail(ZK_ERR_INVALID_ARGUMENT, "terms_out holds %zu values, the plan %zu", termsLen, plan->terms_len);
    auto B = build<R>(ctx, {viewOf(*plan)}, true, normals, streams);
    const auto& P = B->plans[0];
    const View<R> v = viewOf(*plan);
    if (numBermudans != P.nBerm)
      throw fail(ZK_ERR_INVALID_ARGUMENT, "the plan has %u Bermudans, not %zu", P.nBerm, numBermudans);
    // Layout of the regressions: policy term and date of each exercise, continuation term of each date.
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> decide(numBermudans), cont(numBermudans);
    // The two-regressor basis: a policy / continuation record followed by extension records (kind 15) regresses
    // on (x, s) too; its co-terminal swap's bonds are the annuity / float-leg records (kinds 13, 14) right before it.
    std::vector<int> twoD(numBermudans, -1);
    std::map<uint32_t, uint2> coterm;  // term -> range of its bonds in `bonds`
    std::vector<double4> bonds;
    const auto kindAt = [&](uint32_t u) { return static_cast<uint32_t>(v.terms[static_cast<size_t>(u) * kTermStride]) & 15u; };
    for (uint32_t j = 0; j < P.nT; ++j)
      for (uint32_t t = v.indices[j]; t < v.indices[j + 1]; ++t) {
        const auto code = static_cast<uint32_t>(v.terms[static_cast<size_t>(t) * kTermStride]);
        const uint32_t kind = code & 15u, b = bermudanOf(code, P.manyBerm), e = code >> 12u;
        if (kind != 6u && kind != 7u) continue;
        if (b >= numBermudans) throw fail(ZK_ERR_INVALID_PLAN, "an AMC term of Bermudan %u", b);
        const int two = t + 1 < v.indices[j + 1] && kindAt(t + 1) == kBermExt ? 1 : 0;
        if (twoD[b] >= 0 && twoD[b] != two) throw fail(ZK_ERR_INVALID_PLAN, "Bermudan %u mixes one- and two-regressor records", b);
        twoD[b] = two;
        if (two) {
          uint32_t u = t;
          while (u > v.indices[j] && (kindAt(u - 1) == kBermAnnuity || kindAt(u - 1) == kBermCoterm)) --u;
          bool annuity = false;
          const uint32_t at = static_cast<uint32_t>(bonds.size());
          for (; u < t; ++u) {
            const R* r = v.terms + static_cast<size_t>(u) * kTermStride;
            annuity = annuity || kindAt(u) == kBermAnnuity;
            bonds.push_back(make_double4(static_cast<double>(kindAt(u)), static_cast<double>(r[2]), static_cast<double>(r[3]),
                                         static_cast<double>(r[4])));
          }
          if (!annuity) throw fail(ZK_ERR_INVALID_PLAN, "Bermudan %u: a two-regressor record without its co-terminal annuity", b);
          coterm[t] = make_uint2(at, static_cast<uint32_t>(bonds.size()) - at);
        }
        if (kind == 6u) {
          if (e >= static_cast<uint32_t>(kMaxExercises)) throw fail(ZK_ERR_INVALID_PLAN, "exercise index %u", e);
          if (decide[b].size() <= e) decide[b].resize(e + 1, {0xFFFFFFFFu, 0u});
          decide[b][e] = {t, j};
        } else {
          cont[b].push_back({j, t});
        }
      }
    std::vector<AmcFitJob> jobs(numBermudans);
    std::vector<uint32_t> contDates;
    uint32_t slots = 0, eRow = 0;
    for (size_t b = 0; b < numBermudans; ++b) {
      if (degrees[b] > 3) throw fail(ZK_ERR_INVALID_ARGUMENT, "AMC regression degree %u above 3", degrees[b]);
      AmcFitJob& J = jobs[b];
      J = AmcFitJob{};
      J.nP = P.nP, J.nT = P.nT, J.nE = static_cast<uint32_t>(decide[b].size()), J.degree = degrees[b];
      J.twoD = twoD[b] > 0 ? 1u : 0u;
      if (J.nE != P.bermRows[b]) throw fail(ZK_ERR_INVALID_PLAN, "Bermudan %zu: inconsistent exercise terms", b);
      J.eRow = eRow, eRow += J.nE;
      J.slotBase = slots, slots += J.nE + static_cast<uint32_t>(cont[b].size());
      for (uint32_t e = 0; e < J.nE; ++e) {
        if (decide[b][e].first == 0xFFFFFFFFu || (e > 0 && decide[b][e].second <= decide[b][e - 1].second))
          throw fail(ZK_ERR_INVALID_PLAN, "Bermudan %zu: exercise %u missing or out of order", b, e);
        J.exDate[e] = decide[b][e].second;
      }
      J.contBegin = static_cast<uint32_t>(contDates.size()), J.contCount = static_cast<uint32_t>(cont[b].size());
      for (const auto& c : cont[b]) contDates.push_back(c.first);
    }
    // Per fit slot, the range of its co-terminal bonds (two-regressor Bermudans only).
    std::vector<uint2> bondRange(std::max<uint32_t>(slots, 1), make_uint2(0, 0));
    for (size_t b = 0; b < numBermudans; ++b) {
      const AmcFitJob& J = jobs[b];
      if (!J.twoD) continue;
      for (uint32_t e = 0; e < J.nE; ++e) bondRange[J.slotBase + e] = coterm.at(decide[b][e].first);
      for (uint32_t i = 0; i < J.contCount; ++i) bondRange[J.slotBase + J.nE + i] = coterm.at(cont[b][i].second);
    }
    std::copy(v.terms, v.terms + termsLen, termsOut);
    if (numBermudans == 0) return ZK_OK;
    upload(*B, ctx, true, normals, streams);
    execute(*B);
    // Device scratch: jobs, continuation dates, realised values per Bermudan, fitted records, co-terminal bonds and
    // their ranges.
    const size_t jobsBytes = jobs.size() * sizeof(AmcFitJob), datesBytes = std::max<size_t>(contDates.size(), 1) * 4;
    const size_t realisedBytes = numBermudans * static_cast<size_t>(P.nP) * 8, outBytes = static_cast<size_t>(slots) * kFitOut * 8;
    const size_t bondsBytes = std::max<size_t>(bonds.size(), 1) * sizeof(double4), rangeBytes = bondRange.size() * sizeof(uint2);
    const size_t o1 = alignUp(jobsBytes), o2 = o1 + alignUp(datesBytes), o3 = o2 + alignUp(realisedBytes);
    const size_t scratchBytes = bonds.empty() ? 0 : realisedBytes;  // the two-regressor fits' swap rates per path
    const size_t o4 = o3 + alignUp(outBytes), o5 = o4 + alignUp(bondsBytes), o6 = o5 + alignUp(rangeBytes), total = o6 + scratchBytes;
    dmem = takeBlock(ctx, total, dmemBytes);
    if (!dmem) throw fail(ZK_ERR_OUT_OF_MEMORY, "AMC fit: %zu bytes of device memory", total);
    unsigned char* d = static_cast<unsigned char*>(dmem);
    ZK_CUDA(cudaMemcpyAsync(d, jobs.data(), jobsBytes, cudaMemcpyHostToDevice, ctx->stream));
    if (!contDates.empty()) ZK_CUDA(cudaMemcpyAsync(d + o1, contDates.data(), contDates.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    if (!bonds.empty()) {
      ZK_CUDA(cudaMemcpyAsync(d + o4, bonds.data(), bonds.size() * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream));
      ZK_CUDA(cudaMemcpyAsync(d + o5, bondRange.data(), rangeBytes, cudaMemcpyHostToDevice, ctx->stream));
    }
    const uint32_t cluster = P.nP >= 65536 ? 8u : P.nP >= 16384 ? 4u : P.nP >= 4096 ? 2u : 1u;
    const R* sx = reinterpret_cast<const R*>(B->base + B->sinkOff[0]);
    const R* sd = reinterpret_cast<const R*>(B->base + B->sinkOff[1]);
    const R* se = reinterpret_cast<const R*>(B->base + B->sinkOff[2]);
    ZK_CUDA(launchAmcFit<R>(reinterpret_cast<const AmcFitJob*>(d), static_cast<uint32_t>(numBermudans), sx, sd, se,
                            reinterpret_cast<const uint32_t*>(d + o1),
                            bonds.empty() ? nullptr : reinterpret_cast<const double4*>(d + o4),
                            reinterpret_cast<const uint2*>(d + o5), reinterpret_cast<double*>(d + o2),
                            bonds.empty() ? nullptr : reinterpret_cast<double*>(d + o6), reinterpret_cast<double*>(d + o3),
                            ctx->dErr, cluster, ctx->stream));
    std::vector<double> fitted(static_cast<size_t>(slots) * kFitOut);
    uint32_t devErr = 0;
    ZK_CUDA(cudaMemcpyAsync(fitted.data(), d + o3, outBytes, cudaMemcpyDeviceToHost, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(&devErr, ctx->dErr, 4, cudaMemcpyDeviceToHost, ctx->stream));
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
    giveBlock(ctx, static_cast<unsigned char*>(dmem), dmemBytes);
    dmem = nullptr;
    if (devErr != 0) throw fail(ZK_ERR_CUDA, "the AMC fit reported error %u (normal equations not positive definite)", devErr);
    // The records as the reference writes them: center, 1 / scale, c0..c3 (fused_exposure.cpp:118-123).
    // Two-regressor records: cx, 1 / sx, cs, 1 / ss, c0, c1 in the record, c2..c8 in the first extension record's
    // fields 1..7 and c9 in the second's field 1 (the kernel's amcPoly2 reads them so).
    auto write = [&](uint32_t term, const double* f, bool two) {
      R* r = termsOut + static_cast<size_t>(term) * kTermStride;
      if (!two) {
        r[2] = static_cast<R>(f[0]);
        r[3] = static_cast<R>(1.0 / f[1]);
        for (int i = 0; i < 4; ++i) r[4 + i] = static_cast<R>(f[2 + i]);
        return;
      }
      r[2] = static_cast<R>(f[0]), r[3] = static_cast<R>(1.0 / f[1]), r[4] = static_cast<R>(f[2]), r[5] = static_cast<R>(1.0 / f[3]);
      r[6] = static_cast<R>(f[4]), r[7] = static_cast<R>(f[5]);
      R* e1 = r + kTermStride;
      R* e2 = r + 2 * kTermStride;
      for (int i = 0; i < 7; ++i) e1[1 + i] = static_cast<R>(f[6 + i]);
      e2[1] = static_cast<R>(f[13]);
    };
    for (size_t b = 0; b < numBermudans; ++b) {
      const AmcFitJob& J = jobs[b];
      for (uint32_t e = 0; e < J.nE; ++e) write(decide[b][e].first, &fitted[(J.slotBase + e) * kFitOut], J.twoD != 0);
      for (uint32_t i = 0; i < J.contCount; ++i) write(cont[b][i].second, &fitted[(J.slotBase + J.nE + i) * kFitOut], J.twoD != 0);
    }
    return ZK_OK;
  } catch (const Failure& f) {
    if (dmem) {  // the block goes back only once nothing in flight can still use it
      cudaStreamSynchronize(ctx->stream);
      giveBlock(ctx, static_cast<unsigned char*>(dmem), dmemBytes);
    }
    return record(ctx, f);
  }
}
}  // namespace

// ================================================================================================
struct zk_batch {
  std::unique_ptr<Batch<float>> b;
  bool tuned = false;  // the tile shape was autotuned or pinned
  // The execute sequence (simulate, revalue, reduce, row statistics and their timing events) captured once per
  // tile shape in a CUDA graph and replayed; an execute that cannot be captured runs eagerly instead.
  cudaGraphExec_t graph = nullptr;
  int graphPpt = 0;
  bool eager = false;
  ~zk_batch() {
    if (graph) cudaGraphExecDestroy(graph);
  }
};

namespace {
// Captures the batch's execute sequence into b->graph; returns false (and leaves no capture open) if the
// stream cannot be captured.
bool captureExecute(zk_batch* b) {
  Batch<float>& B = *b->b;
  const cudaStream_t s = B.ctx->stream;
  if (!B.ev[0])
    for (auto& e : B.ev) ZK_CUDA(cudaEventCreate(&e));
  if (b->graph) cudaGraphExecDestroy(b->graph), b->graph = nullptr;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  bool ok = true;
  try {
    execute(B, true);
  } catch (const Failure&) {
    ok = false;
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  if (!ok || e != cudaSuccess || !g || cudaGraphInstantiate(&b->graph, g, 0) != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    b->graph = nullptr;
    cudaGetLastError();
    return false;
  }
  cudaGraphDestroy(g);
  b->graphPpt = B.ppt;
  return true;
}
}  // namespace

extern "C" {

int zk_abi_version(void) { return ZK_ABI_VERSION; }

zk_status zk_context_create(int device, zk_context** out) {
  if (!out) return ZK_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return ZK_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return ZK_ERR_INVALID_ARGUMENT;
  auto* ctx = new zk_context();
  ctx->device = device;
  try {
    ZK_CUDA(cudaSetDevice(device));
    ZK_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->ownStream = true;
    ZK_CUDA(cudaMalloc(&ctx->dErr, 16));
  } catch (const Failure& f) {
    delete ctx;
    return f.status;
  }
  *out = ctx;
  return ZK_OK;
}

void zk_context_destroy(zk_context* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->arena) cudaFree(ctx->arena);
  if (ctx->stageIn) cudaFreeHost(ctx->stageIn);
  if (ctx->stageOut) cudaFreeHost(ctx->stageOut);
  if (ctx->dErr) cudaFree(ctx->dErr);
  if (ctx->side) {
    cudaStreamSynchronize(ctx->side);
    cudaStreamDestroy(ctx->side);
  }
  for (auto& blk : ctx->spareBlocks) cudaFree(blk.first);
  if (ctx->cube) cudaFree(ctx->cube);
  if (ctx->presimSteps) cudaFree(ctx->presimSteps);
  for (auto w : ctx->workers) {
    cudaStreamSynchronize(w);
    cudaStreamDestroy(w);
  }
  for (auto e : ctx->workerJoin) cudaEventDestroy(e);
  if (ctx->fork) cudaEventDestroy(ctx->fork);
  if (ctx->join) cudaEventDestroy(ctx->join);
  if (ctx->ownStream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* zk_last_error(const zk_context* ctx) { return ctx ? ctx->lastError.c_str() : "null context"; }

zk_status zk_context_set_stream(zk_context* ctx, void* stream) {
  if (!ctx) return ZK_ERR_INVALID_ARGUMENT;
  if (stream) {
    if (ctx->ownStream && ctx->stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = static_cast<cudaStream_t>(stream);
    ctx->ownStream = false;
  }
  return ZK_OK;
}

zk_status zk_context_set_row_budget(zk_context* ctx, uint64_t bytes) {
  if (!ctx) return ZK_ERR_INVALID_ARGUMENT;
  ctx->rowBudget = bytes;
  return ZK_OK;
}

zk_status zk_context_set_basis(zk_context* ctx, uint32_t mode) {
  if (!ctx || mode > ZK_BASIS_ALL) return ZK_ERR_INVALID_ARGUMENT;
  ctx->basisMode = mode;
  return ZK_OK;
}

zk_status zk_context_set_exact_decisions(zk_context* ctx, double guard) {
  if (!ctx || !(guard >= 0.0) || guard > 1e-2) return ZK_ERR_INVALID_ARGUMENT;
  ctx->exactGuard = guard;
  return ZK_OK;
}

zk_status zk_context_call_timings(const zk_context* ctx, double* ms5) {
  if (!ctx || !ms5) return ZK_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < 5; ++k) ms5[k] = ctx->callMs[k];
  return ZK_OK;
}

zk_status zk_context_exact_stats(zk_context* ctx, uint64_t* flagged_paths, uint64_t* checked_paths) {
  if (!ctx || !flagged_paths || !checked_paths) return ZK_ERR_INVALID_ARGUMENT;
  *flagged_paths = ctx->exactFlagged, *checked_paths = ctx->exactPaths;
  ctx->exactFlagged = ctx->exactPaths = 0;
  return ZK_OK;
}

zk_status zk_debug_basis(const zk_plan_view* plans, size_t n, const double* x, const double* S, const double* xf,
                         double* out, char* err, size_t err_len) {
  auto say = [&](const char* m) {
    if (err && err_len) std::snprintf(err, err_len, "%s", m);
  };
  try {
    if (!plans || n == 0 || !x || !S || !xf || !out) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<Plan<float>> P(n);
    std::vector<BasisPlanIn> in;
    for (size_t i = 0; i < n; ++i) {
      P[i] = parse(viewOf(plans[i]), i);
      in.push_back({P[i].v.terms, P[i].v.indices, P[i].nT, static_cast<uint32_t>(P[i].nTerms), P[i].offCall, P[i].offRep});
    }
    BasisImage img;
    std::string why;
    if (!buildBasis(in, img, why)) throw fail(ZK_ERR_UNSUPPORTED, "%s", why.c_str());
    out[0] = basisCheck(in, img, x, S, xf);
    out[1] = static_cast<double>(img.columns), out[2] = static_cast<double>(img.linearTerms);
    out[3] = img.numFixSlots, out[4] = img.numChunks;
    return ZK_OK;
  } catch (const Failure& f) {
    say(f.message.c_str());
    return f.status;
  } catch (const std::exception& e) {
    say(e.what());
    return ZK_ERR_INVALID_ARGUMENT;
  }
}

namespace {
// The first plan's scenario simulated on the context's stream into the context's cube buffer, so that the factor
// cube is being written while the host validates and lowers the plans; build() hands it to the launch that holds
// plan 0 when that launch needs the same fields (else the launch simulates again).  The step table goes up first;
// the buffers are reused by later calls, which synchronise before they return.
Presim presimulate(zk_context* ctx, const zk_plan_view& v0) {
  Presim pre;
  const Plan<float> P0 = parse(viewOf(v0), 0);
  ScenarioArgs<float> sc;
  CubeArgs<float> cb;
  const uint32_t fields = scenarioOf(P0, P0.probes, 0, sc, cb);
  const size_t cubeBytes = static_cast<size_t>(fields) * P0.nT * P0.nP * 4, stepBytes = static_cast<size_t>(P0.nT) * P0.stepStride * 4;
  if (ctx->cubeBytes < cubeBytes) {
    if (ctx->cube) ZK_CUDA(cudaFree(ctx->cube));
    ctx->cube = nullptr, ctx->cubeBytes = 0;
    if (cudaMalloc(&ctx->cube, cubeBytes) != cudaSuccess) {
      cudaGetLastError();
      return pre;  // no room beside the arena: the batch simulates inside its own
    }
    ctx->cubeBytes = cubeBytes;
  }
  if (ctx->presimStepsBytes < stepBytes) {
    if (ctx->presimSteps) ZK_CUDA(cudaFree(ctx->presimSteps));
    ctx->presimSteps = nullptr, ctx->presimStepsBytes = 0;
    ZK_CUDA(cudaMalloc(&ctx->presimSteps, stepBytes));
    ctx->presimStepsBytes = stepBytes;
  }
  ZK_CUDA(cudaMemcpyAsync(ctx->presimSteps, P0.v.steps, stepBytes, cudaMemcpyHostToDevice, ctx->stream));
  sc.steps = static_cast<const float*>(ctx->presimSteps);
  cb.data = static_cast<float*>(ctx->cube);
  injectPoint(ctx);
  ZK_CUDA(launchSimulate<float>(sc, cb, ctx->stream));
  pre.cube = static_cast<float*>(ctx->cube);
  pre.probes = P0.probes;
  return pre;
}
}  // namespace

zk_status zk_run_plans(zk_context* ctx, const zk_plan_view* plans, size_t n, zk_output* outs) {
  try {
    requireCtx(ctx);
    if (!plans || !outs || n == 0) throw fail(ZK_ERR_INVALID_ARGUMENT, "null or empty plan list");
    std::vector<View<float>> views;
    for (size_t i = 0; i < n; ++i) views.push_back(viewOf(plans[i]));
    BuildOpts bo;
    bo.exact = ctx->exactGuard > 0.0;
    using Clock = std::chrono::steady_clock;
    auto ms = [](Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
    const auto t0 = Clock::now();
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));  // a failed earlier call may have left work on the buffers
    const Presim pre = presimulate(ctx, plans[0]);
    bo.presim = &pre;
    auto B = build<float>(ctx, views, false, nullptr, 0, bo);
    checkOutputs(*B, outs, false);
    const auto t1 = Clock::now();
    upload(*B, ctx, true, nullptr, 0);
    const auto t2 = Clock::now();
    execute(*B);
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
    const auto t3 = Clock::now();
    const auto patches = exactCheck(*B);
    const auto t4 = Clock::now();
    readOutputs(*B, outs);
    applyPatches(patches, outs);
    const auto t5 = Clock::now();
    ctx->callMs[0] = ms(t0, t1), ctx->callMs[1] = ms(t1, t2), ctx->callMs[2] = ms(t2, t3), ctx->callMs[3] = ms(t3, t4);
    ctx->callMs[4] = ms(t4, t5);
    return ZK_OK;
  } catch (const Failure& f) {
    return record(ctx, f);
  } catch (const std::exception& e) {
    return record(ctx, fail(ZK_ERR_CUDA, "%s", e.what()));
  }
}

zk_status zk_run_plan(zk_context* ctx, const zk_plan_view* plan, zk_output* out) { return zk_run_plans(ctx, plan, 1, out); }

zk_status zk_amc_states(zk_context* ctx, const zk_plan_view* plan, float* x, float* deflator, float* exercise, size_t exercise_rows) {
  try {
    requireCtx(ctx);
    if (!plan || !x || !deflator) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    auto B = build<float>(ctx, {viewOf(*plan)}, true, nullptr, 0);
    if (exercise_rows != B->exerciseRows)
      throw fail(ZK_ERR_INVALID_ARGUMENT, "the plan has %u exercise rows, not %zu", B->exerciseRows, exercise_rows);
    if (exercise_rows > 0 && !exercise) throw fail(ZK_ERR_INVALID_ARGUMENT, "null exercise buffer");
    upload(*B, ctx, true, nullptr, 0);
    execute(*B);
    const auto& P = B->plans[0];
    const size_t n = static_cast<size_t>(P.nT) * P.nP;
    ZK_CUDA(cudaMemcpyAsync(x, B->base + B->sinkOff[0], n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(deflator, B->base + B->sinkOff[1], n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (exercise_rows)
      ZK_CUDA(cudaMemcpyAsync(exercise, B->base + B->sinkOff[2], exercise_rows * P.nP * 4, cudaMemcpyDeviceToHost, ctx->stream));
    finish(*B);
    return ZK_OK;
  } catch (const Failure& f) {
    return record(ctx, f);
  }
}


zk_status zk_run_plan_rows(zk_context* ctx, const zk_plan_view* plan, zk_output* out, float* rows) {
  if (!rows) return record(ctx, fail(ZK_ERR_INVALID_ARGUMENT, "null rows buffer"));
  return runInjected<float>(ctx, plan, nullptr, 0, out, rows);
}

zk_status zk_fit_amc(zk_context* ctx, const zk_plan_view* plan, const uint32_t* degrees, size_t num_bermudans, float* terms_out,
                     size_t terms_len) {
  return fitAmc<float>(ctx, plan, nullptr, 0, degrees, num_bermudans, terms_out, terms_len);
}

zk_status zk_fit_amc_f64(zk_context* ctx, const zk_plan_view_f64* plan, const double* normals, size_t streams,
                         const uint32_t* degrees, size_t num_bermudans, double* terms_out, size_t terms_len) {
  return fitAmc<double>(ctx, plan, normals, streams, degrees, num_bermudans, terms_out, terms_len);
}

zk_status zk_gemm_bf16(zk_context* ctx, const uint16_t* A, const uint16_t* B, uint32_t M, uint32_t N, uint32_t K,
                       const float* bias, uint32_t act, float* C) {
  void* d = nullptr;
  try {
    requireCtx(ctx);
    if (!A || !B || !C) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    if (M % 128 || N % 16 || K % 16 || M == 0 || N == 0 || K == 0)
      throw fail(ZK_ERR_INVALID_ARGUMENT, "M must be a multiple of 128, N and K of 16 (got %u, %u, %u)", M, N, K);
    const size_t a = static_cast<size_t>(M) * K * 2, b = static_cast<size_t>(N) * K * 2, c = static_cast<size_t>(M) * N * 4;
    const size_t ob = (a + 255) / 256 * 256, oc = ob + (b + 255) / 256 * 256, obias = oc + (c + 255) / 256 * 256;
    ZK_CUDA(cudaMalloc(&d, obias + N * 4));
    unsigned char* p = static_cast<unsigned char*>(d);
    ZK_CUDA(cudaMemcpyAsync(p, A, a, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(p + ob, B, b, cudaMemcpyHostToDevice, ctx->stream));
    if (bias) ZK_CUDA(cudaMemcpyAsync(p + obias, bias, N * 4, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemsetAsync(ctx->dErr, 0, 4, ctx->stream));
    GemmArgs g{};
    g.A = reinterpret_cast<const __nv_bfloat16*>(p), g.B = reinterpret_cast<const __nv_bfloat16*>(p + ob);
    g.M = M, g.N = N, g.K = K, g.bias = bias ? reinterpret_cast<const float*>(p + obias) : nullptr;
    g.C = reinterpret_cast<float*>(p + oc), g.act = act, g.err = ctx->dErr;
    ZK_CUDA(launchGemm(g, ctx->stream));
    uint32_t devErr = 0;
    ZK_CUDA(cudaMemcpyAsync(C, p + oc, c, cudaMemcpyDeviceToHost, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(&devErr, ctx->dErr, 4, cudaMemcpyDeviceToHost, ctx->stream));
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
    ZK_CUDA(cudaFree(d));
    d = nullptr;
    if (devErr) throw fail(ZK_ERR_DEVICE_TIMEOUT, "the GEMM's wait for its tensor-core operations gave up");
    return ZK_OK;
  } catch (const Failure& f) {
    if (d) cudaFree(d);
    return record(ctx, f);
  }
}

}  // extern "C"

// ---- the learned revaluation surrogate ----
struct zk_surrogate {
  zk_context* ctx = nullptr;
  zk::SurrogateState S;
};

namespace {
zk_context* ctxOf(zk_surrogate* s) {
  if (!s || !s->ctx) throw fail(ZK_ERR_INVALID_ARGUMENT, "null surrogate");
  requireCtx(s->ctx);
  return s->ctx;
}
// A device copy of n host values; the caller frees it.
template <typename T>
T* toDevice(const T* h, size_t n, cudaStream_t st) {
  void* d = nullptr;
  ZK_CUDA(cudaMalloc(&d, std::max<size_t>(n, 1) * sizeof(T)));
  const cudaError_t e = cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    cudaFree(d);
    ZK_CUDA(e);
  }
  return static_cast<T*>(d);
}
void checkErrWord(zk_context* ctx) {
  uint32_t devErr = 0;
  ZK_CUDA(cudaMemcpyAsync(&devErr, ctx->dErr, 4, cudaMemcpyDeviceToHost, ctx->stream));
  ZK_CUDA(cudaStreamSynchronize(ctx->stream));
  if (devErr) throw fail(ZK_ERR_DEVICE_TIMEOUT, "a tensor-core wait gave up (error %u)", devErr);
}
void scaleFromHost(zk_surrogate* s, const float* x, const float* y, size_t n) {
  float sc[32];
  zk::surrogateScaleFrom(s->S, x, y, n, sc);
  ZK_CUDA(cudaMemcpyAsync(s->S.scale, sc, sizeof sc, cudaMemcpyHostToDevice, s->ctx->stream));
  ZK_CUDA(cudaStreamSynchronize(s->ctx->stream));
}
}  // namespace

extern "C" {

zk_status zk_surrogate_create(zk_context* ctx, uint32_t seed, zk_surrogate** out) {
  try {
    requireCtx(ctx);
    if (!out) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    auto s = std::make_unique<zk_surrogate>();
    s->ctx = ctx;
    const cudaError_t e = zk::surrogateCreate(s->S, ctx->stream, ctx->dErr, seed);
    if (e != cudaSuccess) {
      zk::surrogateFree(s->S);
      ZK_CUDA(e);
    }
    *out = s.release();
    return ZK_OK;
  } catch (const Failure& f) {
    return record(ctx, f);
  }
}

void zk_surrogate_destroy(zk_surrogate* s) {
  if (!s) return;
  if (s->ctx) cudaSetDevice(s->ctx->device);
  zk::surrogateFree(s->S);
  delete s;
}

zk_status zk_surrogate_train(zk_surrogate* s, const float* x, const float* y, size_t n, uint32_t epochs, uint32_t batch, float lr,
                             float weight_decay, float* loss_per_epoch) {
  zk_context* ctx = s ? s->ctx : nullptr;
  float *dx = nullptr, *dy = nullptr;
  try {
    ctx = ctxOf(s);
    if (!x || !y || n == 0 || batch == 0) throw fail(ZK_ERR_INVALID_ARGUMENT, "empty training set or batch");
    if (!s->S.scaled) scaleFromHost(s, x, y, n);
    dx = toDevice(x, n * zk::kIn, ctx->stream);
    dy = toDevice(y, n, ctx->stream);
    ZK_CUDA(cudaMemsetAsync(ctx->dErr, 0, 4, ctx->stream));
    for (uint32_t e = 0; e < epochs; ++e) {
      double loss = 0.0;
      ZK_CUDA(zk::surrogateEpoch(s->S, dx, dy, n, batch, lr, weight_decay, true, &loss));
      if (loss_per_epoch) loss_per_epoch[e] = static_cast<float>(loss);
    }
    checkErrWord(ctx);
    cudaFree(dx), cudaFree(dy);
    return ZK_OK;
  } catch (const Failure& f) {
    if (dx) cudaFree(dx);
    if (dy) cudaFree(dy);
    return record(ctx, f);
  }
}

zk_status zk_surrogate_predict(zk_surrogate* s, const float* x, size_t n, float* y) {
  zk_context* ctx = s ? s->ctx : nullptr;
  float *dx = nullptr, *dy = nullptr;
  try {
    ctx = ctxOf(s);
    if (!x || !y) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0) return ZK_OK;
    dx = toDevice(x, n * zk::kIn, ctx->stream);
    ZK_CUDA(cudaMalloc(&dy, n * 4));
    ZK_CUDA(cudaMemsetAsync(ctx->dErr, 0, 4, ctx->stream));
    ZK_CUDA(zk::surrogatePredict(s->S, dx, n, dy));
    ZK_CUDA(cudaMemcpyAsync(y, dy, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    checkErrWord(ctx);
    cudaFree(dx), cudaFree(dy);
    return ZK_OK;
  } catch (const Failure& f) {
    if (dx) cudaFree(dx);
    if (dy) cudaFree(dy);
    return record(ctx, f);
  }
}

zk_status zk_surrogate_gradients(zk_surrogate* s, const float* x, const float* y, size_t n, float* loss, float* grads) {
  zk_context* ctx = s ? s->ctx : nullptr;
  float *dx = nullptr, *dy = nullptr;
  try {
    ctx = ctxOf(s);
    if (!x || !y || !grads || n == 0) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument or empty set");
    if (n > (1u << 20)) throw fail(ZK_ERR_INVALID_ARGUMENT, "gradients of at most 2^20 rows (one batch)");
    if (!s->S.scaled) scaleFromHost(s, x, y, n);
    dx = toDevice(x, n * zk::kIn, ctx->stream);
    dy = toDevice(y, n, ctx->stream);
    ZK_CUDA(cudaMemsetAsync(ctx->dErr, 0, 4, ctx->stream));
    double l = 0.0;
    ZK_CUDA(zk::surrogateEpoch(s->S, dx, dy, n, static_cast<uint32_t>(n), 0.0f, 0.0f, false, &l));
    ZK_CUDA(cudaMemcpyAsync(grads, s->S.grad, zk::SurrogateState::kParams * 4, cudaMemcpyDeviceToHost, ctx->stream));
    checkErrWord(ctx);
    if (loss) *loss = static_cast<float>(l);
    cudaFree(dx), cudaFree(dy);
    return ZK_OK;
  } catch (const Failure& f) {
    if (dx) cudaFree(dx);
    if (dy) cudaFree(dy);
    return record(ctx, f);
  }
}

zk_status zk_surrogate_features(zk_context* ctx, const float* factors, uint32_t nA, uint32_t nR, uint32_t nP, const float* times,
                                const zk_surrogate_trade* trades, uint32_t nTr, const int32_t* resets, const float* periods,
                                const float* bonds, float* X) {
  void* d = nullptr;
  try {
    requireCtx(ctx);
    if (!factors || !times || !trades || !resets || !periods || !X) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    const size_t plane = static_cast<size_t>(nR) * nP, nf = (2 + nA) * plane, rows = plane * nTr;
    for (uint32_t t = 0; t < nTr; ++t)
      if (trades[t].kind > 2) throw fail(ZK_ERR_INVALID_ARGUMENT, "trade %u: kind %u", t, trades[t].kind);
    for (size_t i = 0; i < static_cast<size_t>(nTr) * nR; ++i)
      if (resets[i] >= static_cast<int32_t>(nR)) throw fail(ZK_ERR_INVALID_ARGUMENT, "reset index beyond the reporting dates");
    const size_t o1 = (nf * 4 + 255) / 256 * 256, o2 = o1 + (nR * 4 + 255) / 256 * 256, o3 = o2 + (nTr * 32 + 255) / 256 * 256;
    const size_t o4 = o3 + (nTr * nR * 4 + 255) / 256 * 256, o4b = o4 + (nTr * nR * 8 + 255) / 256 * 256;
    const size_t o5 = o4b + (bonds ? (nTr * nR * 16 + 255) / 256 * 256 : 0);
    ZK_CUDA(cudaMalloc(&d, o5 + std::max<size_t>(rows, 1) * 64));
    unsigned char* b = static_cast<unsigned char*>(d);
    ZK_CUDA(cudaMemcpyAsync(b, factors, nf * 4, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(b + o1, times, nR * 4, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(b + o2, trades, nTr * 32, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(b + o3, resets, nTr * nR * 4, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(b + o4, periods, nTr * nR * 8, cudaMemcpyHostToDevice, ctx->stream));
    if (bonds) ZK_CUDA(cudaMemcpyAsync(b + o4b, bonds, nTr * nR * 16, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(zk::surrogateFeatures(reinterpret_cast<const float*>(b), nA, nR, nP, reinterpret_cast<const float*>(b + o1),
                                  reinterpret_cast<const zk::SurrogateTrade*>(b + o2), reinterpret_cast<const int32_t*>(b + o3),
                                  reinterpret_cast<const float*>(b + o4), bonds ? reinterpret_cast<const float*>(b + o4b) : nullptr, 0,
                                  rows, reinterpret_cast<float*>(b + o5), ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(X, b + o5, rows * 64, cudaMemcpyDeviceToHost, ctx->stream));
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
    ZK_CUDA(cudaFree(d));
    return ZK_OK;
  } catch (const Failure& f) {
    if (d) cudaFree(d);
    return record(ctx, f);
  }
}

zk_status zk_surrogate_book(zk_surrogate* s, const float* factors, uint32_t nA, uint32_t nR, uint32_t nP, const float* times,
                            const zk_surrogate_trade* trades, uint32_t nTr, const int32_t* resets, const float* periods,
                            const float* bonds, uint32_t num_netting_sets, const float* csa, const uint32_t* call_index,
                            double* exposure, float* netted_out, uint32_t paths_out, float* ms) {
  zk_context* ctx = s ? s->ctx : nullptr;
  void* d = nullptr;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  try {
    ctx = ctxOf(s);
    if (!factors || !times || !trades || !resets || !periods || !exposure) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    if (paths_out > nP || (paths_out && !netted_out)) throw fail(ZK_ERR_INVALID_ARGUMENT, "paths_out beyond the paths");
    if (csa && !call_index) throw fail(ZK_ERR_INVALID_ARGUMENT, "a CSA needs the margin-call index of every date");
    if (csa)
      for (uint32_t j = 0; j < nR; ++j)
        if (call_index[j] > j || j - call_index[j] >= 32u) throw fail(ZK_ERR_INVALID_ARGUMENT, "margin-call date %u of date %u", call_index[j], j);
    for (uint32_t t = 0; t < nTr; ++t) {
      if (trades[t].kind > 2) throw fail(ZK_ERR_INVALID_ARGUMENT, "trade %u: kind %u", t, trades[t].kind);
      if (trades[t].netting_set >= num_netting_sets) throw fail(ZK_ERR_INVALID_ARGUMENT, "trade %u: netting set beyond the count", t);
    }
    for (size_t i = 0; i < static_cast<size_t>(nTr) * nR; ++i)
      if (resets[i] >= static_cast<int32_t>(nR)) throw fail(ZK_ERR_INVALID_ARGUMENT, "reset index beyond the reporting dates");
    const size_t plane = static_cast<size_t>(nR) * nP, nf = (2 + nA) * plane;
    const uint32_t chunk = static_cast<uint32_t>(std::max<size_t>(1, (size_t(1) << 23) / std::max<size_t>(plane, 1)));
    const size_t chunkRows = plane * std::min(chunk, std::max(nTr, 1u));
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    const size_t oF = take(nf * 4), oT = take(nR * 4), oTr = take(nTr * 32), oR = take(nTr * nR * 4), oP = take(nTr * nR * 8);
    const size_t oB = take(bonds ? nTr * nR * 16 : 16);
    const size_t oC = take(csa ? num_netting_sets * 16 : 16), oI = take(csa ? nR * 4 : 16);
    const size_t oN = take(static_cast<size_t>(num_netting_sets) * plane * 4), oE = take(num_netting_sets * nR * 16);
    const size_t oX = take(chunkRows * 64), oY = take(chunkRows * 4);
    ZK_CUDA(cudaMalloc(&d, off));
    unsigned char* b = static_cast<unsigned char*>(d);
    ZK_CUDA(cudaMemcpyAsync(b + oF, factors, nf * 4, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(b + oT, times, nR * 4, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(b + oTr, trades, nTr * 32, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(b + oR, resets, nTr * nR * 4, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(b + oP, periods, nTr * nR * 8, cudaMemcpyHostToDevice, ctx->stream));
    if (bonds) ZK_CUDA(cudaMemcpyAsync(b + oB, bonds, nTr * nR * 16, cudaMemcpyHostToDevice, ctx->stream));
    if (csa) {
      ZK_CUDA(cudaMemcpyAsync(b + oC, csa, num_netting_sets * 16, cudaMemcpyHostToDevice, ctx->stream));
      ZK_CUDA(cudaMemcpyAsync(b + oI, call_index, nR * 4, cudaMemcpyHostToDevice, ctx->stream));
    }
    ZK_CUDA(cudaMemsetAsync(b + oN, 0, static_cast<size_t>(num_netting_sets) * plane * 4, ctx->stream));
    ZK_CUDA(cudaMemsetAsync(ctx->dErr, 0, 4, ctx->stream));
    for (auto& e : ev) ZK_CUDA(cudaEventCreate(&e));
    ZK_CUDA(cudaEventRecord(ev[0], ctx->stream));
    ZK_CUDA(zk::surrogateBook(s->S, reinterpret_cast<const float*>(b + oF), nA, nR, nP, reinterpret_cast<const float*>(b + oT),
                              reinterpret_cast<const zk::SurrogateTrade*>(b + oTr), nTr, reinterpret_cast<const int32_t*>(b + oR),
                              reinterpret_cast<const float*>(b + oP), bonds ? reinterpret_cast<const float*>(b + oB) : nullptr,
                              reinterpret_cast<float*>(b + oN), reinterpret_cast<float*>(b + oX),
                              reinterpret_cast<float*>(b + oY), chunk));
    ZK_CUDA(cudaEventRecord(ev[1], ctx->stream));
    if (csa)
      ZK_CUDA(zk::surrogateCollateral(reinterpret_cast<float*>(b + oN), reinterpret_cast<const float*>(b + oC),
                                      reinterpret_cast<const uint32_t*>(b + oI), num_netting_sets, nR, nP, ctx->stream));
    ZK_CUDA(zk::surrogateExposure(reinterpret_cast<const float*>(b + oN), reinterpret_cast<const float*>(b + oF), num_netting_sets, nR,
                                  nP, reinterpret_cast<double*>(b + oE), ctx->stream));
    ZK_CUDA(cudaEventRecord(ev[2], ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(exposure, b + oE, num_netting_sets * nR * 16, cudaMemcpyDeviceToHost, ctx->stream));
    if (paths_out)
      ZK_CUDA(cudaMemcpy2DAsync(netted_out, paths_out * 4, b + oN, nP * 4, paths_out * 4, static_cast<size_t>(num_netting_sets) * nR,
                                cudaMemcpyDeviceToHost, ctx->stream));
    checkErrWord(ctx);
    if (ms) {
      ZK_CUDA(cudaEventElapsedTime(&ms[0], ev[0], ev[1]));
      ZK_CUDA(cudaEventElapsedTime(&ms[1], ev[1], ev[2]));
    }
    for (auto& e : ev) cudaEventDestroy(e);
    ZK_CUDA(cudaFree(d));
    return ZK_OK;
  } catch (const Failure& f) {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (d) cudaFree(d);
    return record(ctx, f);
  }
}

zk_status zk_surrogate_params(zk_surrogate* s, float* get, const float* set, float* scaling_get, const float* scaling_set) {
  zk_context* ctx = s ? s->ctx : nullptr;
  try {
    ctx = ctxOf(s);
    const size_t P = zk::SurrogateState::kParams;
    if (set) {
      ZK_CUDA(cudaMemcpyAsync(s->S.p, set, P * 4, cudaMemcpyHostToDevice, ctx->stream));
      ZK_CUDA(zk::surrogateSync(s->S));
    }
    if (scaling_set) {
      ZK_CUDA(cudaMemcpyAsync(s->S.scale, scaling_set, 32 * 4, cudaMemcpyHostToDevice, ctx->stream));
      s->S.yMean = scaling_set[32], s->S.yScale = scaling_set[33], s->S.scaled = true;
    }
    if (get) ZK_CUDA(cudaMemcpyAsync(get, s->S.p, P * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (scaling_get) ZK_CUDA(cudaMemcpyAsync(scaling_get, s->S.scale, 32 * 4, cudaMemcpyDeviceToHost, ctx->stream));
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
    if (scaling_get) scaling_get[32] = s->S.yMean, scaling_get[33] = s->S.yScale;
    return ZK_OK;
  } catch (const Failure& f) {
    return record(ctx, f);
  }
}

zk_status zk_run_plan_f64(zk_context* ctx, const zk_plan_view_f64* plan, const double* normals, size_t streams, zk_output_f64* out,
                          double* rows) {
  return runInjected<double>(ctx, plan, normals, streams, out, rows);
}

zk_status zk_run_plan_injected(zk_context* ctx, const zk_plan_view* plan, const double* normals, size_t streams, zk_output* out,
                               float* rows) {
  return runInjected<float>(ctx, plan, normals, streams, out, rows);
}

zk_status zk_factor_paths_f64(zk_context* ctx, const zk_plan_view_f64* plan, const double* normals, size_t streams, double* out,
                              size_t out_len) {
  try {
    requireCtx(ctx);
    if (!plan || !out) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    auto B = build<double>(ctx, {viewOf(*plan)}, false, normals, streams);
    const auto& L = B->launches.front();
    const size_t n = static_cast<size_t>(2 + L.sc.nA) * L.sc.nT * L.sc.nP;
    if (out_len != n) throw fail(ZK_ERR_INVALID_ARGUMENT, "out must hold (2 + nA) nT nP = %zu values", n);
    upload(*B, ctx, true, normals, streams);
    ZK_CUDA(cudaMemsetAsync(ctx->dErr, 0, 4, ctx->stream));
    ZK_CUDA(launchSimulate<double>(L.sc, L.cb, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(out, B->base + L.cubeOff, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
    return ZK_OK;
  } catch (const Failure& f) {
    return record(ctx, f);
  }
}

// ---- device-resident batches ----
zk_status zk_batch_create(zk_context* ctx, const zk_plan_view* plans, size_t n, zk_batch** out) {
  try {
    requireCtx(ctx);
    if (!plans || !out || n == 0) throw fail(ZK_ERR_INVALID_ARGUMENT, "null or empty plan list");
    std::vector<View<float>> views;
    for (size_t i = 0; i < n; ++i) views.push_back(viewOf(plans[i]));
    auto b = std::make_unique<zk_batch>();
    b->b = build<float>(ctx, views, false, nullptr, 0);
    upload(*b->b, ctx, false, nullptr, 0);
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = b.release();
    return ZK_OK;
  } catch (const Failure& f) {
    return record(ctx, f);
  }
}

zk_status zk_batch_execute(zk_batch* b) {
  if (!b) return ZK_ERR_INVALID_ARGUMENT;
  try {
    ZK_CUDA(cudaSetDevice(b->b->ctx->device));
    if (!b->tuned) {
      // first execute: time the tile shapes on this batch, keep the fastest (they shape the term-by-term launches
      // only: a batch entirely on the basis kernel keeps the default)
      bool termByTerm = false;
      for (const auto& L : b->b->launches) termByTerm = termByTerm || L.basisCount < L.planIdx.size();
      if (termByTerm) autotune(*b->b);
      b->tuned = true;
    }
    if (!b->eager && (!b->graph || b->graphPpt != b->b->ppt) && !captureExecute(b)) b->eager = true;
    if (b->eager) {
      execute(*b->b);
    } else {
      ZK_CUDA(cudaGraphLaunch(b->graph, b->b->ctx->stream));
      b->b->timed = true;
    }
    return ZK_OK;
  } catch (const Failure& f) {
    return record(b->b->ctx, f);
  }
}

zk_status zk_batch_set_tile_paths(zk_batch* b, uint64_t tile_paths) {
  if (!b) return ZK_ERR_INVALID_ARGUMENT;
  try {
    const uint64_t ppt = tile_paths / kTile;
    if (tile_paths % kTile || (ppt != 1 && ppt != 2 && ppt != 4))
      throw fail(ZK_ERR_INVALID_ARGUMENT, "tile_paths must be 128, 256 or 512");
    for (const auto& L : b->b->launches)
      if (revalueSmemBytes(L.stateWordsMax, L.perTrade, false, static_cast<int>(ppt)) > 200 * 1024)
        throw fail(ZK_ERR_UNSUPPORTED, "this tile shape needs more shared memory than a CTA has");
    ZK_CUDA(cudaSetDevice(b->b->ctx->device));
    setTileShape(*b->b, static_cast<int>(ppt));
    b->tuned = true;
    return ZK_OK;
  } catch (const Failure& f) {
    return record(b->b->ctx, f);
  }
}

zk_status zk_batch_timings(const zk_batch* b, float* ms4) {
  if (!b || !ms4) return ZK_ERR_INVALID_ARGUMENT;
  try {
    Batch<float>& B = *b->b;
    ZK_CUDA(cudaEventSynchronize(B.ev[4]));
    for (int k = 0; k < 4; ++k) ZK_CUDA(cudaEventElapsedTime(&B.ms[k], B.ev[k], B.ev[k + 1]));
    for (int i = 0; i < 4; ++i) ms4[i] = B.ms[i];
    return ZK_OK;
  } catch (const Failure& f) {
    return record(b->b->ctx, f);
  }
}

zk_status zk_batch_read(zk_batch* b, zk_output* outs) {
  if (!b || !outs) return ZK_ERR_INVALID_ARGUMENT;
  try {
    checkOutputs(*b->b, outs, false);
    readOutputs(*b->b, outs);
    return ZK_OK;
  } catch (const Failure& f) {
    return record(b->b->ctx, f);
  }
}

zk_status zk_batch_info_get(const zk_batch* b, zk_batch_info* info) {
  if (!b || !info) return ZK_ERR_INVALID_ARGUMENT;
  const Batch<float>& B = *b->b;
  std::memset(info, 0, sizeof *info);
  info->num_plans = B.plans.size();
  info->num_launch_groups = B.launches.size();
  info->num_paths = B.plans[0].nP;
  info->num_dates = B.plans[0].nT;
  for (const auto& P : B.plans) {
    info->num_terms += P.nTerms;
    info->term_evaluations += P.termEvals;
    info->exp_evaluations += P.expEvals;
    info->table_bytes += P.nIdx * 4 + P.nTerms * 32 + static_cast<uint64_t>(P.nT) * 96 + P.nReq * 32;
    info->row_bytes += static_cast<uint64_t>(P.nR) * P.nP * 4;
  }
  uint64_t kernels = (B.waved ? 0 : 2) + B.im.size();  // reduce, row statistics, one nested-margin launch per margin plan
  auto revalueLaunches = [&](const Batch<float>::Launch& L, size_t first, size_t count) {  // as launchRevalues
    count = std::min(count, L.planIdx.size() - first);
    uint64_t k = 0;
    if (first < L.basisCount && count > 0) {
      const size_t last = std::min(first + count, L.basisCount);
      ++k, count -= last - first, first = last;
    }
    if (count == 0) return k;
    const size_t at = std::min(count, L.splitAt > first ? L.splitAt - first : 0);
    const bool split = L.lean && !L.perTrade && !B.sink && B.ppt > 1 && at < count;
    return k + (split && at > 0 ? 2 : 1);
  };
  for (const auto& L : B.launches) {
    info->num_basis_netting_sets += L.basisCount;
    for (const auto& G : L.groups) {
      const BasisImage& I = G.img;
      info->basis_columns += I.columns, info->basis_terms += I.linearTerms;
      info->basis_bytes += I.dates.size() * 4 + I.kgs.size() * sizeof(BasisKg) + (I.options.size() + I.fixings.size() + I.scale.size()) * 4 +
                           I.chunks.size() * 4 + I.blob.size() * 2 + sizeof(BasisArgs);
    }
    if (!B.waved) {
      kernels += 1 + revalueLaunches(L, 0, L.planIdx.size());  // simulate, then the revalue launches
      continue;
    }
    kernels += 1;  // simulate; per wave its revalue launches, a reduce and (with requests) row statistics
    for (const auto& w : L.waves) kernels += revalueLaunches(L, w.first, w.count) + 1 + (w.rowCount ? 1 : 0);
  }
  info->kernels_per_execute = kernels;
  info->num_waves = 0;
  for (const auto& L : B.launches) info->num_waves += B.waved ? L.waves.size() : 1;
  info->tile_paths = static_cast<uint64_t>(kTile) * B.ppt;
  info->graph_replay = b->graph && !b->eager && b->graphPpt == B.ppt ? 1u : 0u;
  return ZK_OK;
}

void zk_batch_destroy(zk_batch* b) {
  if (!b) return;
  if (b->b && b->b->ctx) {
    cudaSetDevice(b->b->ctx->device);
    cudaStreamSynchronize(b->b->ctx->stream);
  }
  delete b;
}

}  // extern "C"

// ================================================================================================
// Entry point without device allocation.
//
// Some callers cannot call cudaMalloc: a host application that hands all device memory to its own
// pooling allocator up front (a serving process, a framework's caching allocator), or a plug-in that
// runs inside such a host and is not allowed to allocate behind its back.  zk_run_plan_noalloc runs the
// same kernels as zk_run_plan for one plan, but every device buffer it needs (the plan tables, the factor
// cube, the per-tile partials, the path-view rows, the job tables, the error word) lives in the
// file-scope array below, which the CUDA module reserves when it loads on a device.  It creates no
// context, stream or event and allocates no device memory; the host builds its upload image in ordinary
// host memory.
static __device__ __align__(256) unsigned char zkNoAllocScratch[ZK_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex gNoAllocMutex;
unsigned char* gNoAllocBase[kNoAllocMaxDevices] = {};

// The device address of zkNoAllocScratch on `device` (current), looked up once per device.  In host code
// the array's name is only a stand-in; the kernels need this address.  With lazy module loading (the CUDA
// default) the lookup is what loads the module on the device and so reserves the array: a host that gives all
// free device memory to its own pool must make its first call before that.
unsigned char* noAllocBase(int device) {
  std::lock_guard<std::mutex> lock(gNoAllocMutex);
  if (!gNoAllocBase[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, zkNoAllocScratch);
    if (e == cudaErrorMemoryAllocation)
      throw fail(ZK_ERR_OUT_OF_MEMORY, "loading the library's kernels and their %u-byte no-alloc array on device %d: out of memory "
                                       "(make the first call before the host's pool takes the device memory)",
                 static_cast<unsigned>(ZK_NOALLOC_SCRATCH_BYTES), device);
    if (e != cudaSuccess) throw fail(ZK_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch: %s", cudaGetErrorString(e));
    gNoAllocBase[device] = static_cast<unsigned char*>(p);
  }
  return gNoAllocBase[device];
}

// Makes `device` current for the lifetime of the guard and gives the caller's current device back on every exit.
struct DeviceGuard {
  int saved = -1;
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
    ZK_CUDA(cudaSetDevice(device));
  }
  ~DeviceGuard() {
    if (saved >= 0) cudaSetDevice(saved);
  }
};

}  // namespace

extern "C" zk_status zk_run_plan_noalloc(int device, void* stream, const zk_plan_view* plan, zk_output* out, char* err,
                                         size_t err_len) {
  auto report = [&](const Failure& f) {
    if (err && err_len) {
      std::strncpy(err, f.message.c_str(), err_len - 1);
      err[err_len - 1] = 0;
    }
    return f.status;
  };
  try {
    if (!plan || !out) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw fail(ZK_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= n || device >= kNoAllocMaxDevices) throw fail(ZK_ERR_INVALID_ARGUMENT, "device %d out of range", device);
    auto B = build<float>(nullptr, {viewOf(*plan)}, false, nullptr, 0);
    checkOutputs(*B, out, false);
    const size_t errOff = alignUp(B->totalBytes);
    if (errOff + 256 > static_cast<size_t>(ZK_NOALLOC_SCRATCH_BYTES))
      throw fail(ZK_ERR_INVALID_ARGUMENT, "the plan needs %zu bytes of device scratch; zk_run_plan_noalloc has %zu (use zk_run_plan)",
                 errOff + 256, static_cast<size_t>(ZK_NOALLOC_SCRATCH_BYTES));
    DeviceGuard guard(device);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    B->base = noAllocBase(device);
    uint32_t* dErr = reinterpret_cast<uint32_t*>(B->base + errOff);
    fillImage(*B, nullptr, 0);
    ZK_CUDA(cudaMemcpyAsync(B->base, B->image.data(), B->inputBytes, cudaMemcpyHostToDevice, s));
    ZK_CUDA(cudaMemsetAsync(dErr, 0, 4, s));  // the array keeps the previous call's contents
    const uintptr_t base = reinterpret_cast<uintptr_t>(B->base);
    // The kernels and variants of zk_run_plan (launchRevalues), all on the caller's stream.
    for (const auto& L : B->launches) ZK_CUDA(launchSimulate<float>(L.sc, L.cb, s));
    for (const auto& L : B->launches) launchRevalues(*B, L, base, s, nullptr, nullptr, nullptr);
    for (const auto& M : B->im) ZK_CUDA(launchNestedIm<float>(M, s));
    ZK_CUDA(launchReduce<float>(reinterpret_cast<const ReduceJob<float>*>(base + B->reduceOff), static_cast<uint32_t>(B->plans.size()),
                                B->maxReduceN, B->ppt, s));
    ZK_CUDA(launchRowStats<float>(reinterpret_cast<const RowJob<float>*>(base + B->rowOff), B->numRowJobs, dErr, s));
    std::vector<unsigned char> host(B->outBytes);
    uint32_t devErr = 0;
    ZK_CUDA(cudaMemcpyAsync(host.data(), B->base + B->outBegin, B->outBytes, cudaMemcpyDeviceToHost, s));
    ZK_CUDA(cudaMemcpyAsync(&devErr, dErr, 4, cudaMemcpyDeviceToHost, s));
    ZK_CUDA(cudaStreamSynchronize(s));
    throwDeviceError(devErr);
    const auto& P = B->plans[0];
    const auto& D = B->dev[0];
    const float* sums = reinterpret_cast<const float*>(host.data() + (D.sums - B->outBegin));
    const float* vals = reinterpret_cast<const float*>(host.data() + (D.values - B->outBegin));
    std::memcpy(out->sums, sums, static_cast<size_t>(P.nT) * P.nS * sizeof(float));
    std::memcpy(out->values, vals, std::max<uint32_t>(P.v.num_outputs, 1) * sizeof(float));
    return ZK_OK;
  } catch (const Failure& f) {
    return report(f);
  } catch (const std::exception& e) {
    return report(fail(ZK_ERR_CUDA, "%s", e.what()));
  }
}

// ---- failure injection for tests ----
extern "C" zk_status zk_debug_inject(zk_context* ctx, uint32_t what, uint64_t value) {
  if (!ctx) return ZK_ERR_INVALID_ARGUMENT;
  switch (what) {
    case ZK_INJECT_FAIL_LAUNCH:
      ctx->failAtLaunch = value, ctx->launchCount = 0;
      return ZK_OK;
    case ZK_INJECT_ROW_ROUNDS:
      if (value > 16) return record(ctx, fail(ZK_ERR_INVALID_ARGUMENT, "row-statistics rounds %llu above 16",
                                              static_cast<unsigned long long>(value)));
      ctx->rowRounds = static_cast<uint32_t>(value);
      return ZK_OK;
    default:
      return record(ctx, fail(ZK_ERR_INVALID_ARGUMENT, "unknown injection %u", what));
  }
}

// ---- nested exposure: inner paths on the GPU ----
struct zk_nest {
  zk_context* ctx = nullptr;
  unsigned char* dmem = nullptr;  // the program and the outer states
  NestArgs args{};
  size_t numScenarios = 0;
  unsigned char* djobs = nullptr;  // a round's jobs and payoffs, grown on demand
  size_t jobsBytes = 0;
  size_t dmemBytes = 0;
  ~zk_nest() {  // the blocks go back to the context for the next nest
    giveBlock(ctx, dmem, dmemBytes);
    giveBlock(ctx, djobs, jobsBytes);
  }
};

zk_status zk_nest_create(zk_context* ctx, const double* model, size_t model_len, const double* periods, size_t n_periods,
                         const double* terminals, size_t n_terminals, double t, const double* x, const double* spot,
                         const double* known, size_t n_slots, size_t n_scenarios, zk_nest** out) {
  try {
    requireCtx(ctx);
    if (!model || !x || !out || (n_periods && !periods) || (n_terminals && !terminals)) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    if (n_scenarios == 0) throw fail(ZK_ERR_INVALID_ARGUMENT, "no scenarios");
    if (n_slots > kMaxNestSlots) throw fail(ZK_ERR_UNSUPPORTED, "at most %u swaps with a running coupon", kMaxNestSlots);
    zk::host::Model m;
    zk::host::NestProgram P;
    try {
      m = zk::host::decodeModel(model, model_len);
      P = zk::host::nestProgram(m, periods, n_periods, terminals, n_terminals, t);
    } catch (const std::exception& e) {
      throw fail(ZK_ERR_INVALID_ARGUMENT, "%s", e.what());
    }
    const uint32_t nA = static_cast<uint32_t>(P.nA);
    if (nA > 0 && !spot) throw fail(ZK_ERR_INVALID_ARGUMENT, "null spot");
    if (n_slots > 0 && !known) throw fail(ZK_ERR_INVALID_ARGUMENT, "null known fixings");
    for (size_t i = 0; i < n_periods; ++i)
      if (!(periods[6 * i + 5] >= 0.0) || periods[6 * i + 5] >= static_cast<double>(n_slots) || !(periods[6 * i + 2] > 0.0))
        throw fail(ZK_ERR_INVALID_ARGUMENT, "period %zu: slot beyond n_slots or non-positive accrual", i);
    for (size_t f = 0; f < n_terminals; ++f)
      if (!(terminals[6 * f] >= 0.0) || terminals[6 * f] >= static_cast<double>(nA))
        throw fail(ZK_ERR_INVALID_ARGUMENT, "terminal flow %zu: asset beyond the model's assets", f);
    auto N = std::make_unique<zk_nest>();
    N->ctx = ctx, N->numScenarios = n_scenarios;
    // One device block: coef | opBegin | ops | periods | terminals | chol | fixToday | x0 | spot0 | fix0.
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off = alignUp(off + std::max<size_t>(bytes, 16)); return o; };
    const size_t oCoef = take(P.coef.size() * 8), oBegin = take(P.begin.size() * 4), oOps = take(P.ops.size() * 4);
    const size_t oPer = take(P.periods.size() * 8), oTerm = take(P.terminals.size() * 8), oChol = take(P.chol.size() * 8);
    const size_t oToday = take(P.fixToday.size() * 4), oX = take(n_scenarios * 8), oSpot = take(n_scenarios * nA * 8);
    const size_t oFix = take(n_scenarios * n_slots * 8);
    std::vector<unsigned char> img(off, 0);
    auto put = [&](size_t o, const void* src, size_t bytes) { if (bytes) std::memcpy(img.data() + o, src, bytes); };
    put(oCoef, P.coef.data(), P.coef.size() * 8), put(oBegin, P.begin.data(), P.begin.size() * 4);
    put(oOps, P.ops.data(), P.ops.size() * 4), put(oPer, P.periods.data(), P.periods.size() * 8);
    put(oTerm, P.terminals.data(), P.terminals.size() * 8), put(oChol, P.chol.data(), P.chol.size() * 8);
    put(oToday, P.fixToday.data(), P.fixToday.size() * 4), put(oX, x, n_scenarios * 8);
    put(oSpot, spot, n_scenarios * nA * 8), put(oFix, known, n_scenarios * n_slots * 8);
    N->dmem = takeBlock(ctx, off, N->dmemBytes);
    if (!N->dmem) throw fail(ZK_ERR_OUT_OF_MEMORY, "nest: %zu bytes of device memory", off);
    ZK_CUDA(cudaMemcpyAsync(N->dmem, img.data(), off, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
    unsigned char* b = N->dmem;
    NestArgs& A = N->args;
    A.coef = reinterpret_cast<const double*>(b + oCoef), A.opBegin = reinterpret_cast<const uint32_t*>(b + oBegin);
    A.ops = reinterpret_cast<const uint32_t*>(b + oOps), A.periods = reinterpret_cast<const double*>(b + oPer);
    A.terminals = reinterpret_cast<const double*>(b + oTerm), A.chol = reinterpret_cast<const double*>(b + oChol);
    A.fixToday = reinterpret_cast<const uint32_t*>(b + oToday), A.x0 = reinterpret_cast<const double*>(b + oX);
    A.spot0 = reinterpret_cast<const double*>(b + oSpot), A.fix0 = reinterpret_cast<const double*>(b + oFix);
    A.numEvents = static_cast<uint32_t>(P.times.size()), A.nA = nA, A.numSlots = static_cast<uint32_t>(n_slots);
    A.numFixToday = static_cast<uint32_t>(P.fixToday.size());
    *out = N.release();
    return ZK_OK;
  } catch (const Failure& f) {
    return record(ctx, f);
  }
}

zk_status zk_nest_run(zk_nest* nest, const uint64_t* scenario, const uint64_t* seed, const uint64_t* paths, size_t num_jobs, double* out) {
  if (!nest) return ZK_ERR_INVALID_ARGUMENT;
  zk_context* ctx = nest->ctx;
  try {
    requireCtx(ctx);
    if (num_jobs == 0) return ZK_OK;
    if (!scenario || !seed || !paths || !out) throw fail(ZK_ERR_INVALID_ARGUMENT, "null argument");
    if (num_jobs > 0xFFFFFFFFull) throw fail(ZK_ERR_INVALID_ARGUMENT, "too many jobs");
    std::vector<unsigned long long> start(num_jobs);
    unsigned long long total = 0;
    for (size_t k = 0; k < num_jobs; ++k) {
      if (scenario[k] >= nest->numScenarios) throw fail(ZK_ERR_INVALID_ARGUMENT, "job %zu: scenario beyond the outer sample", k);
      start[k] = total;
      total += paths[k];
    }
    if (total == 0) return ZK_OK;
    const size_t jobBytes = alignUp(num_jobs * 8);
    const size_t need = 3 * jobBytes + total * 8;
    if (nest->jobsBytes < need) {
      giveBlock(ctx, nest->djobs, nest->jobsBytes);
      nest->djobs = takeBlock(ctx, need, nest->jobsBytes);
      if (!nest->djobs) {
        nest->jobsBytes = 0;
        throw fail(ZK_ERR_OUT_OF_MEMORY, "nest: %zu bytes of device memory for a round", need);
      }
    }
    unsigned char* d = nest->djobs;
    ZK_CUDA(cudaMemcpyAsync(d, scenario, num_jobs * 8, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(d + jobBytes, seed, num_jobs * 8, cudaMemcpyHostToDevice, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(d + 2 * jobBytes, start.data(), num_jobs * 8, cudaMemcpyHostToDevice, ctx->stream));
    NestArgs A = nest->args;
    A.jobScenario = reinterpret_cast<const unsigned long long*>(d);
    A.jobSeed = reinterpret_cast<const unsigned long long*>(d + jobBytes);
    A.jobStart = reinterpret_cast<const unsigned long long*>(d + 2 * jobBytes);
    A.out = reinterpret_cast<double*>(d + 3 * jobBytes);
    A.totalPaths = total, A.numJobs = static_cast<uint32_t>(num_jobs);
    ZK_CUDA(launchNestInner(A, ctx->stream));
    ZK_CUDA(cudaMemcpyAsync(out, A.out, total * 8, cudaMemcpyDeviceToHost, ctx->stream));
    ZK_CUDA(cudaStreamSynchronize(ctx->stream));
    return ZK_OK;
  } catch (const Failure& f) {
    return record(ctx, f);
  }
}

zk_status zk_zero_bond_coefficients(const double* model, size_t model_len, const double* ts_te, size_t n, double* out) {
  if (!model || (n && (!ts_te || !out))) return ZK_ERR_INVALID_ARGUMENT;
  try {
    const auto m = zk::host::decodeModel(model, model_len);
    for (size_t i = 0; i < n; ++i) {
      const double ts = ts_te[2 * i], te = ts_te[2 * i + 1];
      out[3 * i] = m.hw.curve.discount(te) / m.hw.curve.discount(ts);
      out[3 * i + 1] = 0.5 * (m.hw.V(ts, te) - m.hw.V(0.0, te) + m.hw.V(0.0, ts));
      out[3 * i + 2] = m.hw.B(ts, te);
    }
    return ZK_OK;
  } catch (const std::exception&) {
    return ZK_ERR_INVALID_ARGUMENT;
  }
}

zk_status zk_nest_events(const zk_nest* nest, uint64_t* events) {
  if (!nest || !events) return ZK_ERR_INVALID_ARGUMENT;
  *events = nest->args.numEvents;
  return ZK_OK;
}

void zk_nest_destroy(zk_nest* nest) {
  if (!nest) return;
  cudaSetDevice(nest->ctx->device);
  cudaStreamSynchronize(nest->ctx->stream);  // nothing of the nest's may still run when its blocks are reused
  delete nest;
}
