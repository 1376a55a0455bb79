// ORACLE / TEST INFRASTRUCTURE ONLY.  Not part of the product: only tests/, the smoke check and
// bench.py's CPU-baseline leg load the library this file builds (oracle/_ref/libccr_ref.so).
//
// A C-ABI wrapper around the reference library (svr-net/zlatko, compiled unmodified from its own
// sources by oracle/Makefile).  It decodes the flat model / netting-set / options arrays of
// zlatko_b200/spec.py into the reference's C++ objects and exposes:
//   - gpu::compile (src/gpu/fused_exposure.cpp:214) and the plan's buffers;
//   - gpu::runFusedReference (src/gpu/fused_reference.cpp:628), the reference's FP32 CPU kernels;
//   - gpu::runAmcStates (src/gpu/fused_reference.cpp:609);
//   - gpu::summarise (src/gpu/fused_exposure.cpp:816);
//   - the FP64 ExposureEngine path (src/exposure/exposure_engine.cpp:50-81) either with its own
//     mt19937_64 normals or fed injected normals.  For the latter the ~45-line driver loop of
//     ScenarioGenerator::generate (src/models/scenario_generator.cpp:94-141) is restated below to
//     read the normals from a buffer; every model step, valuation, netting, collateral, profile
//     and CVA function it calls is the reference's own;
//   - the reference's CVA functions (src/cva/cva.cpp) and ccr::quantile (include/ccr/core/math.hpp:39).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <limits>
#include <vector>

#include "ccr/core/math.hpp"
#include "ccr/core/parallel.hpp"
#include "ccr/core/random.hpp"
#include "ccr/cva/cva.hpp"
#include "ccr/exposure/allocation.hpp"
#include "ccr/xva/xva.hpp"
#include "ccr/nested/adaptive_nested.hpp"
#include "ccr/nested/nested_exposure.hpp"
#include "ccr/exposure/collateral.hpp"
#include "ccr/exposure/exposure_engine.hpp"
#include "ccr/exposure/exposure_profile.hpp"
#include "ccr/gpu/fused_exposure.hpp"
#include "ccr/instruments/asset_forward.hpp"
#include "ccr/instruments/bermudan_swaption.hpp"
#include "ccr/instruments/european_option.hpp"
#include "ccr/instruments/interest_rate_swap.hpp"

using namespace ccr;

namespace {

struct Reader {
  const double* p;
  std::size_t n, i = 0;
  double next() {
    if (i >= n) throw std::invalid_argument("spec: truncated array");
    return p[i++];
  }
  std::size_t count() { return static_cast<std::size_t>(next()); }
};

std::shared_ptr<YieldCurve> readCurve(Reader& r) {
  const std::size_t n = r.count();
  std::vector<double> t(n), z(n);
  for (std::size_t k = 0; k < n; ++k) t[k] = r.next(), z[k] = r.next();
  return std::make_shared<YieldCurve>(t, z);
}

struct ModelSpec {
  std::shared_ptr<YieldCurve> curve;
  std::shared_ptr<HullWhite1F> hw;
  std::vector<std::shared_ptr<const LognormalAsset>> assets;
  std::vector<std::shared_ptr<const CirIntensity>> credits;
  std::vector<std::shared_ptr<const CreditCurve>> markets;
  Matrix correlation;
  SimulationConfig sim;
  std::vector<double> base;
};

ModelSpec readModel(const double* a, std::size_t n) {
  Reader r{a, n};
  if (r.next() != 7001.0) throw std::invalid_argument("model: bad magic");
  ModelSpec m;
  m.curve = readCurve(r);
  const double ha = r.next(), hs = r.next();
  m.hw = std::make_shared<HullWhite1F>(m.curve, ha, hs);
  const std::size_t nA = r.count();
  for (std::size_t k = 0; k < nA; ++k) {
    const double spot = r.next(), vol = r.next();
    auto carry = readCurve(r);
    m.assets.push_back(std::make_shared<LognormalAsset>("A" + std::to_string(k), spot, vol, carry));
  }
  const std::size_t nC = r.count();
  for (std::size_t k = 0; k < nC; ++k) {
    const double kappa = r.next(), theta = r.next(), xi = r.next(), y0 = r.next();
    const std::size_t sub = r.count(), nh = r.count();
    std::vector<double> pil(nh), haz(nh);
    for (std::size_t q = 0; q < nh; ++q) pil[q] = r.next(), haz[q] = r.next();
    auto market = std::make_shared<CreditCurve>(pil, haz);
    m.markets.push_back(market);
    m.credits.push_back(std::make_shared<CirIntensity>("C" + std::to_string(k), market, kappa, theta, xi, y0, sub));
  }
  const std::size_t F = r.count();
  if (F > 0) {
    m.correlation = Matrix(F, F);
    for (std::size_t i = 0; i < F; ++i)
      for (std::size_t j = 0; j < F; ++j) m.correlation(i, j) = r.next();
  }
  m.sim.numPaths = r.count();
  m.sim.seed = static_cast<std::uint64_t>(r.next());
  m.sim.antithetic = r.next() != 0.0;
  const std::size_t nb = r.count();
  for (std::size_t k = 0; k < nb; ++k) m.base.push_back(r.next());
  return m;
}

std::vector<double> readSchedule(Reader& r) {
  const std::size_t n = r.count();
  std::vector<double> s(n);
  for (auto& v : s) v = r.next();
  return s;
}

NettingSet readNettingSet(const double* a, std::size_t n) {
  Reader r{a, n};
  if (r.next() != 7002.0) throw std::invalid_argument("netting set: bad magic");
  NettingSet ns;
  ns.id = "ns";
  const std::size_t nt = r.count();
  for (std::size_t k = 0; k < nt; ++k) {
    const int type = static_cast<int>(r.next());
    const std::string id = "t" + std::to_string(k);
    auto dirOf = [](double pay) { return pay != 0.0 ? InterestRateSwap::Direction::PayFixed : InterestRateSwap::Direction::ReceiveFixed; };
    if (type == 0) {
      const double notional = r.next(), fixed = r.next(), pay = r.next();
      ns.trades.push_back(std::make_shared<InterestRateSwap>(id, notional, fixed, readSchedule(r), dirOf(pay)));
    } else if (type == 1) {
      const std::size_t asset = r.count();
      const double notional = r.next(), strike = r.next(), mat = r.next();
      ns.trades.push_back(std::make_shared<AssetForward>(id, "A" + std::to_string(asset), notional, strike, mat));
    } else if (type == 2) {
      const std::size_t asset = r.count();
      const double call = r.next(), notional = r.next(), strike = r.next(), expiry = r.next();
      ns.trades.push_back(std::make_shared<EuropeanOption>(id, "A" + std::to_string(asset), call != 0.0 ? OptionType::Call : OptionType::Put,
                                                           notional, strike, expiry));
    } else if (type == 3) {
      const double notional = r.next(), fixed = r.next(), pay = r.next();
      InterestRateSwap u(id + "/u", notional, fixed, readSchedule(r), dirOf(pay));
      std::vector<double> ex = readSchedule(r);
      const double physical = r.next(), position = r.next();
      const std::size_t degree = r.count();
      ns.trades.push_back(std::make_shared<BermudanSwaption>(id, u, ex, physical != 0.0 ? Settlement::Physical : Settlement::Cash,
                                                             position, degree));
    } else if (type == 4) {
      // Two-schedule swap: the reference has one schedule per swap, and the value is linear in
      // the legs, so it enters as float(K=0) + [fixed leg at K] - [fixed leg at 0].
      const double notional = r.next(), fixed = r.next(), pay = r.next();
      const std::vector<double> fs = readSchedule(r), ls = readSchedule(r);
      ns.trades.push_back(std::make_shared<InterestRateSwap>(id + "/f", notional, 0.0, ls, dirOf(pay)));
      ns.trades.push_back(std::make_shared<InterestRateSwap>(id + "/k", notional, fixed, fs, dirOf(pay)));
      ns.trades.push_back(std::make_shared<InterestRateSwap>(id + "/z", notional, 0.0, fs, dirOf(pay == 0.0 ? 1.0 : 0.0)));
    } else {
      throw std::invalid_argument("netting set: unknown trade type");
    }
  }
  if (r.next() != 0.0) {
    CollateralAgreement c;
    c.thresholdCounterparty = r.next();
    const double own = r.next();
    c.thresholdOwn = own < 0.0 ? std::numeric_limits<double>::infinity() : own;
    c.minimumTransferAmount = r.next();
    c.independentAmount = r.next();
    c.marginPeriodOfRisk = r.next();
    c.type = static_cast<CollateralAgreement::Type>(static_cast<int>(r.next()));
    c.haircut = r.next();
    c.bondMaturity = r.next();
    c.assetIndex = r.count();
    ns.collateral = c;
  }
  return ns;
}

gpu::FusedOptions readOptions(const double* a, std::size_t n) {
  Reader r{a, n};
  if (r.next() != 7003.0) throw std::invalid_argument("options: bad magic");
  gpu::FusedOptions o;
  o.pfeQuantile = r.next();
  o.counterparty = r.count();
  o.perTrade = r.next() != 0.0;
  o.imQuantile = r.next();
  o.imInnerPaths = r.count();
  o.imMarginPeriod = r.next();
  o.imAuditPaths = r.count();
  o.imAuditInnerPaths = r.count();
  o.samples = r.count();
  o.histogramTime = r.next();
  o.histogramBins = r.count();
  o.gross = r.next() != 0.0;
  o.collateralBands = r.next() != 0.0;
  o.tradeViews = r.next() != 0.0;
  o.exerciseViews = r.next() != 0.0;
  o.factorViews = r.next() != 0.0;
  o.bondMaturity = r.next();
  auto seq = [&] {
    const std::size_t k = r.count();
    std::vector<double> v(k);
    for (auto& x : v) x = r.next();
    return v;
  };
  o.extraDates = seq();
  o.bandLevels = seq();
  o.factorBandLevels = seq();
  return o;
}

ExposureEngine makeEngine(const ModelSpec& m) {
  return ExposureEngine(ScenarioGenerator(m.hw, m.assets, m.credits, m.correlation), m.sim, TimeGrid(m.base));
}

void setError(char* err, std::size_t len, const std::exception& e) {
  if (err && len) {
    std::strncpy(err, e.what(), len - 1);
    err[len - 1] = 0;
  }
}

// ---- ScenarioGenerator::generate with injected normals (restated driver loop). ----
// z[(j - 1) * nNormals * nStreams + k * nStreams + stream]: normal k of step j on stream
// `stream` (path p uses stream p >> 1 with the sign of p's parity when antithetic, else p), the
// per-step layout [correlated drivers | HW integral | CIR bridges] of scenario_generator.cpp:69-75.
ScenarioSet generateInjected(const ScenarioGenerator& gen, const TimeGrid& grid, const SimulationConfig& cfg,
                             const double* z, std::size_t nStreams) {
  const std::size_t nT = grid.size(), nP = cfg.numPaths, nA = gen.assets().size(), nC = gen.credits().size();
  const std::size_t nCorr = gen.numFactors();
  std::vector<std::size_t> creditOffset(nC);
  std::size_t nNormals = nCorr + 1;
  for (std::size_t c = 0; c < nC; ++c) creditOffset[c] = nNormals, nNormals += gen.credits()[c]->extraNormals();
  const Matrix L = cholesky(gen.correlation());
  ScenarioSet s;
  s.grid = grid;
  s.numPaths = nP;
  s.rateModel = gen.rateModel();
  s.rateState = Matrix(nP, nT, 0.0);
  s.deflator = Matrix(nP, nT, 1.0);
  s.assetModels = gen.assets();
  s.assetValues.assign(nA, Matrix(nP, nT, 0.0));
  s.creditModels = gen.credits();
  s.intensityState.assign(nC, Matrix(nP, nT, 0.0));
  s.survival.assign(nC, Matrix(nP, nT, 1.0));
  std::vector<double> w(nCorr), step(nNormals);
  for (std::size_t p = 0; p < nP; ++p) {
    const std::size_t stream = cfg.antithetic ? p >> 1 : p;
    const double sign = cfg.antithetic && (p & 1) ? -1.0 : 1.0;
    if (stream >= nStreams) throw std::invalid_argument("injected normals: too few streams");
    double x = 0.0, deflator = 1.0;
    std::vector<double> spot(nA), y(nC), iy(nC, 0.0);
    for (std::size_t a = 0; a < nA; ++a) spot[a] = gen.assets()[a]->spot(), s.assetValues[a](p, 0) = spot[a];
    for (std::size_t c = 0; c < nC; ++c) y[c] = gen.credits()[c]->y0(), s.intensityState[c](p, 0) = y[c];
    for (std::size_t j = 1; j < nT; ++j) {
      const double t0 = grid[j - 1], t1 = grid[j];
      for (std::size_t k = 0; k < nNormals; ++k) step[k] = sign * z[((j - 1) * nNormals + k) * nStreams + stream];
      for (std::size_t i = 0; i < nCorr; ++i) {
        double sum = 0.0;
        for (std::size_t k = 0; k <= i; ++k) sum += L(i, k) * step[k];
        w[i] = sum;
      }
      double integratedRate = 0.0;
      gen.rateModel()->evolve(t0, t1, x, w[0], step[nCorr], x, integratedRate);
      deflator *= std::exp(-integratedRate);
      s.rateState(p, j) = x;
      s.deflator(p, j) = deflator;
      for (std::size_t a = 0; a < nA; ++a) {
        spot[a] = gen.assets()[a]->evolve(t0, t1, spot[a], integratedRate, w[1 + a]);
        s.assetValues[a](p, j) = spot[a];
      }
      for (std::size_t c = 0; c < nC; ++c) {
        gen.credits()[c]->evolve(t1 - t0, w[1 + nA + c], step.data() + creditOffset[c], y[c], iy[c]);
        s.intensityState[c](p, j) = y[c];
        s.survival[c](p, j) = gen.credits()[c]->survival(t1, iy[c]);
      }
    }
  }
  return s;
}

struct EngineRun {
  ExposureResult result;
  std::vector<Matrix> exerciseIndex;  // unused placeholder for symmetry
};

}  // namespace

extern "C" {

// ------------------------------------------------------------------ plans
void* ref_plan_compile(const double* model, std::size_t nm, const double* ns, std::size_t nn, const double* opts,
                       std::size_t no, char* err, std::size_t errlen) {
  try {
    const ModelSpec m = readModel(model, nm);
    const NettingSet n = readNettingSet(ns, nn);
    const gpu::FusedOptions o = readOptions(opts, no);
    return new gpu::FusedPlan(gpu::compile(makeEngine(m), n, o));
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return nullptr;
  }
}

// A FusedPlan made from raw buffers (any plan in the reference's layout, e.g. one compiled by
// zlatko_b200), with numPaths taken from header word 0.  Only the fields the CPU kernels and
// summarise read are set.
void* ref_plan_from_buffers(const std::uint32_t* header, const std::uint32_t* indices, std::size_t nIdx, const float* params,
                            const float* steps, std::size_t nSteps, const float* terms, std::size_t nTerms, const float* requests,
                            std::size_t nReq, std::uint32_t rowsTotal, std::uint32_t numOutputs, const double* times, std::size_t nT,
                            const std::uint64_t* reporting, std::size_t nR) {
  auto* p = new gpu::FusedPlan();
  p->header.assign(header, header + gpu::kHeaderWords);
  p->indices.assign(indices, indices + nIdx);
  p->params.assign(params, params + gpu::kParamCount);
  p->steps.assign(steps, steps + nSteps);
  p->terms.assign(terms, terms + nTerms);
  p->requests.assign(requests, requests + nReq);
  p->rows.total = rowsTotal;
  p->numOutputs = numOutputs;
  p->numPaths = header[0];
  p->statsPerDate = header[16];
  p->times.assign(times, times + nT);
  for (std::size_t k = 0; k < nR; ++k) p->reporting.push_back(reporting[k]);
  p->marketSurvival.assign(nT, 1.0);
  p->numCredits = header[3];
  p->numTradeGroups = header[18];
  p->views.pfe = 0;
  return p;
}

void ref_plan_free(void* p) { delete static_cast<gpu::FusedPlan*>(p); }

// sizes: header, indices, params, steps, terms, requests, rows.total, numOutputs, nT, nR, statsPerDate,
// amc count, unsupported count, numPaths
void ref_plan_sizes(const void* h, std::uint64_t* s) {
  const auto& p = *static_cast<const gpu::FusedPlan*>(h);
  s[0] = p.header.size();
  s[1] = p.indices.size();
  s[2] = p.params.size();
  s[3] = p.steps.size();
  s[4] = p.terms.size();
  s[5] = p.requests.size();
  s[6] = p.rows.total;
  s[7] = p.numOutputs;
  s[8] = p.numDates();
  s[9] = p.reporting.size();
  s[10] = p.statsPerDate;
  s[11] = p.amc.size();
  s[12] = p.unsupported.size();
  s[13] = p.numPaths;
}

void ref_plan_get(const void* h, std::uint32_t* header, std::uint32_t* indices, float* params, float* steps, float* terms,
                  float* requests, double* times, std::uint64_t* reporting, double* marketSurvival) {
  const auto& p = *static_cast<const gpu::FusedPlan*>(h);
  std::memcpy(header, p.header.data(), p.header.size() * 4);
  std::memcpy(indices, p.indices.data(), p.indices.size() * 4);
  std::memcpy(params, p.params.data(), p.params.size() * 4);
  std::memcpy(steps, p.steps.data(), p.steps.size() * 4);
  if (!p.terms.empty()) std::memcpy(terms, p.terms.data(), p.terms.size() * 4);
  if (!p.requests.empty()) std::memcpy(requests, p.requests.data(), p.requests.size() * 4);
  for (std::size_t j = 0; j < p.times.size(); ++j) times[j] = p.times[j], marketSurvival[j] = p.marketSurvival[j];
  for (std::size_t k = 0; k < p.reporting.size(); ++k) reporting[k] = p.reporting[k];
}

// Replaces the plan's term table (e.g. with AMC coefficients fitted elsewhere).
void ref_plan_set_terms(void* h, const float* terms, std::size_t n) {
  auto& p = *static_cast<gpu::FusedPlan*>(h);
  p.terms.assign(terms, terms + n);
}

// Sets the number of paths of a compiled plan (header words 0 and 15), as auditConditionalIm does
// (src/gpu/fused_exposure.cpp:873-877).
void ref_plan_set_paths(void* h, std::size_t numPaths) {
  auto& p = *static_cast<gpu::FusedPlan*>(h);
  p.numPaths = numPaths;
  p.header[0] = static_cast<std::uint32_t>(numPaths);
  p.header[15] = static_cast<std::uint32_t>(p.numWorkgroups());
}

// The reference's FP32 CPU kernels on `threads` threads (0: the default pool).
int ref_run_fused(const void* h, int threads, float* sums, float* values, char* err, std::size_t errlen) {
  try {
    const auto& p = *static_cast<const gpu::FusedPlan*>(h);
    gpu::FusedOutput o;
    if (threads > 0) {
      SpinPool pool(static_cast<std::size_t>(threads - 1));
      o = gpu::runFusedReference(p, pool);
    } else {
      o = gpu::runFusedReference(p);
    }
    std::memcpy(sums, o.sums.data(), o.sums.size() * 4);
    std::memcpy(values, o.values.data(), o.values.size() * 4);
    return 0;
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return 1;
  }
}

// The fused-exposure workgroups only (no reduction): the exposure rows [row][path], as the row-statistics
// kernel reads them, for tests of the row statistics against the same inputs.
int ref_run_rows(const void* h, int threads, float* exposure, char* err, std::size_t errlen) {
  try {
    const auto& p = *static_cast<const gpu::FusedPlan*>(h);
    SpinPool pool(static_cast<std::size_t>(threads > 0 ? threads - 1 : 0));
    const auto s = gpu::runFusedWorkgroups(p, 0, p.numWorkgroups(), pool);
    std::memcpy(exposure, s.exposure.data(), s.exposure.size() * 4);
    return 0;
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return 1;
  }
}

int ref_amc_states(const void* h, int threads, float* x, float* deflator, float* exercise, char* err, std::size_t errlen) {
  try {
    const auto& p = *static_cast<const gpu::FusedPlan*>(h);
    SpinPool pool(static_cast<std::size_t>(threads > 0 ? threads - 1 : 0));
    const auto st = gpu::runAmcStates(p, pool);
    std::memcpy(x, st.x.data(), st.x.size() * 4);
    std::memcpy(deflator, st.deflator.data(), st.deflator.size() * 4);
    if (!st.exercise.empty()) std::memcpy(exercise, st.exercise.data(), st.exercise.size() * 4);
    return 0;
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return 1;
  }
}

// AMC exercise rows of the plan (sum over Bermudans of their exercise dates).
std::uint64_t ref_amc_rows(const void* h) {
  const auto& p = *static_cast<const gpu::FusedPlan*>(h);
  std::uint64_t rows = 0;
  for (const auto& a : p.amc) rows += a.exerciseDates.size();
  return rows;
}

// gpu::summarise: per reporting date EV, EE, ENE, PFE, EE*, ENE*, cvaIncrement, meanSurvival, meanDeflator
// (9 * nR doubles), then pathwiseCva(0.4) in out[9 * nR].
int ref_summarise(const void* h, const float* sums, const float* values, double* out, char* err, std::size_t errlen) {
  try {
    const auto& p = *static_cast<const gpu::FusedPlan*>(h);
    gpu::FusedOutput o;
    o.sums.assign(sums, sums + p.numDates() * p.statsPerDate);
    o.values.assign(values, values + std::max<std::size_t>(1, p.numOutputs));
    const auto r = gpu::summarise(p, o);
    const std::size_t nR = p.reporting.size();
    const std::vector<const std::vector<double>*> cols = {
        &r.profile.expectedValue, &r.profile.expectedExposure, &r.profile.expectedNegativeExposure,
        &r.profile.potentialFutureExposure, &r.profile.discountedExpectedExposure,
        &r.profile.discountedExpectedNegativeExposure, &r.cvaIncrements, &r.meanSurvival, &r.meanDeflator};
    for (std::size_t c = 0; c < cols.size(); ++c)
      for (std::size_t k = 0; k < nR; ++k) out[c * nR + k] = (*cols[c])[k];
    out[9 * nR] = r.pathwiseCva(0.4);
    return 0;
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return 1;
  }
}

// The rest of gpu::summarise's result per reporting date, in blocks of nR doubles (NaN where the result has
// no such series): valueChangeQuantile, conditionalImDiscounted, conditionalImMean, the three
// conditionalImBands, conditionalDiscountedEe, conditionalImAuditRatio, conditionalImDiscountedUncorrected,
// then for each trade group its marginalDiscounted, marginal, incrementalDiscounted, standaloneDiscounted,
// standalone.  out holds (9 + 5 * numTradeGroups) * nR doubles.
int ref_summarise_views(const void* h, const float* sums, const float* values, double* out, std::size_t nOut, char* err,
                        std::size_t errlen) {
  try {
    const auto& p = *static_cast<const gpu::FusedPlan*>(h);
    gpu::FusedOutput o;
    o.sums.assign(sums, sums + p.numDates() * p.statsPerDate);
    o.values.assign(values, values + std::max<std::size_t>(1, p.numOutputs));
    const auto r = gpu::summarise(p, o);
    const std::size_t nR = p.reporting.size();
    if (nOut != (9 + 5 * r.trades.size()) * nR) throw std::invalid_argument("ref_summarise_views: output size");
    std::vector<const std::vector<double>*> cols = {&r.valueChangeQuantile, &r.conditionalImDiscounted, &r.conditionalImMean};
    for (std::size_t b = 0; b < 3; ++b) cols.push_back(b < r.conditionalImBands.size() ? &r.conditionalImBands[b] : nullptr);
    cols.push_back(&r.conditionalDiscountedEe);
    cols.push_back(&r.conditionalImAuditRatio);
    cols.push_back(&r.conditionalImDiscountedUncorrected);
    for (const auto& t : r.trades)
      for (const auto* c : {&t.marginalDiscounted, &t.marginal, &t.incrementalDiscounted, &t.standaloneDiscounted, &t.standalone})
        cols.push_back(c);
    for (std::size_t c = 0; c < cols.size(); ++c)
      for (std::size_t k = 0; k < nR; ++k)
        out[c * nR + k] = cols[c] && cols[c]->size() == nR ? (*cols[c])[k] : std::numeric_limits<double>::quiet_NaN();
    return 0;
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return 1;
  }
}

namespace {
// Flattens a FusedResult into length-prefixed arrays (oracle/ref.py: summarise_full reads them in this order).
struct Flat {
  std::vector<double> d;
  void vec(const std::vector<double>& v) {
    d.push_back(static_cast<double>(v.size()));
    d.insert(d.end(), v.begin(), v.end());
  }
  void mat(const std::vector<std::vector<double>>& m) {
    d.push_back(static_cast<double>(m.size()));
    for (const auto& v : m) vec(v);
  }
  void profile(const ExposureProfile& p) {
    for (const auto* v : {&p.times, &p.expectedValue, &p.expectedExposure, &p.expectedNegativeExposure,
                          &p.potentialFutureExposure, &p.discountedExpectedExposure, &p.discountedExpectedNegativeExposure})
      vec(*v);
  }
};
}  // namespace

// The whole gpu::summarise result (audit included), flattened; returns the number of doubles, writing at most
// cap of them into out (a first call with cap 0 sizes the buffer).
std::int64_t ref_summarise_full(const void* h, const float* sums, const float* values, double* out, std::size_t cap, char* err,
                                std::size_t errlen) {
  try {
    const auto& p = *static_cast<const gpu::FusedPlan*>(h);
    gpu::FusedOutput o;
    o.sums.assign(sums, sums + p.numDates() * p.statsPerDate);
    o.values.assign(values, values + std::max<std::size_t>(1, p.numOutputs));
    const auto r = gpu::summarise(p, o);
    Flat f;
    f.profile(r.profile);
    for (const auto* v : {&r.meanSurvival, &r.marketSurvival, &r.cvaIncrements, &r.conditionalDiscountedEe, &r.meanDeflator,
                          &r.valueChangeQuantile, &r.conditionalImDiscounted, &r.conditionalImMean})
      f.vec(*v);
    f.mat(r.conditionalImBands);
    f.vec(r.conditionalImAuditRatio);
    f.vec(r.conditionalImDiscountedUncorrected);
    f.d.push_back(static_cast<double>(r.trades.size()));
    for (const auto& t : r.trades)
      for (const auto* v : {&t.marginalDiscounted, &t.marginal, &t.incrementalDiscounted, &t.standaloneDiscounted, &t.standalone})
        f.vec(*v);
    f.mat(r.exposureSamples);
    f.mat(r.nettedSamples);
    f.mat(r.collateralSamples);
    f.mat(r.collateralBands);
    f.d.push_back(r.grossProfile ? 1.0 : 0.0);
    if (r.grossProfile) f.profile(*r.grossProfile);
    f.d.push_back(r.histogramTime);
    f.vec(r.histogramEdges);
    f.vec(r.histogramCounts);
    f.d.push_back(static_cast<double>(r.tradeViews.size()));
    for (const auto& t : r.tradeViews) {
      f.profile(t.profile);
      f.mat(t.samples);
      f.mat(t.bands);
      f.vec(t.meanDeflated);
    }
    f.d.push_back(static_cast<double>(r.exercise.size()));
    for (const auto& e : r.exercise) {
      f.vec(e.distribution);
      f.vec(e.sampleIndex);
    }
    f.d.push_back(r.factors ? 1.0 : 0.0);
    if (r.factors) {
      const auto& F = *r.factors;
      f.mat(F.rateSamples);
      f.mat(F.rateBands);
      f.vec(F.rateMean);
      f.vec(F.deflatorMean);
      f.vec(F.bondMean);
      f.d.push_back(static_cast<double>(F.assets.size()));
      for (const auto& a : F.assets) {
        f.mat(a.samples);
        f.mat(a.bands);
        f.vec(a.mean);
        f.vec(a.deflatedMean);
      }
      f.d.push_back(static_cast<double>(F.credits.size()));
      for (const auto& c : F.credits) {
        f.mat(c.intensitySamples);
        f.mat(c.intensityBands);
        f.mat(c.survivalSamples);
        f.vec(c.survivalMean);
      }
      const std::size_t n = F.incrementCorrelation.rows();
      f.d.push_back(static_cast<double>(n));
      for (std::size_t i = 0; i < n; ++i)
        for (std::size_t k = 0; k < n; ++k) f.d.push_back(F.incrementCorrelation(i, k));
    }
    for (std::size_t k = 0; k < f.d.size() && k < cap; ++k) out[k] = f.d[k];
    return static_cast<std::int64_t>(f.d.size());
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return -1;
  }
}

// ---- adaptive nested Monte Carlo (src/nested/adaptive_nested.cpp) ----
// The inner simulator as a C callback: payoffs of `n` inner paths of `scenario` from `seed` into out.
typedef void (*ref_inner_fn)(std::size_t scenario, std::uint64_t seed, double* out, std::size_t n, void* user);

namespace {
nested::AdaptiveOptions adaptiveOptions(const double* o, std::size_t no) {
  nested::AdaptiveOptions a;
  a.trainingFraction = o[0], a.hermiteDegree = static_cast<std::size_t>(o[1]), a.innerBatch = static_cast<std::size_t>(o[2]);
  a.minInnerForVariance = static_cast<std::size_t>(o[3]), a.maxInnerPerScenario = static_cast<std::size_t>(o[4]);
  a.innerBudget = static_cast<std::size_t>(o[5]), a.maxScenariosPerRound = static_cast<std::size_t>(o[6]);
  a.maxRounds = static_cast<std::size_t>(o[7]), a.auditPerBin = static_cast<std::size_t>(o[8]);
  a.minPerBinForMisspecification = static_cast<std::size_t>(o[9]), a.refineOutsideTrainingRange = o[10] != 0.0;
  a.seed = static_cast<std::uint64_t>(o[11]);
  a.binProbabilities.assign(o + 12, o + no);
  return a;
}
}  // namespace

// estimateAdaptive with statistics PositivePart(eeRel, eeAbs) and Quantile(q, positive part, 2.0), flattened:
// estimate[2], baseline[2], regression[2], then length-prefixed training, evaluation, proxy, value, inner, then
// innerPaths, auditInnerPaths, refinedScenarios, auditedScenarios, rounds, unresolved, proxyDegree, proxyBasis,
// stop, then the bins (count, 7 numbers each).  seedHi/seedLo carry the 64-bit seed.  Returns the length.
std::int64_t ref_estimate_adaptive(const double* features, std::size_t n, std::size_t dims, const double* payoff, const double* weight,
                                   ref_inner_fn fn, void* user, double eeRel, double eeAbs, double q, const double* opts,
                                   std::size_t nOpts, std::uint64_t seed, double* out, std::size_t cap, char* err, std::size_t errlen) {
  try {
    nested::OuterSample outer;
    outer.features = Matrix(n, dims);
    for (std::size_t i = 0; i < n; ++i)
      for (std::size_t j = 0; j < dims; ++j) outer.features(i, j) = features[i * dims + j];
    outer.payoff.assign(payoff, payoff + n);
    if (weight) outer.weight.assign(weight, weight + n);
    nested::AdaptiveOptions o = adaptiveOptions(opts, nOpts);
    o.seed = seed;
    const nested::PositivePart ee(eeRel, eeAbs, "EE*");
    const nested::Quantile pfe(q, true, 2.0, "PFE");
    const nested::InnerSimulator inner = [&](std::size_t sc, std::uint64_t sd, double* o2, std::size_t m) { fn(sc, sd, o2, m, user); };
    SpinPool pool(1);
    const auto r = nested::estimateAdaptive(outer, inner, {&ee, &pfe}, o, pool);
    std::vector<double> d;
    auto vec = [&](const auto& v) {
      d.push_back(static_cast<double>(v.size()));
      for (const auto& x : v) d.push_back(static_cast<double>(x));
    };
    for (const auto* v : {&r.estimate, &r.baseline, &r.regression})
      for (double x : *v) d.push_back(x);
    vec(r.training), vec(r.evaluation), vec(r.proxy), vec(r.value), vec(r.inner);
    for (std::size_t x : {r.innerPaths, r.auditInnerPaths, r.refinedScenarios, r.auditedScenarios, r.rounds, r.unresolved,
                          r.proxyDegree, r.proxyBasis})
      d.push_back(static_cast<double>(x));
    d.push_back(static_cast<double>(static_cast<int>(r.stop)));
    d.push_back(static_cast<double>(r.bins.size()));
    for (const auto& b : r.bins)
      for (double x : {b.lowerProbability, b.upperProbability, static_cast<double>(b.scenarios), static_cast<double>(b.refined),
                       b.residualStdDev, b.biasShift, b.biasRms})
        d.push_back(x);
    for (std::size_t k = 0; k < d.size() && k < cap; ++k) out[k] = d[k];
    return static_cast<std::int64_t>(d.size());
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return -1;
  }
}

// estimateUniform with the same two statistics: out = estimate[2], then the value of every scenario.
int ref_estimate_uniform(const double* weight, std::size_t n, ref_inner_fn fn, void* user, const std::uint64_t* scenarios,
                         std::size_t ns, std::size_t perScenario, double eeRel, double eeAbs, double q, std::uint64_t seed, double* out,
                         char* err, std::size_t errlen) {
  try {
    nested::OuterSample outer;
    outer.features = Matrix(n, 1);
    outer.payoff.assign(n, 0.0);
    if (weight) outer.weight.assign(weight, weight + n);
    const nested::PositivePart ee(eeRel, eeAbs, "EE*");
    const nested::Quantile pfe(q, true, 2.0, "PFE");
    const nested::InnerSimulator inner = [&](std::size_t sc, std::uint64_t sd, double* o2, std::size_t m) { fn(sc, sd, o2, m, user); };
    SpinPool pool(1);
    const std::vector<std::size_t> sc(scenarios, scenarios + ns);
    const auto u = nested::estimateUniform(outer, inner, sc, perScenario, {&ee, &pfe}, seed, pool);
    out[0] = u.estimate[0], out[1] = u.estimate[1];
    for (std::size_t k = 0; k < ns; ++k) out[2 + k] = u.value[k];
    return 0;
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return 1;
  }
}

// The reference's counter-based normals and seed mixing, for known answers.
double ref_counter_normal(std::uint64_t seed, std::size_t m) {
  nested::CounterNormals c(seed);
  double v = 0.0;
  for (std::size_t k = 0; k <= m; ++k) v = c.next();
  return v;
}
std::uint64_t ref_derive_seed(std::uint64_t seed, std::uint64_t a, std::uint64_t b, std::uint64_t c) { return nested::deriveSeed(seed, a, b, c); }

// ---- nested exposure (src/nested/nested_exposure.cpp) ----
// The reference's own outer normals: the first n of NormalGenerator(seed), in the order generate() reads them.
void ref_normal_stream(std::uint64_t seed, std::size_t n, double* out) {
  NormalGenerator g(seed);
  g.fill(out, n);
}

// nestedExposure on the model's generator and simulation (paths, seed, antithetic) and the reporting dates, on
// `threads` pool threads; adaptive options as in ref_estimate_adaptive, seed passed apart.  out [nR][16]: time, EE* and PFE of the exact,
// regression, uniform and adaptive estimates, evaluated, inner paths, audit inner paths, refined, rounds, uniform
// inner paths per scenario, live.  Returns the number of points.
std::int64_t ref_nested_exposure(const double* model, std::size_t nm, const double* ns, std::size_t nn, const double* reporting,
                                 std::size_t nr, double pfeQuantile, const double* opts, std::size_t nOpts, std::uint64_t seed,
                                 int uniform, std::size_t threads, double* out, std::size_t cap, char* err, std::size_t errlen) {
  try {
    const ModelSpec m = readModel(model, nm);
    const NettingSet n = readNettingSet(ns, nn);
    const ScenarioGenerator gen(m.hw, m.assets, m.credits, m.correlation);
    nested::NestedExposureOptions o;
    o.pfeQuantile = pfeQuantile;
    o.adaptive = adaptiveOptions(opts, nOpts);
    o.adaptive.seed = seed;
    o.uniform = uniform != 0;
    SpinPool pool(std::max<std::size_t>(threads, 1));
    const auto r = nested::nestedExposure(gen, n, TimeGrid(std::vector<double>(reporting, reporting + nr)), m.sim, o, pool);
    std::size_t k = 0;
    for (const auto& p : r.points)
      for (double v : {p.time, p.eeExact, p.pfeExact, p.eeRegression, p.pfeRegression, p.eeUniform, p.pfeUniform, p.eeAdaptive,
                       p.pfeAdaptive, static_cast<double>(p.evaluated), static_cast<double>(p.innerPaths),
                       static_cast<double>(p.auditInnerPaths), static_cast<double>(p.refined), static_cast<double>(p.rounds),
                       static_cast<double>(p.uniformInnerPerScenario), p.live ? 1.0 : 0.0}) {
        if (k < cap) out[k] = v;
        ++k;
      }
    return static_cast<std::int64_t>(r.points.size());
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return -1;
  }
}

// ------------------------------------------------------------------ FP64 engine
// ExposureEngine::run (exposure_engine.cpp:50-81) on the reference's own normals (normals == nullptr) or
// on injected normals (see generateInjected).  Returns a handle; ref_engine_get copies its matrices.
void* ref_engine_run(const double* model, std::size_t nm, const double* ns, std::size_t nn, double pfeQuantile,
                     const double* normals, std::size_t nStreams, char* err, std::size_t errlen) {
  try {
    const ModelSpec m = readModel(model, nm);
    const NettingSet n = readNettingSet(ns, nn);
    const ExposureEngine engine = makeEngine(m);
    if (!normals) return new ExposureResult(engine.run(n, pfeQuantile));
    if (n.trades.empty()) throw std::invalid_argument("ExposureEngine::run: empty netting set");
    // The steps of ExposureEngine::run with the scenario generated from the injected normals.
    auto* result = new ExposureResult();
    const TimeGrid reporting = engine.reportingGrid(n);
    result->scenarios = generateInjected(engine.generator(), engine.simulationGrid(n), engine.config(), normals, nStreams);
    const ScenarioSet& s = result->scenarios;
    for (double t : reporting.times()) result->reportingIndices.push_back(*s.grid.find(t));
    for (const auto& trade : n.trades) result->tradeValues.push_back(trade->valueCube(s));
    result->nettedValue = netValues(result->tradeValues);
    if (n.collateral) {
      const CollateralAgreement& csa = *n.collateral;
      Matrix price;
      if (csa.type == CollateralAgreement::Type::Bond) {
        price = Matrix(s.numPaths, s.numTimes());
        for (std::size_t p = 0; p < s.numPaths; ++p)
          for (std::size_t j = 0; j < s.numTimes(); ++j) price(p, j) = s.zeroBond(p, j, csa.bondMaturity);
      } else if (csa.type == CollateralAgreement::Type::Asset) {
        price = s.assetValues.at(csa.assetIndex);
      }
      result->collateral = simulateCollateral(csa, result->nettedValue, s.grid, csa.type == CollateralAgreement::Type::Cash ? nullptr : &price);
    } else {
      result->collateral = Matrix(s.numPaths, s.numTimes(), 0.0);
    }
    result->exposureValue = result->nettedValue - result->collateral;
    result->profile = ExposureProfile::compute(selectColumns(result->exposureValue, result->reportingIndices), reporting,
                                              selectColumns(s.deflator, result->reportingIndices), pfeQuantile);
    return result;
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return nullptr;
  }
}

void ref_engine_free(void* h) { delete static_cast<ExposureResult*>(h); }

// nP, nT (simulation dates), nR, nTrades (value cubes), nCredits
void ref_engine_sizes(const void* h, std::uint64_t* s) {
  const auto& r = *static_cast<const ExposureResult*>(h);
  s[0] = r.scenarios.numPaths;
  s[1] = r.scenarios.numTimes();
  s[2] = r.reportingIndices.size();
  s[3] = r.tradeValues.size();
  s[4] = r.scenarios.survival.size();
}

// Any pointer may be null.  Matrices are [path][date] over the simulation grid.
void ref_engine_get(const void* h, double* times, std::uint64_t* reporting, double* profile, double* netted, double* collateral,
                    double* deflator, double* rateState, double* survival, double* trades) {
  const auto& r = *static_cast<const ExposureResult*>(h);
  const auto& s = r.scenarios;
  const std::size_t nP = s.numPaths, nT = s.numTimes(), nR = r.reportingIndices.size();
  auto copy = [&](const Matrix& m, double* out) {
    if (out) std::memcpy(out, m.row(0), nP * nT * sizeof(double));
  };
  if (times)
    for (std::size_t j = 0; j < nT; ++j) times[j] = s.grid[j];
  if (reporting)
    for (std::size_t k = 0; k < nR; ++k) reporting[k] = r.reportingIndices[k];
  if (profile) {
    const auto& p = r.profile;
    const std::vector<const std::vector<double>*> cols = {&p.expectedValue, &p.expectedExposure, &p.expectedNegativeExposure,
                                                          &p.potentialFutureExposure, &p.discountedExpectedExposure,
                                                          &p.discountedExpectedNegativeExposure};
    for (std::size_t c = 0; c < cols.size(); ++c)
      for (std::size_t k = 0; k < nR; ++k) profile[c * nR + k] = (*cols[c])[k];
  }
  copy(r.nettedValue, netted);
  copy(r.collateral, collateral);
  copy(s.deflator, deflator);
  copy(s.rateState, rateState);
  if (survival)
    for (std::size_t c = 0; c < s.survival.size(); ++c) std::memcpy(survival + c * nP * nT, s.survival[c].row(0), nP * nT * sizeof(double));
  if (trades)
    for (std::size_t i = 0; i < r.tradeValues.size(); ++i) std::memcpy(trades + i * nP * nT, r.tradeValues[i].row(0), nP * nT * sizeof(double));
}

// pathwiseCva (cva.cpp:57-77) over the reporting dates.
double ref_engine_pathwise_cva(const void* h, std::size_t credit, double recovery) {
  const auto& r = *static_cast<const ExposureResult*>(h);
  return pathwiseCva(r.scenarios, r.exposureValue, credit, recovery, r.reportingIndices);
}

// ------------------------------------------------------------------ CVA and quantile
double ref_unilateral_cva(const double* times, const double* dee, std::size_t n, const double* pillars, const double* hazards,
                          std::size_t nh, double recovery) {
  const CreditCurve c(std::vector<double>(pillars, pillars + nh), std::vector<double>(hazards, hazards + nh));
  return unilateralCva(std::vector<double>(times, times + n), std::vector<double>(dee, dee + n), c, recovery);
}

void ref_bilateral_cva(const double* times, const double* dee, const double* dene, std::size_t n, const double* cp,
                       const double* ch, std::size_t nc, const double* op, const double* oh, std::size_t no, double rc,
                       double ro, double* out) {
  ExposureProfile p;
  p.times.assign(times, times + n);
  p.discountedExpectedExposure.assign(dee, dee + n);
  p.discountedExpectedNegativeExposure.assign(dene, dene + n);
  const CreditCurve c(std::vector<double>(cp, cp + nc), std::vector<double>(ch, ch + nc));
  const CreditCurve o(std::vector<double>(op, op + no), std::vector<double>(oh, oh + no));
  const BilateralCva b = bilateralCva(p, c, rc, o, ro);
  out[0] = b.cva;
  out[1] = b.dva;
}

// ---- xVA and allocation (src/xva/xva.cpp, src/exposure/allocation.cpp) ----
namespace {
XvaParameters xvaParams(const double* p) {
  XvaParameters x;
  x.fundingSpreadBorrow = p[0], x.fundingSpreadLend = p[1], x.marginFundingSpread = p[2], x.hurdleRate = p[3];
  x.capitalRatio = p[4], x.riskWeight = p[5], x.alpha = p[6];
  return x;
}
CreditCurve curveOf(const double* pillars, const double* hazards, std::size_t n) {
  return CreditCurve(std::vector<double>(pillars, pillars + n), std::vector<double>(hazards, hazards + n));
}
Matrix matrixOf(const double* a, std::size_t rows, std::size_t cols) {
  Matrix m(rows, cols);
  for (std::size_t i = 0; i < rows; ++i)
    for (std::size_t j = 0; j < cols; ++j) m(i, j) = a[i * cols + j];
  return m;
}
}  // namespace

// xva(): out = cva, dva, fca, fba, mva, kva.  dim may be null (no initial margin).
void ref_xva(const double* times, const double* dee, const double* dene, std::size_t n, const double* dim, const double* cp,
             const double* ch, std::size_t nc, double rc, const double* op, const double* oh, std::size_t no, double ro,
             const double* params, double* out) {
  ExposureProfile p;
  p.times.assign(times, times + n);
  p.discountedExpectedExposure.assign(dee, dee + n);
  p.discountedExpectedNegativeExposure.assign(dene, dene + n);
  const std::vector<double> im = dim ? std::vector<double>(dim, dim + n) : std::vector<double>();
  const Xva x = xva(p, im, curveOf(cp, ch, nc), rc, curveOf(op, oh, no), ro, xvaParams(params));
  out[0] = x.cva, out[1] = x.dva, out[2] = x.fca, out[3] = x.fba, out[4] = x.mva, out[5] = x.kva;
}

// allocateExposureXva over `trades` contribution profiles [trade][n]: out[trade][3] = cva, fca, kva.
void ref_allocate_exposure_xva(const double* times, std::size_t n, const double* contributions, std::size_t trades,
                               const double* cp, const double* ch, std::size_t nc, double rc, const double* op, const double* oh,
                               std::size_t no, const double* params, double* out) {
  std::vector<std::vector<double>> c(trades);
  for (std::size_t i = 0; i < trades; ++i) c[i].assign(contributions + i * n, contributions + (i + 1) * n);
  const auto r = allocateExposureXva(std::vector<double>(times, times + n), c, curveOf(cp, ch, nc), rc, curveOf(op, oh, no),
                                     xvaParams(params));
  for (std::size_t i = 0; i < trades; ++i) out[3 * i] = r[i].cva, out[3 * i + 1] = r[i].fca, out[3 * i + 2] = r[i].kva;
}

// initialMarginProfile on values and deflator [paths][dates] and the grid's times: out[dates].
void ref_initial_margin_profile(const double* values, const double* deflator, std::size_t paths, const double* times,
                                std::size_t dates, double q, double mpr, double* out) {
  const auto m = initialMarginProfile(matrixOf(values, paths, dates), TimeGrid(std::vector<double>(times, times + dates)),
                                      matrixOf(deflator, paths, dates), q, mpr);
  for (std::size_t j = 0; j < dates; ++j) out[j] = m[j];
}

// marginalExposureContributions: trade values [trade][paths][dates], netted [paths][dates], deflator (nullable):
// out[trade][dates].
void ref_marginal_contributions(const double* tradeValues, std::size_t trades, const double* netted, const double* deflator,
                                std::size_t paths, std::size_t dates, double* out) {
  std::vector<Matrix> tv;
  for (std::size_t i = 0; i < trades; ++i) tv.push_back(matrixOf(tradeValues + i * paths * dates, paths, dates));
  const Matrix nv = matrixOf(netted, paths, dates);
  const Matrix d = deflator ? matrixOf(deflator, paths, dates) : Matrix();
  const auto c = marginalExposureContributions(tv, nv, deflator ? &d : nullptr);
  for (std::size_t i = 0; i < trades; ++i)
    for (std::size_t j = 0; j < dates; ++j) out[i * dates + j] = c[i][j];
}

// incrementalExposure: out[dates].
void ref_incremental_exposure(const double* netted, const double* newTrade, const double* deflator, std::size_t paths,
                              std::size_t dates, double* out) {
  const Matrix d = deflator ? matrixOf(deflator, paths, dates) : Matrix();
  const auto r = incrementalExposure(matrixOf(netted, paths, dates), matrixOf(newTrade, paths, dates), deflator ? &d : nullptr);
  for (std::size_t j = 0; j < dates; ++j) out[j] = r[j];
}

double ref_quantile(const double* v, std::size_t n, double p) { return quantile(std::vector<double>(v, v + n), p); }

// ExposureProfile::compute on a [path][date] matrix: EV, EE, ENE, PFE, EE*, ENE* (6 * nT) then EPE(horizon),
// effective EPE(1y), max PFE.
void ref_profile(const double* values, const double* deflator, std::size_t nP, const double* times, std::size_t nT,
                 double q, double horizon, double* out) {
  Matrix v(nP, nT), d(nP, nT);
  std::memcpy(v.row(0), values, nP * nT * sizeof(double));
  std::memcpy(d.row(0), deflator, nP * nT * sizeof(double));
  const auto p = ExposureProfile::compute(v, TimeGrid(std::vector<double>(times, times + nT)), d, q);
  const std::vector<const std::vector<double>*> cols = {&p.expectedValue, &p.expectedExposure, &p.expectedNegativeExposure,
                                                        &p.potentialFutureExposure, &p.discountedExpectedExposure,
                                                        &p.discountedExpectedNegativeExposure};
  for (std::size_t c = 0; c < cols.size(); ++c)
    for (std::size_t j = 0; j < nT; ++j) out[c * nT + j] = (*cols[c])[j];
  out[6 * nT] = p.expectedPositiveExposure(horizon);
  out[6 * nT + 1] = p.effectiveExpectedPositiveExposure(1.0);
  out[6 * nT + 2] = p.maxPotentialFutureExposure();
}

// simulateCollateral (collateral.cpp:10-47) on a [path][date] value matrix, cash or with unit prices.
int ref_collateral(const double* values, const double* unitPrice, std::size_t nP, const double* times, std::size_t nT,
                   double hc, double ho, double mta, double ia, double mpr, int type, double haircut, double* out, char* err,
                   std::size_t errlen) {
  try {
    CollateralAgreement c;
    c.thresholdCounterparty = hc;
    c.thresholdOwn = ho < 0.0 ? std::numeric_limits<double>::infinity() : ho;
    c.minimumTransferAmount = mta;
    c.independentAmount = ia;
    c.marginPeriodOfRisk = mpr;
    c.type = static_cast<CollateralAgreement::Type>(type);
    c.haircut = haircut;
    Matrix v(nP, nT), price(nP, nT, 1.0);
    std::memcpy(v.row(0), values, nP * nT * sizeof(double));
    if (unitPrice) std::memcpy(price.row(0), unitPrice, nP * nT * sizeof(double));
    const Matrix r = simulateCollateral(c, v, TimeGrid(std::vector<double>(times, times + nT)), unitPrice ? &price : nullptr);
    std::memcpy(out, r.row(0), nP * nT * sizeof(double));
    return 0;
  } catch (const std::exception& e) {
    setError(err, errlen, e);
    return 1;
  }
}

// The reporting and simulation grids of a netting set (exposure_engine.cpp:35-48) plus the fused extras.
std::size_t ref_grid(const double* model, std::size_t nm, const double* ns, std::size_t nn, const double* opts, std::size_t no,
                     int which, double* out, std::size_t cap) {
  const ModelSpec m = readModel(model, nm);
  const NettingSet n = readNettingSet(ns, nn);
  const ExposureEngine e = makeEngine(m);
  TimeGrid g;
  if (which == 0) g = e.reportingGrid(n);
  else if (which == 1) g = e.simulationGrid(n);
  else g = gpu::simulationGrid(e, n, readOptions(opts, no));
  for (std::size_t k = 0; k < g.size() && k < cap; ++k) out[k] = g[k];
  return g.size();
}

}  // extern "C"
