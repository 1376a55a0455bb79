// Host plan compiler of zlatko_b200: market objects, trades and the compilation of a netting set
// into the fused kernels' tables (a restatement of gpu::compile, src/gpu/fused_exposure.cpp:214-707).
#pragma once

#include <cmath>
#include <cstdint>
#include <optional>
#include <string>
#include <vector>

namespace zk::host {

// Zero curve, continuously compounded, linear in the zero rate, flat beyond the ends
// (src/market/yield_curve.cpp:20-40).
struct Curve {
  std::vector<double> t, r;
  double zero(double x) const;
  double discount(double x) const { return std::exp(-zero(x) * x); }
  double forward(double x) const;  // instantaneous forward f(0, x)
};

// Piecewise-flat hazard curve (src/market/credit_curve.cpp:23-41).
struct Hazard {
  std::vector<double> pillars, hazards;
  double survival(double x) const;
};

struct HullWhite {
  Curve curve;
  double a = 0.03, sigma = 0.01;
  double B(double t, double T) const { return (1.0 - std::exp(-a * (T - t))) / a; }
  double V(double t, double T) const;
  double bond(double t, double T, double x) const;  // P(t, T | x) (hull_white.cpp:27-31)
};

struct Asset {
  double spot = 1.0, vol = 0.0;
  Curve carry;
  double carryDiscount(double t, double T) const { return carry.discount(T) / carry.discount(t); }
};

struct Cir {
  double kappa = 0.5, theta = 0.02, xi = 0.08, y0 = 0.02;
  std::size_t substeps = 8;
  Hazard market;
  double cirSurvival(double t) const;  // cir_intensity.cpp:25-39
  double integratedShift(double t) const { return std::log(cirSurvival(t) / market.survival(t)); }
};

struct Model {
  HullWhite hw;
  std::vector<Asset> assets;
  std::vector<Cir> credits;
  // Stochastic foreign short rates (an extension; the reference's foreign curves are deterministic): foreign[f] is
  // the Hull-White model of asset f's currency, fitted to that asset's carry curve.
  std::vector<HullWhite> foreign;
  std::vector<double> correlation;  // F x F over [rate, assets, credits, foreign rates]; empty: identity
  std::size_t numPaths = 0;
  std::uint64_t seed = 42;
  bool antithetic = true;
  std::vector<double> base;
  std::size_t numFactors() const { return 1 + assets.size() + credits.size() + foreign.size(); }
  // Columns of a step-table row: the reference's 24, then 8 per foreign rate.
  std::size_t stepStride() const { return 24 + 8 * foreign.size(); }
  double correlationOf(std::size_t i, std::size_t j) const {
    return correlation.empty() ? (i == j ? 1.0 : 0.0) : correlation[i * numFactors() + j];
  }
};

struct Swap {
  double notional = 0, fixedRate = 0;
  bool payFixed = true;
  std::vector<double> schedule;
};

struct Trade {
  enum Kind { kSwap, kForward, kOption, kBermudan, kSwapLegs } kind = kSwap;
  Swap swap;                         // swap, or a Bermudan's underlying; kSwapLegs: the floating leg's schedule
  std::vector<double> fixedSchedule; // kSwapLegs: the fixed leg's own schedule
  std::size_t asset = 0;             // forward / option
  double notional = 0, strike = 0, maturity = 0;
  bool call = true;
  std::vector<double> exercise;      // Bermudan
  bool physical = true;
  double position = 1.0;
  std::size_t degree = 3;
  bool twoRegressors = false;        // Bermudan: the regression on the short rate and the co-terminal swap rate
  std::vector<double> eventTimes() const;
};

struct Csa {
  double hc = 0, ho = INFINITY, mta = 0, ia = 0, mpr = 10.0 / 250.0;
  int type = 0;
  double haircut = 0, bondMaturity = 0;
  std::size_t assetIndex = 0;
};

struct NettingSet {
  std::vector<Trade> trades;
  std::optional<Csa> csa;
};

struct Options {
  double pfeQuantile = 0.95;
  std::size_t counterparty = 0;
  bool perTrade = false;
  double imQuantile = 0;
  std::size_t imInnerPaths = 0;
  double imMarginPeriod = 10.0 / 250.0;
  std::size_t imAuditPaths = 0, imAuditInnerPaths = 1024;
  std::size_t samples = 0;
  double histogramTime = -1;
  std::size_t histogramBins = 40;
  bool gross = false, collateralBands = false, tradeViews = false, exerciseViews = false, factorViews = false;
  double bondMaturity = 0;
  std::vector<double> extraDates, bandLevels{0.05, 0.5, 0.95}, factorBandLevels{0.05, 0.25, 0.5, 0.75, 0.95};
};

Model decodeModel(const double* a, std::size_t n);
NettingSet decodeNettingSet(const double* a, std::size_t n);
Options decodeOptions(const double* a, std::size_t n);

// Sorted, de-duplicated dates starting at 0 (src/core/time_grid.cpp:13-66).
struct Grid {
  std::vector<double> t;
  explicit Grid(std::vector<double> times);
  std::size_t atOrBefore(double x) const;
  std::optional<std::size_t> find(double x, double tol = 1e-9) const;
};

struct CompiledPlan {
  std::vector<double> times;
  std::vector<std::uint64_t> reporting;
  std::vector<std::uint32_t> header, indices;
  std::vector<double> params, steps, terms, requests;
  std::vector<float> paramsF, stepsF, termsF, requestsF;
  std::vector<double> marketSurvival;
  std::uint32_t rowsTotal = 0, numOutputs = 0;
  std::size_t numTrades = 0, numBermudans = 0, exerciseRows = 0, statsPerDate = 8;
};

CompiledPlan compile(const Model& m, const NettingSet& ns, const Options& o);

// One row of the step table (m.stepStride() values): the exact transitions of the rate state, its integral, the
// assets and the foreign rates from t0 to t1.
void stepRow(const Model& m, double t0, double t1, double* row);

// The inner paths of the nested exposure from date t (src/nested/nested_exposure.cpp:87-117, 211-244): the event
// dates after t with each one's step from the previous date and its operations, the periods' and terminal flows'
// constants, and the correlation rows of the rate and the assets.  periods are [nPer][6] (ts, te, tau, amount =
// sign x notional, fixed rate, slot: the swap whose fixing the period uses), terminals [nTerm][6] (asset, option,
// call, notional, strike, maturity).
struct NestProgram {
  std::size_t nA = 0;
  std::vector<double> times;           // [E]
  std::vector<double> coef;            // [E][24] step rows
  std::vector<std::uint32_t> begin;    // [E + 1] into ops
  std::vector<std::uint32_t> ops;      // kind << 28 | index: 0 payment, 1 fixing, 2 terminal flow
  std::vector<std::uint32_t> fixToday; // periods that fix at t itself
  std::vector<double> periods;         // [nPer][8]: tau, amount, fixed rate, slot, bond ratio, bond c, bond B, 0
  std::vector<double> terminals;       // [nTerm][8]: asset, option, call, notional, strike
  std::vector<double> chol;            // [(1 + nA)^2] lower
};
NestProgram nestProgram(const Model& m, const double* periods, std::size_t nPer, const double* terminals, std::size_t nTerm,
                        double t);

}  // namespace zk::host
