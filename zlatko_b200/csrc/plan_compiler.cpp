// Host plan compiler of zlatko_b200 (C++17).
//
// Compiles a netting set into the tables the fused kernels run: per-date transition coefficients,
// valuation terms merged per cash-flow date, the index table, CSA and model parameters, path-view
// rows and row-statistics requests.  The table layout and the term semantics are the reference's
// (gpu::compile, src/gpu/fused_exposure.cpp:214-707; term kinds fused_exposure.hpp:131-151), so a
// plan compiled here runs on the reference's own CPU kernels as well, and for every netting set the
// reference accepts the single-precision tables come out identical.  The compiler keeps every
// coefficient in double precision too (the FP64 mode) and lifts the reference's cap of 32 swaps per
// netting set: swap slots are reused once a floating coupon is paid (interval colouring), so only the
// number of coupons alive on one date is bounded.
#include "plan_compiler.h"

#include <algorithm>
#include <cstring>
#include <map>
#include <stdexcept>

#include "../../include/zlatko_b200.h"

namespace zk::host {

namespace {
constexpr std::size_t kMaxAssets = 4, kMaxCredits = 2, kMaxSlots = 32, kMaxNormals = 64, kMaxTradeGroups = 16;
// Bermudans: the reference's kernel prices at most 4 per netting set (fused_exposure.hpp:127); this compiler takes up
// to 256.  Plans with at most 4 keep the reference's tables; above 4 a Bermudan's index carries its high bits in the
// trade-group field of the term code (unused outside per-trade mode) and each Bermudan's exercise terms come
// directly before its own policy record, so the kernel needs one running exercise value per path.
constexpr std::size_t kMaxBermudans = 256, kRegisterBermudans = 4, kMaxExercises = 64, kMaxAmcDegree = 3, kStepStride = 24,
                      kTermStride = 8;
constexpr std::size_t kMaxInnerPaths = 1024, kInnerTop = 16;  // nested initial margin (fused_exposure.hpp:57-58)
constexpr std::size_t kParamCount = 84, kMaxSamples = 64, kPfeBins = 3072, kStatsPerDate = 8, kTradeStats = 5;
constexpr std::uint32_t kNoRow = 0xFFFFFFFFu;
enum Kind { kBond = 0, kFixedFloat = 1, kAsset = 2, kSetFixing = 3, kOption = 4, kBermExercise = 5, kBermDecide = 6,
            kBermContinue = 7, kBermBond = 8, kBermFloat = 9, kProbe = 10,
            // Terms on an asset whose foreign rate is stochastic (an extension; asset index in the extra field):
            // kForeignForward (B_f, c, A_f): c S P_f(t, T | x_f); kForeignOption (B_f, N, A, B, A_f, K, +-sd): Black on
            // S P_f(t, T | x_f) / P(t, T | x) with the reference's volatility.
            kForeignForward = 11, kForeignOption = 12,
            // The two-regressor basis of a Bermudan (an extension): before each policy / continuation record, the
            // co-terminal swap's annuity terms kBermAnnuity (tau, A, B) and float-leg terms kBermCoterm (+-1, A, B)
            // -- the kernel takes s = float leg / annuity -- and after it two kBermExt records holding the rest of
            // its coefficients.
            kBermAnnuity = 13, kBermCoterm = 14, kBermExt = 15 };
enum Op { kRowQuantile = 0, kRowMean = 1, kRowMeanPos = 2, kRowMeanNeg = 3, kRowSamples = 4, kRowHistogram = 5,
          kRowMeanProduct = 6, kRowQuantilePos = 7, kRowMeanPosTimes = 8, kRowMeanNegTimes = 9 };

struct In {
  const double* p;
  std::size_t n, i = 0;
  double d() {
    if (i >= n) throw std::invalid_argument("spec: truncated array");
    return p[i++];
  }
  std::size_t u() {
    const double v = d();
    if (!(v >= 0.0)) throw std::invalid_argument("spec: negative count");
    return static_cast<std::size_t>(v);
  }
};

Curve readCurve(In& in) {
  Curve c;
  const std::size_t n = in.u();
  if (n == 0) throw std::invalid_argument("curve: no pillars");
  for (std::size_t k = 0; k < n; ++k) c.t.push_back(in.d()), c.r.push_back(in.d());
  for (std::size_t k = 1; k < n; ++k)
    if (c.t[k] <= c.t[k - 1]) throw std::invalid_argument("curve: times must increase");
  return c;
}

std::vector<double> readSeq(In& in) {
  std::vector<double> v(in.u());
  for (auto& x : v) x = in.d();
  return v;
}

}  // namespace

// ---------------------------------------------------------------- market
double Curve::zero(double x) const {
  if (x <= t.front()) return r.front();
  if (x >= t.back()) return r.back();
  const std::size_t i = static_cast<std::size_t>(std::upper_bound(t.begin(), t.end(), x) - t.begin());
  const double w = (x - t[i - 1]) / (t[i] - t[i - 1]);
  return r[i - 1] + w * (r[i] - r[i - 1]);
}

double Curve::forward(double x) const {
  double slope = 0.0;
  if (x >= t.front() && x < t.back()) {
    const std::size_t i = static_cast<std::size_t>(std::upper_bound(t.begin(), t.end(), x) - t.begin());
    slope = (r[i] - r[i - 1]) / (t[i] - t[i - 1]);
  }
  return zero(x) + x * slope;
}

double Hazard::survival(double x) const {
  if (x <= 0.0) return 1.0;
  double integral = 0.0, prev = 0.0;
  for (std::size_t i = 0; i < pillars.size(); ++i) {
    const double end = i + 1 == pillars.size() ? x : std::min(x, pillars[i]);
    integral += hazards[i] * (end - prev);
    if (end >= x) break;
    prev = end;
  }
  return std::exp(-integral);
}

// Variance term of the G1++ bond price (Brigo-Mercurio); V(t, T) in hull_white.cpp:21-25.
double HullWhite::V(double t, double T) const {
  const double tau = T - t, e1 = std::exp(-a * tau);
  return sigma * sigma / (a * a) * (tau + 2.0 / a * e1 - 0.5 / a * e1 * e1 - 1.5 / a);
}

double HullWhite::bond(double t, double T, double x) const {
  if (T <= t) return 1.0;
  const double ratio = curve.discount(T) / curve.discount(t);
  return ratio * std::exp(0.5 * (V(t, T) - V(0.0, T) + V(0.0, t)) - B(t, T) * x);
}

// Closed-form E[exp(-int y)] of a CIR process.
double Cir::cirSurvival(double t) const {
  if (t <= 0.0) return 1.0;
  if (xi == 0.0) return std::exp(-(theta * t + (y0 - theta) * (1.0 - std::exp(-kappa * t)) / kappa));
  const double h = std::sqrt(kappa * kappa + 2.0 * xi * xi);
  const double eh = std::exp(h * t) - 1.0;
  const double denom = 2.0 * h + (kappa + h) * eh;
  const double logA = (2.0 * kappa * theta / (xi * xi)) * std::log(2.0 * h * std::exp(0.5 * (kappa + h) * t) / denom);
  return std::exp(logA - 2.0 * eh / denom * y0);
}

std::vector<double> Trade::eventTimes() const {
  switch (kind) {
    case kSwap: return swap.schedule;
    case kSwapLegs: {
      std::vector<double> v = swap.schedule;
      v.insert(v.end(), fixedSchedule.begin(), fixedSchedule.end());
      return v;
    }
    case kForward:
    case kOption: return {maturity};
    default: {
      std::vector<double> v = swap.schedule;
      v.insert(v.end(), exercise.begin(), exercise.end());
      return v;
    }
  }
}

Grid::Grid(std::vector<double> times) {
  times.erase(std::remove_if(times.begin(), times.end(), [](double x) { return x < 0.0 || !std::isfinite(x); }), times.end());
  times.push_back(0.0);
  std::sort(times.begin(), times.end());
  for (double x : times)
    if (t.empty() || x - t.back() > 1e-9) t.push_back(x);
}

std::size_t Grid::atOrBefore(double x) const {
  const auto it = std::upper_bound(t.begin(), t.end(), x + 1e-9);
  return it == t.begin() ? 0 : static_cast<std::size_t>(it - t.begin()) - 1;
}

std::optional<std::size_t> Grid::find(double x, double tol) const {
  const std::size_t i = atOrBefore(x);
  if (std::fabs(t[i] - x) <= tol) return i;
  if (i + 1 < t.size() && std::fabs(t[i + 1] - x) <= tol) return i + 1;
  return std::nullopt;
}

// ---------------------------------------------------------------- decoding (zlatko_b200/spec.py)
Model decodeModel(const double* a, std::size_t n) {
  In in{a, n};
  if (in.d() != 7001.0) throw std::invalid_argument("model: bad magic");
  Model m;
  m.hw.curve = readCurve(in);
  m.hw.a = in.d();
  m.hw.sigma = in.d();
  if (m.hw.a <= 1e-8) throw std::invalid_argument("HullWhite1F: mean reversion must be positive");
  if (m.hw.sigma < 0.0) throw std::invalid_argument("HullWhite1F: volatility must be non-negative");
  const std::size_t nA = in.u();
  for (std::size_t k = 0; k < nA; ++k) {
    Asset s;
    s.spot = in.d();
    s.vol = in.d();
    s.carry = readCurve(in);
    if (s.spot <= 0.0 || s.vol < 0.0) throw std::invalid_argument("asset: spot must be positive, volatility non-negative");
    m.assets.push_back(s);
  }
  const std::size_t nC = in.u();
  for (std::size_t k = 0; k < nC; ++k) {
    Cir c;
    c.kappa = in.d(), c.theta = in.d(), c.xi = in.d(), c.y0 = in.d();
    c.substeps = in.u();
    const std::size_t nh = in.u();
    for (std::size_t q = 0; q < nh; ++q) c.market.pillars.push_back(in.d()), c.market.hazards.push_back(in.d());
    if (c.kappa <= 0.0 || c.theta < 0.0 || c.xi < 0.0 || c.y0 < 0.0 || c.substeps == 0 || nh == 0)
      throw std::invalid_argument("CirIntensity: invalid parameters");
    m.credits.push_back(c);
  }
  const std::size_t F = in.u();
  if (F > 8) throw std::invalid_argument("correlation matrix has wrong dimension");
  for (std::size_t k = 0; k < F * F; ++k) m.correlation.push_back(in.d());
  m.numPaths = in.u();
  m.seed = static_cast<std::uint64_t>(in.d());
  m.antithetic = in.d() != 0.0;
  m.base = readSeq(in);
  if (in.i < in.n) {  // stochastic foreign rates (the spec module's extension block)
    if (in.d() != 7011.0) throw std::invalid_argument("model: unknown trailing block");
    const std::size_t nF = in.u();
    if (nF > nA || nF > 2) throw std::invalid_argument("model: at most two stochastic foreign rates, one per leading asset");
    for (std::size_t f = 0; f < nF; ++f) {
      HullWhite h;
      h.curve = m.assets[f].carry;
      h.a = in.d(), h.sigma = in.d();
      if (h.a <= 1e-8 || h.sigma < 0.0) throw std::invalid_argument("foreign HullWhite1F: invalid parameters");
      m.foreign.push_back(h);
    }
  }
  if (F > 0 && F != m.numFactors()) throw std::invalid_argument("correlation matrix has wrong dimension");
  return m;
}

NettingSet decodeNettingSet(const double* a, std::size_t n) {
  In in{a, n};
  if (in.d() != 7002.0) throw std::invalid_argument("netting set: bad magic");
  NettingSet ns;
  const std::size_t nt = in.u();
  auto readSwap = [&](Swap& s) {
    s.notional = in.d();
    s.fixedRate = in.d();
    s.payFixed = in.d() != 0.0;
    s.schedule = readSeq(in);
    if (s.schedule.size() < 2) throw std::invalid_argument("InterestRateSwap: schedule needs at least two dates");
    for (std::size_t k = 1; k < s.schedule.size(); ++k)
      if (s.schedule[k] <= s.schedule[k - 1]) throw std::invalid_argument("InterestRateSwap: schedule must be strictly increasing");
  };
  for (std::size_t k = 0; k < nt; ++k) {
    const int type = static_cast<int>(in.d());
    Trade t;
    if (type == 0) {
      t.kind = Trade::kSwap;
      readSwap(t.swap);
    } else if (type == 1 || type == 2) {
      t.kind = type == 1 ? Trade::kForward : Trade::kOption;
      t.asset = in.u();
      if (type == 2) t.call = in.d() != 0.0;
      t.notional = in.d();
      t.strike = in.d();
      t.maturity = in.d();
      if (t.maturity <= 0.0) throw std::invalid_argument("maturity must be positive");
    } else if (type == 3) {
      t.kind = Trade::kBermudan;
      readSwap(t.swap);
      t.exercise = readSeq(in);
      std::sort(t.exercise.begin(), t.exercise.end());
      t.physical = in.d() != 0.0;
      t.position = in.d();
      t.degree = in.u();
      if (t.degree >= 10) t.twoRegressors = true, t.degree -= 10;  // this library's two-regressor basis
      if (t.exercise.empty()) throw std::invalid_argument("BermudanSwaption: no exercise dates");
    } else if (type == 4) {  // swap with its own fixed and floating schedules
      t.kind = Trade::kSwapLegs;
      t.swap.notional = in.d();
      t.swap.fixedRate = in.d();
      t.swap.payFixed = in.d() != 0.0;
      t.fixedSchedule = readSeq(in);
      t.swap.schedule = readSeq(in);
      for (const auto* sch : {&t.fixedSchedule, &t.swap.schedule}) {
        if (sch->size() < 2) throw std::invalid_argument("swap legs: a schedule needs at least two dates");
        for (std::size_t q = 1; q < sch->size(); ++q)
          if ((*sch)[q] <= (*sch)[q - 1]) throw std::invalid_argument("swap legs: schedules must be strictly increasing");
      }
    } else {
      throw std::invalid_argument("netting set: unknown trade type");
    }
    ns.trades.push_back(t);
  }
  if (in.d() != 0.0) {
    Csa c;
    c.hc = in.d();
    const double own = in.d();
    c.ho = own < 0.0 ? INFINITY : own;
    c.mta = in.d();
    c.ia = in.d();
    c.mpr = in.d();
    c.type = static_cast<int>(in.d());
    c.haircut = in.d();
    c.bondMaturity = in.d();
    c.assetIndex = in.u();
    ns.csa = c;
  }
  return ns;
}

Options decodeOptions(const double* a, std::size_t n) {
  In in{a, n};
  if (in.d() != 7003.0) throw std::invalid_argument("options: bad magic");
  Options o;
  o.pfeQuantile = in.d();
  o.counterparty = in.u();
  o.perTrade = in.d() != 0.0;
  o.imQuantile = in.d();
  o.imInnerPaths = in.u();
  o.imMarginPeriod = in.d();
  o.imAuditPaths = in.u();
  o.imAuditInnerPaths = in.u();
  o.samples = in.u();
  o.histogramTime = in.d();
  o.histogramBins = in.u();
  o.gross = in.d() != 0.0;
  o.collateralBands = in.d() != 0.0;
  o.tradeViews = in.d() != 0.0;
  o.exerciseViews = in.d() != 0.0;
  o.factorViews = in.d() != 0.0;
  o.bondMaturity = in.d();
  o.extraDates = readSeq(in);
  o.bandLevels = readSeq(in);
  o.factorBandLevels = readSeq(in);
  return o;
}

// ---------------------------------------------------------------- compile
namespace {

struct Term {
  int kind;
  double slot, c, A, B, p1, p2, p3;
  std::size_t trade, bermudan, extra;
  bool merged = false;  // a merged bond / asset record: trade-independent fields dropped
  double ts = 0.0, te = 0.0;  // the floating period of a fixing / running-coupon term
};

bool sameBond(const Term& a, const Term& b) { return a.A == b.A && a.B == b.B; }

// Merges the terms of one date in double precision (the rules of mergeTerms, fused_exposure.cpp:45-100):
// bonds of one (A, B) summed; a running coupon with the bond of its payment date folded into p1;
// forwards on one asset summed; options, AMC terms and fixings kept, fixings last.
std::vector<Term> merge(const std::vector<Term>& in, bool manyBermudans = false) {
  std::vector<Term> floating, bonds, assets, options, fixings, exercise, amc, foreignFwd;
  for (const Term& r : in) {
    switch (r.kind) {
      case kBond: {
        auto it = std::find_if(bonds.begin(), bonds.end(), [&](const Term& b) { return sameBond(b, r); });
        if (it == bonds.end()) bonds.push_back(r);
        else it->c += r.c;
        break;
      }
      case kFixedFloat: {
        auto it = std::find_if(floating.begin(), floating.end(), [&](const Term& f) { return f.slot == r.slot && sameBond(f, r); });
        if (it == floating.end()) floating.push_back(r);
        else it->c += r.c, it->p1 += r.p1;
        break;
      }
      case kAsset: {
        auto it = std::find_if(assets.begin(), assets.end(), [&](const Term& a) { return a.slot == r.slot; });
        const double cA = r.c * r.A;
        if (it == assets.end()) {
          Term a{kAsset, r.slot, cA, 1.0, 0.0, 0.0, 0.0, 0.0, 0, 0, 0, true};
          assets.push_back(a);
        } else {
          it->c += cA;
        }
        break;
      }
      case kSetFixing: fixings.push_back(r); break;
      case kOption: options.push_back(r); break;
      case kForeignForward: {
        auto it = std::find_if(foreignFwd.begin(), foreignFwd.end(),
                               [&](const Term& a) { return a.extra == r.extra && a.slot == r.slot && a.A == r.A; });
        if (it == foreignFwd.end()) foreignFwd.push_back(r);
        else it->c += r.c;
        break;
      }
      case kForeignOption: options.push_back(r); break;
      case kBermExercise: {
        auto it = std::find_if(exercise.begin(), exercise.end(), [&](const Term& b) { return b.bermudan == r.bermudan && sameBond(b, r); });
        if (it == exercise.end()) exercise.push_back(r);
        else it->c += r.c;
        break;
      }
      default: amc.push_back(r);
    }
  }
  std::vector<Term> out;
  for (Term& f : floating) {
    auto it = std::find_if(bonds.begin(), bonds.end(), [&](const Term& b) { return sameBond(b, f); });
    if (it != bonds.end()) f.p1 += it->c, bonds.erase(it);
    out.push_back(f);
  }
  for (const Term& b : bonds) {
    if (b.c == 0.0) continue;
    out.push_back(Term{kBond, 0.0, b.c * b.A, 1.0, b.B, 0.0, 0.0, 0.0, 0, 0, 0, true});
  }
  for (const Term& a : assets)
    if (a.c != 0.0) out.push_back(a);
  for (const Term& a : foreignFwd)
    if (a.c != 0.0) out.push_back(a);
  out.insert(out.end(), options.begin(), options.end());
  if (!manyBermudans) {
    out.insert(out.end(), exercise.begin(), exercise.end());
    out.insert(out.end(), amc.begin(), amc.end());
  } else {  // Bermudan by Bermudan: its exercise terms, then its policy, continuation and exercised-tail records
    std::vector<std::size_t> ids;
    for (const Term& r : exercise) ids.push_back(r.bermudan);
    for (const Term& r : amc) ids.push_back(r.bermudan);
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    for (std::size_t b : ids) {
      for (const Term& r : exercise)
        if (r.bermudan == b) out.push_back(r);
      for (const Term& r : amc)
        if (r.bermudan == b) out.push_back(r);
    }
  }
  out.insert(out.end(), fixings.begin(), fixings.end());
  return out;
}

std::vector<double> cholesky(const std::vector<double>& a, std::size_t n) {
  std::vector<double> l(n * n, 0.0);
  for (std::size_t i = 0; i < n; ++i)
    for (std::size_t j = 0; j <= i; ++j) {
      if (std::fabs(a[i * n + j] - a[j * n + i]) > 1e-10) throw std::invalid_argument("cholesky: matrix must be symmetric");
      double sum = a[i * n + j];
      for (std::size_t k = 0; k < j; ++k) sum -= l[i * n + k] * l[j * n + k];
      if (i == j) {
        if (sum <= 0.0) throw std::invalid_argument("cholesky: matrix is not positive definite");
        l[i * n + i] = std::sqrt(sum);
      } else {
        l[i * n + j] = sum / l[j * n + j];
      }
    }
  return l;
}

std::uint32_t floatBits(float f) {
  std::uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

}  // namespace

// The exact step from t0 to t1 of the Hull-White state and its integral (hull_white.cpp:40-68) and of every
// lognormal asset (lognormal_asset.cpp:17-22), as one row of the step table: [0] e^{-a dt}, [1] sd of x,
// [2] [3] the integral's loadings on the x and independent normals, [4] the integral of the shift, [5]
// (1 - e^{-a dt}) / a, [6] dt, [8 + k] the log carry ratio, [12 + k] vol sqrt(dt), [16 + k] vol^2 dt / 2, [20 + c]
// the CIR++ shift integrated to t1.
void stepRow(const Model& m, double t0, double t1, double* row) {
  const HullWhite& hw = m.hw;
  const double a = hw.a, sigma = hw.sigma;
  const double dt = t1 - t0, e = std::exp(-a * dt), s2 = sigma * sigma;
  const double varX = s2 * (1 - e * e) / (2 * a);
  const double varI = s2 / (a * a) * (dt - 2 * (1 - e) / a + (1 - e * e) / (2 * a));
  const double cov = s2 / (2 * a * a) * (1 - e) * (1 - e);
  const double sdX = std::sqrt(varX), c1 = sdX > 0 ? cov / sdX : 0.0, c2 = std::sqrt(std::max(varI - c1 * c1, 0.0));
  const double g2 = dt - 2 / a * (std::exp(-a * t0) - std::exp(-a * t1)) + 0.5 / a * (std::exp(-2 * a * t0) - std::exp(-2 * a * t1));
  row[0] = e, row[1] = sdX, row[2] = c1, row[3] = c2;
  row[4] = std::log(hw.curve.discount(t0) / hw.curve.discount(t1)) + s2 / (2 * a * a) * g2;
  row[5] = (1 - e) / a, row[6] = dt;
  for (std::size_t k = 0; k < m.assets.size(); ++k) {
    const Asset& s = m.assets[k];
    row[8 + k] = std::log(s.carry.discount(t0) / s.carry.discount(t1));
    row[12 + k] = s.vol * std::sqrt(dt);
    row[16 + k] = 0.5 * s.vol * s.vol * dt;
  }
  for (std::size_t c = 0; c < m.credits.size(); ++c) row[20 + c] = m.credits[c].integratedShift(t1);
  // Stochastic foreign rate f (an extension): x_f of the foreign Hull-White model under the domestic measure, with
  // the quanto drift -rho(f, S_f) sigma_f sigma_S of its asset's volatility, and the integral of r_f = x_f + phi_f,
  // stepped exactly as the domestic rate: [0] e^{-a dt}, [1] sd of x_f, [2] [3] the integral's loadings, [4] the
  // integral of phi_f, [5] (1 - e^{-a dt}) / a, [6] the drift's contribution to x_f, [7] to its integral.
  for (std::size_t f = 0; f < m.foreign.size(); ++f) {
    const HullWhite& h = m.foreign[f];
    const double af = h.a, sf = h.sigma, ef = std::exp(-af * dt), s2f = sf * sf;
    const double vX = s2f * (1 - ef * ef) / (2 * af);
    const double vI = s2f / (af * af) * (dt - 2 * (1 - ef) / af + (1 - ef * ef) / (2 * af));
    const double cv = s2f / (2 * af * af) * (1 - ef) * (1 - ef);
    const double sd = std::sqrt(vX), k1 = sd > 0 ? cv / sd : 0.0, k2 = std::sqrt(std::max(vI - k1 * k1, 0.0));
    const double g = dt - 2 / af * (std::exp(-af * t0) - std::exp(-af * t1)) + 0.5 / af * (std::exp(-2 * af * t0) - std::exp(-2 * af * t1));
    const std::size_t fi = 1 + m.assets.size() + m.credits.size() + f;
    const double q = m.correlationOf(fi, 1 + f) * sf * m.assets[f].vol;
    double* r = row + 24 + 8 * f;
    r[0] = ef, r[1] = sd, r[2] = k1, r[3] = k2;
    r[4] = std::log(h.curve.discount(t0) / h.curve.discount(t1)) + s2f / (2 * af * af) * g;
    r[5] = (1 - ef) / af;
    r[6] = -q * (1 - ef) / af;
    r[7] = -q / af * (dt - (1 - ef) / af);
  }
}

NestProgram nestProgram(const Model& m, const double* periods, std::size_t nPer, const double* terminals, std::size_t nTerm, double t) {
  constexpr double kEps = 1e-10;  // the trades' tolerance for "on or before t" (nested_exposure.cpp:19)
  if (!m.foreign.empty()) throw std::invalid_argument("the nested exposure runs the reference's model: no stochastic foreign rates");
  NestProgram P;
  P.nA = m.assets.size();
  // Event dates after t (nested_exposure.cpp:87-117): fixings after t, payments and terminal flows after t.
  std::vector<double> times;
  for (std::size_t i = 0; i < nPer; ++i) {
    const double* q = periods + 6 * i;
    if (q[1] <= t + kEps) continue;
    if (q[0] > t + kEps) times.push_back(q[0]);
    times.push_back(q[1]);
  }
  for (std::size_t f = 0; f < nTerm; ++f)
    if (terminals[6 * f + 5] > t + kEps) times.push_back(terminals[6 * f + 5]);
  std::sort(times.begin(), times.end());
  for (double u : times)
    if (P.times.empty() || u > P.times.back() + 1e-9) P.times.push_back(u);
  const std::size_t E = P.times.size();
  auto at = [&](double u) {
    for (std::size_t e = 0; e < E; ++e)
      if (std::fabs(P.times[e] - u) <= 1e-9) return e;
    throw std::logic_error("nested exposure: event date not in the program");
  };
  std::vector<std::vector<std::uint32_t>> pay(E), fix(E), term(E);
  for (std::size_t i = 0; i < nPer; ++i) {
    const double* q = periods + 6 * i;
    if (q[1] <= t + kEps) continue;
    if (q[0] > t + kEps) fix[at(q[0])].push_back(static_cast<std::uint32_t>(i));
    else if (q[0] >= t - kEps) P.fixToday.push_back(static_cast<std::uint32_t>(i));  // fixed today, from x at t
    pay[at(q[1])].push_back(static_cast<std::uint32_t>(i));
  }
  for (std::size_t f = 0; f < nTerm; ++f)
    if (terminals[6 * f + 5] > t + kEps) term[at(terminals[6 * f + 5])].push_back(static_cast<std::uint32_t>(f));
  // The step of every event from the previous one (t first), and the event's operations in the reference's
  // order: payments, then fixings, then terminal flows.
  P.coef.assign(E * kStepStride, 0.0);
  P.begin.push_back(0);
  double prev = t;
  for (std::size_t e = 0; e < E; ++e) {
    stepRow(m, prev, P.times[e], &P.coef[e * kStepStride]);
    P.coef[e * kStepStride + 7] = m.hw.a;  // the inner step forms x (1 - e^{-a dt}) / a as the reference does
    prev = P.times[e];
    for (auto i : pay[e]) P.ops.push_back(i);
    for (auto i : fix[e]) P.ops.push_back((1u << 28) | i);
    for (auto f : term[e]) P.ops.push_back((2u << 28) | f);
    P.begin.push_back(static_cast<std::uint32_t>(P.ops.size()));
  }
  // Periods: tau, amount, fixed rate, slot, and the zero bond P(ts, te | x) = ratio exp(c - B x) of the fixing
  // (hull_white.cpp:27-31); terminal flows: asset, option, call, notional, strike.
  P.periods.assign(nPer * 8, 0.0);
  for (std::size_t i = 0; i < nPer; ++i) {
    const double* q = periods + 6 * i;
    double* r = &P.periods[8 * i];
    const double ts = q[0], te = q[1];
    r[0] = q[2], r[1] = q[3], r[2] = q[4], r[3] = q[5];
    if (te > ts) {
      r[4] = m.hw.curve.discount(te) / m.hw.curve.discount(ts);
      r[5] = 0.5 * (m.hw.V(ts, te) - m.hw.V(0.0, te) + m.hw.V(0.0, ts));
      r[6] = m.hw.B(ts, te);
    }
  }
  P.terminals.assign(nTerm * 8, 0.0);
  for (std::size_t f = 0; f < nTerm; ++f)
    for (int k = 0; k < 5; ++k) P.terminals[8 * f + k] = terminals[6 * f + k];
  // The first 1 + nA rows of the correlation's Cholesky factor (nested_exposure.cpp:136, 215-222).
  const std::size_t F = m.numFactors(), r = 1 + P.nA;
  std::vector<double> corr(F * F, 0.0);
  for (std::size_t i = 0; i < F; ++i) corr[i * F + i] = 1.0;
  if (!m.correlation.empty()) corr = m.correlation;
  const std::vector<double> chol = cholesky(corr, F);
  P.chol.assign(r * r, 0.0);
  for (std::size_t i = 0; i < r; ++i)
    for (std::size_t k = 0; k <= i; ++k) P.chol[i * r + k] = chol[i * F + k];
  return P;
}

CompiledPlan compile(const Model& m, const NettingSet& ns, const Options& o) {
  Options eff = o;
  if (o.gross || o.tradeViews) eff.perTrade = true;
  if (eff.perTrade && ns.trades.size() > kMaxTradeGroups) throw std::invalid_argument("per-trade statistics on the GPU support at most 16 trades");
  if (o.imQuantile < 0.0 || o.imQuantile > 1.0) throw std::invalid_argument("imQuantile must be in [0, 1]");
  if (o.imInnerPaths > 0) {
    // The kernel keeps the kInnerTop largest inner samples: the quantile's order statistic must be among them
    // (gpu::compile, fused_exposure.cpp:233-247).
    auto checkInner = [&](std::size_t n) {
      if (n > kMaxInnerPaths || n < 2) throw std::invalid_argument("nested initial margin: 2 to 1024 inner paths");
      const double rank = o.imQuantile * static_cast<double>(n - 1);
      if (static_cast<double>(n - 1) - std::floor(rank) >= static_cast<double>(kInnerTop - 1))
        throw std::invalid_argument("nested initial margin: the quantile needs more inner paths (keeps the 16 largest)");
    };
    checkInner(o.imInnerPaths);
    if (o.imAuditPaths > 0) {
      checkInner(o.imAuditInnerPaths);
      if (o.imAuditInnerPaths <= o.imInnerPaths)
        throw std::invalid_argument("nested initial margin: the audit needs more inner paths than the kernel");
    }
  }
  if (m.assets.size() > kMaxAssets) throw std::invalid_argument("GPU kernel supports at most 4 assets");
  if (m.credits.size() > kMaxCredits) throw std::invalid_argument("GPU kernel supports at most 2 credits");
  for (const auto& c : m.credits)
    if (c.substeps != m.credits.front().substeps) throw std::invalid_argument("GPU kernel needs the same CIR substeps for all credits");
  if (!m.credits.empty() && o.counterparty >= m.credits.size()) throw std::invalid_argument("counterparty index out of range");
  if (m.numPaths == 0) throw std::invalid_argument("numPaths must be positive");
  for (const auto& t : ns.trades)
    if ((t.kind == Trade::kForward || t.kind == Trade::kOption) && t.asset >= m.assets.size()) throw std::invalid_argument("unknown asset");

  // Grids: reporting = base + trade events; simulation = + t - MPR under a CSA, + extra dates.
  std::vector<double> events = m.base;
  for (const auto& t : ns.trades) {
    const auto e = t.eventTimes();
    events.insert(events.end(), e.begin(), e.end());
  }
  const Grid reporting(events);
  std::vector<double> sim = reporting.t;
  if (ns.csa && ns.csa->mpr > 0.0)
    for (double x : reporting.t)
      if (x > ns.csa->mpr) sim.push_back(x - ns.csa->mpr);
  // Nested initial margin: inner paths run from every reporting date t to t + MPR, so t + MPR joins the grid.
  if (o.imInnerPaths > 0) {
    const double horizon = reporting.t.back();
    for (double x : reporting.t)
      if (x + o.imMarginPeriod <= horizon + 1e-10) sim.push_back(x + o.imMarginPeriod);
  }
  sim.insert(sim.end(), o.extraDates.begin(), o.extraDates.end());
  const Grid grid(sim);
  const std::size_t nT = grid.t.size();
  const HullWhite& hw = m.hw;

  CompiledPlan P;
  P.times = grid.t;
  const std::size_t perTradeGroups = eff.perTrade ? ns.trades.size() : 0;
  P.statsPerDate = (kStatsPerDate + kTradeStats * perTradeGroups + 3) / 4 * 4;
  P.numTrades = ns.trades.size();

  // ---- step coefficients (the exact transitions of hull_white.cpp:40-68 and lognormal_asset.cpp:17-22)
  const std::size_t stride = m.stepStride();
  P.steps.assign(nT * stride, 0.0);
  for (std::size_t j = 1; j < nT; ++j) stepRow(m, grid.t[j - 1], grid.t[j], &P.steps[j * stride]);
  if (!m.foreign.empty() && o.imInnerPaths > 0)
    throw std::invalid_argument("the nested initial margin runs the reference's model: no stochastic foreign rates");

  // ---- valuation terms per date
  std::vector<std::vector<Term>> at(nT);
  auto bondA = [&](double t, double T) { return hw.bond(t, T, 0.0); };
  auto bondB = [&](double t, double T) { return T <= t ? 0.0 : hw.B(t, T); };
  std::size_t tradeIndex = 0;
  auto add = [&](std::size_t j, int kind, double slot, double c, double A, double B, double p1 = 0, double p2 = 0, double p3 = 0) {
    at[j].push_back(Term{kind, slot, c, A, B, p1, p2, p3, tradeIndex, 0, 0});
  };
  auto addAmc = [&](std::size_t j, int kind, std::size_t b, std::size_t extra, double slot, double c, double A, double B, double p1 = 0) {
    at[j].push_back(Term{kind, slot, c, A, B, p1, 0.0, 0.0, tradeIndex, b, extra});
  };
  std::size_t swapSlots = 0, bermudans = 0;
  struct AmcInfo { std::vector<std::size_t> exerciseDates; };
  std::vector<AmcInfo> amc;
  for (; tradeIndex < ns.trades.size(); ++tradeIndex) {
    const Trade& tr = ns.trades[tradeIndex];
    if (tr.kind == Trade::kSwap) {
      const double sign = tr.swap.payFixed ? 1.0 : -1.0, n = tr.swap.notional, k = tr.swap.fixedRate;
      const auto& sch = tr.swap.schedule;
      const double slot = static_cast<double>(swapSlots++);
      for (std::size_t i = 1; i < sch.size(); ++i) {
        const double ts = sch[i - 1], te = sch[i], tau = te - ts;
        // The fixing is recovered on the path at the last date on or before ts, after the previous
        // period's terms of that date (fixings merge last).
        const std::size_t kf = grid.atOrBefore(ts);
        add(kf, kSetFixing, slot, tau, bondA(grid.t[kf], ts) / bondA(grid.t[kf], te), bondB(grid.t[kf], ts) - bondB(grid.t[kf], te));
        at[kf].back().ts = ts, at[kf].back().te = te;
        for (std::size_t j = 0; j < nT; ++j) {
          const double t = grid.t[j];
          if (te <= t + 1e-10) continue;
          if (ts >= t - 1e-10) {
            add(j, kBond, 0, sign * n, bondA(t, ts), bondB(t, ts));
            add(j, kBond, 0, -sign * n * (1 + k * tau), bondA(t, te), bondB(t, te));
          } else {
            add(j, kFixedFloat, slot, sign * n * tau, bondA(t, te), bondB(t, te));
            at[j].back().ts = ts, at[j].back().te = te;
            add(j, kBond, 0, -sign * n * k * tau, bondA(t, te), bondB(t, te));
          }
        }
      }
    } else if (tr.kind == Trade::kSwapLegs) {
      // The floating leg exactly as a swap with a zero fixed rate on its schedule (fixings recovered on the
      // path, running coupon with one exponential); the fixed leg as one coupon bond per fixed period.  The
      // value equals the reference's decomposition float(K = 0) + [swap(K) - swap(0)] on the fixed schedule.
      const double sign = tr.swap.payFixed ? 1.0 : -1.0, n = tr.swap.notional, k = tr.swap.fixedRate;
      const auto& sch = tr.swap.schedule;
      const double slot = static_cast<double>(swapSlots++);
      for (std::size_t i = 1; i < sch.size(); ++i) {
        const double ts = sch[i - 1], te = sch[i], tau = te - ts;
        const std::size_t kf = grid.atOrBefore(ts);
        add(kf, kSetFixing, slot, tau, bondA(grid.t[kf], ts) / bondA(grid.t[kf], te), bondB(grid.t[kf], ts) - bondB(grid.t[kf], te));
        at[kf].back().ts = ts, at[kf].back().te = te;
        for (std::size_t j = 0; j < nT; ++j) {
          const double t = grid.t[j];
          if (te <= t + 1e-10) continue;
          if (ts >= t - 1e-10) {
            add(j, kBond, 0, sign * n, bondA(t, ts), bondB(t, ts));
            add(j, kBond, 0, -sign * n, bondA(t, te), bondB(t, te));
          } else {
            add(j, kFixedFloat, slot, sign * n * tau, bondA(t, te), bondB(t, te));
            at[j].back().ts = ts, at[j].back().te = te;
          }
        }
      }
      const auto& fs = tr.fixedSchedule;
      for (std::size_t i = 1; i < fs.size(); ++i) {
        const double te = fs[i], tau = te - fs[i - 1];
        for (std::size_t j = 0; j < nT; ++j) {
          const double t = grid.t[j];
          if (te <= t + 1e-10) continue;
          add(j, kBond, 0, -sign * n * k * tau, bondA(t, te), bondB(t, te));
        }
      }
    } else if (tr.kind == Trade::kForward) {
      const Asset& s = m.assets[tr.asset];
      for (std::size_t j = 0; j < nT; ++j) {
        const double t = grid.t[j];
        if (t >= tr.maturity - 1e-10) continue;
        if (tr.asset < m.foreign.size()) {
          const HullWhite& h = m.foreign[tr.asset];
          at[j].push_back(Term{kForeignForward, h.B(t, tr.maturity), tr.notional, h.bond(t, tr.maturity, 0.0), 0.0, 0.0, 0.0, 0.0,
                               tradeIndex, 0, tr.asset});
        } else {
          add(j, kAsset, static_cast<double>(tr.asset), tr.notional, s.carryDiscount(t, tr.maturity), 0.0);
        }
        add(j, kBond, 0, -tr.notional * tr.strike, bondA(t, tr.maturity), bondB(t, tr.maturity));
      }
    } else if (tr.kind == Trade::kOption) {
      const Asset& s = m.assets[tr.asset];
      if (tr.strike <= 0.0) throw std::invalid_argument("EuropeanOption: invalid expiry or strike");
      for (std::size_t j = 0; j < nT; ++j) {
        const double t = grid.t[j];
        if (t >= tr.maturity - 1e-10) continue;
        const double sd = s.vol * std::sqrt(tr.maturity - t);
        if (tr.asset < m.foreign.size()) {
          const HullWhite& h = m.foreign[tr.asset];
          at[j].push_back(Term{kForeignOption, h.B(t, tr.maturity), tr.notional, bondA(t, tr.maturity), bondB(t, tr.maturity),
                               h.bond(t, tr.maturity, 0.0), tr.strike, tr.call ? sd : -sd, tradeIndex, 0, tr.asset});
        } else {
          add(j, kOption, static_cast<double>(tr.asset), tr.notional, bondA(t, tr.maturity), bondB(t, tr.maturity),
              s.carryDiscount(t, tr.maturity), tr.strike, tr.call ? sd : -sd);
        }
      }
    } else {
      if (bermudans >= kMaxBermudans) throw std::invalid_argument("the GPU kernel prices at most 256 Bermudan swaptions per netting set");
      if (tr.exercise.size() > kMaxExercises) throw std::invalid_argument("too many exercise dates for the GPU kernel");
      if (tr.degree > kMaxAmcDegree) throw std::invalid_argument("AMC regression degree above 3 on the GPU");
      const std::size_t b = bermudans++;
      const double sign = tr.swap.payFixed ? 1.0 : -1.0, n = tr.swap.notional, k = tr.swap.fixedRate, pos = tr.position;
      const auto& sch = tr.swap.schedule;
      const auto& ex = tr.exercise;
      const std::size_t nE = ex.size();
      // Two-regressor basis: the co-terminal swap from `start` (its annuity and its float leg at time t), before the
      // policy or continuation record; after it, the records of its coefficients beyond the second.
      auto coterminal = [&](std::size_t j, double t, double start) {
        if (!tr.twoRegressors) return;
        std::size_t first = sch.size();
        for (std::size_t i = 1; i < sch.size(); ++i)
          if (sch[i - 1] >= start - 1e-10) {
            if (first == sch.size()) first = i;
            addAmc(j, kBermAnnuity, b, 0, 0.0, sch[i] - sch[i - 1], bondA(t, sch[i]), bondB(t, sch[i]));
          }
        if (first == sch.size()) throw std::invalid_argument("Bermudan: an exercise date at or after the last period");
        addAmc(j, kBermCoterm, b, 0, 0.0, 1.0, bondA(t, sch[first - 1]), bondB(t, sch[first - 1]));
        addAmc(j, kBermCoterm, b, 0, 0.0, -1.0, bondA(t, sch.back()), bondB(t, sch.back()));
      };
      auto extension = [&](std::size_t j) {
        if (!tr.twoRegressors) return;
        addAmc(j, kBermExt, b, 0, 0.0, 0.0, 0.0, 0.0);
        addAmc(j, kBermExt, b, 0, 0.0, 0.0, 0.0, 0.0);
      };
      if (tr.twoRegressors && o.imInnerPaths > 0)
        throw std::invalid_argument("the nested initial margin of a Bermudan with the two-regressor basis");
      for (double e : ex)
        if (!std::any_of(sch.begin(), sch.end() - 1, [e](double x) { return std::fabs(x - e) < 1e-8; }))
          throw std::invalid_argument("BermudanSwaption: exercise dates must be start dates of the underlying periods");
      AmcInfo info;
      for (double e : ex) {
        const auto idx = grid.find(e, 1e-8);
        if (!idx) throw std::invalid_argument("Bermudan exercise date not on the simulation grid");
        info.exerciseDates.push_back(*idx);
      }
      std::vector<long> lastEx(sch.size() - 1, -1);
      for (std::size_t i = 1; i < sch.size(); ++i)
        for (std::size_t e = 0; e < nE; ++e)
          if (ex[e] <= sch[i - 1] + 1e-10) lastEx[i - 1] = static_cast<long>(e);
      const double slot = static_cast<double>(swapSlots++);
      if (tr.physical)
        for (std::size_t i = 1; i < sch.size(); ++i) {
          if (lastEx[i - 1] < 0) continue;
          const double ts = sch[i - 1], te = sch[i];
          const std::size_t kf = grid.atOrBefore(ts);
          add(kf, kSetFixing, slot, te - ts, bondA(grid.t[kf], ts) / bondA(grid.t[kf], te), bondB(grid.t[kf], ts) - bondB(grid.t[kf], te));
          at[kf].back().ts = ts, at[kf].back().te = te;
        }
      for (std::size_t j = 0; j < nT; ++j) {
        const double t = grid.t[j];
        std::size_t next = 0;
        while (next < nE && ex[next] <= t + 1e-10) ++next;
        for (std::size_t e = 0; e < nE; ++e) {
          if (info.exerciseDates[e] != j) continue;
          for (std::size_t i = 1; i < sch.size(); ++i) {
            const double ts = sch[i - 1], te = sch[i], tau = te - ts;
            if (ts < ex[e] - 1e-10) continue;
            addAmc(j, kBermExercise, b, e, 0.0, sign * n, bondA(t, ts), bondB(t, ts));
            addAmc(j, kBermExercise, b, e, 0.0, -sign * n * (1 + k * tau), bondA(t, te), bondB(t, te));
          }
          coterminal(j, t, ex[e]);
          addAmc(j, kBermDecide, b, e, 0.0, 0.0, 0.0, 0.0);
          extension(j);
        }
        if (next < nE) {
          coterminal(j, t, ex[next]);
          addAmc(j, kBermContinue, b, 0, pos, 0.0, 0.0, 0.0);
          extension(j);
        }
        if (tr.physical)
          for (std::size_t i = 1; i < sch.size(); ++i) {
            if (lastEx[i - 1] < 0) continue;
            const double ts = sch[i - 1], te = sch[i], tau = te - ts;
            if (te <= t + 1e-10) continue;
            const auto kMax = static_cast<std::size_t>(lastEx[i - 1]);
            if (ts >= t - 1e-10) {
              addAmc(j, kBermBond, b, kMax, 0.0, pos * sign * n, bondA(t, ts), bondB(t, ts));
              addAmc(j, kBermBond, b, kMax, 0.0, -pos * sign * n * (1 + k * tau), bondA(t, te), bondB(t, te));
            } else {
              addAmc(j, kBermFloat, b, kMax, slot, pos * sign * n * tau, bondA(t, te), bondB(t, te), -pos * sign * n * k * tau);
              at[j].back().ts = ts, at[j].back().te = te;
            }
          }
      }
      amc.push_back(info);
      P.exerciseRows += nE;
    }
  }
  P.numBermudans = amc.size();
  const bool manyBermudans = amc.size() > kRegisterBermudans;
  if (amc.size() > 16 && perTradeGroups > 0) throw std::invalid_argument("per-trade views of more than 16 Bermudans");
  if (manyBermudans && o.imInnerPaths > 0) throw std::invalid_argument("the nested initial margin of more than 4 Bermudans");

  // ---- swap slots.  Up to 32 swaps keep one slot each (the reference's numbering, identical tables).
  // Beyond that a slot is keyed by the floating period (ts, te) instead of the swap: the fixing of a
  // period is the same for every swap, so coupons of one period share a slot (and merge), duplicate
  // fixings are dropped, and a slot is reused once its period is paid (interval colouring).
  if (swapSlots > kMaxSlots) {
    std::map<std::pair<double, double>, std::size_t> keyOf;
    for (const auto& terms : at)
      for (const Term& r : terms)
        if (r.kind == kSetFixing || r.kind == kFixedFloat || r.kind == kBermFloat) keyOf.emplace(std::make_pair(r.ts, r.te), 0);
    std::size_t nk = 0;
    for (auto& kv : keyOf) kv.second = nk++;
    std::vector<std::size_t> first(nk, nT), last(nk, 0);
    for (std::size_t j = 0; j < nT; ++j)
      for (const Term& r : at[j])
        if (r.kind == kSetFixing || r.kind == kFixedFloat || r.kind == kBermFloat) {
          const std::size_t key = keyOf[{r.ts, r.te}];
          first[key] = std::min(first[key], j), last[key] = std::max(last[key], j);
        }
    std::vector<std::size_t> order(nk);
    for (std::size_t q = 0; q < nk; ++q) order[q] = q;
    std::stable_sort(order.begin(), order.end(), [&](std::size_t x, std::size_t y) { return first[x] < first[y]; });
    std::vector<std::size_t> busyUntil, colour(nk, 0);
    for (std::size_t q : order) {
      std::size_t c = 0;
      while (c < busyUntil.size() && busyUntil[c] > first[q]) ++c;
      if (c == busyUntil.size()) busyUntil.push_back(0);
      busyUntil[c] = last[q];
      colour[q] = c;
    }
    if (busyUntil.size() > kMaxSlots) throw std::invalid_argument("more than 32 floating periods alive on one date in a netting set");
    for (auto& terms : at) {
      std::vector<Term> kept;
      for (Term& r : terms) {
        if (r.kind == kSetFixing || r.kind == kFixedFloat || r.kind == kBermFloat) r.slot = static_cast<double>(colour[keyOf[{r.ts, r.te}]]);
        if (r.kind == kSetFixing &&
            std::any_of(kept.begin(), kept.end(), [&](const Term& q) { return q.kind == kSetFixing && q.slot == r.slot; }))
          continue;  // the same period's fixing, already recorded on this date
        kept.push_back(r);
      }
      terms.swap(kept);
    }
  }

  // ---- rows and requests of the path views (fused_exposure.cpp:435-609)
  std::vector<std::size_t> repDates;
  for (std::size_t j = 0; j < nT; ++j)
    if (reporting.find(grid.t[j])) repDates.push_back(j);
  const auto nR = static_cast<std::uint32_t>(repDates.size());
  const std::size_t nTr = perTradeGroups;
  const std::size_t S = std::min(o.samples, std::min<std::size_t>(kMaxSamples, m.numPaths));
  std::uint32_t nextRow = 0;
  auto block = [&](std::uint32_t rows) { const std::uint32_t r = nextRow; nextRow += rows; return r; };
  struct Rows { std::uint32_t exposure = 0, valueChange = kNoRow, exposureValue = kNoRow, netted = kNoRow, collateral = kNoRow,
                gross = kNoRow, trades = kNoRow, exercise = kNoRow, conditionalIm = kNoRow; } L;
  const bool hasCsa = ns.csa.has_value(), im = o.imQuantile > 0.0, histogram = o.histogramTime >= 0.0;
  L.exposure = block(nR);
  if (im) L.valueChange = block(nR);
  if (S > 0 || histogram) L.exposureValue = block(nR);
  if (S > 0) L.netted = block(nR);
  if (hasCsa && (S > 0 || o.collateralBands)) L.collateral = block(nR);
  if (o.gross) L.gross = block(nR);
  if (o.tradeViews) L.trades = block(static_cast<std::uint32_t>(nTr * nR));
  if (o.exerciseViews && !amc.empty()) L.exercise = block(static_cast<std::uint32_t>(amc.size()));
  if (o.imInnerPaths > 0) L.conditionalIm = block(nR);
  auto probe = [&](std::size_t j, std::uint32_t row, int what, std::size_t index, double offset = 0.0, double A = 0.0, double B = 0.0) {
    at[j].push_back(Term{kProbe, static_cast<double>(what + 16 * static_cast<int>(index)), offset, A, B, static_cast<double>(row), 0.0, 0.0, 0, 0, 0});
  };
  std::uint32_t deflatorRows = kNoRow;
  if (o.gross || o.tradeViews || o.factorViews || o.imInnerPaths > 0) {
    deflatorRows = block(nR);
    for (std::uint32_t r = 0; r < nR; ++r) probe(repDates[r], deflatorRows + r, 1, 0);
  }
  struct { std::uint32_t x = kNoRow, bond = kNoRow; std::vector<std::uint32_t> asset, deflated, intensity, survival, increments; } F;
  if (o.factorViews) {
    F.x = block(nR);
    F.bond = block(nR);
    for (std::uint32_t r = 0; r < nR; ++r) {
      const std::size_t j = repDates[r];
      const double T = std::max(o.bondMaturity, grid.t[j]);
      probe(j, F.x + r, 0, 0);
      probe(j, F.bond + r, 7, 0, 0.0, bondA(grid.t[j], T), bondB(grid.t[j], T));
    }
    for (std::size_t ai = 0; ai < m.assets.size(); ++ai) {
      F.asset.push_back(block(nR));
      F.deflated.push_back(block(nR));
      for (std::uint32_t r = 0; r < nR; ++r) probe(repDates[r], F.asset.back() + r, 2, ai), probe(repDates[r], F.deflated.back() + r, 6, ai);
    }
    for (std::size_t c = 0; c < m.credits.size(); ++c) {
      F.intensity.push_back(block(nR));
      F.survival.push_back(block(nR));
      for (std::uint32_t r = 0; r < nR; ++r) probe(repDates[r], F.intensity.back() + r, 4, c), probe(repDates[r], F.survival.back() + r, 5, c);
    }
    if (nT > 1) {
      F.increments.push_back(block(1));
      probe(1, F.increments.back(), 0, 0);
      for (std::size_t ai = 0; ai < m.assets.size(); ++ai) F.increments.push_back(block(1)), probe(1, F.increments.back(), 3, ai);
      for (std::size_t c = 0; c < m.credits.size(); ++c) F.increments.push_back(block(1)), probe(1, F.increments.back(), 4, c, -m.credits[c].y0);
    }
  }
  P.rowsTotal = nextRow;
  auto request = [&](int op, std::uint32_t row, std::uint32_t count = 1, double level = 0.0, std::uint32_t row2 = 0, double lo = 0.0, double hi = 0.0) {
    const std::size_t out = P.numOutputs;
    for (double v : {double(op), double(row), double(row2), double(count), level, lo, hi, double(out)}) P.requests.push_back(v);
    P.numOutputs += op == kRowHistogram ? count + 2 : count;
  };
  auto perDate = [&](int op, std::uint32_t base, std::uint32_t count = 1, double level = 0.0, std::uint32_t row2Base = 0) {
    for (std::uint32_t r = 0; r < nR; ++r) request(op, base + r, count, level, row2Base == 0 ? 0 : row2Base + r);
  };
  auto profileOf = [&](std::uint32_t base) {
    perDate(kRowMean, base);
    perDate(kRowMeanPos, base);
    perDate(kRowMeanNeg, base);
    perDate(kRowQuantilePos, base, 1, o.pfeQuantile);
    perDate(kRowMeanPosTimes, base, 1, 0.0, deflatorRows);
    perDate(kRowMeanNegTimes, base, 1, 0.0, deflatorRows);
  };
  perDate(kRowQuantile, L.exposure, 1, o.pfeQuantile);
  if (im) perDate(kRowQuantile, L.valueChange, 1, o.imQuantile);
  if (S > 0) {
    perDate(kRowSamples, L.exposureValue, static_cast<std::uint32_t>(S));
    perDate(kRowSamples, L.netted, static_cast<std::uint32_t>(S));
    if (L.collateral != kNoRow) perDate(kRowSamples, L.collateral, static_cast<std::uint32_t>(S));
  }
  if (L.conditionalIm != kNoRow) {
    perDate(kRowMeanProduct, L.conditionalIm, 1, 0.0, deflatorRows);
    perDate(kRowMean, L.conditionalIm);
    for (double q : {0.05, 0.5, 0.95}) perDate(kRowQuantile, L.conditionalIm, 1, q);
  }
  if (o.collateralBands && L.collateral != kNoRow)
    for (double q : o.bandLevels) perDate(kRowQuantile, L.collateral, 1, q);
  if (o.gross) profileOf(L.gross);
  if (histogram) {
    std::size_t rank = 0;
    for (std::size_t r = 0; r < nR; ++r)
      if (grid.t[repDates[r]] <= o.histogramTime + 1e-10) rank = r;
    const std::size_t bins = std::max<std::size_t>(1, std::min<std::size_t>(o.histogramBins, kPfeBins));
    request(kRowHistogram, L.exposureValue + static_cast<std::uint32_t>(rank), static_cast<std::uint32_t>(bins));
  }
  if (o.tradeViews)
    for (std::size_t i = 0; i < nTr; ++i) {
      const auto base = L.trades + static_cast<std::uint32_t>(i * nR);
      profileOf(base);
      if (S > 0) perDate(kRowSamples, base, static_cast<std::uint32_t>(S));
      for (double q : o.bandLevels) perDate(kRowQuantile, base, 1, q);
      perDate(kRowMeanProduct, base, 1, 0.0, deflatorRows);
    }
  if (L.exercise != kNoRow)
    for (std::size_t b = 0; b < amc.size(); ++b) {
      const auto row = L.exercise + static_cast<std::uint32_t>(b);
      const double nE = static_cast<double>(amc[b].exerciseDates.size());
      request(kRowHistogram, row, static_cast<std::uint32_t>(nE + 1), 0.0, 0, -1.5, nE - 0.5);
      if (S > 0) request(kRowSamples, row, static_cast<std::uint32_t>(S));
    }
  if (o.factorViews) {
    if (S > 0) perDate(kRowSamples, F.x, static_cast<std::uint32_t>(S));
    for (double q : o.factorBandLevels) perDate(kRowQuantile, F.x, 1, q);
    perDate(kRowMean, F.x);
    perDate(kRowMean, deflatorRows);
    perDate(kRowMean, F.bond);
    for (std::size_t ai = 0; ai < m.assets.size(); ++ai) {
      if (S > 0) perDate(kRowSamples, F.asset[ai], static_cast<std::uint32_t>(S));
      for (double q : o.factorBandLevels) perDate(kRowQuantile, F.asset[ai], 1, q);
      perDate(kRowMean, F.asset[ai]);
      perDate(kRowMean, F.deflated[ai]);
    }
    for (std::size_t c = 0; c < m.credits.size(); ++c) {
      if (S > 0) perDate(kRowSamples, F.intensity[c], static_cast<std::uint32_t>(S)), perDate(kRowSamples, F.survival[c], static_cast<std::uint32_t>(S));
      for (double q : o.factorBandLevels) perDate(kRowQuantile, F.intensity[c], 1, q);
      perDate(kRowMean, F.survival[c]);
    }
    for (auto row : F.increments) request(kRowMean, row);
    for (auto ra : F.increments)
      for (auto rb : F.increments) request(kRowMeanProduct, ra, 1, 0.0, rb);
  }

  // ---- index table and merged terms
  const std::size_t offCall = nT + 1, offRep = offCall + nT, offIm = offRep + nT;
  P.indices.assign(offIm + nT, kNoRow);
  for (std::size_t j = 0; j < offIm; ++j) P.indices[j] = 0u;
  if (o.imInnerPaths > 0)
    for (std::size_t r = 0; r < nR; ++r)
      if (const auto target = grid.find(grid.t[repDates[r]] + o.imMarginPeriod, 1e-8))
        P.indices[offIm + repDates[r]] = static_cast<std::uint32_t>(*target);
  for (std::size_t j = 0; j < nT; ++j) {
    P.indices[j] = static_cast<std::uint32_t>(P.terms.size() / kTermStride);
    auto emit = [&](const std::vector<Term>& recs, std::size_t group) {
      for (const Term& r : merge(recs, manyBermudans)) {
        const std::size_t b = r.merged ? 0 : r.bermudan;
        const double extra = r.merged ? 0.0 : static_cast<double>(r.extra);
        // Bermudan b: low 4 bits in the reference's field, high bits in the trade-group field (never per-trade here).
        P.terms.push_back(static_cast<double>(r.kind) + 16.0 * static_cast<double>(group + (b >> 4)) +
                          256.0 * static_cast<double>(b & 15) + 4096.0 * extra);
        for (double v : {r.slot, r.c, r.A, r.B, r.p1, r.p2, r.p3}) P.terms.push_back(v);
      }
    };
    if (perTradeGroups == 0) {
      emit(at[j], 0);
    } else {
      for (std::size_t g = 0; g < perTradeGroups; ++g) {
        std::vector<Term> grp;
        for (const Term& r : at[j])
          if (r.trade == g) grp.push_back(r);
        emit(grp, g);
      }
    }
  }
  P.indices[nT] = static_cast<std::uint32_t>(P.terms.size() / kTermStride);
  const double mpr = hasCsa ? ns.csa->mpr : 0.0;
  for (std::size_t j = 0; j < nT; ++j) {
    P.indices[offCall + j] = static_cast<std::uint32_t>(grid.atOrBefore(std::max(grid.t[j] - mpr, 0.0)));
    if (reporting.find(grid.t[j])) {
      P.reporting.push_back(j);
      P.indices[offRep + j] = static_cast<std::uint32_t>(P.reporting.size());
    }
  }

  // ---- parameters: CIR x2 | CSA | spots | Cholesky rows | collateral security
  const std::size_t nCorr = m.numFactors();
  std::size_t numNormals = nCorr + 1 + m.foreign.size();  // drivers | rate integral | foreign integrals | CIR bridges
  for (const auto& c : m.credits) numNormals += c.substeps - 1;
  if (numNormals > kMaxNormals) throw std::invalid_argument("too many normals per step for the GPU kernel");
  std::vector<double> corr = m.correlation;
  if (corr.empty()) {
    corr.assign(nCorr * nCorr, 0.0);
    for (std::size_t i = 0; i < nCorr; ++i) corr[i * nCorr + i] = 1.0;
  }
  for (std::size_t i = 0; i < nCorr; ++i)
    if (std::fabs(corr[i * nCorr + i] - 1.0) > 1e-12) throw std::invalid_argument("correlation matrix must have unit diagonal");
  const std::vector<double> chol = cholesky(corr, nCorr);
  P.params.assign(kParamCount, 0.0);
  for (std::size_t c = 0; c < m.credits.size(); ++c) {
    P.params[4 * c] = m.credits[c].kappa, P.params[4 * c + 1] = m.credits[c].theta;
    P.params[4 * c + 2] = m.credits[c].xi, P.params[4 * c + 3] = m.credits[c].y0;
  }
  if (hasCsa) {
    const Csa& c = *ns.csa;
    if (c.hc < 0.0 || c.ho < 0.0 || c.mta < 0.0 || c.mpr < 0.0 || c.haircut < 0.0 || c.haircut >= 1.0)
      throw std::invalid_argument("simulateCollateral: invalid collateral agreement");
    P.params[8] = c.hc;
    P.params[9] = std::isfinite(c.ho) ? c.ho : -1.0;
    P.params[10] = c.mta;
    P.params[11] = c.ia;
    const std::size_t off = 16 + 64;
    P.params[off] = c.type;
    P.params[off + 1] = static_cast<double>(c.assetIndex);
    P.params[off + 2] = c.type == 0 ? 0.0 : c.haircut;
    if (c.type == 2 && c.assetIndex >= m.assets.size()) throw std::invalid_argument("collateral asset index out of range");
    if (c.type == 1) {
      if (c.bondMaturity < grid.t.back() - 1e-10) throw std::invalid_argument("the collateral bond must mature after the horizon");
      for (std::size_t j = 0; j < nT; ++j) {
        P.steps[j * stride + 22] = bondA(grid.t[j], c.bondMaturity);
        P.steps[j * stride + 23] = bondB(grid.t[j], c.bondMaturity);
      }
    }
  }
  for (std::size_t k = 0; k < m.assets.size(); ++k) P.params[12 + k] = m.assets[k].spot;
  for (std::size_t i = 0; i < nCorr; ++i)
    for (std::size_t k = 0; k <= i; ++k) P.params[16 + i * 8 + k] = chol[i * nCorr + k];
  for (double t : P.times) P.marketSurvival.push_back(m.credits.empty() ? 1.0 : m.credits[o.counterparty].market.survival(t));

  const std::size_t numWG = (m.numPaths + 63) / 64;
  P.header = {static_cast<std::uint32_t>(m.numPaths), static_cast<std::uint32_t>(nT), static_cast<std::uint32_t>(m.assets.size()),
              static_cast<std::uint32_t>(m.credits.size()), static_cast<std::uint32_t>(m.credits.empty() ? 1 : m.credits.front().substeps),
              static_cast<std::uint32_t>(numNormals), static_cast<std::uint32_t>(m.seed % 4294967296ull), m.antithetic ? 1u : 0u,
              hasCsa ? 1u : 0u, static_cast<std::uint32_t>(o.counterparty), static_cast<std::uint32_t>(stride / 4),
              static_cast<std::uint32_t>(nCorr), static_cast<std::uint32_t>(offCall), static_cast<std::uint32_t>(offRep),
              floatBits(static_cast<float>(o.pfeQuantile)), static_cast<std::uint32_t>(numWG), static_cast<std::uint32_t>(P.statsPerDate),
              nR, static_cast<std::uint32_t>(perTradeGroups), L.valueChange, L.exposureValue, L.netted, L.collateral, L.gross,
              L.trades, L.exercise, static_cast<std::uint32_t>(P.requests.size() / 8), static_cast<std::uint32_t>(amc.size()),
              L.exposure, L.conditionalIm, static_cast<std::uint32_t>(o.imInnerPaths),
              floatBits(static_cast<float>(o.imQuantile))};
  auto toF = [](const std::vector<double>& v) {
    std::vector<float> f(v.size());
    for (std::size_t k = 0; k < v.size(); ++k) f[k] = static_cast<float>(v[k]);
    return f;
  };
  P.paramsF = toF(P.params);
  P.stepsF = toF(P.steps);
  P.termsF = toF(P.terms);
  P.requestsF = toF(P.requests);
  return P;
}

}  // namespace zk::host

// ---------------------------------------------------------------- C ABI
struct zk_plan {
  zk::host::CompiledPlan p;
};

extern "C" {

zk_status zk_compile(const double* model, size_t model_len, const double* netting_set, size_t ns_len, const double* options,
                     size_t options_len, zk_plan** out, char* err, size_t err_len) {
  if (!out || !model || !netting_set || !options) return ZK_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  try {
    const auto m = zk::host::decodeModel(model, model_len);
    const auto n = zk::host::decodeNettingSet(netting_set, ns_len);
    const auto o = zk::host::decodeOptions(options, options_len);
    auto* p = new zk_plan{zk::host::compile(m, n, o)};
    *out = p;
    return ZK_OK;
  } catch (const std::exception& e) {
    if (err && err_len) {
      std::strncpy(err, e.what(), err_len - 1);
      err[err_len - 1] = 0;
    }
    return ZK_ERR_INVALID_PLAN;
  }
}

zk_status zk_plan_view_of(const zk_plan* p, zk_plan_view* v) {
  if (!p || !v) return ZK_ERR_INVALID_ARGUMENT;
  const auto& c = p->p;
  *v = {c.header.data(), c.header.size(), c.indices.data(), c.indices.size(), c.paramsF.data(), c.paramsF.size(),
        c.stepsF.data(), c.stepsF.size(), c.termsF.data(), c.termsF.size(), c.requestsF.data(), c.requestsF.size(),
        c.rowsTotal, c.numOutputs};
  return ZK_OK;
}

zk_status zk_plan_view_f64_of(const zk_plan* p, zk_plan_view_f64* v) {
  if (!p || !v) return ZK_ERR_INVALID_ARGUMENT;
  const auto& c = p->p;
  *v = {c.header.data(), c.header.size(), c.indices.data(), c.indices.size(), c.params.data(), c.params.size(),
        c.steps.data(), c.steps.size(), c.terms.data(), c.terms.size(), c.requests.data(), c.requests.size(),
        c.rowsTotal, c.numOutputs};
  return ZK_OK;
}

zk_status zk_plan_dates(const zk_plan* p, double* times, size_t nT, uint64_t* reporting, size_t nR) {
  if (!p) return ZK_ERR_INVALID_ARGUMENT;
  const auto& c = p->p;
  if (nT != c.times.size() || nR != c.reporting.size()) return ZK_ERR_INVALID_ARGUMENT;
  if (times) std::copy(c.times.begin(), c.times.end(), times);
  if (reporting) std::copy(c.reporting.begin(), c.reporting.end(), reporting);
  return ZK_OK;
}

zk_status zk_plan_sizes(const zk_plan* p, uint64_t* s) {
  if (!p || !s) return ZK_ERR_INVALID_ARGUMENT;
  const auto& c = p->p;
  s[0] = c.times.size();
  s[1] = c.reporting.size();
  s[2] = c.statsPerDate;
  s[3] = c.numTrades;
  s[4] = c.numBermudans;
  s[5] = c.exerciseRows;
  return ZK_OK;
}

void zk_plan_destroy(zk_plan* p) { delete p; }

}  // extern "C"
