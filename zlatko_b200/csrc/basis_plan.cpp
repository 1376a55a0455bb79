// The linear revaluation of a group of netting sets as a matrix product: the host lowering (buildBasis) and its
// host check (basisCheck).  The term records are the reference's (include/ccr/gpu/fused_exposure.hpp:96-127; the
// kinds it merges in mergeTerms, src/gpu/fused_exposure.cpp:45-100), read the way the term-by-term kernel reads
// them after lowerTerms: bonds c A 2^(b x), floating coupons (c A fix + p1 A) 2^(b x) with the fixing read before
// the date's own fixings are set, asset forwards c S A, foreign forwards c S A_f 2^(b_f x_f), and Black options.
#include "basis_plan.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>

#include "zk_device.cuh"

namespace zk {
namespace {

constexpr double kLog2e = 1.4426950408889634;

uint32_t bitsOf(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  return u;
}

double fromHalf(uint16_t h) {
  const double s = (h & 0x8000u) ? -1.0 : 1.0;
  const int E = (h >> 10) & 31, M = h & 1023;
  if (E == 0) return s * std::ldexp(static_cast<double>(M), -24);
  return s * std::ldexp(static_cast<double>(1024 + M), E - 25);
}

float bOf(float B) { return static_cast<float>(-static_cast<double>(B) * kLog2e); }

// Black price in double (the check compares two sums of the same prices, not the formula).
double blackD(double F, double K, double sd, double df, bool call) {
  const double s = call ? 1.0 : -1.0;
  if (sd <= 1e-7 || F <= 0.0) return df * std::max(s * (F - K), 0.0);
  const double d1 = std::log(F / K) / sd + 0.5 * sd, d2 = d1 - sd;
  auto N = [](double z) { return 0.5 * std::erfc(-z / std::sqrt(2.0)); };
  return df * s * (F * N(s * d1) - K * N(s * d2));
}

// The unscaled Black price of an option record on one path state.
double optionPrice(const float* r, double x, const double* S, const double* xf) {
  const uint32_t code = static_cast<uint32_t>(r[0]), kind = code & 15u;
  const double b0 = static_cast<double>(r[3]) * std::exp(-static_cast<double>(r[4]) * x);
  const double p3 = r[7];
  if (kind == kOption) {
    const uint32_t a = static_cast<uint32_t>(r[1]) & 3u;
    return blackD(S[a] * static_cast<double>(r[5]) / b0, r[6], std::fabs(p3), b0, p3 > 0.0);
  }
  const uint32_t a = std::min<uint32_t>(code >> 12u, 1u);
  const double q = static_cast<double>(r[5]) * std::exp(-static_cast<double>(r[1]) * xf[a]);
  return blackD(S[a] * q / b0, r[6], std::fabs(p3), b0, p3 > 0.0);
}

// The same price from a basis option record (appendOption).
double basisOptionPrice(const float* o, bool foreign, double x, const double* S, const double* xf) {
  const uint32_t flags = static_cast<uint32_t>(o[9]), a = flags & 3u;
  const double b0 = static_cast<double>(o[0]) * std::exp(-static_cast<double>(o[1]) * x);
  const double q = foreign ? static_cast<double>(o[2]) * std::exp(-static_cast<double>(o[3]) * xf[std::min(a, 1u)]) : o[2];
  return blackD(S[a] * q / b0, o[4], o[8], b0, (flags & 4u) != 0);
}

struct FixKey {
  uint32_t j, A, b, invc;
  bool operator<(const FixKey& o) const { return std::tie(j, A, b, invc) < std::tie(o.j, o.A, o.b, o.invc); }
};
struct Fix {
  uint32_t j;
  float A, b, invc;
  uint32_t lastUse = 0;
  bool used = false;
  int slot = -1;
};

uint32_t kindOf(const float* r) { return static_cast<uint32_t>(r[0]) & 15u; }

// Binary16 of a float with round-to-nearest-even, by the exponent rebias (|f| below the FP16 maximum).
uint16_t f2h(float f) {
  uint32_t x = bitsOf(f);
  const uint32_t sign = (x >> 16) & 0x8000u;
  x &= 0x7FFFFFFFu;
  if (x >= 0x477FF000u) return static_cast<uint16_t>(sign | 0x7BFFu);  // not reached: coefficients are below 2^15
  if (x < 0x38800000u) {                                                // below 2^-14: a subnormal half or zero
    float a;
    std::memcpy(&a, &x, 4);
    return static_cast<uint16_t>(sign | static_cast<uint32_t>(std::nearbyint(a * 16777216.0f)));
  }
  const uint32_t y = x - 0x38000000u;  // exponent bias 127 -> 15
  return static_cast<uint16_t>(sign | ((y + 0xFFFu + ((y >> 13) & 1u)) >> 13));
}

// A Black option term as the basis kernel prices it: A, B, P_f (rec[5]), B_f (foreign options), K, 1 / K,
// 1 / sd (0 where sd <= 1e-7: the intrinsic value), sd / 2, sd, flags (asset | 4 call), 0, 0 -- the divisions by K
// and sd of the reference's formula (fused_kernels.cpp:209-215) done once here.
void appendOption(const float* r, bool foreign, std::vector<float>& out) {
  const uint32_t code = static_cast<uint32_t>(r[0]);
  const uint32_t asset = foreign ? std::min<uint32_t>(code >> 12u, 1u) : static_cast<uint32_t>(r[1]) & 3u;
  const float K = r[6], sd = std::fabs(r[7]);
  const bool call = r[7] > 0.0f;
  const float v[kBasisOptWords] = {r[3], r[4], r[5], foreign ? r[1] : 0.0f, K, 1.0f / K, sd <= 1e-7f ? 0.0f : 1.0f / sd,
                                   0.5f * sd, sd, static_cast<float>(asset | (call ? 4u : 0u)), 0.0f, 0.0f};
  out.insert(out.end(), v, v + kBasisOptWords);
}

// One date's part of the image (built independently of the other dates).
struct DateOut {
  std::vector<BasisKg> kgs;
  std::vector<float> options;
  std::vector<size_t> chunkAt;         // halves from the date's first chunk
  std::vector<uint32_t> chunkSteps;
  std::vector<uint16_t> blob;
  std::vector<float> scale = std::vector<float>(kBasisRows, 1.0f);
  uint64_t linearTerms = 0;
  std::string why;
};

// A linear term's contribution: the column it lands in (type, asset or fixing, b bits, option record bits), the
// netting set, the coefficient.
struct Ent {
  std::array<uint32_t, 11> key;
  uint32_t n;
  double v;
};

void buildDate(const std::vector<BasisPlanIn>& plans, const std::vector<Fix>& fixes,
               const std::vector<std::vector<int>>& couponKey, uint32_t j, DateOut& D) {
  std::vector<Ent> ents;
  auto push = [&](uint32_t type, uint32_t a, uint32_t b, const float* opt, size_t n, double v) {
    Ent e;
    e.key.fill(0u);
    e.key[0] = type, e.key[1] = a, e.key[2] = b;
    if (opt)
      for (int q = 0; q < 8; ++q) e.key[3 + q] = q == 2 ? 0u : bitsOf(opt[q]);  // c is the coefficient
    e.n = static_cast<uint32_t>(n), e.v = v;
    ents.push_back(e);
  };
  for (size_t n = 0; n < plans.size(); ++n) {
    const auto& P = plans[n];
    for (uint32_t t = P.indices[j]; t < P.indices[j + 1]; ++t) {
      const float* r = P.terms + static_cast<size_t>(t) * kTermStride;
      const uint32_t code = static_cast<uint32_t>(r[0]), kind = code & 15u;
      const double c = r[2], A = r[3];
      switch (kind) {
        case kBond:
          push(kColBond, 0, bitsOf(bOf(r[4])), nullptr, n, c * A), ++D.linearTerms;
          break;
        case kFixedFloat: {
          const uint32_t b = bitsOf(bOf(r[4]));
          push(kColBond, 0, b, nullptr, n, static_cast<double>(r[5]) * A);
          const int k = couponKey[n][t];
          if (k >= 0) push(kColCoupon, static_cast<uint32_t>(fixes[k].slot), b, nullptr, n, c * A);
          ++D.linearTerms;
          break;
        }
        case kAsset:
          push(kColSpot, static_cast<uint32_t>(r[1]) & 3u, 0, nullptr, n, c * A), ++D.linearTerms;
          break;
        case kForeignForward:
          push(kColForeign, std::min<uint32_t>(code >> 12u, 1u), bitsOf(bOf(r[1])), nullptr, n, c * A), ++D.linearTerms;
          break;
        case kOption:
        case kForeignOption:
          push(kind == kOption ? kColOption : kColForeignOption, 0, 0, r, n, c), ++D.linearTerms;
          break;
        default:
          break;  // fixings: the fixing keys
      }
    }
  }
  // columns: the distinct keys in order (type first: the types' runs follow each other); a column's
  // coefficients summed in plan term order
  std::stable_sort(ents.begin(), ents.end(), [](const Ent& a, const Ent& b) { return a.key < b.key; });
  std::vector<size_t> colStart;  // first entry of each column
  for (size_t i = 0; i < ents.size(); ++i)
    if (i == 0 || ents[i].key != ents[i - 1].key) colStart.push_back(i);
  colStart.push_back(ents.size());
  const size_t nCols = colStart.size() - 1;
  std::vector<double> coef(nCols * kBasisRows, 0.0);
  for (size_t c = 0; c < nCols; ++c)
    for (size_t i = colStart[c]; i < colStart[c + 1]; ++i) coef[c * kBasisRows + ents[i].n] += ents[i].v;
  // k-groups: each type's run padded to whole groups with repeats of its first column (finite values, zero
  // coefficients); an even number of groups in all (16-column MMA steps)
  std::vector<int> colOfSlot;  // column position -> key column, -1 for padding
  size_t c = 0;
  while (c < nCols) {
    const uint32_t type = ents[colStart[c]].key[0], asset = ents[colStart[c]].key[1];
    // a run: the columns of one type (foreign bonds and FX rates: of one asset, so a k-group reads one rate)
    const bool perAsset = type == kColForeign || type == kColSpot;
    size_t e = c;
    while (e < nCols && ents[colStart[e]].key[0] == type && (!perAsset || ents[colStart[e]].key[1] == asset)) ++e;
    const bool opt = type == kColOption || type == kColForeignOption;
    const size_t optFirst = D.options.size() / kBasisOptWords;
    if (opt) {
      for (size_t q = c; q < e; ++q) {
        const auto& k = ents[colStart[q]].key;
        float r[8];
        for (int w = 0; w < 8; ++w) std::memcpy(&r[w], &k[3 + w], 4);
        appendOption(r, type == kColForeignOption, D.options);
      }
      if (D.options.size() / kBasisOptWords > 0x10000u) {
        D.why = "more than 65,536 options on one date";
        return;
      }
    }
    for (size_t s0 = c; s0 < e; s0 += 8) {
      BasisKg g;
      std::memset(&g, 0, sizeof g);
      g.type = type;
      g.mult = type == kColCoupon ? kCouponScale : opt ? kOptionScale : 1.0f;
      for (int q = 0; q < 8; ++q) {
        const bool real = s0 + q < e;
        const size_t col = real ? s0 + q : c;
        const auto& k = ents[colStart[col]].key;
        float b;
        std::memcpy(&b, &k[2], 4);
        g.b[q] = b;
        g.sel[q] = static_cast<uint16_t>(opt ? optFirst + (col - c) : k[1]);
        colOfSlot.push_back(real ? static_cast<int>(col) : -1);
      }
      D.kgs.push_back(g);
    }
    c = e;
  }
  if (D.kgs.size() % 2) {
    BasisKg g;
    std::memset(&g, 0, sizeof g);
    g.type = kColBond, g.mult = 1.0f;
    D.kgs.push_back(g);
    for (int q = 0; q < 8; ++q) colOfSlot.push_back(-1);
  }
  const size_t numKg = D.kgs.size();
  // per netting set of the date: the largest |C / mult| lands in [2^14, 2^15)
  std::vector<double> inv(kBasisRows, 1.0);
  for (size_t n = 0; n < plans.size(); ++n) {
    double mx = 0.0;
    for (size_t q = 0; q < colOfSlot.size(); ++q)
      if (colOfSlot[q] >= 0) mx = std::max(mx, std::fabs(coef[static_cast<size_t>(colOfSlot[q]) * kBasisRows + n]) / D.kgs[q / 8].mult);
    if (mx > 0.0) {
      if (!std::isfinite(mx)) {
        D.why = "a non-finite coefficient";
        return;
      }
      const int s = std::ilogb(mx) - 14;
      if (s < -126 || s > 127) {
        D.why = "a coefficient outside the single-precision scale range";
        return;
      }
      D.scale[n] = std::ldexp(1.0f, s);
      inv[n] = std::ldexp(1.0, -s);
    }
  }
  // chunks of up to 8 k-groups: the hi image then the lo image, K-major over the 128 rows
  for (size_t c0 = 0; c0 < numKg; c0 += kBasisChunkKg) {
    const size_t kgs = std::min<size_t>(kBasisChunkKg, numKg - c0);
    const size_t at = D.blob.size();
    D.chunkAt.push_back(at);
    D.chunkSteps.push_back(static_cast<uint32_t>(kgs / 2));
    D.blob.resize(at + kgs * 1024 * 2, 0);
    uint16_t* hi = D.blob.data() + at;
    uint16_t* lo = hi + kgs * 1024;
    for (size_t g = 0; g < kgs; ++g)
      for (int e = 0; e < 8; ++e) {
        const size_t q = (c0 + g) * 8 + e;
        const int kc = colOfSlot[q];
        if (kc < 0) continue;
        const double m = 1.0 / D.kgs[c0 + g].mult;
        for (size_t n = 0; n < plans.size(); ++n) {
          const double v = coef[static_cast<size_t>(kc) * kBasisRows + n] * m * inv[n];
          const uint16_t h = f2h(static_cast<float>(v));
          const uint16_t l = f2h(static_cast<float>(v - fromHalf(h)));
          const size_t off = g * 1024 + (n & 7) * 8 + (n >> 3) * 64 + e;
          hi[off] = h, lo[off] = l;
        }
      }
  }
}

}  // namespace

bool buildBasis(const std::vector<BasisPlanIn>& plans, BasisImage& out, std::string& why, const ParallelFor& parallel) {
  out = BasisImage();
  const size_t nNs = plans.size();
  if (nNs == 0 || nNs > static_cast<size_t>(kBasisRows)) return why = "group size outside 1..128", false;
  const uint32_t nT = plans[0].nT;
  for (const auto& p : plans) {
    if (p.nT != nT) return why = "netting sets on different date grids", false;
    for (uint32_t j = 0; j < nT; ++j)
      if (p.indices[p.offCall + j] != plans[0].indices[plans[0].offCall + j] ||
          p.indices[p.offRep + j] != plans[0].indices[plans[0].offRep + j])
        return why = "netting sets with different margin-call or reporting dates", false;
    for (uint32_t t = 0; t < p.nTerms; ++t) {
      const float* r = p.terms + static_cast<size_t>(t) * kTermStride;
      const uint32_t code = static_cast<uint32_t>(r[0]), kind = code & 15u;
      const bool linear = kind == kBond || kind == kFixedFloat || kind == kAsset || kind == kSetFixing || kind == kOption;
      if (!(linear && (code >> 4u) == 0u) && kind != kForeignForward && kind != kForeignOption)
        return why = "a term kind the basis does not lower", false;
    }
  }
  // ---- fixings: one key per distinct (date, A, b, 1/c) set; a floating coupon reads the key its swap slot held
  // before the date's own fixings ----
  std::map<FixKey, uint32_t> fixIds;
  std::vector<Fix> fixes;
  std::vector<std::vector<int>> slotKey(nNs, std::vector<int>(kMaxSwapSlots, -1));
  // couponKey[n][t]: the fixing key a coupon term reads (-1: none set yet, the fixing is zero)
  std::vector<std::vector<int>> couponKey(nNs);
  for (size_t n = 0; n < nNs; ++n) {
    const auto& P = plans[n];
    couponKey[n].assign(P.nTerms, -1);
    for (uint32_t j = 0; j < nT; ++j) {
      for (uint32_t t = P.indices[j]; t < P.indices[j + 1]; ++t) {
        const float* r = P.terms + static_cast<size_t>(t) * kTermStride;
        if (kindOf(r) != kFixedFloat) continue;
        const uint32_t slot = static_cast<uint32_t>(r[1]);
        if (slot >= static_cast<uint32_t>(kMaxSwapSlots)) return why = "swap slot beyond 32", false;
        const int k = slotKey[n][slot];
        couponKey[n][t] = k;
        if (k >= 0) fixes[k].used = true, fixes[k].lastUse = std::max(fixes[k].lastUse, j);
      }
      for (uint32_t t = P.indices[j]; t < P.indices[j + 1]; ++t) {
        const float* r = P.terms + static_cast<size_t>(t) * kTermStride;
        if (kindOf(r) != kSetFixing) continue;
        const uint32_t slot = static_cast<uint32_t>(r[1]);
        if (slot >= static_cast<uint32_t>(kMaxSwapSlots)) return why = "swap slot beyond 32", false;
        const float b = bOf(r[4]), invc = static_cast<float>(1.0 / static_cast<double>(r[2]));
        const FixKey key{j, bitsOf(r[3]), bitsOf(b), bitsOf(invc)};
        auto it = fixIds.find(key);
        if (it == fixIds.end()) {
          it = fixIds.emplace(key, static_cast<uint32_t>(fixes.size())).first;
          Fix f;
          f.j = j, f.A = r[3], f.b = b, f.invc = invc, f.lastUse = j;
          fixes.push_back(f);
        }
        slotKey[n][slot] = static_cast<int>(it->second);
      }
    }
  }
  // Slots: a key written while its date's coupons are read (after them in the kernel) may take the slot of a key
  // whose last reader is that date or earlier.
  {
    std::vector<uint32_t> order;
    for (uint32_t k = 0; k < fixes.size(); ++k)
      if (fixes[k].used) order.push_back(k);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return fixes[a].j < fixes[b].j; });
    std::vector<uint32_t> freeFrom;  // per slot: the last reader's date of its key
    for (uint32_t k : order) {
      int s = -1;
      for (size_t q = 0; q < freeFrom.size(); ++q)
        if (freeFrom[q] <= fixes[k].j) {
          s = static_cast<int>(q);
          break;
        }
      if (s < 0) {
        s = static_cast<int>(freeFrom.size());
        freeFrom.push_back(0);
      }
      freeFrom[s] = fixes[k].lastUse;
      fixes[k].slot = s;
    }
    if (freeFrom.size() > static_cast<size_t>(kBasisMaxFix)) return why = "more than 64 fixings live at once", false;
    out.numFixSlots = static_cast<uint32_t>(freeFrom.size());
  }
  out.numNs = static_cast<uint32_t>(nNs), out.nT = nT;
  // ---- per date (independent of each other): columns, k-groups, option records, chunks and scales ----
  std::vector<DateOut> per(nT);
  auto one = [&](size_t j) { buildDate(plans, fixes, couponKey, static_cast<uint32_t>(j), per[j]); };
  if (parallel) {
    parallel(nT, one);
  } else {
    for (size_t j = 0; j < nT; ++j) one(j);
  }
  // ---- merged in date order ----
  out.dates.assign(static_cast<size_t>(nT) * kBasisDateWords, 0u);
  out.scale.assign(static_cast<size_t>(nT) * kBasisRows, 1.0f);
  std::vector<std::vector<uint32_t>> fixesAt(nT);
  for (uint32_t k = 0; k < fixes.size(); ++k)
    if (fixes[k].used) fixesAt[fixes[k].j].push_back(k);
  size_t blobTotal = 0;
  for (const auto& D : per) blobTotal += D.blob.size();
  if (blobTotal * 2 >= (1ull << 32)) return why = "basis tables above 4 GB", false;
  out.blob.reserve(blobTotal);
  for (uint32_t j = 0; j < nT; ++j) {
    const DateOut& D = per[j];
    if (!D.why.empty()) return why = D.why, false;
    uint32_t* d = &out.dates[static_cast<size_t>(j) * kBasisDateWords];
    d[bdCall] = plans[0].indices[plans[0].offCall + j];
    d[bdRep] = plans[0].indices[plans[0].offRep + j];
    d[bdFixBegin] = static_cast<uint32_t>(out.fixings.size() / 4);
    for (uint32_t k : fixesAt[j]) {
      const Fix& f = fixes[k];
      out.fixings.push_back(f.A), out.fixings.push_back(f.b), out.fixings.push_back(f.invc);
      out.fixings.push_back(static_cast<float>(f.slot));
    }
    d[bdFixEnd] = static_cast<uint32_t>(out.fixings.size() / 4);
    d[bdKg] = static_cast<uint32_t>(out.kgs.size());
    d[bdKgs] = static_cast<uint32_t>(D.kgs.size());
    out.kgs.insert(out.kgs.end(), D.kgs.begin(), D.kgs.end());
    d[bdOpt] = static_cast<uint32_t>(out.options.size() / kBasisOptWords);
    d[bdOpts] = static_cast<uint32_t>(D.options.size() / kBasisOptWords);
    out.descBytes = std::max<uint32_t>(out.descBytes, static_cast<uint32_t>((D.kgs.size() * sizeof(BasisKg) + D.options.size() * 4 + 1023) / 1024 * 1024));
    out.options.insert(out.options.end(), D.options.begin(), D.options.end());
    d[bdChunk] = out.numChunks;
    d[bdChunks] = static_cast<uint32_t>(D.chunkSteps.size());
    for (size_t c = 0; c < D.chunkSteps.size(); ++c) {
      out.chunks.push_back(static_cast<uint32_t>((out.blob.size() + D.chunkAt[c]) * 2));
      out.chunks.push_back(D.chunkSteps[c]);
    }
    out.numChunks += static_cast<uint32_t>(D.chunkSteps.size());
    out.blob.insert(out.blob.end(), D.blob.begin(), D.blob.end());
    std::copy(D.scale.begin(), D.scale.end(), out.scale.begin() + static_cast<size_t>(j) * kBasisRows);
    out.linearTerms += D.linearTerms, out.columns += 8ull * D.kgs.size();
  }
  if (basisSmemBytes(out.descBytes, out.numFixSlots) > kBasisMaxSmem)
    return why = "a date's basis columns, option records and fixings beyond the kernel's shared memory", false;
  uint32_t next = nT;
  for (uint32_t j = nT; j-- > 0;) {
    uint32_t* d = &out.dates[static_cast<size_t>(j) * kBasisDateWords];
    d[bdNextRep] = next;
    if (d[bdRep] > 0) next = j;
    d[bdPrevChunks] = j > 0 ? out.dates[static_cast<size_t>(j - 1) * kBasisDateWords + bdChunks] : 0u;
  }
  return true;
}

double basisCheck(const std::vector<BasisPlanIn>& plans, const BasisImage& img, const double* x, const double* S,
                  const double* xf) {
  const uint32_t nT = img.nT;
  const size_t nNs = plans.size();
  std::vector<double> fixImg(std::max<uint32_t>(img.numFixSlots, 1), 0.0);
  std::vector<std::vector<double>> fixPlan(nNs, std::vector<double>(kMaxSwapSlots, 0.0));
  std::vector<double> worst(nNs, 0.0), gross(nNs, 1e-300);
  for (uint32_t j = 0; j < nT; ++j) {
    const uint32_t* d = &img.dates[static_cast<size_t>(j) * kBasisDateWords];
    const double xj = x[j];
    const double* Sj = S + 4 * static_cast<size_t>(j);
    const double* xfj = xf + 2 * static_cast<size_t>(j);
    // the image: every column's function, times hi + lo, times the date's scale
    std::vector<double> vImg(nNs, 0.0), gImg(nNs, 0.0);
    uint32_t chunk = d[bdChunk];
    for (uint32_t g = 0; g < d[bdKgs]; ++g) {
      const BasisKg& K = img.kgs[d[bdKg] + g];
      const uint32_t c = chunk + g / kBasisChunkKg, gl = g % kBasisChunkKg;
      const uint32_t steps = img.chunks[2 * c + 1];
      const uint16_t* hi = img.blob.data() + img.chunks[2 * c] / 2;
      const uint16_t* lo = hi + static_cast<size_t>(steps) * 2 * 1024;
      for (int e = 0; e < 8; ++e) {
        double phi;
        switch (K.type) {
          case kColBond: phi = std::exp2(static_cast<double>(K.b[e]) * xj); break;
          case kColCoupon: phi = K.mult * fixImg[K.sel[e]] * std::exp2(static_cast<double>(K.b[e]) * xj); break;
          case kColForeign: phi = Sj[K.sel[e]] * std::exp2(static_cast<double>(K.b[e]) * xfj[K.sel[e]]); break;
          case kColSpot: phi = Sj[K.sel[e]]; break;
          default:
            phi = K.mult * basisOptionPrice(&img.options[(static_cast<size_t>(d[bdOpt]) + K.sel[e]) * kBasisOptWords],
                                            K.type == kColForeignOption, xj, Sj, xfj);
        }
        for (size_t n = 0; n < nNs; ++n) {
          const size_t off = static_cast<size_t>(gl) * 1024 + (n & 7) * 8 + (n >> 3) * 64 + e;
          const double w = (fromHalf(hi[off]) + fromHalf(lo[off])) * img.scale[static_cast<size_t>(j) * kBasisRows + n];
          vImg[n] += w * phi;
          gImg[n] += std::fabs(w * phi);
        }
      }
    }
    for (uint32_t f = d[bdFixBegin]; f < d[bdFixEnd]; ++f) {
      const float* r = &img.fixings[4 * static_cast<size_t>(f)];
      fixImg[static_cast<size_t>(r[3])] = (r[0] * std::exp2(static_cast<double>(r[1]) * xj) - 1.0) * r[2];
    }
    // term by term
    for (size_t n = 0; n < nNs; ++n) {
      const auto& P = plans[n];
      double v = 0.0;
      for (uint32_t t = P.indices[j]; t < P.indices[j + 1]; ++t) {
        const float* r = P.terms + static_cast<size_t>(t) * kTermStride;
        const uint32_t code = static_cast<uint32_t>(r[0]), kind = code & 15u;
        const double c = r[2], A = r[3];
        switch (kind) {
          case kBond: v += c * A * std::exp2(static_cast<double>(bOf(r[4])) * xj); break;
          case kFixedFloat:
            v += (c * A * fixPlan[n][static_cast<uint32_t>(r[1])] + static_cast<double>(r[5]) * A) *
                 std::exp2(static_cast<double>(bOf(r[4])) * xj);
            break;
          case kAsset: v += c * A * Sj[static_cast<uint32_t>(r[1]) & 3u]; break;
          case kForeignForward: {
            const uint32_t a = std::min<uint32_t>(code >> 12u, 1u);
            v += c * A * Sj[a] * std::exp2(static_cast<double>(bOf(r[1])) * xfj[a]);
            break;
          }
          case kOption:
          case kForeignOption: v += c * optionPrice(r, xj, Sj, xfj); break;
          default: break;
        }
      }
      for (uint32_t t = P.indices[j]; t < P.indices[j + 1]; ++t) {
        const float* r = P.terms + static_cast<size_t>(t) * kTermStride;
        if (kindOf(r) != kSetFixing) continue;
        const double invc = static_cast<float>(1.0 / static_cast<double>(r[2]));
        fixPlan[n][static_cast<uint32_t>(r[1])] = (r[3] * std::exp2(static_cast<double>(bOf(r[4])) * xj) - 1.0) * invc;
      }
      worst[n] = std::max(worst[n], std::fabs(vImg[n] - v));
      gross[n] = std::max(gross[n], gImg[n]);
    }
  }
  double r = 0.0;
  for (size_t n = 0; n < nNs; ++n) r = std::max(r, worst[n] / gross[n]);
  return r;
}

}  // namespace zk
