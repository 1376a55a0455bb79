/* ORACLE / TEST INFRASTRUCTURE ONLY.  Plain-C restatement of the reference's fused exposure pipeline in
 * single precision (the CPU mirror of its GPU kernels, src/gpu/fused_reference.cpp), on a plan in the
 * reference's binary layout (include/ccr/gpu/fused_exposure.hpp:131-226).  The statement order of every
 * float expression follows the reference so that, compiled without FMA contraction against the same libm,
 * the statistics come out bit for bit; the row statistics' quantile is the exact interpolated empirical
 * quantile of ccr::quantile (include/ccr/core/math.hpp:39-47) instead of the reference kernel's histogram
 * approximation of it.  Only the tests and the smoke check call this file. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

enum { INNER_TOP = 16, WG = 64, STATS = 8, TRADE_STATS = 5, MAX_ASSETS = 4, MAX_CREDITS = 2, MAX_SLOTS = 32, MAX_NORMALS = 64,
       MAX_TRADES = 16, MAX_BERM = 4, CHOL = 8, STEP = 24, TERM = 8, REQ = 8 };
#define NO_ROW 0xFFFFFFFFu
#define NOT_EXERCISED 0xFFFFFFFFu

/* PCG hash (fused_reference.cpp:19-23). */
static uint32_t pcg_hash(uint32_t v) {
  const uint32_t state = v * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}

/* Box-Muller pair k of date j on a path stream (fused_reference.cpp:26-34). */
static void normal_pair(uint32_t stream, uint32_t j, uint32_t k, float* out) {
  const uint32_t h1 = pcg_hash(stream ^ pcg_hash(j * 131u + k));
  const uint32_t h2 = pcg_hash(h1 ^ 0x68E31DA4u);
  const float u1 = ((float)(h1 >> 8u) + 0.5f) / 16777216.0f;
  const float u2 = ((float)(h2 >> 8u) + 0.5f) / 16777216.0f;
  const float radius = sqrtf(-2.0f * logf(u1)), angle = 6.2831853f * u2;
  out[0] = radius * cosf(angle);
  out[1] = radius * sinf(angle);
}

static float maxf(float a, float b) { return a < b ? b : a; }
static float minf(float a, float b) { return b < a ? b : a; }

/* Abramowitz-Stegun 7.1.26 normal CDF (fused_reference.cpp:36-42). */
static float norm_cdf(float x) {
  const float z = fabsf(x) * 0.70710678f;
  const float t = 1.0f / (1.0f + 0.3275911f * z);
  const float poly = ((((1.061405429f * t - 1.453152027f) * t + 1.421413741f) * t - 0.284496736f) * t + 0.254829592f) * t;
  const float e = 1.0f - poly * expf(-z * z);
  return x >= 0.0f ? 0.5f * (1.0f + e) : 0.5f * (1.0f - e);
}

/* df * Black (fused_reference.cpp:44-50). */
static float black76(float F, float K, float sd, float df, int call) {
  const float s = call ? 1.0f : -1.0f;
  if (sd <= 1e-7f || F <= 0.0f) return df * maxf(s * (F - K), 0.0f);
  const float d1 = logf(F / K) / sd + 0.5f * sd;
  const float d2 = d1 - sd;
  return df * s * (F * norm_cdf(s * d1) - K * norm_cdf(s * d2));
}

/* Per-trade statistic (fused_reference.cpp:79-88). */
static float trade_stat(uint32_t m, float vi, float v, float D) {
  const float pos = v > 0.0f ? 1.0f : 0.0f;
  switch (m) {
    case 0: return D * vi * pos;
    case 1: return vi * pos;
    case 2: return D * (maxf(v, 0.0f) - maxf(v - vi, 0.0f));
    case 3: return D * maxf(vi, 0.0f);
    default: return maxf(vi, 0.0f);
  }
}

/* AMC regression polynomial (fused_reference.cpp:104-107). */
static float amc_poly(const float* rec, float x) {
  const float z = (x - rec[2]) * rec[3];
  return ((rec[7] * z + rec[6]) * z + rec[5]) * z + rec[4];
}

/* The regression of a policy / continuation record: the polynomial above in x or, when extension records (kind 15)
 * follow it, the two-regressor basis of this library (an extension with no reference code behind it) in x and the
 * co-terminal swap rate s = flt / ann summed from the annuity (13) and float-leg (14) records before it: cx, 1 / sx,
 * cs, 1 / ss, c0, c1 in the record, c2..c8 in the first extension's fields 1..7, c9 in the second's field 1. */
static float amc_value(const float* rec, int twoD, float x, float ann, float flt) {
  if (!twoD) return amc_poly(rec, x);
  const float* e1 = rec + TERM;
  const float* e2 = rec + 2 * TERM;
  const float s = ann != 0.0f ? flt / ann : 0.0f;
  const float z = (x - rec[2]) * rec[3], w = (s - rec[4]) * rec[5];
  const float zz = z * z, zw = z * w, ww = w * w;
  return rec[6] + rec[7] * z + e1[1] * w + e1[2] * zz + e1[3] * zw + e1[4] * ww + e1[5] * zz * z + e1[6] * zz * w +
         e1[7] * zw * w + e2[1] * ww * w;
}

typedef struct PlanS {
  const uint32_t *H, *I;
  const float *FP, *ST, *T;
  uint32_t nP, nT, nA, nC, sub, nNormals, seed, anti, hasCsa, cpty, nCorr, offCall, offRep, nS, nR, nTr;
  uint32_t rowDV, rowE, rowV, rowC, rowGross, rowTrades, rowEx, nBerm, rowEP;
  uint32_t rowIm, nInner;
  float imLevel;
} Plan;

/* Nested Monte Carlo for the conditional initial margin (fused_reference.cpp:108-196): one inner path's state
 * and its exact step from date j - 1 to j on its own stream (the outer step with the inner normals). */
typedef struct {
  float x, lnD, lnS[MAX_ASSETS], S[MAX_ASSETS], y[MAX_CREDITS], Y[MAX_CREDITS];
} InnerPath;

struct PlanS;
static void inner_step(const struct PlanS* v, InnerPath* st, uint32_t j, uint32_t stream, float sign);
static float inner_value(const struct PlanS* v, const InnerPath* st, float* fix, uint32_t* ex, uint32_t j);

/* The AMC regression pass records x and the deflator on every date and each exercise value instead of
 * deciding exercise (fused_reference.cpp:89-97, 275-281). */
typedef struct {
  float *x, *deflator, *exercise;
  size_t nP;
  const uint32_t* offsets; /* first exercise row of each Bermudan */
} Sink;

/* One path through every date (fused_reference.cpp:198-422): statistics into stats[nT][nS], rows into
 * expo[row * stride], netted value and collateral price into vals[2 nT]. */
static void simulate_path(const Plan* v, uint32_t p, float* stats, float* expo, size_t stride, float* vals,
                          const Sink* sink) {
  const float* FP = v->FP;
  float sign = 1.0f;
  uint32_t pathStream = p;
  if (v->anti) {
    pathStream = p >> 1u;
    if ((p & 1u) == 1u) sign = -1.0f;
  }
  const uint32_t stream = pcg_hash(pcg_hash(v->seed) ^ pcg_hash(pathStream + 0x9E3779B9u));
  float x = 0.0f, lnD = 0.0f, D = 1.0f;
  float S[MAX_ASSETS], lnS[MAX_ASSETS] = {0, 0, 0, 0}, y[MAX_CREDITS], Y[MAX_CREDITS], fix[MAX_SLOTS], z[MAX_NORMALS], w[CHOL];
  memset(fix, 0, sizeof fix);
  memset(z, 0, sizeof z);
  for (int a = 0; a < MAX_ASSETS; ++a) S[a] = FP[12 + a];
  for (int c = 0; c < MAX_CREDITS; ++c) y[c] = FP[4 * c + 3], Y[c] = 0.0f;
  float held = 0.0f, prevDE = 0.0f, prevQ = 1.0f, prevRV = 0.0f;
  uint32_t exercised[MAX_BERM] = {NOT_EXERCISED, NOT_EXERCISED, NOT_EXERCISED, NOT_EXERCISED};
  const float ia = FP[11], mta = FP[10];
  for (uint32_t j = 0; j < v->nT; ++j) {
    float Q = 1.0f;
    if (j > 0) {
      const float* step = v->ST + (size_t)j * STEP;
      const uint32_t nZ = 4 * ((v->nNormals + 3) / 4);
      for (uint32_t k = 0; k < nZ; k += 2) normal_pair(stream, j, k / 2, &z[k]);
      for (uint32_t k = 0; k < nZ; ++k) z[k] *= sign;
      for (int i = 0; i < CHOL; ++i) {
        const float* row = &FP[16 + i * CHOL];
        const float d0 = row[0] * z[0] + row[1] * z[1] + row[2] * z[2] + row[3] * z[3];
        const float d1 = row[4] * z[4] + row[5] * z[5] + row[6] * z[6] + row[7] * z[7];
        w[i] = d0 + d1;
      }
      /* Hull-White exact step (hull_white.cpp:40-68) with the plan's coefficients. */
      const float integrated = x * step[5] + step[2] * w[0] + step[3] * z[v->nCorr] + step[4];
      x = x * step[0] + step[1] * w[0];
      lnD = lnD - integrated;
      D = expf(lnD);
      for (int a = 0; a < MAX_ASSETS; ++a) {
        lnS[a] = lnS[a] + (integrated - step[8 + a] - step[16 + a] + step[12 + a] * w[1 + a]);
        S[a] = FP[12 + a] * expf(lnS[a]);
      }
      /* CIR++ on Brownian-bridge sub-steps, full truncation (cir_intensity.cpp:49-66). */
      const float dt = step[6];
      uint32_t off = v->nCorr + 1;
      for (uint32_t c = 0; c < v->nC; ++c) {
        const float kappa = FP[4 * c], theta = FP[4 * c + 1], xi = FP[4 * c + 2];
        const float h = dt / (float)v->sub;
        float rem = sqrtf(dt) * w[1 + v->nA + c], remT = dt, yy = y[c], YY = Y[c];
        for (uint32_t s = 0; s < v->sub; ++s) {
          float dW = rem;
          if (s + 1 < v->sub) dW = h / remT * rem + sqrtf(maxf(h * (remT - h) / remT, 0.0f)) * z[off + s];
          rem -= dW;
          remT -= h;
          const float yp = maxf(yy, 0.0f);
          const float yn = yy + kappa * (theta - yp) * h + xi * sqrtf(yp) * dW;
          YY += 0.5f * (yp + maxf(yn, 0.0f)) * h;
          yy = yn;
        }
        y[c] = yy;
        Y[c] = YY;
        off += v->sub - 1;
      }
      if (v->nC > 0) Q = expf(-Y[v->cpty] - step[20 + v->cpty]);
    }

    float value = 0.0f, vt[MAX_TRADES], ev[MAX_BERM] = {0, 0, 0, 0}, ann = 0.0f, flt = 0.0f;
    memset(vt, 0, sizeof vt);
    const uint32_t nTr = v->nTr < MAX_TRADES ? v->nTr : MAX_TRADES;
    if (sink) sink->x[(size_t)j * sink->nP + p] = x, sink->deflator[(size_t)j * sink->nP + p] = D;
    for (uint32_t t = v->I[j]; t < v->I[j + 1]; ++t) {
      const float* rec = v->T + (size_t)t * TERM;
      const uint32_t code = (uint32_t)rec[0];
      const uint32_t kind = code & 15u, extra = code >> 12u;
      uint32_t bm = (code >> 8u) & 15u;
      if (bm > MAX_BERM - 1) bm = MAX_BERM - 1;
      const uint32_t slot = (uint32_t)rec[1];
      const float c = rec[2];
      const float bond = rec[3] * expf(-rec[4] * x);  /* only the kinds that read it use it */
      float term = 0.0f;
      switch (kind) {
        case 0: term = c * bond; break;
        case 1: term = (c * fix[slot] + rec[5]) * bond; break;
        case 2: term = c * S[slot] * rec[3]; break;
        case 3: fix[slot] = (bond - 1.0f) / c; break;
        case 4: {
          const float p3 = rec[7];
          term = c * black76(S[slot] * rec[5] / bond, rec[6], fabsf(p3), bond, p3 > 0.0f);
          break;
        }
        case 5: ev[bm] += c * bond; break;
        case 6: {
          const int twoD = t + 1 < v->I[j + 1] && ((uint32_t)rec[TERM] & 15u) == 15u;
          if (sink)
            sink->exercise[((size_t)sink->offsets[bm] + extra) * sink->nP + p] = ev[bm];
          else if (exercised[bm] == NOT_EXERCISED && ev[bm] > 0.0f && ev[bm] > amc_value(rec, twoD, x, ann, flt))
            exercised[bm] = extra;
          ann = flt = 0.0f;
          break;
        }
        case 7: {
          const int twoD = t + 1 < v->I[j + 1] && ((uint32_t)rec[TERM] & 15u) == 15u;
          if (exercised[bm] == NOT_EXERCISED) term = rec[1] * maxf(amc_value(rec, twoD, x, ann, flt), 0.0f);
          ann = flt = 0.0f;
          break;
        }
        case 13: ann += c * bond; break;
        case 14: flt += c * bond; break;
        case 15: break;
        case 8:
          if (exercised[bm] != NOT_EXERCISED && exercised[bm] <= extra) term = c * bond;
          break;
        case 10: { /* probe of a risk factor into row p1 */
          const uint32_t what = slot & 15u, ix = (slot >> 4u) < 3u ? (slot >> 4u) : 3u, ic = ix < 1u ? ix : 1u;
          float q;
          switch (what) {
            case 0: q = x; break;
            case 1: q = D; break;
            case 2: q = S[ix]; break;
            case 3: q = lnS[ix]; break;
            case 4: q = y[ic]; break;
            case 5: q = j == 0 ? 1.0f : expf(-Y[ic] - v->ST[(size_t)j * STEP + 20 + ic]); break;
            case 6: q = D * S[ix]; break;
            default: q = D * bond;
          }
          expo[(size_t)rec[5] * stride] = q + c;
          break;
        }
        default: /* kBermFloat */
          if (exercised[bm] != NOT_EXERCISED && exercised[bm] <= extra) term = (c * fix[slot] + rec[5]) * bond;
      }
      if (v->nTr > 0) {
        const uint32_t g = (code >> 4u) & 15u;
        vt[g < MAX_TRADES - 1 ? g : MAX_TRADES - 1] += term;
      } else {
        value += term;
      }
    }
    for (uint32_t i = 0; i < nTr; ++i) value += vt[i];

    /* CSA: collateral called on the value at t - MPR (collateral.cpp:10-47). */
    float collateral = 0.0f;
    vals[j] = value;
    if (v->hasCsa) {
      const float* ca = &FP[16 + CHOL * CHOL];
      const uint32_t ctype = (uint32_t)ca[0];
      float price = 1.0f;
      if (ctype == 1) price = v->ST[(size_t)j * STEP + 22] * expf(-v->ST[(size_t)j * STEP + 23] * x);
      else if (ctype == 2) price = S[(uint32_t)ca[1] < 3u ? (uint32_t)ca[1] : 3u];
      vals[v->nT + j] = price;
      const uint32_t callJ = v->I[v->offCall + j];
      const float vc = callJ != j ? vals[callJ] : value, pc = callJ != j ? vals[v->nT + callJ] : price;
      const float keep = ctype != 0 ? 1.0f - ca[2] : 1.0f;
      const float hc = FP[8], hb = FP[9];
      float required = 0.0f;
      if (vc > hc) required += vc - hc;
      if (hb >= 0.0f && -vc > hb) required -= -vc - hb;
      if (j == 0 || fabsf(required - held * keep * pc) >= mta) held = required / (keep * pc);
      collateral = held * price + ia;
    }
    const float e = value - collateral, ep = maxf(e, 0.0f), en = minf(e, 0.0f);
    const uint32_t rs = v->I[v->offRep + j];
    if (rs > 0) {
      const size_t k = rs - 1;
#define PUT(base, offset, val) \
  if ((base) != NO_ROW) expo[((size_t)(base) + (offset)) * stride] = (val)
      PUT(v->rowEP, k, ep);
      PUT(v->rowDV, k, rs == 1 ? 0.0f : fabsf(value - prevRV));
      PUT(v->rowE, k, e);
      PUT(v->rowV, k, value);
      PUT(v->rowC, k, collateral);
      if (v->rowGross != NO_ROW) {
        float gross = 0.0f;
        for (uint32_t i = 0; i < nTr; ++i) gross += maxf(vt[i], 0.0f);
        PUT(v->rowGross, k, gross);
      }
      if (v->rowTrades != NO_ROW)
        for (uint32_t i = 0; i < nTr; ++i) PUT(v->rowTrades, (size_t)i * v->nR + k, vt[i]);
#undef PUT
    }
    /* Nested Monte Carlo: the conditional initial margin of this path on this reporting date, the imLevel
     * quantile of |V_inner(t + MPR) - V(t)| over nInner inner paths from the grid's kInnerTop largest samples
     * (fused_reference.cpp:356-393). */
    if (rs > 0 && v->nInner > 0) {
      const uint32_t target = v->I[v->offRep + v->nT + j];
      float im = 0.0f;
      if (target != NO_ROW) {
        float top[INNER_TOP];
        memset(top, 0, sizeof top);
        InnerPath start;
        memset(&start, 0, sizeof start);
        start.x = x, start.lnD = lnD;
        for (int a = 0; a < MAX_ASSETS; ++a) start.lnS[a] = lnS[a], start.S[a] = S[a];
        for (int c = 0; c < MAX_CREDITS; ++c) start.y[c] = y[c], start.Y[c] = Y[c];
        for (uint32_t i = 0; i < v->nInner; ++i) {
          InnerPath st = start;
          float f2[MAX_SLOTS];
          uint32_t e2[MAX_BERM];
          memcpy(f2, fix, sizeof f2);
          memcpy(e2, exercised, sizeof e2);
          const uint32_t istream = pcg_hash(stream ^ pcg_hash(0x85EBCA6Bu + (i >> 1u) * 0x9E3779B9u + j));
          const float isign = (i & 1u) == 1u ? -1.0f : 1.0f;
          float vi = value;
          for (uint32_t jj = j + 1; jj <= target; ++jj) {
            inner_step(v, &st, jj, istream, isign);
            vi = inner_value(v, &st, f2, e2, jj);
          }
          float cur = fabsf(vi - value);
          for (uint32_t k = 0; k < INNER_TOP; ++k)
            if (cur > top[k]) {
              const float t = top[k];
              top[k] = cur, cur = t;
            }
        }
        const float rank = v->imLevel * (float)(v->nInner - 1);
        const uint32_t k = (uint32_t)floorf(rank);
        const uint32_t hiIdx = v->nInner - 1 - k < INNER_TOP - 1 ? v->nInner - 1 - k : INNER_TOP - 1;
        const float ok = top[hiIdx], ok1 = hiIdx > 0 ? top[hiIdx - 1] : ok;
        im = ok + (rank - (float)k) * (ok1 - ok);
      }
      if (v->rowIm != NO_ROW) expo[((size_t)v->rowIm + rs - 1) * stride] = im;
    }
    if (v->rowEx != NO_ROW)
      for (uint32_t i = 0; i < v->nBerm && i < MAX_BERM; ++i)
        expo[((size_t)v->rowEx + i) * stride] = exercised[i] == NOT_EXERCISED ? -1.0f : (float)exercised[i];
    float cvaInc = 0.0f;
    if (rs > 0) {
      prevRV = value;
      const float de = D * ep;
      if (j > 0) cvaInc = 0.5f * (prevDE + de) * (prevQ - Q);
      prevDE = de;
      prevQ = Q;
    }
    float* st = &stats[(size_t)j * v->nS];
    st[0] = e, st[1] = ep, st[2] = en, st[3] = D * ep, st[4] = D * en, st[5] = cvaInc, st[6] = Q, st[7] = D;
    for (uint32_t k = STATS; k < v->nS; ++k) {
      const uint32_t i = (k - STATS) / TRADE_STATS;
      st[k] = i < nTr ? trade_stat((k - STATS) % TRADE_STATS, vt[i], value, D) : 0.0f;
    }
  }
}

static void inner_step(const Plan* v, InnerPath* st, uint32_t j, uint32_t stream, float sign) {
  const float* FP = v->FP;
  const float* step = v->ST + (size_t)j * STEP;
  float z[MAX_NORMALS], w[CHOL];
  memset(z, 0, sizeof z);
  const uint32_t nZ = 4 * ((v->nNormals + 3) / 4);
  for (uint32_t k = 0; k < nZ; k += 2) normal_pair(stream, j, k / 2, &z[k]);
  for (uint32_t k = 0; k < nZ; ++k) z[k] *= sign;
  for (int i = 0; i < CHOL; ++i) {
    const float* row = &FP[16 + i * CHOL];
    const float d0 = row[0] * z[0] + row[1] * z[1] + row[2] * z[2] + row[3] * z[3];
    const float d1 = row[4] * z[4] + row[5] * z[5] + row[6] * z[6] + row[7] * z[7];
    w[i] = d0 + d1;
  }
  const float integrated = st->x * step[5] + step[2] * w[0] + step[3] * z[v->nCorr] + step[4];
  st->x = st->x * step[0] + step[1] * w[0];
  st->lnD = st->lnD - integrated;
  for (int a = 0; a < MAX_ASSETS; ++a) {
    st->lnS[a] = st->lnS[a] + (integrated - step[8 + a] - step[16 + a] + step[12 + a] * w[1 + a]);
    st->S[a] = FP[12 + a] * expf(st->lnS[a]);
  }
  const float dt = step[6];
  uint32_t off = v->nCorr + 1;
  for (uint32_t c = 0; c < v->nC; ++c) {
    const float kappa = FP[4 * c], theta = FP[4 * c + 1], xi = FP[4 * c + 2];
    const float h = dt / (float)v->sub;
    float rem = sqrtf(dt) * w[1 + v->nA + c], remT = dt, yy = st->y[c], YY = st->Y[c];
    for (uint32_t s = 0; s < v->sub; ++s) {
      float dW = rem;
      if (s + 1 < v->sub) dW = h / remT * rem + sqrtf(maxf(h * (remT - h) / remT, 0.0f)) * z[off + s];
      rem -= dW;
      remT -= h;
      const float yp = maxf(yy, 0.0f);
      const float yn = yy + kappa * (theta - yp) * h + xi * sqrtf(yp) * dW;
      YY += 0.5f * (yp + maxf(yn, 0.0f)) * h;
      yy = yn;
    }
    st->y[c] = yy;
    st->Y[c] = YY;
    off += v->sub - 1;
  }
}

/* The netting set's value on an inner path (no trade groups, no probes). */
static float inner_value(const Plan* v, const InnerPath* st, float* fix, uint32_t* ex, uint32_t j) {
  float value = 0.0f, ev[MAX_BERM] = {0, 0, 0, 0};
  const float x = st->x;
  for (uint32_t t = v->I[j]; t < v->I[j + 1]; ++t) {
    const float* rec = v->T + (size_t)t * TERM;
    const uint32_t code = (uint32_t)rec[0];
    const uint32_t kind = code & 15u, extra = code >> 12u;
    uint32_t bm = (code >> 8u) & 15u;
    if (bm > MAX_BERM - 1) bm = MAX_BERM - 1;
    const uint32_t slot = (uint32_t)rec[1];
    const float c = rec[2];
    const float bond = rec[3] * expf(-rec[4] * x);
    switch (kind) {
      case 0: value += c * bond; break;
      case 1: value += (fix[slot] * c + rec[5]) * bond; break;
      case 2: value += c * st->S[slot] * rec[3]; break;
      case 3: fix[slot] = (bond - 1.0f) / c; break;
      case 4: {
        const float p3 = rec[7];
        value += c * black76(st->S[slot] * rec[5] / bond, rec[6], fabsf(p3), bond, p3 > 0.0f);
        break;
      }
      case 5: ev[bm] += c * bond; break;
      case 6:
        if (ex[bm] == NOT_EXERCISED && ev[bm] > 0.0f && ev[bm] > amc_poly(rec, x)) ex[bm] = extra;
        break;
      case 7:
        if (ex[bm] == NOT_EXERCISED) value += rec[1] * maxf(amc_poly(rec, x), 0.0f);
        break;
      case 8:
        if (ex[bm] != NOT_EXERCISED && ex[bm] <= extra) value += c * bond;
        break;
      case 9:
        if (ex[bm] != NOT_EXERCISED && ex[bm] <= extra) value += (fix[slot] * c + rec[5]) * bond;
        break;
      default: break;
    }
  }
  return value;
}

static int cmp_double(const void* a, const void* b) {
  const double x = *(const double*)a, y = *(const double*)b;
  return x < y ? -1 : x > y ? 1 : 0;
}

/* ccr::quantile (math.hpp:39-47): sort, then interpolate between order statistics floor(h), floor(h) + 1. */
double orc_quantile(const double* values, size_t n, double p) {
  if (n == 0) return NAN;
  double* s = (double*)malloc(n * sizeof(double));
  memcpy(s, values, n * sizeof(double));
  qsort(s, n, sizeof(double), cmp_double);
  const double h = p * (double)(n - 1);
  const size_t lo = (size_t)floor(h), hi = lo + 1 < n ? lo + 1 : n - 1;
  const double r = s[lo] + (h - (double)lo) * (s[hi] - s[lo]);
  free(s);
  return r;
}

/* The header fields the path reads (fused_reference.cpp:64-75, fused_kernels.cpp:32-41). */
static int read_plan(Plan* v, const uint32_t* header, const uint32_t* indices, const float* params, const float* steps,
                     const float* terms, char* err, size_t errLen) {
  memset(v, 0, sizeof *v);
  v->H = header, v->I = indices, v->FP = params, v->ST = steps, v->T = terms;
  v->nP = header[0], v->nT = header[1], v->nA = header[2], v->nC = header[3], v->sub = header[4];
  v->nNormals = header[5], v->seed = header[6], v->anti = header[7] == 1u, v->hasCsa = header[8] == 1u;
  v->cpty = header[9], v->nCorr = header[11], v->offCall = header[12], v->offRep = header[13], v->nS = header[16];
  v->nR = header[17], v->nTr = header[18], v->rowDV = header[19], v->rowE = header[20], v->rowV = header[21];
  v->rowC = header[22], v->rowGross = header[23], v->rowTrades = header[24], v->rowEx = header[25];
  v->nBerm = header[27], v->rowEP = header[28], v->rowIm = header[29], v->nInner = header[30];
  memcpy(&v->imLevel, &header[31], sizeof(float));
  if (v->nP == 0 || v->nT == 0) {
    if (err && errLen) snprintf(err, errLen, "empty plan");
    return 1;
  }
  if (v->nBerm > MAX_BERM) { /* the reference's kernel prices at most 4 Bermudans per netting set */
    if (err && errLen) snprintf(err, errLen, "the restated kernels run the reference's plans (at most 4 Bermudans)");
    return 1;
  }
  if (header[10] != STEP / 4) { /* the reference's plans only: no stochastic foreign rates */
    if (err && errLen) snprintf(err, errLen, "the restated kernels run the reference's plans (24-value step rows)");
    return 1;
  }
  return 0;
}

int orc_run_fused(const uint32_t* header, const uint32_t* indices, size_t nIdx, const float* params, const float* steps,
                  const float* terms, size_t nTerms, const float* requests, size_t nReq, uint32_t rowsTotal,
                  uint32_t numOutputs, float* sums, float* values, float* rowsOut, char* err, size_t errLen) {
  (void)nIdx;
  (void)nTerms;
  Plan v;
  if (read_plan(&v, header, indices, params, steps, terms, err, errLen)) return 1;
  const size_t nT = v.nT, nS = v.nS, nP = v.nP, numWG = (nP + WG - 1) / WG, n = nT * nS;
  float* rows = (float*)calloc((size_t)(rowsTotal ? rowsTotal : 1) * nP, sizeof(float));
  float* partials = (float*)calloc(numWG * n, sizeof(float));
  float* stats = (float*)malloc((size_t)WG * n * sizeof(float));
  float* red = (float*)malloc((size_t)WG * nS * sizeof(float));
  float* vals = (float*)malloc(2 * nT * sizeof(float));
  /* Workgroups of 64 paths; inactive paths contribute zeros; tree reduction per date
   * (fused_reference.cpp:444-464). */
  for (size_t g = 0; g < numWG; ++g) {
    memset(stats, 0, (size_t)WG * n * sizeof(float));
    for (uint32_t l = 0; l < WG; ++l) {
      const size_t p = g * WG + l;
      if (p >= nP) break;
      simulate_path(&v, (uint32_t)p, &stats[l * n], rows + p, nP, vals, NULL);
    }
    for (size_t j = 0; j < nT; ++j) {
      for (uint32_t l = 0; l < WG; ++l)
        for (size_t f = 0; f < nS; ++f) red[l * nS + f] = stats[(l * nT + j) * nS + f];
      for (uint32_t s = WG / 2; s > 0; s >>= 1)
        for (uint32_t l = 0; l < s; ++l)
          for (size_t f = 0; f < nS; ++f) red[l * nS + f] += red[(l + s) * nS + f];
      for (size_t f = 0; f < nS; ++f) partials[(g * nT + j) * nS + f] = red[f];
    }
  }
  /* Compensated sum over workgroups in order, divided by the paths (fused_reference.cpp:481-496). */
  for (size_t i = 0; i < n; ++i) {
    float sum = 0.0f, comp = 0.0f;
    for (size_t g = 0; g < numWG; ++g) {
      const float yv = partials[g * n + i] - comp;
      const float tv = sum + yv;
      comp = (tv - sum) - yv;
      sum = tv;
    }
    sums[i] = sum / (float)nP;
  }
  /* Row statistics (fused_reference.cpp:499-605), with the exact quantile. */
  const size_t nOut = numOutputs ? numOutputs : 1;
  memset(values, 0, nOut * sizeof(float));
  double* buf = (double*)malloc(nP * sizeof(double));
  for (size_t q = 0; q < nReq; ++q) {
    const float* rq = requests + q * REQ;
    const uint32_t op = (uint32_t)rq[0], row = (uint32_t)rq[1], row2 = (uint32_t)rq[2], count = (uint32_t)rq[3];
    float* o = values + (size_t)rq[7];
    const float* X = rows + (size_t)row * nP;
    const float* Yr = rows + (size_t)row2 * nP;
    if (op == 4) {
      for (uint32_t k = 0; k < count && k < nP; ++k) o[k] = X[k];
      continue;
    }
    if (op != 0 && op != 5 && op != 7) {
      float sum = 0.0f, comp = 0.0f;
      for (size_t p = 0; p < nP; ++p) {
        const float x = X[p];
        float f = x;
        if (op == 2) f = maxf(x, 0.0f);
        else if (op == 3) f = minf(x, 0.0f);
        else if (op == 6) f = x * Yr[p];
        else if (op == 8) f = maxf(x, 0.0f) * Yr[p];
        else if (op == 9) f = minf(x, 0.0f) * Yr[p];
        const float yv = f - comp, tv = sum + yv;
        comp = (tv - sum) - yv;
        sum = tv;
      }
      o[0] = sum / (float)nP;
      continue;
    }
    if (op == 5) { /* histogram of `count` bins */
      float lo = 3.402823466e38f, hi = -lo;
      for (size_t p = 0; p < nP; ++p) lo = minf(lo, X[p]), hi = maxf(hi, X[p]);
      if (rq[5] != rq[6]) lo = rq[5], hi = rq[6];
      const float span = maxf(hi - lo, 1e-30f);
      uint32_t* hist = (uint32_t*)calloc(count, sizeof(uint32_t));
      for (size_t p = 0; p < nP; ++p) {
        const float f = maxf((X[p] - lo) / span, 0.0f) * (float)count;
        uint32_t b = f >= 4294967040.0f ? 0xFFFFFFFFu : (uint32_t)f;
        if (b > count - 1) b = count - 1;
        ++hist[b];
      }
      for (uint32_t b = 0; b < count; ++b) o[b] = (float)hist[b];
      o[count] = lo, o[count + 1] = hi;
      free(hist);
      continue;
    }
    for (size_t p = 0; p < nP; ++p) buf[p] = op == 7 ? (double)maxf(X[p], 0.0f) : (double)X[p];
    o[0] = (float)orc_quantile(buf, nP, (double)rq[4]);
  }
  if (rowsOut) memcpy(rowsOut, rows, (size_t)rowsTotal * nP * sizeof(float));
  free(buf);
  free(rows);
  free(partials);
  free(stats);
  free(red);
  free(vals);
  return 0;
}

int orc_amc_states(const uint32_t* header, const uint32_t* indices, const float* params, const float* steps,
                   const float* terms, uint32_t rowsTotal, const uint32_t* offsets, float* x, float* deflator,
                   float* exercise, char* err, size_t errLen) {
  Plan v;
  if (read_plan(&v, header, indices, params, steps, terms, err, errLen)) return 1;
  const Sink sink = {x, deflator, exercise, v.nP, offsets};
  const size_t nT = v.nT, nS = v.nS;
  float* stats = (float*)malloc(nT * nS * sizeof(float));
  float* expo = (float*)calloc((size_t)rowsTotal + 1, sizeof(float));
  float* vals = (float*)malloc(2 * nT * sizeof(float));
  for (uint32_t p = 0; p < v.nP; ++p) simulate_path(&v, p, stats, expo, 1, vals, &sink);
  free(stats), free(expo), free(vals);
  return 0;
}
