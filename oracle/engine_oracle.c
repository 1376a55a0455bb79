/* ORACLE / TEST INFRASTRUCTURE ONLY.  Plain-C restatement, in double precision, of the reference's
 * exposure engine (src/exposure/exposure_engine.cpp:50-81) run on injected standard normals:
 *   scenario generation   scenario_generator.cpp:94-141 (driver loop), hull_white.cpp:40-68,
 *                         lognormal_asset.cpp:16-21, cir_intensity.cpp:25-66, matrix.cpp:49-68
 *   grids                 time_grid.cpp:13-66, exposure_engine.cpp:35-48
 *   valuation             interest_rate_swap.cpp:51-83, asset_forward.cpp:13-25, european_option.cpp:21-35,
 *                         math.hpp:15-30 (Black), bermudan_swaption.cpp:49-146 (Longstaff-Schwartz on the
 *                         short-rate state, with the regression of amc_oracle.c)
 *   netting, collateral   exposure_engine.cpp:9-14, collateral.cpp:10-47
 *   statistics and CVA    exposure_profile.cpp:10-83, math.hpp:39-47, cva.cpp:11-77, credit_curve.cpp:23-35
 * The netting-set / model arrays are the flat encodings the package's spec module writes. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define TIME_TOL 1e-9

typedef struct {
  size_t n;
  double *t, *r;
} Curve;
typedef struct {
  size_t n;
  double *pillar, *hazard;
} Hazard;
typedef struct {
  double spot, vol;
  Curve carry;
} Asset;
typedef struct {
  double kappa, theta, xi, y0;
  size_t sub;
  Hazard market;
} Credit;
typedef struct {
  int kind; /* 0 swap, 1 forward, 2 option, 3 Bermudan swaption on the swap */
  double notional, fixed, strike, maturity;
  int payFixed, call;
  size_t asset, nSched;
  double* sched;
  /* Bermudan: sorted exercise times, settlement, position, regression degree */
  size_t nEx;
  double* ex;
  int physical, degree;
  double position;
} Trade;
typedef struct {
  int has, type;
  double hc, ho, mta, ia, mpr, haircut, bondMaturity;
  size_t asset;
} Csa;

typedef struct {
  const double* a;
  size_t n, i;
  int bad;
} Reader;

static double next(Reader* r) {
  if (r->i >= r->n) {
    r->bad = 1;
    return 0.0;
  }
  return r->a[r->i++];
}
static size_t count(Reader* r) {
  const double v = next(r);
  return v > 0 ? (size_t)v : 0;
}

static void read_curve(Reader* r, Curve* c) {
  c->n = count(r);
  c->t = (double*)calloc(c->n + 1, sizeof(double));
  c->r = (double*)calloc(c->n + 1, sizeof(double));
  for (size_t k = 0; k < c->n; ++k) c->t[k] = next(r), c->r[k] = next(r);
}

/* Zero rate linear in t, flat outside the pillars (yield_curve.cpp:20-27). */
static double zero_rate(const Curve* c, double t) {
  if (t <= c->t[0]) return c->r[0];
  if (t >= c->t[c->n - 1]) return c->r[c->n - 1];
  size_t i = 1;
  while (i < c->n && c->t[i] <= t) ++i; /* first pillar above t */
  const double w = (t - c->t[i - 1]) / (c->t[i] - c->t[i - 1]);
  return c->r[i - 1] + w * (c->r[i] - c->r[i - 1]);
}
static double discount(const Curve* c, double t) { return exp(-zero_rate(c, t) * t); }

/* Piecewise-flat hazard survival (credit_curve.cpp:23-35). */
static double hazard_survival(const Hazard* h, double t) {
  if (t <= 0.0) return 1.0;
  double integral = 0.0, prev = 0.0;
  for (size_t i = 0; i < h->n; ++i) {
    const int last = i + 1 == h->n;
    const double end = last ? t : (t < h->pillar[i] ? t : h->pillar[i]);
    integral += h->hazard[i] * (end - prev);
    if (end >= t) break;
    prev = end;
  }
  return exp(-integral);
}

/* ---- Hull-White one factor (hull_white.cpp:19-68) */
typedef struct {
  Curve curve;
  double a, sigma;
} HW;

static double hw_B(const HW* m, double t, double T) { return (1.0 - exp(-m->a * (T - t))) / m->a; }
static double hw_V(const HW* m, double t, double T) {
  const double tau = T - t, e1 = exp(-m->a * tau);
  return m->sigma * m->sigma / (m->a * m->a) * (tau + 2.0 / m->a * e1 - 0.5 / m->a * e1 * e1 - 1.5 / m->a);
}
static double hw_bond(const HW* m, double t, double T, double x) {
  if (T <= t) return 1.0;
  const double ratio = discount(&m->curve, T) / discount(&m->curve, t);
  return ratio * exp(0.5 * (hw_V(m, t, T) - hw_V(m, 0.0, T) + hw_V(m, 0.0, t)) - hw_B(m, t, T) * x);
}
/* Exact joint step of x and of its integral over [t0, t1]; returns the integrated short rate. */
static double hw_evolve(const HW* m, double t0, double t1, double z1, double z2, double* x) {
  const double a = m->a, dt = t1 - t0, e = exp(-a * dt), s2 = m->sigma * m->sigma;
  const double varX = s2 * (1.0 - e * e) / (2.0 * a);
  const double varI = s2 / (a * a) * (dt - 2.0 * (1.0 - e) / a + (1.0 - e * e) / (2.0 * a));
  const double cov = s2 / (2.0 * a * a) * (1.0 - e) * (1.0 - e);
  const double sdX = sqrt(varX), x0 = *x;
  *x = x0 * e + sdX * z1;
  double c1 = 0.0, c2 = sqrt(varI > 0.0 ? varI : 0.0);
  if (sdX > 0.0) {
    c1 = cov / sdX;
    const double r = varI - c1 * c1;
    c2 = sqrt(r > 0.0 ? r : 0.0);
  }
  const double intX = x0 * (1.0 - e) / a + c1 * z1 + c2 * z2;
  const double g2 = dt - 2.0 / a * (exp(-a * t0) - exp(-a * t1)) + 0.5 / a * (exp(-2.0 * a * t0) - exp(-2.0 * a * t1));
  const double intPhi = log(discount(&m->curve, t0) / discount(&m->curve, t1)) + s2 / (2.0 * a * a) * g2;
  return intX + intPhi;
}

/* The foreign rate's step under the domestic measure: hw_evolve with the quanto drift -q of x_f,
 * q = rho(x_f, S_f) sigma_f sigma_S, added to the state and to its integral (an extension: the reference's
 * foreign curves are deterministic). */
static double hw_evolve_drift(const HW* m, double t0, double t1, double z1, double z2, double q, double* x) {
  const double a = m->a, dt = t1 - t0, e = exp(-a * dt);
  const double integrated = hw_evolve(m, t0, t1, z1, z2, x);
  *x -= q * (1.0 - e) / a;
  return integrated - q / a * (dt - (1.0 - e) / a);
}

/* ---- CIR++ intensity (cir_intensity.cpp:25-66) */
static double cir_survival(const Credit* c, double t) {
  if (t <= 0.0) return 1.0;
  if (c->xi == 0.0) return exp(-(c->theta * t + (c->y0 - c->theta) * (1.0 - exp(-c->kappa * t)) / c->kappa));
  const double h = sqrt(c->kappa * c->kappa + 2.0 * c->xi * c->xi), eh = exp(h * t) - 1.0;
  const double denom = 2.0 * h + (c->kappa + h) * eh;
  const double logA = (2.0 * c->kappa * c->theta / (c->xi * c->xi)) * log(2.0 * h * exp(0.5 * (c->kappa + h) * t) / denom);
  return exp(logA - 2.0 * eh / denom * c->y0);
}
static double credit_survival(const Credit* c, double t, double iy) {
  return exp(-iy - log(cir_survival(c, t) / hazard_survival(&c->market, t)));
}
static void cir_evolve(const Credit* c, double dt, double z, const double* extra, double* y, double* iy) {
  const double h = dt / (double)c->sub;
  double rem = sqrt(dt) * z, remT = dt;
  for (size_t s = 0; s < c->sub; ++s) {
    double dW = rem;
    if (s + 1 < c->sub) dW = h / remT * rem + sqrt(h * (remT - h) / remT) * extra[s];
    rem -= dW;
    remT -= h;
    const double yp = *y > 0.0 ? *y : 0.0;
    const double yn = *y + c->kappa * (c->theta - yp) * h + c->xi * sqrt(yp) * dW;
    *iy += 0.5 * (yp + (yn > 0.0 ? yn : 0.0)) * h;
    *y = yn;
  }
}

/* ---- time grids (time_grid.cpp:13-66) */
typedef struct {
  size_t n;
  double* t;
} Grid;

static int cmp_d(const void* a, const void* b) {
  const double x = *(const double*)a, y = *(const double*)b;
  return x < y ? -1 : x > y ? 1 : 0;
}
/* Keeps finite t >= 0, adds 0, sorts, drops times within the tolerance of the previous kept one. */
static Grid make_grid(const double* in, size_t n) {
  double* t = (double*)malloc((n + 1) * sizeof(double));
  size_t m = 0;
  for (size_t i = 0; i < n; ++i)
    if (in[i] >= 0.0 && isfinite(in[i])) t[m++] = in[i];
  t[m++] = 0.0;
  qsort(t, m, sizeof(double), cmp_d);
  Grid g = {0, (double*)malloc(m * sizeof(double))};
  for (size_t i = 0; i < m; ++i)
    if (g.n == 0 || t[i] - g.t[g.n - 1] > TIME_TOL) g.t[g.n++] = t[i];
  free(t);
  return g;
}
static size_t at_or_before(const Grid* g, double t) {
  size_t k = 0; /* number of grid times <= t + tol */
  while (k < g->n && g->t[k] <= t + TIME_TOL) ++k;
  return k == 0 ? 0 : k - 1;
}
static long find_time(const Grid* g, double t) {
  const size_t i = at_or_before(g, t);
  if (fabs(g->t[i] - t) <= TIME_TOL) return (long)i;
  if (i + 1 < g->n && fabs(g->t[i + 1] - t) <= TIME_TOL) return (long)(i + 1);
  return -1;
}

/* ---- valuation */
static double norm_cdf(double x) { return 0.5 * erfc(-x / sqrt(2.0)); }
static double black(int call, double F, double K, double sd, double df) {
  const double s = call ? 1.0 : -1.0;
  if (sd <= 1e-14 || F <= 0.0 || K <= 0.0) {
    const double v = s * (F - K);
    return df * (v > 0.0 ? v : 0.0);
  }
  const double d1 = log(F / K) / sd + 0.5 * sd, d2 = d1 - sd;
  return df * s * (F * norm_cdf(s * d1) - K * norm_cdf(s * d2));
}

typedef struct {
  HW hw;
  size_t nA, nC, F, nP, nBase;
  Asset* assets;
  Credit* credits;
  double *corr, *base;
  int antithetic;
  /* Stochastic foreign rates (an extension of the reference's model, whose foreign curves are deterministic):
   * foreign[f] is the Hull-White model of asset f's currency on that asset's carry curve, XF[f] its state
   * [path][date] once simulated. */
  size_t nF;
  HW foreign[2];
  double* XF[2];
} Model;

typedef struct {
  size_t nTr;
  Trade* tr;
  Csa csa;
} Netting;

static int fail(char* err, size_t len, const char* msg) {
  if (err && len) snprintf(err, len, "%s", msg);
  return 1;
}

static void read_sched(Reader* r, Trade* t) {
  t->nSched = count(r);
  t->sched = (double*)calloc(t->nSched + 1, sizeof(double));
  for (size_t k = 0; k < t->nSched; ++k) t->sched[k] = next(r);
}

static int read_model(const double* a, size_t n, Model* m, char* err, size_t len) {
  Reader r = {a, n, 0, 0};
  memset(m, 0, sizeof *m);
  if (next(&r) != 7001.0) return fail(err, len, "model: bad magic");
  read_curve(&r, &m->hw.curve);
  m->hw.a = next(&r), m->hw.sigma = next(&r);
  m->nA = count(&r);
  m->assets = (Asset*)calloc(m->nA + 1, sizeof(Asset));
  for (size_t k = 0; k < m->nA; ++k) {
    m->assets[k].spot = next(&r), m->assets[k].vol = next(&r);
    read_curve(&r, &m->assets[k].carry);
  }
  m->nC = count(&r);
  m->credits = (Credit*)calloc(m->nC + 1, sizeof(Credit));
  for (size_t k = 0; k < m->nC; ++k) {
    Credit* c = &m->credits[k];
    c->kappa = next(&r), c->theta = next(&r), c->xi = next(&r), c->y0 = next(&r);
    c->sub = count(&r);
    c->market.n = count(&r);
    c->market.pillar = (double*)calloc(c->market.n + 1, sizeof(double));
    c->market.hazard = (double*)calloc(c->market.n + 1, sizeof(double));
    for (size_t q = 0; q < c->market.n; ++q) c->market.pillar[q] = next(&r), c->market.hazard[q] = next(&r);
  }
  const size_t f = count(&r);
  if (f > 8) return fail(err, len, "model: correlation matrix has wrong dimension");
  double* given = (double*)calloc(f * f + 1, sizeof(double));
  for (size_t i = 0; i < f * f; ++i) given[i] = next(&r);
  m->nP = count(&r);
  next(&r); /* seed: unused with injected normals */
  m->antithetic = next(&r) != 0.0;
  m->nBase = count(&r);
  m->base = (double*)calloc(m->nBase + 1, sizeof(double));
  for (size_t k = 0; k < m->nBase; ++k) m->base[k] = next(&r);
  if (r.i < r.n) { /* the foreign-rate block: 7011, nF, (a, sigma) per leading asset */
    if (next(&r) != 7011.0) return free(given), fail(err, len, "model: unknown trailing block");
    m->nF = count(&r);
    if (m->nF > 2 || m->nF > m->nA) return free(given), fail(err, len, "model: at most two foreign rates, one per leading asset");
    for (size_t q = 0; q < m->nF; ++q) {
      m->foreign[q].curve = m->assets[q].carry; /* shared with the asset: freed once, with the asset */
      m->foreign[q].a = next(&r), m->foreign[q].sigma = next(&r);
    }
  }
  m->F = 1 + m->nA + m->nC + m->nF;
  m->corr = (double*)calloc(m->F * m->F, sizeof(double));
  if (f == 0) {
    for (size_t i = 0; i < m->F; ++i) m->corr[i * m->F + i] = 1.0;
  } else if (f != m->F) {
    free(given);
    return fail(err, len, "model: correlation matrix has wrong dimension");
  } else {
    for (size_t i = 0; i < f * f; ++i) m->corr[i] = given[i];
  }
  free(given);
  if (r.bad) return fail(err, len, "spec: truncated array");
  if (m->hw.curve.n == 0 || m->hw.a <= 1e-8 || m->hw.sigma < 0.0) return fail(err, len, "model: invalid rate model");
  for (size_t k = 0; k < m->nC; ++k)
    if (m->credits[k].sub == 0 || m->credits[k].market.n == 0) return fail(err, len, "model: invalid credit");
  return 0;
}

static Trade swap_of(double notional, double fixed, int payFixed, const double* s, size_t n) {
  Trade t;
  memset(&t, 0, sizeof t);
  t.kind = 0, t.notional = notional, t.fixed = fixed, t.payFixed = payFixed, t.nSched = n;
  t.sched = (double*)malloc((n + 1) * sizeof(double));
  memcpy(t.sched, s, n * sizeof(double));
  return t;
}

static int read_netting(const double* a, size_t n, Netting* ns, char* err, size_t len) {
  Reader r = {a, n, 0, 0};
  memset(ns, 0, sizeof *ns);
  if (next(&r) != 7002.0) return fail(err, len, "netting set: bad magic");
  const size_t nt = count(&r);
  ns->tr = (Trade*)calloc(3 * nt + 1, sizeof(Trade));
  for (size_t k = 0; k < nt && !r.bad; ++k) {
    const int type = (int)next(&r);
    Trade* t = &ns->tr[ns->nTr];
    if (type == 0) {
      t->kind = 0, t->notional = next(&r), t->fixed = next(&r), t->payFixed = next(&r) != 0.0;
      read_sched(&r, t);
      ++ns->nTr;
    } else if (type == 1) {
      t->kind = 1, t->asset = count(&r), t->notional = next(&r), t->strike = next(&r), t->maturity = next(&r);
      ++ns->nTr;
    } else if (type == 2) {
      t->kind = 2, t->asset = count(&r), t->call = next(&r) != 0.0, t->notional = next(&r), t->strike = next(&r);
      t->maturity = next(&r);
      ++ns->nTr;
    } else if (type == 4) {
      /* Two schedules: float(K = 0, floating schedule) + swap(K, fixed schedule) - swap(0, fixed schedule). */
      Trade fixed, flt;
      memset(&fixed, 0, sizeof fixed), memset(&flt, 0, sizeof flt);
      const double notional = next(&r), K = next(&r);
      const int pay = next(&r) != 0.0;
      read_sched(&r, &fixed);
      read_sched(&r, &flt);
      ns->tr[ns->nTr++] = swap_of(notional, 0.0, pay, flt.sched, flt.nSched);
      ns->tr[ns->nTr++] = swap_of(notional, K, pay, fixed.sched, fixed.nSched);
      ns->tr[ns->nTr++] = swap_of(notional, 0.0, !pay, fixed.sched, fixed.nSched);
      free(fixed.sched), free(flt.sched);
    } else if (type == 3) {
      t->kind = 3, t->notional = next(&r), t->fixed = next(&r), t->payFixed = next(&r) != 0.0;
      read_sched(&r, t);
      t->nEx = count(&r);
      t->ex = (double*)calloc(t->nEx + 1, sizeof(double));
      for (size_t q = 0; q < t->nEx; ++q) t->ex[q] = next(&r);
      qsort(t->ex, t->nEx, sizeof(double), cmp_d);
      t->physical = next(&r) != 0.0, t->position = next(&r), t->degree = (int)count(&r);
      ++ns->nTr;
    } else {
      return fail(err, len, "netting set: unknown trade type");
    }
  }
  if (next(&r) != 0.0) {
    Csa* c = &ns->csa;
    c->has = 1, c->hc = next(&r);
    const double own = next(&r);
    c->ho = own < 0.0 ? INFINITY : own;
    c->mta = next(&r), c->ia = next(&r), c->mpr = next(&r), c->type = (int)next(&r), c->haircut = next(&r);
    c->bondMaturity = next(&r), c->asset = count(&r);
  }
  if (r.bad) return fail(err, len, "spec: truncated array");
  if (ns->nTr == 0) return fail(err, len, "ExposureEngine::run: empty netting set");
  for (size_t k = 0; k < ns->nTr; ++k) {
    const Trade* t = &ns->tr[k];
    if (t->kind == 3) {
      if (t->nEx == 0) return fail(err, len, "BermudanSwaption: no exercise dates");
      for (size_t q = 0; q < t->nEx; ++q) {
        int on = 0;
        for (size_t i = 0; i + 1 < t->nSched; ++i) on |= fabs(t->sched[i] - t->ex[q]) < 1e-8;
        if (!on) return fail(err, len, "BermudanSwaption: exercise dates must be start dates of the underlying periods");
      }
    }
    if (t->kind == 0 || t->kind == 3) {
      if (t->nSched < 2 || t->sched[0] < 0.0) return fail(err, len, "InterestRateSwap: invalid schedule");
      for (size_t i = 1; i < t->nSched; ++i)
        if (t->sched[i] <= t->sched[i - 1]) return fail(err, len, "InterestRateSwap: schedule must be strictly increasing");
    } else if (t->kind == 1 && t->maturity <= 0.0) {
      return fail(err, len, "AssetForward: maturity must be positive");
    } else if (t->kind == 2 && (t->maturity <= 0.0 || t->strike <= 0.0)) {
      return fail(err, len, "EuropeanOption: invalid expiry or strike");
    }
  }
  return 0;
}

/* Lower Cholesky factor (matrix.cpp:49-68). */
static int cholesky(const double* A, size_t n, double* L) {
  memset(L, 0, n * n * sizeof(double));
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j <= i; ++j) {
      if (fabs(A[i * n + j] - A[j * n + i]) > 1e-10) return 1;
      double s = A[i * n + j];
      for (size_t k = 0; k < j; ++k) s -= L[i * n + k] * L[j * n + k];
      if (i == j) {
        if (s <= 0.0) return 1;
        L[i * n + i] = sqrt(s);
      } else {
        L[i * n + j] = s / L[j * n + j];
      }
    }
  return 0;
}

/* Value of trade k on every path at grid index j (interest_rate_swap.cpp:51-83, asset_forward.cpp:13-25,
 * european_option.cpp:21-35).  X[p * nT + j] is the rate state, S the asset cube of the trade's asset. */
static void value_at(const Model* m, const Trade* tr, const Grid* g, size_t j, const double* X, double* const* S,
                     size_t nP, double* out) {
  const size_t nT = g->n;
  const double t = g->t[j];
  for (size_t p = 0; p < nP; ++p) out[p] = 0.0;
  if (tr->kind == 0) {
    const double sgn = tr->payFixed ? 1.0 : -1.0;
    if (t >= tr->sched[tr->nSched - 1] - 1e-10) return;
    for (size_t i = 1; i < tr->nSched; ++i) {
      const double ts = tr->sched[i - 1], te = tr->sched[i];
      if (te <= t + 1e-10) continue;
      const double tau = te - ts;
      if (ts >= t - 1e-10) {
        for (size_t p = 0; p < nP; ++p) {
          const double x = X[p * nT + j], pe = hw_bond(&m->hw, t, te, x);
          const double flt = hw_bond(&m->hw, t, ts, x) - pe;
          out[p] += sgn * tr->notional * (flt - tr->fixed * tau * pe);
        }
      } else {
        const size_t k = at_or_before(g, ts);
        const double tk = g->t[k];
        for (size_t p = 0; p < nP; ++p) {
          const double xk = X[p * nT + k];
          const double fixing = (hw_bond(&m->hw, tk, ts, xk) / hw_bond(&m->hw, tk, te, xk) - 1.0) / tau;
          const double pe = hw_bond(&m->hw, t, te, X[p * nT + j]);
          out[p] += sgn * tr->notional * (fixing - tr->fixed) * tau * pe;
        }
      }
    }
    return;
  }
  if (t >= tr->maturity - 1e-10) return;
  const Asset* as = &m->assets[tr->asset];
  const double carry = discount(&as->carry, tr->maturity) / discount(&as->carry, t);
  /* The foreign discount bond: the deterministic carry, or with a stochastic foreign rate P_f(t, T | x_f). */
  const int stochastic = tr->asset < m->nF;
#define FOREIGN_BOND(p) (stochastic ? hw_bond(&m->foreign[tr->asset], t, tr->maturity, m->XF[tr->asset][(p) * nT + j]) : carry)
  if (tr->kind == 1) {
    for (size_t p = 0; p < nP; ++p)
      out[p] = tr->notional * (S[tr->asset][p * nT + j] * FOREIGN_BOND(p) - tr->strike * hw_bond(&m->hw, t, tr->maturity, X[p * nT + j]));
    return;
  }
  const double sd = as->vol * sqrt(tr->maturity - t);
  for (size_t p = 0; p < nP; ++p) {
    const double df = hw_bond(&m->hw, t, tr->maturity, X[p * nT + j]);
    const double fwd = S[tr->asset][p * nT + j] * FOREIGN_BOND(p) / df;
    out[p] = tr->notional * black(tr->call, fwd, tr->strike, sd, df);
  }
#undef FOREIGN_BOND
}

/* The co-terminal swap rate of a tail swap at time t on short-rate state x: (P(t, T_0) - P(t, T_n)) / sum_i tau_i
 * P(t, T_i) over its schedule T_0 < .. < T_n -- the second regressor of the two-regressor basis (an extension of the
 * reference, whose regression is on x alone). */
static double coterminal_rate(const Model* m, const Trade* tail, double t, double x) {
  double ann = 0.0;
  for (size_t i = 1; i < tail->nSched; ++i)
    ann += (tail->sched[i] - tail->sched[i - 1]) * hw_bond(&m->hw, t, tail->sched[i], x);
  const double flt = hw_bond(&m->hw, t, tail->sched[0], x) - hw_bond(&m->hw, t, tail->sched[tail->nSched - 1], x);
  return ann > 0.0 ? flt / ann : 0.0;
}

/* A Bermudan swaption on every path and date (bermudan_swaption.cpp:49-146): exercise values of the tail swaps,
 * backward Longstaff-Schwartz over the exercise dates on the short-rate state, first exercise per path, then
 * on every date the tail swap (exercised, physical), nothing (exercised, cash) or the regressed continuation. */
static void bermudan_cube(const Model* m, const Trade* tr, const Grid* g, const double* X, const double* Dm, size_t nP,
                          double* out, double* exIndex) {
  const size_t nT = g->n, nE = tr->nEx;
  size_t* jEx = (size_t*)malloc(nE * sizeof(size_t));
  Trade* tails = (Trade*)calloc(nE, sizeof(Trade));
  for (size_t k = 0; k < nE; ++k) {
    jEx[k] = (size_t)find_time(g, tr->ex[k]);
    size_t first = 0;
    while (first < tr->nSched && tr->sched[first] < tr->ex[k] - 1e-10) ++first;
    tails[k] = swap_of(tr->notional, tr->fixed, tr->payFixed, tr->sched + first, tr->nSched - first);
  }
  double* exValue = (double*)malloc(nE * nP * sizeof(double));
  for (size_t k = 0; k < nE; ++k) value_at(m, &tails[k], g, jEx[k], X, NULL, nP, exValue + k * nP);
  double* strategy = (double*)calloc((nE + 1) * nP, sizeof(double));
  unsigned char* exercise = (unsigned char*)calloc(nE * nP, 1);
  double *realised = (double*)calloc(nP, sizeof(double)), *target = (double*)malloc(nP * sizeof(double));
  double* x = (double*)malloc(nP * sizeof(double));
  unsigned char* itm = (unsigned char*)malloc(nP);
  orc_regression reg;
  orc_regression2 reg2;
  /* degree >= 10: the two-regressor basis of degree - 10 on (x, co-terminal swap rate) */
  const int twoD = tr->degree >= 10, deg = twoD ? tr->degree - 10 : tr->degree;
  double* sw = (double*)malloc(nP * sizeof(double));
  for (size_t k = nE; k-- > 0;) {
    const size_t j = jEx[k];
    for (size_t p = 0; p < nP; ++p) {
      x[p] = X[p * nT + j];
      target[p] = realised[p] / Dm[p * nT + j];
      itm[p] = exValue[k * nP + p] > 0.0;
      if (twoD) sw[p] = coterminal_rate(m, &tails[k], g->t[j], x[p]);
    }
    if (twoD) orc_reg2_fit(&reg2, deg, x, sw, target, itm, nP);
    else orc_reg_fit(&reg, deg, x, target, itm, nP);
    for (size_t p = 0; p < nP; ++p) {
      const double e = exValue[k * nP + p];
      const double c = twoD ? orc_reg2_predict(&reg2, x[p], sw[p]) : orc_reg_predict(&reg, x[p]);
      if (e > 0.0 && e > c) exercise[k * nP + p] = 1, realised[p] = Dm[p * nT + j] * e;
    }
    memcpy(strategy + k * nP, realised, nP * sizeof(double));
  }
  for (size_t p = 0; p < nP; ++p) {
    exIndex[p] = -1.0;
    for (size_t k = 0; k < nE; ++k)
      if (exercise[k * nP + p]) {
        exIndex[p] = (double)k;
        break;
      }
  }
  double *cont = (double*)malloc(nP * sizeof(double)), *tailv = (double*)malloc(nE * nP * sizeof(double));
  for (size_t j = 0; j < nT; ++j) {
    const double t = g->t[j];
    size_t nextK = 0;
    while (nextK < nE && tr->ex[nextK] <= t + 1e-10) ++nextK;
    if (nextK < nE) {
      for (size_t p = 0; p < nP; ++p) {
        x[p] = X[p * nT + j], target[p] = strategy[nextK * nP + p] / Dm[p * nT + j];
        if (twoD) sw[p] = coterminal_rate(m, &tails[nextK], t, x[p]);
      }
      if (twoD) orc_reg2_fit(&reg2, deg, x, sw, target, NULL, nP);
      else orc_reg_fit(&reg, deg, x, target, NULL, nP);
      for (size_t p = 0; p < nP; ++p) {
        const double c = twoD ? orc_reg2_predict(&reg2, x[p], sw[p]) : orc_reg_predict(&reg, x[p]);
        cont[p] = c > 0.0 ? c : 0.0;
      }
    } else {
      for (size_t p = 0; p < nP; ++p) cont[p] = 0.0;
    }
    if (tr->physical)
      for (size_t k = 0; k < nextK; ++k) value_at(m, &tails[k], g, j, X, NULL, nP, tailv + k * nP);
    for (size_t p = 0; p < nP; ++p) {
      const double k = exIndex[p];
      double v;
      if (k >= 0.0 && (size_t)k < nextK) v = tr->physical ? tailv[(size_t)k * nP + p] : 0.0;
      else v = cont[p];
      out[p * nT + j] = tr->position * v;
    }
  }
  for (size_t k = 0; k < nE; ++k) free(tails[k].sched);
  free(tails), free(jEx), free(exValue), free(strategy), free(exercise), free(realised), free(target), free(x);
  free(itm), free(cont), free(tailv), free(sw);
}

static double required_collateral(double v, double hc, double ho) {
  double c = 0.0;
  if (v > hc) c += v - hc;
  if (isfinite(ho) && -v > ho) c -= -v - ho;
  return c;
}

int orc_collateral(const double* values, const double* unitPrice, size_t nP, const double* times, size_t nT, double hc,
                   double ho, double mta, double ia, double mpr, int type, double haircut, double* out) {
  if (ho < 0.0) ho = INFINITY;
  if (hc < 0.0 || mta < 0.0 || mpr < 0.0 || haircut < 0.0 || haircut >= 1.0) return 1;
  const int securities = type != 0;
  if (securities && !unitPrice) return 1;
  const Grid g = {nT, (double*)times};
  size_t* call = (size_t*)malloc((nT ? nT : 1) * sizeof(size_t));
  for (size_t j = 0; j < nT; ++j) call[j] = at_or_before(&g, times[j] - mpr > 0.0 ? times[j] - mpr : 0.0);
  const double keep = securities ? 1.0 - haircut : 1.0;
  for (size_t p = 0; p < nP; ++p) {
    const double* V = values + p * nT;
    const double* P = securities ? unitPrice + p * nT : NULL;
#define PRICE(j) (securities ? P[j] : 1.0)
    double units = required_collateral(V[call[0]], hc, ho) / (keep * PRICE(call[0]));
    for (size_t j = 0; j < nT; ++j) {
      const size_t c = call[j];
      const double target = required_collateral(V[c], hc, ho);
      if (fabs(target - units * keep * PRICE(c)) >= mta) units = target / (keep * PRICE(c));
      out[p * nT + j] = units * PRICE(j) + ia;
    }
#undef PRICE
  }
  free(call);
  return 0;
}

static double time_average(const double* t, const double* v, size_t n, double horizon) {
  double integral = 0.0, end = 0.0;
  for (size_t j = 1; j < n && t[j] <= horizon + 1e-10; ++j) {
    integral += v[j] * (t[j] - t[j - 1]);
    end = t[j];
  }
  return end > 0.0 ? integral / end : (n == 0 ? 0.0 : v[0]);
}

void orc_profile(const double* values, const double* deflator, size_t nP, const double* times, size_t nT, double q,
                 double horizon, double* out) {
  double* pos = (double*)malloc((nP ? nP : 1) * sizeof(double));
  const double n = (double)nP;
  for (size_t j = 0; j < nT; ++j) {
    double sum = 0.0, ee = 0.0, ene = 0.0, dee = 0.0, dene = 0.0;
    for (size_t p = 0; p < nP; ++p) {
      const double v = values[p * nT + j], d = deflator[p * nT + j];
      sum += v;
      pos[p] = v > 0.0 ? v : 0.0;
      ee += pos[p];
      ene += v < 0.0 ? v : 0.0;
      dee += d * pos[p];
      dene += d * (v < 0.0 ? v : 0.0);
    }
    out[j] = sum / n, out[nT + j] = ee / n, out[2 * nT + j] = ene / n;
    out[3 * nT + j] = orc_quantile(pos, nP, q);
    out[4 * nT + j] = dee / n, out[5 * nT + j] = dene / n;
  }
  free(pos);
  double* eff = (double*)malloc((nT ? nT : 1) * sizeof(double));
  double running = 0.0, mx = 0.0;
  for (size_t j = 0; j < nT; ++j) {
    running = running > out[nT + j] ? running : out[nT + j];
    eff[j] = running;
    if (j == 0 || out[3 * nT + j] > mx) mx = out[3 * nT + j];
  }
  out[6 * nT] = time_average(times, out + nT, nT, horizon);
  out[6 * nT + 1] = time_average(times, eff, nT, 1.0);
  out[6 * nT + 2] = nT ? mx : 0.0;
  free(eff);
}

static double default_prob(const Hazard* h, double t1, double t2) { return hazard_survival(h, t1) - hazard_survival(h, t2); }

double orc_unilateral_cva(const double* times, const double* dee, size_t n, const double* pillars, const double* hazards,
                          size_t nh, double recovery) {
  const Hazard h = {nh, (double*)pillars, (double*)hazards};
  double cva = 0.0; /* the term at index 0 is zero and is summed first, as the term structure is */
  for (size_t i = 1; i < n; ++i) cva += (1.0 - recovery) * (0.5 * (dee[i - 1] + dee[i])) * default_prob(&h, times[i - 1], times[i]);
  return cva;
}

void orc_bilateral_cva(const double* times, const double* dee, const double* dene, size_t n, const double* cp,
                       const double* ch, size_t nc, const double* op, const double* oh, size_t no, double rc, double ro,
                       double* out) {
  const Hazard c = {nc, (double*)cp, (double*)ch}, o = {no, (double*)op, (double*)oh};
  double cva = 0.0, dva = 0.0;
  for (size_t i = 1; i < n; ++i) {
    const double mid = 0.5 * (times[i - 1] + times[i]);
    cva += (1.0 - rc) * 0.5 * (dee[i - 1] + dee[i]) * hazard_survival(&o, mid) * default_prob(&c, times[i - 1], times[i]);
    dva += (1.0 - ro) * 0.5 * (-dene[i - 1] - dene[i]) * hazard_survival(&c, mid) * default_prob(&o, times[i - 1], times[i]);
  }
  out[0] = cva, out[1] = dva;
}

double orc_pathwise_cva(const double* exposure, const double* deflator, const double* survival, size_t nP, size_t nT,
                        const uint64_t* dates, size_t nDates, double recovery) {
  double total = 0.0;
  for (size_t p = 0; p < nP; ++p) {
    const double* E = exposure + p * nT;
    const double* D = deflator + p * nT;
    const double* Q = survival + p * nT;
    double prev = D[dates[0]] * (E[dates[0]] > 0.0 ? E[dates[0]] : 0.0);
    for (size_t k = 1; k < nDates; ++k) {
      const size_t i0 = dates[k - 1], i1 = dates[k];
      const double cur = D[i1] * (E[i1] > 0.0 ? E[i1] : 0.0);
      total += 0.5 * (prev + cur) * (Q[i0] - Q[i1]);
      prev = cur;
    }
  }
  return (1.0 - recovery) * total / (double)nP;
}

static void free_model(Model* m) {
  free(m->hw.curve.t), free(m->hw.curve.r);
  for (size_t k = 0; k < m->nA; ++k) free(m->assets[k].carry.t), free(m->assets[k].carry.r);
  for (size_t k = 0; k < m->nC; ++k) free(m->credits[k].market.pillar), free(m->credits[k].market.hazard);
  free(m->assets), free(m->credits), free(m->corr), free(m->base);
}
static void free_netting(Netting* n) {
  for (size_t k = 0; k < n->nTr; ++k) free(n->tr[k].sched), free(n->tr[k].ex);
  free(n->tr);
}

int orc_engine_run(const double* model, size_t nm, const double* ns, size_t nn, double pfeQuantile, const double* z,
                   size_t streams, size_t cap, double* times, uint64_t* reporting, size_t* sizes, double* profile,
                   double* netted, double* collateral, double* deflator, double* survival, double* exercise, char* err,
                   size_t errLen) {
  Model m;
  Netting n;
  int rc = read_model(model, nm, &m, err, errLen);
  if (rc) return free_model(&m), rc;
  rc = read_netting(ns, nn, &n, err, errLen);
  if (rc) return free_model(&m), free_netting(&n), rc;
  for (size_t k = 0; k < n.nTr; ++k)
    if ((n.tr[k].kind == 1 || n.tr[k].kind == 2) && n.tr[k].asset >= m.nA) {
      free_model(&m), free_netting(&n);
      return fail(err, errLen, "ScenarioSet: unknown asset");
    }

  /* Reporting grid: base grid with every trade's event times; simulation grid: plus t - MPR under a CSA
   * (exposure_engine.cpp:35-48, time_grid.cpp:44-55). */
  size_t nEv = m.nBase;
  for (size_t k = 0; k < n.nTr; ++k) nEv += n.tr[k].kind == 0 ? n.tr[k].nSched : n.tr[k].kind == 3 ? n.tr[k].nSched + n.tr[k].nEx : 1;
  double* ev = (double*)malloc((nEv + 1) * sizeof(double));
  size_t q = 0;
  for (size_t k = 0; k < m.nBase; ++k) ev[q++] = m.base[k];
  const Grid base = make_grid(ev, q);
  memcpy(ev, base.t, base.n * sizeof(double));
  q = base.n;
  free(base.t);
  for (size_t k = 0; k < n.nTr; ++k) {
    if (n.tr[k].kind == 0 || n.tr[k].kind == 3) {
      for (size_t i = 0; i < n.tr[k].nSched; ++i) ev[q++] = n.tr[k].sched[i];
      for (size_t i = 0; n.tr[k].kind == 3 && i < n.tr[k].nEx; ++i) ev[q++] = n.tr[k].ex[i];
    } else {
      ev[q++] = n.tr[k].maturity;
    }
  }
  const Grid rep = make_grid(ev, q);
  free(ev);
  Grid sim;
  if (n.csa.has && n.csa.mpr > 0.0) {
    double* t2 = (double*)malloc(2 * rep.n * sizeof(double));
    size_t c = 0;
    for (size_t j = 0; j < rep.n; ++j) t2[c++] = rep.t[j];
    for (size_t j = 0; j < rep.n; ++j)
      if (rep.t[j] > n.csa.mpr) t2[c++] = rep.t[j] - n.csa.mpr;
    sim = make_grid(t2, c);
    free(t2);
  } else {
    sim = make_grid(rep.t, rep.n);
  }
  const size_t nT = sim.n, nR = rep.n, nP = m.nP, nA = m.nA, nC = m.nC, F = m.F;
  sizes[0] = nT, sizes[1] = nR;
  if (nT > cap || nR > cap) {
    free_model(&m), free_netting(&n), free(rep.t), free(sim.t);
    return fail(err, errLen, "engine: grid larger than the output capacity");
  }
  for (size_t j = 0; j < nT; ++j) times[j] = sim.t[j];
  for (size_t k = 0; k < nR; ++k) reporting[k] = (uint64_t)find_time(&sim, rep.t[k]);

  /* Scenarios from the injected normals: normal k of step j on stream s at z[((j - 1) nNormals + k) streams + s];
   * path p reads stream p >> 1 with sign (-1)^(p & 1) when antithetic (scenario_generator.cpp:94-141). */
  const size_t nF = m.nF;
  size_t nNormals = F + 1 + nF; /* drivers | rate integral | foreign rate integrals | CIR bridges */
  size_t* cOff = (size_t*)calloc(nC + 1, sizeof(size_t));
  for (size_t c = 0; c < nC; ++c) cOff[c] = nNormals, nNormals += m.credits[c].sub - 1;
  double* L = (double*)malloc(F * F * sizeof(double));
  if (cholesky(m.corr, F, L)) {
    free_model(&m), free_netting(&n), free(rep.t), free(sim.t), free(cOff), free(L);
    return fail(err, errLen, "cholesky: correlation is not symmetric positive definite");
  }
  double* X = (double*)calloc(nP * nT, sizeof(double));
  double* Dm = (double*)malloc(nP * nT * sizeof(double));
  double** S = (double**)calloc(nA + 1, sizeof(double*));
  for (size_t a = 0; a < nA; ++a) S[a] = (double*)calloc(nP * nT, sizeof(double));
  double* Q0 = (double*)malloc(nP * nT * sizeof(double));
  for (size_t f = 0; f < nF; ++f) m.XF[f] = (double*)calloc(nP * nT, sizeof(double));
  double xf[2] = {0.0, 0.0}, intF[2] = {0.0, 0.0};
  double *w = (double*)malloc(F * sizeof(double)), *step = (double*)malloc(nNormals * sizeof(double));
  double *spot = (double*)calloc(nA + 1, sizeof(double)), *y = (double*)calloc(nC + 1, sizeof(double));
  double* iy = (double*)calloc(nC + 1, sizeof(double));
  int bad = 0;
  for (size_t p = 0; p < nP && !bad; ++p) {
    const size_t s = m.antithetic ? p >> 1 : p;
    const double sign = m.antithetic && (p & 1) ? -1.0 : 1.0;
    if (s >= streams) {
      bad = 1;
      break;
    }
    double x = 0.0, defl = 1.0;
    xf[0] = xf[1] = 0.0;
    Dm[p * nT] = 1.0, Q0[p * nT] = 1.0;
    for (size_t a = 0; a < nA; ++a) spot[a] = m.assets[a].spot, S[a][p * nT] = spot[a];
    for (size_t c = 0; c < nC; ++c) y[c] = m.credits[c].y0, iy[c] = 0.0;
    for (size_t j = 1; j < nT; ++j) {
      const double t0 = sim.t[j - 1], t1 = sim.t[j];
      for (size_t k = 0; k < nNormals; ++k) step[k] = sign * z[((j - 1) * nNormals + k) * streams + s];
      for (size_t i = 0; i < F; ++i) {
        double sum = 0.0;
        for (size_t k = 0; k <= i; ++k) sum += L[i * F + k] * step[k];
        w[i] = sum;
      }
      const double integrated = hw_evolve(&m.hw, t0, t1, w[0], step[F], &x);
      defl *= exp(-integrated);
      X[p * nT + j] = x, Dm[p * nT + j] = defl;
      for (size_t f = 0; f < nF; ++f) {
        const size_t fi = 1 + nA + nC + f;
        const double q = m.corr[fi * F + 1 + f] * m.foreign[f].sigma * m.assets[f].vol;
        intF[f] = hw_evolve_drift(&m.foreign[f], t0, t1, w[fi], step[F + 1 + f], q, &xf[f]);
        m.XF[f][p * nT + j] = xf[f];
      }
      for (size_t a = 0; a < nA; ++a) {
        const Asset* as = &m.assets[a];
        const double dt = t1 - t0, carry = a < nF ? intF[a] : log(discount(&as->carry, t0) / discount(&as->carry, t1));
        const double drift = integrated - carry - 0.5 * as->vol * as->vol * dt;
        spot[a] = spot[a] * exp(drift + as->vol * sqrt(dt) * w[1 + a]);
        S[a][p * nT + j] = spot[a];
      }
      for (size_t c = 0; c < nC; ++c) {
        cir_evolve(&m.credits[c], t1 - t0, w[1 + nA + c], step + cOff[c], &y[c], &iy[c]);
        if (c == 0) Q0[p * nT + j] = credit_survival(&m.credits[0], t1, iy[0]);
      }
      if (nC == 0) Q0[p * nT + j] = 1.0;
    }
  }
  free(w), free(step), free(spot), free(y), free(iy), free(cOff), free(L);
  if (bad) {
    rc = fail(err, errLen, "injected normals: too few streams");
    goto done;
  }

  /* Trade values, netted in trade order; collateral; exposure; profile on the reporting dates. */
  {
    double* V = (double*)calloc(nP * nT, sizeof(double));
    double* slice = (double*)malloc(nP * sizeof(double));
    double* cube = (double*)malloc(nP * nT * sizeof(double));
    double* exIdx = (double*)malloc(nP * sizeof(double));
    size_t berm = 0;
    for (size_t k = 0; k < n.nTr; ++k) {
      if (n.tr[k].kind == 3) {
        bermudan_cube(&m, &n.tr[k], &sim, X, Dm, nP, cube, exIdx);
        if (exercise) memcpy(exercise + berm * nP, exIdx, nP * sizeof(double));
        ++berm;
      }
      for (size_t j = 0; j < nT; ++j) {
        if (n.tr[k].kind == 3)
          for (size_t p = 0; p < nP; ++p) slice[p] = cube[p * nT + j];
        else
          value_at(&m, &n.tr[k], &sim, j, X, S, nP, slice);
        for (size_t p = 0; p < nP; ++p) V[p * nT + j] = k == 0 ? slice[p] : V[p * nT + j] + slice[p];
      }
    }
    free(slice), free(cube), free(exIdx);
    double* C = (double*)calloc(nP * nT, sizeof(double));
    if (n.csa.has) {
      double* price = NULL;
      if (n.csa.type == 1) {
        if (n.csa.bondMaturity < sim.t[nT - 1] - 1e-10) {
          free(V), free(C);
          rc = fail(err, errLen, "the collateral bond must mature after the horizon");
          goto done;
        }
        price = (double*)malloc(nP * nT * sizeof(double));
        for (size_t p = 0; p < nP; ++p)
          for (size_t j = 0; j < nT; ++j) price[p * nT + j] = hw_bond(&m.hw, sim.t[j], n.csa.bondMaturity, X[p * nT + j]);
      } else if (n.csa.type == 2) {
        if (n.csa.asset >= nA) {
          free(V), free(C);
          rc = fail(err, errLen, "collateral asset out of range");
          goto done;
        }
        price = (double*)malloc(nP * nT * sizeof(double));
        memcpy(price, S[n.csa.asset], nP * nT * sizeof(double));
      }
      if (orc_collateral(V, price, nP, sim.t, nT, n.csa.hc, n.csa.ho, n.csa.mta, n.csa.ia, n.csa.mpr, n.csa.type,
                         n.csa.haircut, C)) {
        free(price), free(V), free(C);
        rc = fail(err, errLen, "simulateCollateral: invalid collateral agreement");
        goto done;
      }
      free(price);
    }
    double* E = (double*)malloc(nP * nR * sizeof(double));
    double* DR = (double*)malloc(nP * nR * sizeof(double));
    for (size_t p = 0; p < nP; ++p)
      for (size_t k = 0; k < nR; ++k) {
        const size_t j = reporting[k];
        E[p * nR + k] = V[p * nT + j] - C[p * nT + j];
        DR[p * nR + k] = Dm[p * nT + j];
      }
    double* prof = (double*)malloc((6 * nR + 3) * sizeof(double));
    orc_profile(E, DR, nP, rep.t, nR, pfeQuantile, 0.0, prof);
    if (profile) memcpy(profile, prof, 6 * nR * sizeof(double));
    if (netted) memcpy(netted, V, nP * nT * sizeof(double));
    if (collateral) memcpy(collateral, C, nP * nT * sizeof(double));
    if (deflator) memcpy(deflator, Dm, nP * nT * sizeof(double));
    if (survival) memcpy(survival, Q0, nP * nT * sizeof(double));
    free(prof), free(E), free(DR), free(V), free(C);
  }
done:
  for (size_t f = 0; f < nF; ++f) free(m.XF[f]);
  for (size_t a = 0; a < nA; ++a) free(S[a]);
  free(S), free(X), free(Dm), free(Q0);
  free(rep.t), free(sim.t);
  free_model(&m), free_netting(&n);
  return rc;
}
