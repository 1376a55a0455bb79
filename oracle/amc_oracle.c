/* ORACLE / TEST INFRASTRUCTURE ONLY.  Plain-C restatement of the reference's Longstaff-Schwartz pieces:
 *   orc_reg_fit / orc_reg_predict   PolynomialRegression::fit / predict (src/core/regression.cpp:29-98) with
 *                                   leastSquares (:8-27) and solveLinearSystem (src/core/matrix.cpp:70-96):
 *                                   masked standardisation, degree fallback, ridge 1e-12 n, normal equations
 *                                   solved by Gaussian elimination with partial pivoting;
 *   orc_fit_amc                     fitAmc (src/gpu/fused_exposure.cpp:103-156): the policy and continuation
 *                                   coefficients of a plan's Bermudans, fitted in double precision on the
 *                                   single-precision states of the AMC pass (runAmcStates), backwards over the
 *                                   exercise dates;
 *   orc_reg2_fit / orc_reg2_predict the two-regressor basis of this library (short rate and co-terminal swap
 *                                   rate), an extension with no reference code behind it (oracle.h).
 * The sums run in path order, as the reference's, so the fitted coefficients are the reference's bits. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

enum { TERM = 8, MAX_BERM = 4, MAX_DEG = 3 };

/* Normal equations of the standardised monomial design, solved by elimination with partial pivoting. */
static void least_squares(const double* x, const double* y, const unsigned char* mask, size_t n, double center,
                          double scale, int degree, size_t count, double* coef) {
  const int k = degree + 1;
  double A[(MAX_DEG + 1) * (MAX_DEG + 1)] = {0}, b[MAX_DEG + 1] = {0}, row[MAX_DEG + 1];
  for (size_t i = 0; i < n; ++i) {
    if (mask && !mask[i]) continue;
    const double z = (x[i] - center) / scale;
    double power = 1.0;
    for (int d = 0; d < k; ++d) row[d] = power, power *= z;
    for (int a = 0; a < k; ++a) {
      b[a] += row[a] * y[i];
      for (int c = 0; c <= a; ++c) A[a * k + c] += row[a] * row[c];
    }
  }
  const double ridge = 1e-12 * (double)count;
  for (int a = 0; a < k; ++a) {
    for (int c = 0; c < a; ++c) A[c * k + a] = A[a * k + c];
    A[a * k + a] += ridge;
  }
  for (int col = 0; col < k; ++col) {
    int pivot = col;
    for (int r = col + 1; r < k; ++r)
      if (fabs(A[r * k + col]) > fabs(A[pivot * k + col])) pivot = r;
    if (pivot != col) {
      for (int c = 0; c < k; ++c) {
        const double t = A[col * k + c];
        A[col * k + c] = A[pivot * k + c], A[pivot * k + c] = t;
      }
      const double t = b[col];
      b[col] = b[pivot], b[pivot] = t;
    }
    for (int r = col + 1; r < k; ++r) {
      const double f = A[r * k + col] / A[col * k + col];
      if (f == 0.0) continue;
      for (int c = col; c < k; ++c) A[r * k + c] -= f * A[col * k + c];
      b[r] -= f * b[col];
    }
  }
  for (int i = k; i-- > 0;) {
    double s = b[i];
    for (int c = i + 1; c < k; ++c) s -= A[i * k + c] * coef[c];
    coef[i] = s / A[i * k + i];
  }
}

void orc_reg_fit(orc_regression* r, int degree, const double* x, const double* y, const unsigned char* mask, size_t n) {
  size_t count = 0;
  double sx = 0.0, sxx = 0.0, sy = 0.0;
  for (size_t i = 0; i < n; ++i) {
    if (mask && !mask[i]) continue;
    ++count;
    sx += x[i];
    sxx += x[i] * x[i];
    sy += y[i];
  }
  memset(r->coef, 0, sizeof r->coef);
  if (count == 0) {
    r->center = 0.0, r->scale = 1.0, r->ncoef = 1;
    return;
  }
  r->center = sx / (double)count;
  const double var = sxx / (double)count - r->center * r->center;
  r->scale = sqrt(var > 0.0 ? var : 0.0);
  int deg = degree;
  if (r->scale < 1e-12 * (fabs(r->center) > 1.0 ? fabs(r->center) : 1.0)) deg = 0;
  if (count < 2 * (size_t)(deg + 1)) deg = count >= 4 ? (int)(count / 2) - 1 : 0;
  if (deg == 0) {
    r->scale = 1.0, r->ncoef = 1, r->coef[0] = sy / (double)count;
    return;
  }
  r->ncoef = deg + 1;
  least_squares(x, y, mask, n, r->center, r->scale, deg, count, r->coef);
}

double orc_reg_predict(const orc_regression* r, double x) {
  const double z = (x - r->center) / r->scale;
  double v = 0.0;
  for (int d = r->ncoef; d-- > 0;) v = v * z + r->coef[d];
  return v;
}

int orc_basis2(double z, double w, int degree, double* out) {
  const double v[10] = {1.0, z, w, z * z, z * w, w * w, z * z * z, z * z * w, z * w * w, w * w * w};
  const int count = degree <= 0 ? 1 : degree == 1 ? 3 : degree == 2 ? 6 : 10;
  for (int i = 0; i < 10; ++i) out[i] = i < count ? v[i] : 0.0;
  return count;
}

void orc_reg2_fit(orc_regression2* r, int degree, const double* x, const double* s, const double* y, const unsigned char* mask,
                  size_t n) {
  size_t count = 0;
  double sx = 0.0, sxx = 0.0, ss = 0.0, sss = 0.0, sy = 0.0;
  for (size_t i = 0; i < n; ++i) {
    if (mask && !mask[i]) continue;
    ++count;
    sx += x[i], sxx += x[i] * x[i], ss += s[i], sss += s[i] * s[i], sy += y[i];
  }
  memset(r, 0, sizeof *r);
  r->sx = r->ss = 1.0;
  if (count == 0) {
    r->degree = -1;
    return;
  }
  const double cnt = (double)count;
  r->cx = sx / cnt, r->cs = ss / cnt;
  const double vx = sxx / cnt - r->cx * r->cx, vs = sss / cnt - r->cs * r->cs;
  r->sx = sqrt(vx > 0.0 ? vx : 0.0), r->ss = sqrt(vs > 0.0 ? vs : 0.0);
  int deg = degree;
  if (r->sx < 1e-12 * (fabs(r->cx) > 1.0 ? fabs(r->cx) : 1.0) || r->ss < 1e-12 * (fabs(r->cs) > 1.0 ? fabs(r->cs) : 1.0)) deg = 0;
  while (deg > 0 && cnt < 2.0 * (deg == 1 ? 3 : deg == 2 ? 6 : 10)) --deg;
  if (deg == 0) {
    r->sx = r->ss = 1.0, r->cx = r->cs = 0.0, r->coef[0] = sy / cnt, r->degree = 0;
    return;
  }
  double A[100] = {0}, b[10] = {0}, row[10];
  const int k = orc_basis2(0.0, 0.0, deg, row);
  for (size_t i = 0; i < n; ++i) {
    if (mask && !mask[i]) continue;
    orc_basis2((x[i] - r->cx) / r->sx, (s[i] - r->cs) / r->ss, deg, row);
    for (int a = 0; a < k; ++a) {
      b[a] += row[a] * y[i];
      for (int c = 0; c <= a; ++c) A[a * 10 + c] += row[a] * row[c];
    }
  }
  /* The two regressors can be nearly collinear (in a one-factor model the swap rate is a smooth function of the short
   * rate; the graded Gram's condition number then reaches 1e17): a ridge of 1e-6 n on the standardised basis keeps the
   * solution stable to the summation order (predictions to ~1e-11) at a negligible bias where the data are
   * well conditioned (eigenvalues O(n)). */
  const double ridge = 1e-6 * cnt;
  double L[100] = {0}, z[10];
  for (int a = 0; a < k; ++a) A[a * 10 + a] += ridge;
  for (int i = 0; i < k; ++i)
    for (int j = 0; j <= i; ++j) {
      double v = A[i * 10 + j];
      for (int m = 0; m < j; ++m) v -= L[i * 10 + m] * L[j * 10 + m];
      L[i * 10 + j] = i == j ? sqrt(v > 0.0 ? v : 1.0) : v / L[j * 10 + j];
    }
  for (int i = 0; i < k; ++i) {
    double v = b[i];
    for (int j = 0; j < i; ++j) v -= L[i * 10 + j] * z[j];
    z[i] = v / L[i * 10 + i];
  }
  for (int i = k; i-- > 0;) {
    double v = z[i];
    for (int j = i + 1; j < k; ++j) v -= L[j * 10 + i] * r->coef[j];
    r->coef[i] = v / L[i * 10 + i];
  }
  r->degree = deg;
}

double orc_reg2_predict(const orc_regression2* r, double x, double s) {
  if (r->degree < 0) return 0.0;
  double row[10];
  const int k = orc_basis2((x - r->cx) / r->sx, (s - r->cs) / r->ss, r->degree, row);
  double v = 0.0;
  for (int i = 0; i < k; ++i) v += r->coef[i] * row[i];
  return v;
}

/* The record a fit leaves in a policy or continuation term (fused_exposure.cpp:118-123). */
static void write_term(float* rec, const orc_regression* r) {
  rec[2] = (float)r->center;
  rec[3] = (float)(1.0 / r->scale);
  for (int d = 0; d < 4; ++d) rec[4 + d] = d < r->ncoef ? (float)r->coef[d] : 0.0f;
}

int orc_fit_amc(const uint32_t* header, const uint32_t* indices, const float* params, const float* steps, float* terms,
                uint32_t rowsTotal, const uint32_t* degrees, size_t numBermudans, char* err, size_t errLen) {
  const uint32_t nP = header[0], nT = header[1];
  /* Where the regressions live: the policy term of each exercise, the continuation term of each date. */
  long decide[MAX_BERM][64], exDate[MAX_BERM][64], *cont[MAX_BERM];
  uint32_t nE[MAX_BERM] = {0, 0, 0, 0};
  for (int b = 0; b < MAX_BERM; ++b) {
    cont[b] = (long*)malloc(nT * sizeof(long));
    for (uint32_t j = 0; j < nT; ++j) cont[b][j] = -1;
  }
  int rc = 0;
  for (uint32_t j = 0; j < nT && !rc; ++j)
    for (uint32_t t = indices[j]; t < indices[j + 1]; ++t) {
      const uint32_t code = (uint32_t)terms[(size_t)t * TERM], kind = code & 15u, e = code >> 12u;
      uint32_t b = (code >> 8u) & 15u;
      if (kind != 6u && kind != 7u) continue;
      if (b >= numBermudans || b >= MAX_BERM || e >= 64u) {
        if (err && errLen) snprintf(err, errLen, "AMC term of an unknown Bermudan or exercise");
        rc = 1;
        break;
      }
      if (kind == 6u) {
        decide[b][e] = t, exDate[b][e] = j;
        if (e + 1 > nE[b]) nE[b] = e + 1;
      } else {
        cont[b][j] = t;
      }
    }
  uint32_t offsets[MAX_BERM + 1] = {0};
  for (int b = 0; b < MAX_BERM; ++b) offsets[b + 1] = offsets[b] + nE[b];
  float *x = NULL, *D = NULL, *E = NULL;
  if (!rc) {
    x = (float*)malloc((size_t)nT * nP * sizeof(float));
    D = (float*)malloc((size_t)nT * nP * sizeof(float));
    E = (float*)malloc(((size_t)offsets[MAX_BERM] + 1) * nP * sizeof(float));
    rc = orc_amc_states(header, indices, params, steps, terms, rowsTotal, offsets, x, D, E, err, errLen);
  }
  if (!rc) {
    double *xs = (double*)malloc(nP * sizeof(double)), *target = (double*)malloc(nP * sizeof(double));
    double* realised = (double*)malloc(nP * sizeof(double));
    unsigned char* mask = (unsigned char*)malloc(nP);
    for (size_t b = 0; b < numBermudans && b < MAX_BERM; ++b) {
      const uint32_t n = nE[b];
      double* strategy = (double*)calloc(((size_t)n + 1) * nP, sizeof(double));
      orc_regression reg;
      for (uint32_t p = 0; p < nP; ++p) realised[p] = 0.0;
      for (uint32_t k = n; k-- > 0;) {
        const size_t j = (size_t)exDate[b][k];
        const float* Ek = E + ((size_t)offsets[b] + k) * nP;
        for (uint32_t p = 0; p < nP; ++p) {
          xs[p] = x[j * nP + p];
          target[p] = realised[p] / D[j * nP + p];
          mask[p] = Ek[p] > 0.0f;
        }
        orc_reg_fit(&reg, (int)degrees[b], xs, target, mask, nP);
        write_term(terms + (size_t)decide[b][k] * TERM, &reg);
        for (uint32_t p = 0; p < nP; ++p)
          if (Ek[p] > 0.0f && Ek[p] > orc_reg_predict(&reg, xs[p])) realised[p] = D[j * nP + p] * Ek[p];
        memcpy(strategy + (size_t)k * nP, realised, nP * sizeof(double));
      }
      for (uint32_t j = 0; j < nT; ++j) {
        if (cont[b][j] < 0) continue;
        uint32_t next = 0;
        while (next < n && (uint32_t)exDate[b][next] <= j) ++next;
        const double* s = strategy + (size_t)next * nP;
        for (uint32_t p = 0; p < nP; ++p) xs[p] = x[(size_t)j * nP + p], target[p] = s[p] / D[(size_t)j * nP + p];
        orc_reg_fit(&reg, (int)degrees[b], xs, target, NULL, nP);
        write_term(terms + (size_t)cont[b][j] * TERM, &reg);
      }
      free(strategy);
    }
    free(xs), free(target), free(realised), free(mask);
  }
  for (int b = 0; b < MAX_BERM; ++b) free(cont[b]);
  free(x), free(D), free(E);
  return rc;
}
