/* ORACLE / TEST INFRASTRUCTURE ONLY (not part of the product): a plain-C restatement of the
 * reference's algorithm for the exposure path, used by the tests and by the smoke check as the checker.
 *
 *   orc_run_fused     the fused pipeline on a plan in the reference's layout, in single precision:
 *                     fused-exposure per path, workgroup tree reduction, compensated sum over
 *                     workgroups (src/gpu/fused_reference.cpp:198-607), with the row statistics'
 *                     quantile computed exactly as ccr::quantile (include/ccr/core/math.hpp:39-47).
 *   orc_amc_states, orc_fit_amc   the AMC state pass and the Longstaff-Schwartz fit of a plan's Bermudans
 *                     (fused_reference.cpp:609-626, fused_exposure.cpp:103-156; amc_oracle.c).
 *   orc_engine_run    the FP64 exposure engine (src/exposure/exposure_engine.cpp:50-81) on injected
 *                     normals: scenario generation, swap / forward / option / Bermudan valuation, netting,
 *                     collateral, exposure profile.
 *   orc_quantile, orc_collateral, orc_profile, orc_unilateral_cva, orc_bilateral_cva: the building
 *                     blocks (math.hpp:39, collateral.cpp:10-47, exposure_profile.cpp:10-60, cva.cpp:11-48).
 */
#ifndef ZK_ORACLE_H
#define ZK_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Returns 0, or 1 with a message in err. rows (nullable) receives [rowsTotal][nP]. */
int orc_run_fused(const uint32_t* header, const uint32_t* indices, size_t nIdx, const float* params, const float* steps,
                  const float* terms, size_t nTerms, const float* requests, size_t nReq, uint32_t rowsTotal,
                  uint32_t numOutputs, float* sums, float* values, float* rows, char* err, size_t errLen);

/* gpu::runAmcStates (fused_reference.cpp:609-626): x and deflator [date][path]; exercise values
 * [offsets[b] + e][path] for exercise e of Bermudan b. */
int orc_amc_states(const uint32_t* header, const uint32_t* indices, const float* params, const float* steps,
                   const float* terms, uint32_t rowsTotal, const uint32_t* offsets, float* x, float* deflator,
                   float* exercise, char* err, size_t errLen);

/* PolynomialRegression (regression.cpp:29-98): predict(x) = sum_d coef[d] ((x - center) / scale)^d. */
typedef struct orc_regression {
  double center, scale, coef[4];
  int ncoef;
} orc_regression;
void orc_reg_fit(orc_regression* r, int degree, const double* x, const double* y, const unsigned char* mask, size_t n);
double orc_reg_predict(const orc_regression* r, double x);

/* The two-regressor basis (an extension of the reference, whose regression is on the short rate alone; no reference
 * code pins it): the graded monomials of total degree <= 3 in the standardised short rate z and co-terminal swap
 * rate w -- 1, z, w, z^2, z w, w^2, z^3, z^2 w, z w^2, w^3 -- fitted by the normal equations with the ridge 1e-6 n,
 * solved by Cholesky.  The degree falls to 0 (the mean) when either regressor is degenerate and while the samples
 * are fewer than twice the basis. */
typedef struct orc_regression2 {
  double cx, sx, cs, ss;  /* centers and scales */
  double coef[10];        /* graded order; zero beyond the degree */
  int degree;             /* -1: no sample (predicts 0) */
} orc_regression2;
void orc_reg2_fit(orc_regression2* r, int degree, const double* x, const double* s, const double* y, const unsigned char* mask,
                  size_t n);
double orc_reg2_predict(const orc_regression2* r, double x, double s);
/* The basis of degree <= 3 at (z, w), graded, into out[10] (zero beyond the degree); the number of functions. */
int orc_basis2(double z, double w, int degree, double* out);

/* fitAmc (fused_exposure.cpp:103-156): fills the policy and continuation records of terms in place, from the
 * AMC pass of the plan; degrees[b] is the regression degree of Bermudan b. */
int orc_fit_amc(const uint32_t* header, const uint32_t* indices, const float* params, const float* steps, float* terms,
                uint32_t rowsTotal, const uint32_t* degrees, size_t numBermudans, char* err, size_t errLen);

/* Engine on injected normals z[((j - 1) * nNormals + k) * streams + s].  Sizes: sizes[0] = nT (simulation
 * dates), sizes[1] = nR; times has room for cap dates, reporting for cap indices.  Per-path outputs
 * (nullable) are [path][date] over the simulation grid; survival is that of credit 0; exercise is
 * [bermudan][path], the first exercise taken (-1: never).  profile holds EV, EE, ENE, PFE, EE*, ENE* over
 * the reporting dates (6 * nR). */
int orc_engine_run(const double* model, size_t nm, const double* ns, size_t nn, double pfeQuantile, const double* normals,
                   size_t streams, size_t cap, double* times, uint64_t* reporting, size_t* sizes, double* profile,
                   double* netted, double* collateral, double* deflator, double* survival, double* exercise, char* err,
                   size_t errLen);

double orc_quantile(const double* v, size_t n, double p);
/* values, unitPrice (nullable): [path][date]; out: [path][date] collateral held. */
int orc_collateral(const double* values, const double* unitPrice, size_t nP, const double* times, size_t nT, double hc,
                   double ho, double mta, double ia, double mpr, int type, double haircut, double* out);
/* EV, EE, ENE, PFE, EE*, ENE* (6 * nT), then EPE(horizon), effective EPE(1y), max PFE. */
void orc_profile(const double* values, const double* deflator, size_t nP, const double* times, size_t nT, double q,
                 double horizon, double* out);
double orc_unilateral_cva(const double* times, const double* dee, size_t n, const double* pillars, const double* hazards,
                          size_t nh, double recovery);
void orc_bilateral_cva(const double* times, const double* dee, const double* dene, size_t n, const double* cp,
                       const double* ch, size_t nc, const double* op, const double* oh, size_t no, double rc, double ro,
                       double* out);
/* pathwiseCva (cva.cpp:57-77): exposure, deflator, survival [path][date]; dates index the columns. */
double orc_pathwise_cva(const double* exposure, const double* deflator, const double* survival, size_t nP, size_t nT,
                        const uint64_t* dates, size_t nDates, double recovery);

#ifdef __cplusplus
}
#endif
#endif
