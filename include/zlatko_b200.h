/* zlatko_b200: the counterparty-exposure hot path of svr-net/zlatko on one NVIDIA B200 (sm_100a).
 *
 * The reference compiles a netting set into a gpu::FusedPlan (flat tables) and hands it to a
 * backend functor that returns a gpu::FusedOutput (src/app/analyses.cpp:2148-2177, the seam of
 * analyseFused; the two reference backends are the WebGPU read-back at analyses.cpp:2179 and
 * runFusedReference at analyses.cpp:2196).  This library is a third backend behind that seam:
 * it takes the plan's buffers verbatim and fills the output in the reference's layout.
 *
 * Every entry point returns a zk_status and never throws across the ABI; zk_last_error() gives the
 * message.  ZK_ERR_INVALID_PLAN and ZK_ERR_UNSUPPORTED are the cases where the reference throws
 * std::invalid_argument (PlanView, src/gpu/fused_reference.cpp:64-75; finishFused :473-478;
 * compile, src/gpu/fused_exposure.cpp:219-230).  Calls on one context are serialised on the
 * context's stream; a context is not thread-safe (guard it with a mutex or use one per thread).
 * There is no CPU fallback: without a CUDA device zk_context_create fails with ZK_ERR_NO_DEVICE.
 */
#ifndef ZLATKO_B200_H
#define ZLATKO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZK_ABI_VERSION 1

typedef enum zk_status {
  ZK_OK = 0,
  ZK_ERR_INVALID_ARGUMENT = 1, /* null pointer, wrong buffer length */
  ZK_ERR_INVALID_PLAN = 2,     /* malformed or inconsistent plan tables */
  ZK_ERR_UNSUPPORTED = 3,      /* a plan feature this library does not run (message says which) */
  ZK_ERR_OUT_OF_MEMORY = 4,
  ZK_ERR_CUDA = 5,             /* a CUDA runtime error (launch failure, ...) */
  ZK_ERR_DEVICE_TIMEOUT = 6,   /* a bounded wait inside a kernel gave up; the context stays usable */
  ZK_ERR_NO_DEVICE = 7
} zk_status;

typedef struct zk_context zk_context;

/* The GPU buffers of a reference gpu::FusedPlan (include/ccr/gpu/fused_exposure.hpp:152-226), in
 * the reference's exact binary layout.  All lengths count elements. */
typedef struct zk_plan_view {
  const uint32_t* header;  size_t header_len;   /* kHeaderWords = 32 (fused_kernels.cpp:32-41)           */
  const uint32_t* indices; size_t indices_len;  /* termStart[nT+1] | callIndex[nT] | reportingSlot[nT] | imTarget[nT] */
  const float* params;     size_t params_len;   /* kParamCount = 84: CIR x2 | CSA | spots | Cholesky 8x8 | collateral */
  const float* steps;      size_t steps_len;    /* nT * kStepStride (24)                                  */
  const float* terms;      size_t terms_len;    /* numTerms * kTermStride (8)                             */
  const float* requests;   size_t requests_len; /* numRequests * kRequestStride (8)                       */
  uint32_t rows_total;                          /* FusedPlan::rows.total                                  */
  uint32_t num_outputs;                         /* FusedPlan::numOutputs                                  */
} zk_plan_view;

/* gpu::FusedOutput (fused_exposure.hpp:223-226): sums[nT * statsPerDate] (already divided by the
 * number of paths) and values[max(1, numOutputs)].  The caller owns both buffers. */
typedef struct zk_output {
  float* sums;   size_t sums_len;
  float* values; size_t values_len;
} zk_output;

/* Double-precision plan (the FP64 mode): the same layout with double tables, as produced by
 * zk_compile.  The reference's own plans are single precision; this mode exists to check the
 * kernels against the reference's FP64 ExposureEngine on identical normals. */
typedef struct zk_plan_view_f64 {
  const uint32_t* header;  size_t header_len;
  const uint32_t* indices; size_t indices_len;
  const double* params;    size_t params_len;
  const double* steps;     size_t steps_len;
  const double* terms;     size_t terms_len;
  const double* requests;  size_t requests_len;
  uint32_t rows_total;
  uint32_t num_outputs;
} zk_plan_view_f64;

typedef struct zk_output_f64 {
  double* sums;   size_t sums_len;
  double* values; size_t values_len;
} zk_output_f64;

/* ---- context ---------------------------------------------------------------------------------- */
zk_status zk_context_create(int device, zk_context** out);
void zk_context_destroy(zk_context* ctx);
const char* zk_last_error(const zk_context* ctx);
int zk_abi_version(void);
/* Runs the context's work on `stream` (a cudaStream_t; NULL: the context's own stream).  A book whose netting
 * sets differ widely in shared-memory state forks its large-state revalue launch onto a second stream the
 * context owns and joins it back with events, so work on `stream` stays ordered as usual (and a graph
 * captured from `stream` holds both branches). */
zk_status zk_context_set_stream(zk_context* ctx, void* stream);
/* Device memory a call or batch of this context may give to per-path rows and warp partials at once (bytes; 0, the
 * default: all netting sets at once while that takes under 70% of the free device memory, else 60% of it).  A
 * book whose rows exceed it runs its netting sets in waves that reuse one region: each wave's reduce and row
 * statistics follow its revalue launch, and the outputs are the same bits as in one wave.  (The reference's
 * kernels keep every netting set's rows, EXPO[rows][P], at once: fused_exposure.hpp:214-216.) */
zk_status zk_context_set_row_budget(zk_context* ctx, uint64_t bytes);
/* Which netting sets of a call or batch run on the tensor-core basis kernel: single-precision plans of bonds,
 * floating coupons, FX forwards and options, with no CSA or a cash CSA looking back at most one date and no rows
 * besides the exposure rows, grouped by identical margin-call and reporting dates into groups of at most 128.
 * On a date every distinct bond, fixing x bond, foreign bond x FX rate, FX rate and option of a group is evaluated
 * once per path and the netting sets' values are one FP16 hi/lo product on the tensor cores (about 22 bits of
 * each coefficient and basis value).  ZK_BASIS_AUTO (the default): groups of at least 24 netting sets;
 * ZK_BASIS_OFF: none (every netting set term by term, as the reference's kernel); ZK_BASIS_ALL: every eligible
 * netting set.  No counterpart in the reference. */
#define ZK_BASIS_AUTO 0u
#define ZK_BASIS_OFF 1u
#define ZK_BASIS_ALL 2u
zk_status zk_context_set_basis(zk_context* ctx, uint32_t mode);

/* Exact decisions: with guard > 0, zk_run_plan, zk_run_plans and zk_run_plan_rows take every margin call and
 * exercise decision as the FP64 mode takes it on the same normals.  The FP32 revalue kernel flags each path with a
 * decision whose margin (| |required - held| - MTA | for a call, |e| and |e - continuation| for an exercise) lies
 * within guard times a bound on the netting set's gross term value on that date; the flagged paths run again in
 * FP64 and in FP32, and their rows and share of the date statistics are replaced by the FP64 ones (the row
 * statistics recomputed).  The basis kernel is not used while it is on; plans with the nested initial margin are
 * not checked; a book whose rows exceed the row budget is refused (ZK_ERR_UNSUPPORTED).  guard = 0 (the default):
 * off, the reference kernel's single-precision decisions.  On the tested workloads 1e-7 already left no decision
 * apart; 3e-7 re-runs 0.2-9% of the paths.
 * zk_context_exact_stats returns (and clears) the paths flagged and the paths checked since the last call.
 * No counterpart in the reference (collateral.cpp:42, bermudan_swaption.cpp:87 are the rules). */
zk_status zk_context_set_exact_decisions(zk_context* ctx, double guard);
zk_status zk_context_exact_stats(zk_context* ctx, uint64_t* flagged_paths, uint64_t* checked_paths);

/* Host wall time in milliseconds of the last zk_run_plans / zk_run_plan call, by phase: [0] validate and lower the
 * plans (the basis groups included), [1] fill and send the inputs, [2] the device run, [3] the exact-decision check,
 * [4] the read-back into the caller's buffers.  No counterpart in the reference. */
zk_status zk_context_call_timings(const zk_context* ctx, double* ms5);

/* ---- the drop-in backend ------------------------------------------------------------------------ */
/* Replaces gpu::runFusedReference(plan) (src/gpu/fused_reference.cpp:628-630): the fused-exposure,
 * reduce-partials and row-statistics kernels (src/gpu/fused_kernels.cpp:224-530, :538-563,
 * :565-771) on the GPU.  Host buffers in, host buffers out. */
zk_status zk_run_plan(zk_context* ctx, const zk_plan_view* plan, zk_output* out);

/* zk_run_plan plus the per-path rows the fused kernel wrote, rows[row][path] (rows_total * nP floats): the
 * exposure slice of the reference's runFusedWorkgroups (FusedSlice::exposure, fused_reference.cpp:426-466). */
zk_status zk_run_plan_rows(zk_context* ctx, const zk_plan_view* plan, zk_output* out, float* rows);

/* Many plans in one launch (the reference's book mode, analyses.cpp:1604-2050 runs one plan per
 * netting set).  Plans that share the scenario (paths, dates, models, seed, Cholesky) share one
 * simulation of the risk factors on the GPU; the rest run as separate launches. */
zk_status zk_run_plans(zk_context* ctx, const zk_plan_view* plans, size_t n, zk_output* outs);

/* Replaces gpu::runAmcStates (src/gpu/fused_reference.cpp:609-626): x and the deflator on every date
 * ([date][path]) and the exercise value of every Bermudan exercise ([row][path], rows in Bermudan
 * then exercise order; exercise_rows must equal the plan's total number of exercise dates). */
zk_status zk_amc_states(zk_context* ctx, const zk_plan_view* plan, float* x, float* deflator, float* exercise,
                        size_t exercise_rows);

/* Replaces the Longstaff-Schwartz fit that the reference's gpu::compile runs on its CPU kernels (fitAmc,
 * src/gpu/fused_exposure.cpp:103-156): the AMC state pass on the GPU, then the policy regression of every
 * exercise (in-the-money paths, backwards) and the continuation regression of every date, in double
 * precision with FP64 Cholesky solves, one thread-block cluster per Bermudan.  terms_out (terms_len =
 * plan->terms_len) receives the plan's term table with the fitted policy and continuation records;
 * degrees[b] (<= 3) is the regression degree of Bermudan b, num_bermudans the plan's count (header[27]). */
zk_status zk_fit_amc(zk_context* ctx, const zk_plan_view* plan, const uint32_t* degrees, size_t num_bermudans, float* terms_out,
                     size_t terms_len);
/* The same fit in the FP64 mode, on the FP64 state pass (normals as in zk_run_plan_f64; nullable). */
zk_status zk_fit_amc_f64(zk_context* ctx, const zk_plan_view_f64* plan, const double* normals, size_t streams,
                         const uint32_t* degrees, size_t num_bermudans, double* terms_out, size_t terms_len);

/* FP64 mode.  `normals` (nullable) injects the standard normals instead of the counter-based
 * generator: normals[((j - 1) * nNormals + k) * streams + s] is normal k of step j on stream s; path p
 * reads stream p >> 1 with sign (-1)^(p & 1) when the plan is antithetic, else stream p.  `rows`
 * (nullable, rows_total * nP doubles) receives the per-path rows the fused kernel writes. */
zk_status zk_run_plan_f64(zk_context* ctx, const zk_plan_view_f64* plan, const double* normals, size_t streams,
                          zk_output_f64* out, double* rows);
/* FP32 with injected normals (converted to float), for the error of the FP32 path against FP64. */
zk_status zk_run_plan_injected(zk_context* ctx, const zk_plan_view* plan, const double* normals, size_t streams,
                               zk_output* out, float* rows);

/* The simulated risk factors of a plan in the FP64 mode (normals as in zk_run_plan_f64; nullable): out
 * [2 + nA][nT][nP] = the Hull-White state x, the deflator D and every asset level S_a on every date and path. */
zk_status zk_factor_paths_f64(zk_context* ctx, const zk_plan_view_f64* plan, const double* normals, size_t streams, double* out,
                              size_t out_len);

/* ---- nested exposure: the inner simulations (src/nested/nested_exposure.cpp:211-244 runs them on the CPU) ---- */
/* The inner paths of one reporting date t of a netting set, on the GPU: from the outer scenarios' states at t,
 * exact Hull-White and lognormal steps (FP64) to every later event date, coupons and terminal flows
 * discounted to t, the normals of the reference's CounterNormals.  model: the flat model of zk_compile;
 * periods [n_periods][6] (ts, te, tau, amount = +-notional, fixed rate, slot: the swap whose running coupon
 * the period uses, < 64); terminals [n_terminals][6] (asset, option, call, notional, strike, maturity);
 * x [n_scenarios], spot [n_scenarios][nA] and known [n_scenarios][n_slots] (the fixing of each slot's
 * coupon running at t, 0 where none) the outer states at t. */
typedef struct zk_nest zk_nest;
zk_status zk_nest_create(zk_context* ctx, const double* model, size_t model_len, const double* periods, size_t n_periods,
                         const double* terminals, size_t n_terminals, double t, const double* x, const double* spot,
                         const double* known, size_t n_slots, size_t n_scenarios, zk_nest** out);
/* One round of jobs: job k runs paths[k] inner paths of scenario[k] on the normal stream seed[k] (inner path q
 * from normal q x events x (nA + 2)); out receives the payoffs job after job (sum of paths values). */
zk_status zk_nest_run(zk_nest* nest, const uint64_t* scenario, const uint64_t* seed, const uint64_t* paths, size_t num_jobs,
                      double* out);
/* The zero-bond coefficients of the model's Hull-White curve: P(ts, te | x) = ratio exp(c - B x) for each pair
 * (ts, te) of ts_te [n][2]; out [n][3] = ratio, c, B (hull_white.cpp:27-31). */
zk_status zk_zero_bond_coefficients(const double* model, size_t model_len, const double* ts_te, size_t n, double* out);
/* The number of event dates after t (0: nothing is paid after t). */
zk_status zk_nest_events(const zk_nest* nest, uint64_t* events);
/* Returns the nest's device memory to its context, which reuses it for later nests and frees it with the
 * context: destroy every nest before its context. */
void zk_nest_destroy(zk_nest* nest);

/* ---- the adaptive nest's proxy (HermiteProxy, src/nested/adaptive_nested.cpp:145-277; host code) ---- */
/* Least squares of y on the Hermite products of the standardised features up to total degree `degree`
 * (lowered until every basis function has two training rows), ridge relative to the mean diagonal, HC0
 * sandwich covariance; the reference's arithmetic order, so its bits.  features [n_rows][dims] row-major,
 * y [n_rows]; rows [n_train] the training rows (HermiteProxy::fit).  Errors (fewer than two rows, more than
 * 2000 basis functions, singular equations) return ZK_ERR_INVALID_ARGUMENT with the message in err. */
typedef struct zk_hermite zk_hermite;
zk_status zk_hermite_fit(const double* features, size_t n_rows, size_t dims, const double* y, const uint64_t* rows, size_t n_train,
                         uint32_t degree, double ridge, zk_hermite** out, char* err, size_t err_len);
/* value[k] and variance[k] (>= 0) of feature row rows[k] of features [n_rows][dims] (HermiteProxy::predict),
 * row-parallel on the host; a row index >= n_rows or a dims other than the fit's is ZK_ERR_INVALID_ARGUMENT. */
zk_status zk_hermite_predict(const zk_hermite* proxy, const double* features, size_t n_rows, size_t dims, const uint64_t* rows,
                             size_t n, double* value, double* variance);
/* degree_and_basis[0] = the fitted degree, [1] = the number of basis functions. */
zk_status zk_hermite_info(const zk_hermite* proxy, uint64_t* degree_and_basis);
void zk_hermite_destroy(zk_hermite* proxy);
/* out[k] = erfc(x[k]) of the C library (the reference's normalCdf, include/ccr/core/math.hpp:15, is
 * 0.5 erfc(-x / sqrt 2)): the estimator's misclassification probabilities of all scenarios in one call. */
zk_status zk_erfc_array(const double* x, size_t n, double* out);

/* ---- without device allocation (no counterpart in the reference) ----------------------------------- */
/* For callers that cannot call cudaMalloc: a host that hands all device memory to its own pooling
 * allocator up front (a serving process, a framework's caching allocator), or a plug-in that runs
 * inside such a host.  Runs one plan like zk_run_plan (host buffers in and out) but allocates no device
 * memory and needs no context: every device buffer lives in one fixed array of
 * ZK_NOALLOC_SCRATCH_BYTES that the library reserves on each GPU where it is loaded and holds until the
 * process exits.  A plan that needs more scratch is rejected with ZK_ERR_INVALID_ARGUMENT (use
 * zk_run_plan).  `stream` may be NULL (the legacy default stream).  The first call on a device looks up
 * the array's device address; make that first call before any stream capture.  With CUDA's lazy module
 * loading (the default) that lookup is also what loads the library's kernels on the device and reserves
 * the array, so a host that hands all free device memory to its own pool must make its first call before
 * that (or load modules eagerly, CUDA_MODULE_LOADING=EAGER); otherwise the call fails with
 * ZK_ERR_OUT_OF_MEMORY.  The call makes `device` current while it runs and gives the caller's current
 * device back before it returns.  Every call reuses the same array, so calls that overlap on the GPU (on
 * other streams or from other threads) race: the caller must serialise them.  On failure the message is
 * copied to err (err_len bytes). */
#define ZK_NOALLOC_SCRATCH_BYTES (32u << 20)
zk_status zk_run_plan_noalloc(int device, void* stream, const zk_plan_view* plan, zk_output* out, char* err, size_t err_len);

/* ---- failure injection for tests (host side; no counterpart in the reference) ---------------------- */
/* ZK_INJECT_FAIL_LAUNCH: the value-th kernel launch of the context's eager calls from now on fails with
 * ZK_ERR_CUDA instead of launching (once; 0 clears it), leaving the launches before it in flight and the
 * context usable.  ZK_INJECT_ROW_ROUNDS: caps the row statistics' quantile search at value narrowing rounds
 * (16, the default, restores it); a quantile that needs more makes the call fail with ZK_ERR_CUDA. */
#define ZK_INJECT_FAIL_LAUNCH 1u
#define ZK_INJECT_ROW_ROUNDS 2u
zk_status zk_debug_inject(zk_context* ctx, uint32_t what, uint64_t value);
/* Host check of the basis lowering (no GPU): lowers the n plans as one group and evaluates both the lowered
 * group and the plans term by term in double along one path of factor values x[nT], S[nT][4], xf[nT][2].
 * out[0]: the largest difference relative to the netting set's gross basis sum; out[1]: basis columns over all
 * dates; out[2]: linear terms and options over all dates; out[3]: fixing slots; out[4]: coefficient chunks.
 * ZK_ERR_UNSUPPORTED (with the reason in err) when the plans do not lower. */
zk_status zk_debug_basis(const zk_plan_view* plans, size_t n, const double* x, const double* S, const double* xf,
                         double* out, char* err, size_t err_len);

/* ---- device-resident batches (inputs uploaded once; used to time the kernels alone) -------------- */
typedef struct zk_batch zk_batch;
typedef struct zk_batch_info {
  uint64_t num_plans, num_launch_groups, num_paths, num_dates, num_trades_hint;
  uint64_t num_terms;            /* term records over all plans and dates                         */
  uint64_t term_evaluations;     /* sum over plans and dates of the terms a path evaluates         */
  uint64_t exp_evaluations;      /* of which need an exponential                                  */
  uint64_t table_bytes;          /* bytes of plan tables on the device                            */
  uint64_t row_bytes;            /* bytes of per-path rows (PFE inputs) written per execute        */
  uint64_t kernels_per_execute;  /* kernel launches of one zk_batch_execute                         */
  uint64_t tile_paths;           /* paths per revalue CTA, chosen by the autotuner at creation     */
  uint64_t graph_replay;         /* 1 once executes replay a captured CUDA graph, 0 while eager    */
  uint64_t num_waves;            /* waves of netting sets within the row budget (1 per launch group without) */
  uint64_t num_basis_netting_sets; /* netting sets revalued by the tensor-core basis kernel (zk_context_set_basis) */
  uint64_t basis_columns;        /* basis functions a path evaluates over all dates, summed over the basis groups */
  uint64_t basis_terms;          /* the linear terms and options those columns stand for (all dates and groups)   */
  uint64_t basis_bytes;          /* bytes of the basis groups' tables (coefficient images, columns, options, ...) */
} zk_batch_info;

/* Uploads the plans.  The first zk_batch_execute autotunes the tile shape (paths per revalue CTA) on
 * them, a few timed runs, unless zk_batch_set_tile_paths pinned one. */
zk_status zk_batch_create(zk_context* ctx, const zk_plan_view* plans, size_t n, zk_batch** out);
/* After the tile shape is settled, the execute sequence is captured once in a CUDA graph and replayed (the
 * context's stream must be capturable; otherwise executes stay eager). */
zk_status zk_batch_execute(zk_batch* b);
/* Pins the tile shape: paths per revalue CTA, 128 x (1, 2 or 4) in single precision. */
zk_status zk_batch_set_tile_paths(zk_batch* b, uint64_t tile_paths);
/* Milliseconds of the last execute by kernel: [0] risk-factor simulation, [1] revalue / net /
 * collateralise / reduce per tile, [2] reduce of the partials, [3] row statistics, measured with CUDA
 * events on the context stream.  A batch that runs in waves counts its waves' reduce and row statistics in [1]. */
zk_status zk_batch_timings(const zk_batch* b, float* ms4);
zk_status zk_batch_read(zk_batch* b, zk_output* outs);
zk_status zk_batch_info_get(const zk_batch* b, zk_batch_info* info);
void zk_batch_destroy(zk_batch* b);

/* ---- the surrogate's tensor-core GEMM (no counterpart in the reference) --------------------------------- */
/* C[M][N] = A[M][K] B[N][K]^T (+ bias[N], SiLU if act == 1): bf16 operands (raw bit patterns), FP32 result,
 * on the fifth-generation tensor cores (tcgen05.mma, FP32 accumulation in TMEM).  M % 128 == 0, N % 16 == 0,
 * K % 16 == 0.  Host buffers; bias nullable. */
zk_status zk_gemm_bf16(zk_context* ctx, const uint16_t* A, const uint16_t* B, uint32_t M, uint32_t N, uint32_t K,
                       const float* bias, uint32_t act, float* C);

/* ---- the learned revaluation surrogate (no counterpart in the reference) -------------------------------- */
/* A 16 -> 128 -> 128 -> 128 -> 1 perceptron (SiLU), BF16 weights and activations, FP32 accumulation, trained
 * and evaluated on the tensor cores by this library's kernels.  Inputs x are [n][16] floats, targets and
 * predictions [n] floats, all host buffers; inputs and targets are standardised with the moments of the first
 * training (or gradient) set.  Parameters flatten as W1[128][16] b1[128] W2[128][128] b2 W3[128][128] b3
 * w4[128] b4 (ZK_SURROGATE_PARAMS floats); the scaling as mean[16], 1/sd[16], target mean, target sd. */
#define ZK_SURROGATE_PARAMS 35329u
typedef struct zk_surrogate zk_surrogate;
zk_status zk_surrogate_create(zk_context* ctx, uint32_t seed, zk_surrogate** out);
void zk_surrogate_destroy(zk_surrogate* s);
/* Adam over `epochs` passes in batches of `batch` rows (mean squared error in standardised units). */
zk_status zk_surrogate_train(zk_surrogate* s, const float* x, const float* y, size_t n, uint32_t epochs, uint32_t batch, float lr,
                             float weight_decay, float* loss_per_epoch);
zk_status zk_surrogate_predict(zk_surrogate* s, const float* x, size_t n, float* y);
/* Loss and gradient of the mean squared error over n rows (one batch, n <= 2^20) at the current parameters. */
zk_status zk_surrogate_gradients(zk_surrogate* s, const float* x, const float* y, size_t n, float* loss, float* grads);
/* Reads (get, scaling_get[34]) and / or replaces (set, scaling_set[34]) the FP32 parameters and the scaling. */
zk_status zk_surrogate_params(zk_surrogate* s, float* get, const float* set, float* scaling_get, const float* scaling_set);

/* A trade of a book the surrogate revalues: kind 0 interest-rate swap (sign +1 pay fixed, -1 receive; strike
 * = fixed rate), 1 FX forward (sign +1), 2 FX option (sign +1 call, -1 put); asset = FX factor (forward,
 * option); maturity in years; the surrogate predicts the value per unit notional. */
typedef struct zk_surrogate_trade {
  uint32_t netting_set, kind, asset;
  int32_t sign;
  float notional, strike, maturity, pad;
} zk_surrogate_trade;
/* Features of every (trade, reporting date, path): X[nTr][nR][nP][16] (the training inputs).  factors is
 * [2 + nA][nR][nP] on the reporting dates: the deflator, the Hull-White state x, then ln S of each FX factor;
 * resets[nTr][nR] is the reporting-date index of the reset of the swap period running on each date (-1: none),
 * periods[nTr][nR][2] that period's start and end; bonds (nullable) [nTr][nR][4] = (ln A, B) of the zero bond to
 * the trade's maturity and of the one to the end of its running period, P(t, T | x) = A exp(-B x): features 14
 * and 15 (zero without). */
zk_status zk_surrogate_features(zk_context* ctx, const float* factors, uint32_t nA, uint32_t nR, uint32_t nP, const float* times,
                                const zk_surrogate_trade* trades, uint32_t nTr, const int32_t* resets, const float* periods,
                                const float* bonds, float* X);
/* Revaluation of a book by the surrogate on the GPU: features, tensor-core inference and netting per netting
 * set, then exposure[num_netting_sets][nR][2] = (EE, EE*) on the nR dates given; netted_out (nullable,
 * [num_netting_sets][nR][paths_out]) receives the netted values of the first paths_out paths; ms[2] (nullable) the
 * device time of the revaluation and of the exposure reduction.  csa (nullable, [num_netting_sets][4] = hc, ho
 * (< 0: none), mta (< 0: no CSA), ia) applies each netting set's cash CSA on its netted values before the reduction,
 * the collateral called on the value at date call_index[j] (at most 31 dates before j; collateral.cpp:10-47):
 * pass every simulation date, margin-call dates included, and netted_out then holds V - collateral. */
zk_status zk_surrogate_book(zk_surrogate* s, const float* factors, uint32_t nA, uint32_t nR, uint32_t nP, const float* times,
                            const zk_surrogate_trade* trades, uint32_t nTr, const int32_t* resets, const float* periods,
                            const float* bonds, uint32_t num_netting_sets, const float* csa, const uint32_t* call_index,
                            double* exposure, float* netted_out, uint32_t paths_out, float* ms);

/* Measured rate of the special-function unit's ex2 (billions per second on the whole GPU), the ceiling
 * of the fused kernel's bond exponentials (a roofline denominator; not part of the reference). */
zk_status zk_peak_ex2(int device, double* giga_per_s);

/* ---- plan compiler (host, C++17) ------------------------------------------------------------------ */
/* Restates gpu::compile (src/gpu/fused_exposure.cpp:214-707) from the flat model / netting-set /
 * options arrays of zlatko_b200/spec.py, in double precision, without the reference's per-plan caps
 * on swaps.  zk_plan_view_of gives the single-precision tables (the reference's layout). */
typedef struct zk_plan zk_plan;
zk_status zk_compile(const double* model, size_t model_len, const double* netting_set, size_t ns_len,
                     const double* options, size_t options_len, zk_plan** out, char* err, size_t err_len);
zk_status zk_plan_view_of(const zk_plan* p, zk_plan_view* view);
zk_status zk_plan_view_f64_of(const zk_plan* p, zk_plan_view_f64* view);
/* Simulation dates (nT) and reporting-date indices (nR) of a compiled plan. */
zk_status zk_plan_dates(const zk_plan* p, double* times, size_t nT, uint64_t* reporting, size_t nR);
/* Number of simulation dates, reporting dates, stats per date, trades, bermudans, exercise rows. */
zk_status zk_plan_sizes(const zk_plan* p, uint64_t* sizes6);
void zk_plan_destroy(zk_plan* p);

#ifdef __cplusplus
}
#endif
#endif /* ZLATKO_B200_H */
