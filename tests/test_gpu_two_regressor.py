"""GPU parity of the two-regressor Longstaff-Schwartz basis (short rate and co-terminal swap rate; this library's
extension of the reference's one-regressor fit), through zk_fit_amc / zk_fit_amc_f64 and the fused kernel.

FP64 mode: on identical normals, the GPU's FP64 state pass, cluster fit (FP64 Gram sums, FP64 Cholesky) and
revaluation against the FP64 engine with the same basis (oracle/engine_oracle.c): every exercise decision identical,
path for path, and the exposure profile within 1e-9.

FP32 mode: the GPU fit on its own AMC pass against the oracle's plan-level fit (restated.fit_amc2) on the oracle's
pass, each plan then run by its own evaluator (the fused kernel; oracle/fused_oracle.c).  In a one-factor model the
co-terminal swap rate is a smooth function of the short rate, so the two regressors are nearly collinear and the
fitted coefficients themselves are ill-conditioned (large and cancelling); what the fit determines well is the
regression's prediction.  The test compares what the records are used for: the exercise decisions (a path whose
exercise value lies within rounding of the regression can go either way) and the exposure profile.
"""
import numpy as np
import pytest

from oracle import restated
from setups import bermudan, gpu_setup
from zlatko_b200 import gpu
from zlatko_b200 import spec as S

pytestmark = pytest.mark.gpu


def book(paths, csa=False):
    m, ns = gpu_setup(paths, csa)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0, 4.0), physical=True, degree=3, basis="rate_swap"))
    ns.trades.append(bermudan(exercise=(2.0, 3.0), physical=False, position=-0.5, degree=2, pay=True, basis="rate_swap"))
    ns.trades.append(bermudan(exercise=(1.0, 3.0), physical=True, degree=1, basis="rate_swap"))
    return m, ns


def normals(plan, seed):
    streams = (plan.num_paths + 1) // 2
    return np.random.default_rng(seed).standard_normal((plan.num_dates - 1) * int(plan.header[5]) * streams), streams


@pytest.mark.parametrize("csa", [False, True])
def test_fp64_two_regressor_decisions_match_the_engine(ctx, csa):
    m, ns = book(3000, csa)
    p = gpu.compile(m, ns, S.Options(exercise_views=True, samples=1))
    z, streams = normals(p, 7)
    f = ctx.fit_amc_f64(p, z, streams)
    sums, vals, rows = ctx.run_f64(f, z, streams, rows=True)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, m.num_paths)
    ex = int(p.header[25])
    for b in range(3):
        assert np.array_equal(rows[ex + b], e.exercise[b]), f"Bermudan {b}: exercise decisions differ"
    from zlatko_b200.summary import summarise

    res = summarise(f, sums, vals)
    for k in ("ev", "ee", "ene", "pfe", "dee", "dene"):
        scale = max(np.abs(e.profile[k]).max(), 1e-12)
        assert np.abs(res[k] - e.profile[k]).max() <= 1e-9 * scale, k


@pytest.mark.parametrize("paths", [6000, 70000])  # 70,000 paths: clusters of 8 CTAs per Bermudan
def test_fp32_two_regressor_fit_against_the_oracle_fit(ctx, paths):
    m, ns = book(paths)
    p = gpu.compile(m, ns, S.Options(exercise_views=True))
    g = ctx.fit_amc(p)
    o = restated.fit_amc2(p, p.amc_degrees)
    tg, to = np.asarray(g.terms).reshape(-1, 8), o.reshape(-1, 8)
    kind = to[:, 0].astype(np.int64) & 15
    fitted = (kind == 6) | (kind == 7) | (kind == 15)
    assert np.array_equal(tg[~fitted], to[~fitted])  # nothing but the regression records changes
    assert np.array_equal(tg[fitted][:, 0], to[fitted][:, 0])
    # The centers and scales are means and deviations: well conditioned.
    reg = (kind == 6) | (kind == 7)
    for col in (2, 3, 4, 5):
        a, b = tg[reg][:, col].astype(np.float64), to[reg][:, col].astype(np.float64)
        assert np.abs(a - b).max() <= 2e-3 * np.abs(b).max(), col
    po = gpu.Plan.from_arrays(p.header, p.indices, p.params, p.steps, o, p.requests, p.rows_total, p.num_outputs,
                              p.times, p.reporting)
    sums_g, _, rows_g = ctx.run(g, rows=True)
    sums_o, _, rows_o = restated.run_plan(po, rows=True)
    ex = int(p.header[25])
    mism = int((rows_g[ex:ex + 3] != rows_o[ex:ex + 3]).sum())
    assert mism <= 1e-2 * paths * 3, f"{mism} of {3 * paths} exercise decisions differ"
    nS = p.stats_per_date
    ee_g, ee_o = (np.asarray(s, np.float64).reshape(-1, nS)[:, 1] for s in (sums_g, sums_o))
    assert np.abs(ee_g - ee_o).max() <= 1e-2 * np.abs(ee_o).max()


def test_two_regressor_plan_runs_with_one_regressor_bermudans(ctx):
    """A book mixing both bases: each Bermudan's records are fitted with its own basis in one launch."""
    m, ns = gpu_setup(4000, False)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0), degree=3, basis="rate_swap"))
    ns.trades.append(bermudan(exercise=(2.0, 3.0), degree=2, pay=True))
    p = gpu.compile(m, ns, S.Options(exercise_views=True, samples=1))
    z, streams = normals(p, 9)
    f = ctx.fit_amc_f64(p, z, streams)
    _, _, rows = ctx.run_f64(f, z, streams, rows=True)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, m.num_paths)
    ex = int(p.header[25])
    for b in range(2):
        assert np.array_equal(rows[ex + b], e.exercise[b]), f"Bermudan {b}: exercise decisions differ"


def test_bermudan_book_with_the_two_regressor_basis_in_fp64(ctx):
    """Two netting sets (8 Bermudans, 10y annual, exercise 1y-9y) of the AMC book with the two-regressor basis at
    20,000 paths: every exercise decision equal to the FP64 engine's with the same basis."""
    from zlatko_b200 import workloads

    m, books, _ = workloads.bermudan_book(20_000, basis="rate_swap")
    for ns in books[:2]:
        p = gpu.compile(m, ns, S.Options(exercise_views=True, samples=1))
        z, streams = normals(p, 13)
        f = ctx.fit_amc_f64(p, z, streams)
        _, _, rows = ctx.run_f64(f, z, streams, rows=True)
        e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, m.num_paths)
        ex = int(p.header[25])
        for b in range(len(ns.trades)):
            assert np.array_equal(rows[ex + b], e.exercise[b]), f"Bermudan {b}: exercise decisions differ"
