"""GPU parity on the workloads the benchmark measures, not only on the small set-ups.

- The swap portfolio at full size (20 two-schedule swaps, HW(0.03, 0.01), flat 2%, 10,000 paths on 60 monthly
  dates): the FP32 kernels against the restated FP32 kernels of the reference, and the FP64 mode against the
  restated FP64 ExposureEngine on identical normals (1e-9, per path).
- The correlated CSA book, all 100 netting sets in one zk_run_plans batch -- on the tensor-core basis kernel, and
  term by term (the large- and small-state launches, the cash-CSA variant, the side stream) -- against the
  restated FP32 kernels, netting set by netting set; and a
  few of its netting sets in the FP64 mode against the FP64 engine, every margin call decided the same way.
- The Bermudan book (10y swaptions, annual exercise, degree 3): the FP64 fit and revaluation against the FP64
  engine's Longstaff-Schwartz on identical normals, every exercise decision the same.
- The error of the FP32 path against the FP64 mode, output by output, below the Monte Carlo standard error.
"""
import numpy as np
import pytest

from oracle import restated
from test_gpu_parity import RTOL, check_sums, check_values, injected_normals
from zlatko_b200 import gpu, precision, workloads
from zlatko_b200 import spec as S
from zlatko_b200.summary import summarise, unilateral_cva

pytestmark = pytest.mark.gpu

BOOK_PATHS = 8192  # a margin call decided on the other side of the MTA rule moves a mean by MTA / paths


def _engine_profile_check(p, sums, vals, rows, e, csa):
    res = summarise(p, sums, vals)
    for k in ("ev", "ee", "ene", "pfe", "dee", "dene"):
        scale = max(np.abs(e.profile[k]).max(), 1e-12)
        assert np.abs(res[k] - e.profile[k]).max() <= 1e-9 * scale, k
    H, rep = p.header, e.reporting
    scale = np.abs(e.netted).max()
    assert np.abs(rows[H[21]:H[21] + len(rep)].T - e.netted[:, rep]).max() <= 1e-9 * scale
    if csa:  # every margin call decided as the engine decides it
        assert np.abs(rows[H[22]:H[22] + len(rep)].T - e.collateral[:, rep]).max() <= 1e-9 * scale
    return res


# ---------------------------------------------------------------- the swap portfolio, full size
def test_swap_portfolio_full_size_against_the_oracle(ctx):
    m, ns, o = workloads.swap_portfolio(10_000)
    p = gpu.compile(m, ns, o)
    assert p.num_paths == 10_000 and len(p.reporting) == 61
    sg, vg = ctx.run(p)
    sr, vr = restated.run_plan(p)
    check_sums(p, sg, sr)
    check_values(p, vg, vr)
    a, b = summarise(p, sg, vg), summarise(p, sr, vr)
    cp = m.credits[0]
    cva_g = unilateral_cva(a["times"], a["dee"], cp.pillars, cp.hazards, 0.4)
    cva_r = unilateral_cva(b["times"], b["dee"], cp.pillars, cp.hazards, 0.4)
    assert abs(cva_g - cva_r) <= RTOL * abs(cva_r)


def test_swap_portfolio_full_size_fp64_against_the_engine(ctx):
    m, ns, _ = workloads.swap_portfolio(10_000)
    p = gpu.compile(m, ns, S.Options(samples=1, pfe_quantile=0.975))
    z, streams = injected_normals(p, 21)
    sums, vals, rows = ctx.run_f64(p, z, streams, rows=True)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.975, z, streams, m.num_paths)
    res = _engine_profile_check(p, sums, vals, rows, e, False)
    cp = m.credits[0]
    cva = unilateral_cva(res["times"], res["dee"], cp.pillars, cp.hazards, 0.4)
    cva_e = unilateral_cva(res["times"], e.profile["dee"], cp.pillars, cp.hazards, 0.4)
    assert abs(cva - cva_e) <= 1e-9 * abs(cva_e)


# ---------------------------------------------------------------- the correlated CSA book
@pytest.fixture(scope="module")
def book():
    m, books, o, trades = workloads.correlated_csa_book(BOOK_PATHS, foreign_rates=False)
    plans = [gpu.compile(m, b, o) for b in books]
    return m, books, o, plans, [restated.run_plan(p) for p in plans]


@pytest.mark.parametrize("basis", [gpu.Context.BASIS_AUTO, gpu.Context.BASIS_OFF])
def test_correlated_book_in_one_batch_against_the_oracle(ctx, book, basis):
    """With the basis kernel (the default: the 100 netting sets as one tensor-core group) and term by term."""
    m, books, o, plans, oracle = book
    assert len(plans) == 100
    ctx.set_basis(basis)
    try:
        got = ctx.run_many(plans)
        b = ctx.batch(plans)
        try:
            info = b.info()
        finally:
            b.close()
    finally:
        ctx.set_basis(gpu.Context.BASIS_AUTO)
    assert info.num_launch_groups == 1  # one shared simulation for the 100 netting sets
    assert info.num_basis_netting_sets == (100 if basis == gpu.Context.BASIS_AUTO else 0)
    for i, (p, (sg, vg), (sr, vr)) in enumerate(zip(plans, got, oracle)):
        try:
            check_sums(p, sg, sr)
            check_values(p, vg, vr)
        except AssertionError as exc:
            raise AssertionError(f"netting set {i} ({len(books[i].trades)} trades): {exc}") from None


@pytest.mark.parametrize("which", ["largest", "median", "smallest"])
def test_correlated_book_fp64_against_the_engine(ctx, which):
    m, books, _, _ = workloads.correlated_csa_book(1024)
    order = sorted(range(len(books)), key=lambda i: len(books[i].trades))
    ns = books[{"largest": order[-1], "median": order[len(order) // 2], "smallest": order[0]}[which]]
    p = gpu.compile(m, ns, S.Options(samples=1, pfe_quantile=0.975))
    z, streams = injected_normals(p, 33)
    sums, vals, rows = ctx.run_f64(p, z, streams, rows=True)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.975, z, streams, m.num_paths)
    _engine_profile_check(p, sums, vals, rows, e, True)


# ---------------------------------------------------------------- the Bermudan book
def test_bermudan_book_fp64_decisions_match_the_engine(ctx):
    m, books, _ = workloads.bermudan_book(4000)
    for ns in books[:2]:
        p = gpu.compile(m, ns, S.Options(exercise_views=True, samples=1))
        z, streams = injected_normals(p, 9)
        f = ctx.fit_amc_f64(p, z, streams)
        sums, vals, rows = ctx.run_f64(f, z, streams, rows=True)
        e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, m.num_paths)
        ex = int(p.header[25])
        for b in range(len(ns.trades)):
            assert np.array_equal(rows[ex + b], e.exercise[b]), f"Bermudan {b}: exercise decisions differ"
        _engine_profile_check(f, sums, vals, rows, e, False)


# ---------------------------------------------------------------- reduced precision against FP64
def test_fp32_error_is_below_the_monte_carlo_error_on_the_book(ctx):
    m, books, o, _ = workloads.correlated_csa_book(8192)
    own = S.Credit(1e-6, 0.0, 0.0, 0.0, [1.0], [0.005], substeps=1)
    r = precision.compare(ctx, m, books, o, own)
    for key, v in r["outputs"].items():
        assert v["max_err_over_se"] < 1.0, (key, v)
        assert v["max_rel_err_without_mc_error"] <= 1e-4, (key, v)  # date 0: single-precision rounding only
