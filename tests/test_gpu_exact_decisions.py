"""Exact decisions in single precision (zk_context_set_exact_decisions): every margin call and exercise decision of
the FP32 path taken as the FP64 mode takes it on the same counter-based normals.

The FP32 kernel flags each path with a decision inside the guard band (a bound on the single-precision rounding of
the rule's margin); those paths run again in FP64 and replace their rows and their share of the statistics.  The
reference for "the same decision" is the FP64 mode on the same plan tables (the single-precision tables widened to
double, so the only difference is the arithmetic): the margin-call rule |required - held| >= MTA
(src/exposure/collateral.cpp:42) and the exercise rule e > 0 and e > continuation
(src/instruments/bermudan_swaption.cpp:87).  Without the check a fraction of a percent of paths decides otherwise
(tests/test_gpu_decisions.py); with it, none.
"""
import dataclasses

import numpy as np
import pytest

from setups import gpu_setup
from zlatko_b200 import gpu, workloads
from zlatko_b200 import spec as S

pytestmark = pytest.mark.gpu

# The guard relative to the netting set's gross term value: 1e-7 already left no decision apart on these
# workloads; 3e-7 re-runs 0.2-9% of their paths in FP64.
GUARD = 3e-7


def widened(p):
    """The plan with FP64 tables equal to its FP32 tables."""
    t = {"params": p.params, "steps": p.steps, "terms": p.terms, "requests": p.requests}
    return dataclasses.replace(p, tables64={k: np.asarray(v, np.float64).copy() for k, v in t.items()})


@pytest.fixture
def exact(ctx):
    ctx.set_exact_decisions(GUARD)
    ctx.exact_stats()
    yield ctx
    ctx.set_exact_decisions(0.0)


def _csa_cases():
    m, ns = gpu_setup(8000, True)
    yield m, ns
    mb, books, _, _ = workloads.correlated_csa_book(8192)
    order = sorted(range(len(books)), key=lambda i: len(books[i].trades))
    for i in (order[len(order) // 2], order[-3], order[-1]):
        yield mb, books[i]


def test_margin_calls_are_the_fp64_calls(exact):
    ctx = exact
    flagged = checked = apart_without = 0
    for m, ns in _csa_cases():
        p = gpu.compile(m, ns, S.Options(samples=1, pfe_quantile=0.975))
        H, nR = p.header, p.num_reporting
        _, _, r64 = ctx.run_f64(widened(p), rows=True)
        s32, v32, r32 = ctx.run(p, rows=True)
        f, n = ctx.exact_stats()
        flagged, checked = flagged + f, checked + n
        c64 = r64[H[22]:H[22] + nR]
        # A call taken on one side only moves the collateral by about the MTA; equal calls leave rounding.
        apart = np.abs(r32[H[22]:H[22] + nR].astype(np.float64) - c64) > 0.1 * ns.csa.mta
        assert not apart.any(), f"{int(apart.any(axis=0).sum())} paths with a margin call FP64 does not make"
        # Without the check some paths call otherwise; the statistics stay the FP32 path's, with the re-run paths'
        # share in FP64.
        ctx.set_exact_decisions(0.0)
        s_off, _, r_off = ctx.run(p, rows=True)
        ctx.set_exact_decisions(GUARD)
        apart_without += int((np.abs(r_off[H[22]:H[22] + nR].astype(np.float64) - c64) > 0.1 * ns.csa.mta).any(axis=0).sum())
        g, o = s32.reshape(-1, p.stats_per_date).astype(np.float64), s_off.reshape(-1, p.stats_per_date).astype(np.float64)
        for k in range(p.stats_per_date):
            scale = max(np.abs(o[:, k]).max(), 1e-30)
            assert np.abs(g[:, k] - o[:, k]).max() <= 1e-3 * scale, k
    assert checked > 0 and 0 < flagged <= 0.1 * checked, (flagged, checked)
    assert apart_without > 0  # the check has something to do on these workloads


def test_exercise_decisions_are_the_fp64_decisions(exact):
    ctx = exact
    m, books, _ = workloads.bermudan_book(8000)
    for ns in books[:2]:
        p = gpu.compile(m, ns, S.Options(exercise_views=True))
        f = ctx.fit_amc_f64(p)
        p32 = gpu.Plan.from_arrays(p.header, p.indices, p.params, p.steps, f.tables64["terms"].astype(np.float32), p.requests,
                                   p.rows_total, p.num_outputs, p.times, p.reporting)
        _, _, r64 = ctx.run_f64(widened(p32), rows=True)
        _, _, r32 = ctx.run(p32, rows=True)
        ex = int(p.header[25])
        for b in range(len(ns.trades)):
            assert np.array_equal(r32[ex + b].astype(np.float64), r64[ex + b]), f"Bermudan {b}: exercise decisions differ"


def test_a_book_of_plans_is_checked_plan_by_plan(exact):
    """Several flagged plans in one zk_run_plans call: each plan's result equals its result alone."""
    ctx = exact
    mb, books, _, _ = workloads.correlated_csa_book(4096)
    order = sorted(range(len(books)), key=lambda i: len(books[i].trades))
    plans = [gpu.compile(mb, books[i], S.Options(pfe_quantile=0.975)) for i in order[-6:]]
    together = ctx.run_many(plans)
    f, n = ctx.exact_stats()
    assert f > 0 and n == sum(p.num_paths for p in plans)
    for p, (s, v) in zip(plans, together):
        s1, v1 = ctx.run(p)
        assert np.array_equal(s, s1) and np.array_equal(v, v1)
