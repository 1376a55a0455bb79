"""The tensor-core basis kernel (basisRevalueKernel) against the term-by-term kernel and the oracle.

Its parity with the restated FP32 kernels of the reference on the 100-netting-set book is
tests/test_gpu_workloads.py::test_correlated_book_in_one_batch_against_the_oracle; its FP32 error against the FP64
mode, output by output, is test_fp32_error_is_below_the_monte_carlo_error_on_the_book (both run it by default).
Here, against the term-by-term kernel (BASIS_OFF) on the same counter-based normals:

- the three-currency book at a ragged path count (not a multiple of 128 or 4): every statistic and every PFE at
  1e-3 of its scale (a margin call decided on the other side of the MTA rule on one path of 4,099 moves a small
  netting set's ENE by MTA / paths, 2e-4 of its scale; the parity test against the oracle on 2,048 paths is the
  tight one);
- per path: the exposure rows agree to single-precision rounding except on the paths whose margin call sits on
  the MTA boundary within that rounding (fewer than 1%), where the two kernels may decide differently;
- groups (at the same 1e-3): 130 netting sets run as two groups of 65; netting sets the kernel does not run (per-trade views, FX
  collateral) run term by term in the same call;
- a batch: the graph replay and waves of groups give the same bits as one eager execute.
"""
import numpy as np
import pytest

from test_gpu_parity import check_sums, check_values
from zlatko_b200 import gpu, workloads
from zlatko_b200 import spec as S

pytestmark = pytest.mark.gpu

RTOL_CSA = 1e-3  # a few margin calls decided on the other side of the MTA rule


def _both(ctx, plans, mode=gpu.Context.BASIS_AUTO):
    ctx.set_basis(mode)
    try:
        a = ctx.run_many(plans)
    finally:
        ctx.set_basis(gpu.Context.BASIS_OFF)
    try:
        b = ctx.run_many(plans)
    finally:
        ctx.set_basis(gpu.Context.BASIS_AUTO)
    return a, b


@pytest.fixture(scope="module")
def book3():
    m, books, o, _ = workloads.correlated_csa_book(4099, foreign_rates=True)
    return m, books, o, [gpu.compile(m, b, o) for b in books]


def test_three_currency_book_against_the_term_kernel(ctx, book3):
    m, books, o, plans = book3
    got, ref = _both(ctx, plans)
    for i, (p, (sg, vg), (sr, vr)) in enumerate(zip(plans, got, ref)):
        try:
            check_sums(p, sg, sr, RTOL_CSA)
            check_values(p, vg, vr, RTOL_CSA)
        except AssertionError as exc:
            raise AssertionError(f"netting set {i} ({len(books[i].trades)} trades): {exc}") from None


def test_exposure_rows_differ_only_at_margin_boundaries(ctx, book3):
    m, books, o, plans = book3
    order = sorted(range(len(books)), key=lambda i: len(books[i].trades))
    for i in (order[-1], order[len(order) // 2], order[0]):
        p = plans[i]
        ctx.set_basis(gpu.Context.BASIS_ALL)  # a group of one
        try:
            _, _, ra = ctx.run(p, rows=True)
        finally:
            ctx.set_basis(gpu.Context.BASIS_OFF)
        try:
            _, _, rb = ctx.run(p, rows=True)
        finally:
            ctx.set_basis(gpu.Context.BASIS_AUTO)
        H = p.header
        a = ra[H[28]:H[28] + len(p.reporting)].astype(np.float64)
        b = rb[H[28]:H[28] + len(p.reporting)].astype(np.float64)
        scale = np.abs(b).max()
        diff = np.abs(a - b)
        moved = (diff > 1e-4 * scale).any(axis=0)  # paths with a margin call decided differently somewhere
        assert moved.mean() < 0.01, (i, moved.mean())
        assert np.median(diff) <= 1e-6 * scale
        assert np.abs(a - b)[:, ~moved].max() <= 1e-4 * scale


@pytest.fixture(scope="module")
def book200():
    m, books, o, _ = workloads.correlated_csa_book(8192, netting_sets=200, num_trades=3000, foreign_rates=True)
    return m, books, o


def test_two_groups_and_the_rest_term_by_term(ctx, book200):
    """Statistics at 1e-3 (a PFE moves by a gap between order statistics when one path's margin call goes the other
    way: the per-path comparison above covers the rows the quantiles come from)."""
    m, books, o = book200
    plans = [gpu.compile(m, b, o) for b in books[:130]]  # two groups of 65
    # not on the basis kernel: per-trade views; collateral in an FX rate
    plans.append(gpu.compile(m, books[130], S.Options(pfe_quantile=0.975, trade_views=True)))
    fx = S.NettingSet(books[131].trades, S.Csa(1e5, 1e5, 1e4, 0.0, 10.0 / 250.0, kind=2, asset_index=0))
    plans.append(gpu.compile(m, fx, o))
    got, ref = _both(ctx, plans)
    for i, (p, (sg, vg), (sr, vr)) in enumerate(zip(plans, got, ref)):
        try:
            check_sums(p, sg, sr, RTOL_CSA)
        except AssertionError as exc:
            raise AssertionError(f"plan {i}: {exc}") from None
    b = ctx.batch(plans)
    try:
        info = b.info()
    finally:
        b.close()
    assert info.num_basis_netting_sets == 130


def test_batch_graph_and_waves_keep_the_bits(ctx, book200):
    m, books, o = book200
    plans = [gpu.compile(m, b, o) for b in books]  # two groups of 100
    b = ctx.batch(plans)
    try:
        b.execute()
        first = b.read()
        b.execute()  # the captured graph
        again = b.read()
        info = b.info()
    finally:
        b.close()
    assert info.num_basis_netting_sets == 200
    for (s1, v1), (s2, v2) in zip(first, again):
        assert np.array_equal(s1, s2) and np.array_equal(v1, v2)
    # rows and partials of ~6 MB per netting set: under a 100 MB budget each group is a wave (never split)
    ctx.set_row_budget(100 << 20)
    try:
        bw = ctx.batch(plans)
        try:
            bw.execute()
            w = bw.read()
            assert bw.info().num_waves == 2
        finally:
            bw.close()
    finally:
        ctx.set_row_budget(0)
    for (s1, v1), (s2, v2) in zip(first, w):
        assert np.array_equal(s1, s2) and np.array_equal(v1, v2)
