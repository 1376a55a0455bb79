"""GPU parity: the CUDA kernels (zk_run_plan and friends) against the oracle.

The oracle is the plain-C restatement of the reference's path (oracle/restated.py), which is pinned bit for bit
to the reference itself (tests/test_oracle_pins.py), plus the golden fixtures the reference computed
(tests/golden/).  Plans come from this package's compiler (pinned table-for-table to the reference's
gpu::compile by tests/test_compiler.py) or, where the reference fits something this package does not (the AMC
regression of a Bermudan), from the reference's own tables stored in a fixture.

Tolerances.  The FP32 kernels draw the same counter-based normals as the reference; the two differ only by the
rounding of single-precision transcendental functions (CUDA's against glibc's), so statistics agree to about
1e-6 of their scale; the tests allow 2e-4 of each statistic's scale (and 1e-3 for the few path-level view
statistics that sit on a histogram edge).  Quantiles are exact on both sides, so they differ only through the
exposure rows.  FP64 mode against the FP64 engine on identical normals: 1e-9 relative.
"""
import os

import numpy as np
import pytest

from oracle import restated
from setups import bermudan, gpu_model, gpu_netting_set, gpu_setup, swap_book
from zlatko_b200 import gpu
from zlatko_b200 import spec as S

pytestmark = pytest.mark.gpu

RTOL = 2e-4
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def check_sums(plan, sums_g, sums_r, rtol=RTOL):
    nS = plan.stats_per_date
    g = np.asarray(sums_g, np.float64).reshape(-1, nS)
    r = np.asarray(sums_r, np.float64).reshape(-1, nS)
    floor = 1e-6 * np.abs(r).max()  # statistics that are zero up to rounding noise (e.g. E[D max(V_i, 0)] of a short option)
    for k in range(nS):
        scale = max(np.abs(r[:, k]).max(), floor, 1e-30)
        err = np.abs(g[:, k] - r[:, k]).max()
        assert err <= rtol * scale, f"statistic {k}: error {err:.3e} vs scale {scale:.3e}"


def check_values(plan, vals_g, vals_r, rtol=RTOL):
    """Means are compared on the scale of all outputs of the same kind (like a statistic over its dates): a mean
    of products that nearly cancel (a trade's deflated value on one date) carries the rounding of its terms."""
    n = max(1, plan.num_outputs)
    g, r = np.asarray(vals_g[:n], np.float64), np.asarray(vals_r[:n], np.float64)
    reqs = plan.requests.reshape(-1, 8)
    op_scale = {}
    for q in reqs:
        if int(q[0]) in (1, 2, 3, 6, 8, 9):
            op_scale[int(q[0])] = max(op_scale.get(int(q[0]), 0.0), abs(r[int(q[7])]))
    for q in reqs:
        op, count, out = int(q[0]), int(q[3]), int(q[7])
        width = count if op == 4 else count + 2 if op == 5 else 1
        a, b = g[out:out + width], r[out:out + width]
        if op == 5:  # histogram: counts may move across a bin edge by a path or two
            assert abs(a[:count].sum() - b[:count].sum()) < 0.5
            assert np.abs(a[:count] - b[:count]).sum() <= max(4.0, 1e-3 * plan.num_paths)
            continue
        scale = max(np.abs(r).max() if op in (0, 7) else op_scale.get(op, np.abs(b).max()), 1e-12)
        assert np.abs(a - b).max() <= max(rtol, 1e-3 if op in (0, 4, 7) else rtol) * scale, (op, a, b)


def run_both(ctx, m, ns, o=None):
    p = gpu.compile(m, ns, o or S.Options())
    sg, vg = ctx.run(p)
    sr, vr = restated.run_plan(p)
    return p, (sg, vg), (sr, vr)


def fixture(name):
    f = np.load(os.path.join(GOLDEN, name + ".npz"))
    plan = gpu.Plan.from_arrays(f["header"], f["indices"], f["params"], f["steps"], f["terms"], f["requests"],
                                int(f["rows_total"]), int(f["num_outputs"]), f["times"], f["reporting"])
    return f, plan


def with_paths(plan: gpu.Plan, n: int) -> gpu.Plan:
    """The same plan on n paths (header[0]; header[15] is the reference's count of 64-path workgroups)."""
    h = plan.header.copy()
    h[0], h[15] = n, (n + 63) // 64
    return gpu.Plan.from_arrays(h, plan.indices, plan.params, plan.steps, plan.terms, plan.requests, plan.rows_total,
                                plan.num_outputs, plan.times, plan.reporting)


@pytest.mark.parametrize("csa", [False, True])
def test_fused_matches_oracle(ctx, csa):
    m, ns = gpu_setup(8000, csa)
    p, (sg, vg), (sr, vr) = run_both(ctx, m, ns)
    check_sums(p, sg, sr)
    check_values(p, vg, vr)
    # The summaries (EE, PFE, CVA inputs per reporting date) of both read-backs agree too.
    from zlatko_b200.summary import summarise

    a, b = summarise(p, sg, vg), summarise(p, sr, vr)
    for k in ("ee", "ene", "pfe", "dee", "dene", "mean_survival"):
        assert np.abs(a[k] - b[k]).max() <= RTOL * max(np.abs(b[k]).max(), 1e-12), k


def test_per_trade_and_margin_quantile(ctx):
    m, ns = gpu_setup(8000, False)
    p, (sg, vg), (sr, vr) = run_both(ctx, m, ns, S.Options(per_trade=True, im_quantile=0.99))
    assert p.stats_per_date == 24
    check_sums(p, sg, sr)
    check_values(p, vg, vr)


def test_path_views(ctx):
    m, ns = gpu_setup(8000, True)
    o = S.Options(samples=12, histogram_time=2.0, gross=True, collateral_bands=True, trade_views=True)
    p, (sg, vg), (sr, vr) = run_both(ctx, m, ns, o)
    check_sums(p, sg, sr)
    check_values(p, vg, vr)


def test_factor_views_probes(ctx):
    m, _ = gpu_setup(8000, False)
    o = S.Options(factor_views=True, samples=5, bond_maturity=8.0)
    p, (sg, vg), (sr, vr) = run_both(ctx, m, S.NettingSet([]), o)
    check_sums(p, sg, sr)
    check_values(p, vg, vr)


@pytest.mark.parametrize("kind", [1, 2])
def test_securities_collateral(ctx, kind):
    m, ns = gpu_setup(8000, True)
    ns.csa.kind, ns.csa.haircut, ns.csa.bond_maturity, ns.csa.mpr = kind, 0.02 if kind == 1 else 0.15, 10.0, 20.0 / 250.0
    p, (sg, vg), (sr, vr) = run_both(ctx, m, ns)
    check_sums(p, sg, sr)
    check_values(p, vg, vr)


def test_two_schedule_swap_book(ctx):
    m = gpu_model(6000, seed=3)
    m.base_grid = [k / 12 for k in range(1, 61)]
    p, (sg, vg), (sr, vr) = run_both(ctx, m, swap_book(25, seed=9, csa=S.Csa(1e5, 1e5, 1e4)), S.Options(pfe_quantile=0.975))
    check_sums(p, sg, sr)
    check_values(p, vg, vr)


@pytest.mark.parametrize("name", ["fused_plain", "fused_csa_views", "fused_bond_collateral", "fused_asset_collateral",
                                  "fused_bermudan", "fused_swap_book", "fused_nested_im"])
def test_golden_fixtures(ctx, name):
    """The reference's own tables run on the GPU reproduce the reference's own outputs.  These fixtures have a
    few hundred paths, so one margin call that CUDA's and glibc's single-precision exponentials decide
    differently on a path sitting at the minimum-transfer boundary moves a mean by MTA / paths (~4e-4 of EE
    with securities collateral); the collateralised and Bermudan fixtures allow 1e-3."""
    f, p = fixture(name)
    sg, vg = ctx.run(p)
    loose = name in ("fused_bermudan", "fused_bond_collateral", "fused_asset_collateral", "fused_nested_im")
    check_sums(p, sg, f["sums"], rtol=1e-3 if loose else RTOL)
    exact = f["values"].copy()
    for q in p.requests.reshape(-1, 8):  # quantiles: the exact ccr::quantile of the reference's rows
        if int(q[0]) in (0, 7):
            exact[int(q[7])] = f["exact_quantiles"][int(q[7])]
    check_values(p, vg, exact, rtol=1e-3 if loose else RTOL)


# ---------------------------------------------------------------- nested initial margin
IM_OPTIONS = [S.Options(im_quantile=0.99, im_inner_paths=64, samples=2),
              S.Options(per_trade=True, im_quantile=0.95, im_inner_paths=40),  # lanes 8..31 run one inner path
              S.Options(im_quantile=1.0, im_inner_paths=33)]                   # the largest sample: order statistic 0


def check_im_rows(p, rg, rr, tol):
    """The margin rows [nR][paths]: each path's margin is an order statistic of |V_inner - V| over its inner paths,
    a continuous function of the values, so it moves with their rounding (CUDA's against glibc's single-precision
    exponentials); an inner Bermudan exercise decided differently at its boundary moves one sample, so the bound
    on single paths is on 99.9% of them, the mean of every date holds on all."""
    im, nR = int(p.header[29]), p.num_reporting
    a, b = rg[im:im + nR].astype(np.float64), rr[im:im + nR].astype(np.float64)
    scale = np.abs(b).max()
    assert scale > 0 and np.isfinite(a).all()
    err = np.abs(a - b)
    assert np.quantile(err, 0.999) <= tol * scale, np.quantile(err, 0.999) / scale
    assert np.abs(a.mean(1) - b.mean(1)).max() <= tol * scale


@pytest.mark.parametrize("csa", [False, True])
@pytest.mark.parametrize("oi", range(len(IM_OPTIONS)))
def test_nested_initial_margin(ctx, csa, oi):
    m, ns = gpu_setup(1500, csa)
    p = gpu.compile(m, ns, IM_OPTIONS[oi])
    sg, vg, rg = ctx.run(p, rows=True)
    sr, vr, rr = restated.run_plan(p, rows=True)
    check_sums(p, sg, sr)
    check_values(p, vg, vr, rtol=1e-3 if csa else RTOL)
    check_im_rows(p, rg, rr, 1e-3 if csa else RTOL)


def test_nested_initial_margin_with_bermudans_and_1024_inner_paths(ctx):
    m, ns = gpu_setup(256, True)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0, 4.0), physical=True, degree=2))
    ns.trades.append(bermudan(exercise=(2.0, 3.0), physical=False, position=-0.5, degree=3))
    p = gpu.compile(m, ns, S.Options(im_quantile=0.99, im_inner_paths=1024), fit=ctx)
    sg, vg, rg = ctx.run(p, rows=True)
    sr, vr, rr = restated.run_plan(p, rows=True)
    check_sums(p, sg, sr, rtol=1e-3)
    check_im_rows(p, rg, rr, 1e-3)


def test_nested_initial_margin_audit_on_the_gpu(ctx):
    """gpu::summarise's audit of the margin (two more runs on the first paths, with the kernel's and with more
    inner paths) with the GPU as its backend, against the same audit on the oracle."""
    m, ns = gpu_setup(1200, True)
    p = gpu.compile(m, ns, S.Options(per_trade=True, im_quantile=0.99, im_inner_paths=64, im_audit_paths=256,
                                     im_audit_inner_paths=512))
    sg, vg = ctx.run(p)
    sr, vr = restated.run_plan(p)
    from zlatko_b200.summary import summarise

    a, b = ctx.summarise(p, sg, vg), summarise(p, sr, vr, run=restated.run_plan)
    assert np.any(b["conditional_im_audit_ratio"] != 1.0)
    assert np.abs(a["conditional_im_audit_ratio"] - b["conditional_im_audit_ratio"]).max() <= 1e-3
    for k in ("conditional_im_discounted", "conditional_im_mean", "conditional_im_discounted_uncorrected"):
        assert np.abs(a[k] - b[k]).max() <= 1e-3 * np.abs(b[k]).max(), k


def test_nested_initial_margin_in_a_batch_and_a_graph(ctx):
    """Batched with plans without the margin (one shared scenario), replayed from the captured graph: the same
    bits as the single run."""
    m, ns = gpu_setup(2000, True)
    p_im = gpu.compile(m, ns, S.Options(im_quantile=0.99, im_inner_paths=64))
    p_plain = gpu.compile(m, ns, S.Options())
    s1, v1 = ctx.run(p_im)
    b = ctx.batch([p_plain, p_im, p_plain])
    try:
        for _ in range(3):
            b.execute()
            out = b.read()
            assert np.array_equal(out[1][0], s1) and np.array_equal(out[1][1][: p_im.num_outputs], v1[: p_im.num_outputs])
    finally:
        b.close()


@pytest.mark.parametrize("physical", [True, False])
def test_bermudan_amc_terms(ctx, physical):
    """Bermudans priced by the reference-fitted policy and continuation terms: the same exercise decisions as the
    oracle on the same tables, on 4000 paths."""
    f, p = fixture("fused_bermudan")
    p = with_paths(p, 4000)
    if not physical:  # the same policy, settled in cash: drop the exercised-tail terms of the underlying
        t = p.terms.reshape(-1, 8).copy()
        kind = t[:, 0].astype(np.int64) & 15
        t[(kind == 8) | (kind == 9), 2] = 0.0
        t[(kind == 9), 5] = 0.0
        p = gpu.Plan.from_arrays(p.header, p.indices, p.params, p.steps, t.reshape(-1), p.requests, p.rows_total,
                                 p.num_outputs, p.times, p.reporting)
    sg, vg = ctx.run(p)
    sr, vr = restated.run_plan(p)
    check_sums(p, sg, sr, rtol=1e-3)
    check_values(p, vg, vr, rtol=1e-3)


def test_amc_state_pass_matches_oracle(ctx):
    f, p = fixture("fused_bermudan")
    p = with_paths(p, 2000)
    rows = int(restated.exercise_offsets(p.terms)[-1])
    xg, dg, eg = ctx.amc_states(p, rows)
    xr, dr, er = restated.amc_states(p)
    assert np.abs(xg - xr).max() <= 1e-5 * np.abs(xr).max()
    assert np.abs(dg - dr).max() <= 1e-5
    assert np.abs(eg - er).max() <= 2e-4 * np.abs(er).max()


def test_batch_equals_single_plans(ctx):
    """Netting sets sharing a scenario run in one launch; each result equals its own single-plan run."""
    m = gpu_model(3000)
    m.base_grid = [k / 12 for k in range(1, 61)]
    books = [swap_book(n, seed=s) for n, s in ((3, 1), (7, 2), (1, 3), (12, 4))]
    books[1].csa = S.Csa(1e5, 1e5, 1e4)
    plans = [gpu.compile(m, b, S.Options(pfe_quantile=0.975)) for b in books]
    many = ctx.run_many(plans)
    for p, (s, v) in zip(plans, many):
        s1, v1 = ctx.run(p)
        assert np.array_equal(s, s1) and np.array_equal(v, v1)


def test_results_do_not_depend_on_the_tile_shape(ctx):
    """Every tile shape the autotuner may pick gives the same bits (the partials are reduced in path order)."""
    m = gpu_model(5000)
    m.base_grid = [k / 12 for k in range(1, 61)]
    plans = [gpu.compile(m, swap_book(9, seed=s, csa=S.Csa(1e5, 1e5, 1e4) if s else None), S.Options()) for s in (0, 1)]
    out = []
    for tile in (128, 256, 512):
        b = ctx.batch(plans)
        try:
            b.set_tile_paths(tile)
            b.execute()
            out.append(b.read())
        finally:
            b.close()
    for r in out[1:]:
        for (s0, v0), (s1, v1) in zip(out[0], r):
            assert np.array_equal(s0, s1) and np.array_equal(v0, v1)


def test_large_and_small_state_netting_sets_share_a_batch(ctx):
    """A netting set with 30 running-coupon slots (more shared-memory state than the variant with more resident
    CTAs allows) and two small ones: with 2 or 4 paths per thread the batch revalues them in two launches, the
    small ones on the kernel compiled for more resident CTAs.  Every tile shape gives the same bits, and so does
    each plan run alone."""
    m = gpu_model(3000)
    m.base_grid = [k / 12 for k in range(1, 61)]
    csa = S.Csa(1e5, 1e5, 1e4)  # every plan on the same dates (margin-call dates included): one launch group
    books = [swap_book(3, seed=1, csa=csa), swap_book(30, seed=5, csa=csa), swap_book(9, seed=2, csa=csa)]
    plans = [gpu.compile(m, b, S.Options(pfe_quantile=0.975)) for b in books]
    out = []
    for tile in (128, 256, 512):
        b = ctx.batch(plans)
        try:
            b.set_tile_paths(tile)
            b.execute()
            out.append(b.read())
            if tile > 128:
                assert b.info().kernels_per_execute == 5  # simulate, two revalue launches, reduce, row statistics
        finally:
            b.close()
    for r in out[1:]:
        for (s0, v0), (s1, v1) in zip(out[0], r):
            assert np.array_equal(s0, s1) and np.array_equal(v0, v1)
    for p, (s, v) in zip(plans, out[1]):
        s1, v1 = ctx.run(p)
        assert np.array_equal(s, s1) and np.array_equal(v, v1)


def test_batch_replays_a_cuda_graph_with_the_same_bits(ctx):
    """After the tile shape settles, a batch's executes replay one captured CUDA graph: same results as the
    eager first execute and as single-plan runs."""
    m = gpu_model(3000)
    m.base_grid = [k / 12 for k in range(1, 61)]
    plans = [gpu.compile(m, swap_book(n, seed=s, csa=S.Csa(1e5, 1e5, 1e4)), S.Options()) for n, s in ((5, 1), (9, 2))]
    b = ctx.batch(plans)
    try:
        b.execute()  # autotunes, then captures
        first = b.read()
        assert b.info().graph_replay == 1
        for _ in range(3):
            b.execute()
        again = b.read()
        assert np.all(b.timings() > 0)
    finally:
        b.close()
    for (s0, v0), (s1, v1), p in zip(first, again, plans):
        s2, v2 = ctx.run(p)
        assert np.array_equal(s0, s1) and np.array_equal(v0, v1)
        assert np.array_equal(s0, s2) and np.array_equal(v0, v2)


def test_pfe_is_the_exact_interpolated_quantile(ctx):
    """The row-statistics kernel returns ccr::quantile of the rows the fused kernel wrote (exactly, up to
    the final rounding to float)."""
    m, ns = gpu_setup(5000, True)
    for level in (0.5, 0.95, 0.975, 0.99):
        p = gpu.compile(m, ns, S.Options(pfe_quantile=level))
        streams = (p.num_paths + 1) // 2
        z = np.random.default_rng(11).standard_normal((p.num_dates - 1) * int(p.header[5]) * streams)
        sums, vals, rows = ctx.run_injected(p, z, streams, rows=True)
        for k in range(p.num_reporting):
            # The plan carries the level in single precision (requests are f32), as the reference's kernel reads it.
            exact = restated.quantile(rows[int(p.header[28]) + k].astype(np.float64), float(np.float32(level)))
            assert vals[k] == np.float32(exact) or abs(vals[k] - exact) <= 1e-7 * max(abs(exact), 1.0)


@pytest.mark.parametrize("paths", [8192, 30001, 65536])
def test_exact_quantile_on_long_rows(ctx, paths):
    """Levels in the zero mass of the exposure rows, the median, the tails and both ends, on a row length read 16
    bytes per load (8,192), one that is not (30,001) and one long enough for the histogram's first range to come
    from a sample of the row (65,536): the exact interpolated quantile."""
    m, ns = gpu_setup(paths, True)
    for level in (0.0, 0.3, 0.5, 0.9, 0.975, 0.999, 1.0):
        p = gpu.compile(m, ns, S.Options(pfe_quantile=level))
        sums, vals, rows = ctx.run(p, rows=True)
        for k in range(p.num_reporting):
            exact = restated.quantile(rows[int(p.header[28]) + k].astype(np.float64), float(np.float32(level)))
            assert vals[k] == np.float32(exact) or abs(vals[k] - exact) <= 1e-7 * max(abs(exact), 1.0), (level, k)


def test_quantile_edge_cases(ctx):
    """Rows with ties, one distinct value and very few paths: still the exact interpolated quantile."""
    for paths in (1, 2, 3, 64, 65):
        m, _ = gpu_setup(paths, False)
        p = gpu.compile(m, S.NettingSet([]), S.Options(factor_views=True, samples=min(paths, 3), pfe_quantile=0.95))
        sg, vg = ctx.run(p)
        sr, vr = restated.run_plan(p)
        check_values(p, vg, vr)
        assert np.isfinite(vg[: max(1, p.num_outputs)]).all()


def test_invalid_plans_are_rejected(ctx):
    from zlatko_b200._native import ZkError

    m, ns = gpu_setup(500, False)
    p = gpu.compile(m, ns, S.Options())
    bad = gpu.Plan.from_arrays(p.header[:20], p.indices, p.params, p.steps, p.terms, p.requests, p.rows_total,
                               p.num_outputs, p.times, p.reporting)
    with pytest.raises(ZkError, match="INVALID_PLAN"):
        ctx.run(bad)
    t = p.terms.copy().reshape(-1, 8)
    t[0, 1] = 40.0  # a swap slot beyond 32 on a fixing term
    t[0, 0] = 3.0
    bad2 = gpu.Plan.from_arrays(p.header, p.indices, p.params, p.steps, t.reshape(-1), p.requests, p.rows_total,
                                p.num_outputs, p.times, p.reporting)
    with pytest.raises(ZkError, match="INVALID_PLAN"):
        ctx.run(bad2)
    pim = gpu.compile(m, ns, S.Options(im_quantile=0.99, im_inner_paths=64))
    h = pim.header.copy()
    h[30] = 2048  # nested initial margin: more inner paths than the reference's 1024
    with pytest.raises(ZkError, match="INVALID_PLAN"):
        ctx.run(gpu.Plan.from_arrays(h, pim.indices, pim.params, pim.steps, pim.terms, pim.requests, pim.rows_total,
                                     pim.num_outputs, pim.times, pim.reporting))
    idx = pim.indices.copy()
    nT = pim.num_dates
    rep = np.nonzero(idx[2 * nT + 1:3 * nT + 1])[0]
    idx[3 * nT + 1 + rep[1]] = rep[1]  # an initial-margin target on its own date
    with pytest.raises(ZkError, match="INVALID_PLAN"):
        ctx.run(gpu.Plan.from_arrays(pim.header, idx, pim.params, pim.steps, pim.terms, pim.requests, pim.rows_total,
                                     pim.num_outputs, pim.times, pim.reporting))
    # The context stays usable after errors.
    s, v = ctx.run(p)
    assert np.isfinite(s).all()


# ---------------------------------------------------------------- FP64 mode against the FP64 engine
def injected_normals(plan: gpu.Plan, seed: int):
    streams = (plan.num_paths + 1) // 2
    z = np.random.default_rng(seed).standard_normal((plan.num_dates - 1) * int(plan.header[5]) * streams)
    return z, streams


@pytest.mark.parametrize("csa", [False, True])
def test_fp64_matches_engine_on_identical_normals(ctx, csa):
    m, ns = gpu_setup(2000, csa)
    o = S.Options(samples=1, pfe_quantile=0.95)
    p = gpu.compile(m, ns, o)
    z, streams = injected_normals(p, 5)
    sums, vals, rows = ctx.run_f64(p, z, streams, rows=True)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, m.num_paths)
    assert np.array_equal(e.times, p.times)
    from zlatko_b200.summary import summarise

    res = summarise(p, sums, vals)
    for k in ("ev", "ee", "ene", "pfe", "dee", "dene"):
        scale = max(np.abs(e.profile[k]).max(), 1e-12)
        assert np.abs(res[k] - e.profile[k]).max() <= 1e-9 * scale, k
    # Per-path netted values, collateral and exposure on every reporting date.
    H = p.header
    rep = e.reporting
    scale = np.abs(e.netted).max()
    assert np.abs(rows[H[21]:H[21] + len(rep)].T - e.netted[:, rep]).max() <= 1e-9 * scale
    if csa:
        coll = rows[H[22]:H[22] + len(rep)].T
        assert np.abs(coll - e.collateral[:, rep]).max() <= 1e-9 * scale  # every margin call decided the same way
    # Pathwise CVA with the simulated survival.
    pcva = 0.6 * np.nansum(res["cva_inc"])
    assert abs(pcva - e.pathwise_cva_04) <= 1e-9 * abs(e.pathwise_cva_04)


@pytest.mark.parametrize("csa", [False, True])
def test_fp64_matches_golden_engine(ctx, csa):
    """The FP64 mode on the normals of a golden engine fixture reproduces the reference engine's profile."""
    f = np.load(os.path.join(GOLDEN, "engine_csa.npz" if csa else "engine_plain.npz"))
    m, ns = gpu_setup(256, csa)  # the set-up the fixture was made from
    assert np.array_equal(S.encode_model(m), f["model"]) and np.array_equal(S.encode_netting_set(ns), f["netting_set"])
    p = gpu.compile(m, ns, S.Options(samples=1))
    streams = int(f["streams"])
    z = np.random.default_rng(int(f["seed"])).standard_normal((p.num_dates - 1) * int(f["num_normals"]) * streams)
    sums, vals, rows = ctx.run_f64(p, z, streams, rows=True)
    from zlatko_b200.summary import summarise

    res = summarise(p, sums, vals)
    for i, k in enumerate(("ev", "ee", "ene", "pfe", "dee", "dene")):
        scale = max(np.abs(f["profile"][i]).max(), 1e-12)
        assert np.abs(res[k] - f["profile"][i]).max() <= 1e-9 * scale, k
    H, nR = p.header, len(f["reporting"])
    scale = np.abs(f["netted"]).max()
    assert np.abs(rows[H[21]:H[21] + nR].T - f["netted"]).max() <= 1e-9 * scale
    assert abs(0.6 * np.nansum(res["cva_inc"]) - float(f["pathwise_cva_04"])) <= 1e-9 * abs(float(f["pathwise_cva_04"]))


# ---------------------------------------------------------------- a book on common scenarios
def test_book_on_the_gpu_matches_the_oracle(ctx):
    """A book of four netting sets of two counterparties (zlatko_b200.book): one zk_run_plans call on the GPU, the
    combined profile, the xVA per netting set and the per-trade allocation against the same book on the oracle."""
    from test_book import OWN, small_book
    from zlatko_b200 import book as B

    m, nets, cps = small_book()
    m.num_paths = 4000
    plans = B.compile_book(m, nets, cps, S.Options(per_trade=True))
    g = B.run_book(plans, m, cps, OWN, ctx=ctx)
    r = B.run_book(plans, m, cps, OWN, run=restated.run_plan)
    for k in B.ADDITIVE:
        assert np.abs(g.total[k] - r.total[k]).max() <= RTOL * np.abs(r.total[k]).max(), k
    for k in ("cva", "dva", "fca", "fba", "kva"):
        assert abs(g.xva_total[k] - r.xva_total[k]) <= 1e-3 * abs(r.xva_total[k]), k
    for ag, ar in zip(g.allocation, r.allocation):
        scale = max(abs(t["cva"]) for t in ar)
        assert max(abs(a["cva"] - b["cva"]) for a, b in zip(ag, ar)) <= 1e-3 * scale
