"""Pins of the oracle (CPU only).  The plain-C restatement of the reference's path (oracle/restated.py) is checked

  1. against the known-answer tests of the reference's own test suite (tests/test_core.cpp:56-67,
     tests/test_exposure.cpp:14-73, tests/test_cva.cpp:12-42), restated here with their inputs and answers;
  2. against the golden fixtures under tests/golden/, which the reference computed (make_golden.py):
     bit for bit on the statistics, exactly on the quantiles;
  3. where the reference is built in this container (oracle/_ref/libccr_ref.so), against the reference itself on
     every option set of the compiler tests, the AMC state pass, the FP64 engine and its building blocks.

It also pins this package's plan compiler to the reference's tables stored in the fixtures, so the compiler is
checked on machines without the reference too.
"""
import math
import os

import numpy as np
import pytest

from oracle import ref, restated
from setups import bermudan, gpu_setup
from zlatko_b200 import gpu
from zlatko_b200 import spec as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FUSED = ["fused_plain", "fused_csa_views", "fused_bond_collateral", "fused_asset_collateral", "fused_bermudan",
         "fused_swap_book", "fused_nested_im"]
needs_ref = pytest.mark.skipif(not ref.available(), reason="the reference is not built in this container")


def _load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def _run(f, rows=False):
    return restated.run_fused(f["header"], f["indices"], f["params"], f["steps"], f["terms"], f["requests"],
                              int(f["rows_total"]), int(f["num_outputs"]), rows)


def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


# ------------------------------------------------------------------ 1. the reference's known-answer tests
def test_quantile_known_answers():
    # tests/test_core.cpp:63-64
    assert restated.quantile([1, 2, 3, 4, 5], 0.5) == 3.0
    assert abs(restated.quantile([1, 2, 3, 4, 5], 0.9) - 4.6) <= 1e-12
    # order does not matter; one sample; the ends
    assert restated.quantile([5, 1, 4, 2, 3], 0.9) == restated.quantile([1, 2, 3, 4, 5], 0.9)
    assert restated.quantile([7.0], 0.99) == 7.0
    assert restated.quantile([1, 2, 3], 0.0) == 1.0 and restated.quantile([1, 2, 3], 1.0) == 3.0


def test_profile_known_answers():
    # tests/test_exposure.cpp:14-40: two paths, three dates.
    v = np.array([[2.0, 4.0, -3.0], [-1.0, 1.0, 6.0]])
    p = restated.profile(v, np.ones_like(v), [0.0, 0.5, 1.0], 1.0, 1.0)
    assert list(p["ee"]) == [1.0, 2.5, 3.0]
    assert p["ene"][0] == -0.5 and p["ene"][2] == -1.5
    assert p["pfe"][1] == 4.0 and p["max_pfe"] == 6.0
    assert abs(p["epe"] - 2.75) <= 1e-15
    w = np.array([[1.0, 3.0, 2.0]])
    p2 = restated.profile(w, np.ones_like(w), [0.0, 0.5, 1.0], 0.95, 1.0)
    assert abs(p2["eepe"] - 3.0) <= 1e-15 and p2["eepe"] >= p2["epe"]


def test_collateral_known_answers():
    # tests/test_exposure.cpp:42-73: thresholds 2 / 4, MTA 1, no lag; then a lag of one date; then one-way with IA.
    t = [0.0, 0.1, 0.2, 0.3]
    v = np.array([[5.0, 12.0, 12.5, -20.0]])
    c = restated.collateral(v, t, 2.0, 4.0, 1.0, 0.0, 0.0)
    assert list(c[0]) == [3.0, 10.0, 10.0, -16.0]
    lagged = restated.collateral(v, t, 2.0, 4.0, 0.0, 0.0, 0.1)
    assert np.allclose(lagged[0, 1:], [3.0, 10.0, 10.5], rtol=0, atol=1e-12)
    one_way = restated.collateral(v, t, 0.0, -1.0, 0.0, 1.5, 0.0)
    assert one_way[0, 3] == 1.5 and one_way[0, 1] == 13.5
    with pytest.raises(ValueError):
        restated.collateral(v, t, -1.0, 4.0, 0.0, 0.0, 0.0)


def test_cva_known_answers():
    # tests/test_cva.cpp:12-23: constant discounted EE of 100 on a quarterly grid to 5y.
    times = [0.25 * i for i in range(21)]
    ee = [100.0] * 21
    surv5 = math.exp(-(0.01 * 2.0 + 0.03 * 3.0))
    assert abs(restated.unilateral_cva(times, ee, [2.0, 5.0], [0.01, 0.03], 0.4) - 0.6 * 100.0 * (1.0 - surv5)) <= 1e-10
    # tests/test_cva.cpp:25-42: bilateral limits.
    t = [0.5 * i for i in range(11)]
    dee, dene = [50.0] * 11, [-30.0] * 11
    cva, dva = restated.bilateral_cva(t, dee, dene, ([1.0], [0.02]), ([1.0], [0.0]), 0.4, 0.4)
    assert abs(cva - restated.unilateral_cva(t, dee, [1.0], [0.02], 0.4)) <= 1e-12 and dva == 0.0
    cva2, dva2 = restated.bilateral_cva(t, dee, dene, ([1.0], [0.02]), ([1.0], [0.01]), 0.4, 0.4)
    assert cva2 < cva and dva2 > 0.0


# ------------------------------------------------------------------ 2. the golden fixtures
@pytest.mark.parametrize("name", FUSED)
def test_restatement_reproduces_golden_fused(name):
    f = _load(name)
    sums, values = _run(f)
    assert np.array_equal(_bits(sums), _bits(f["sums"])), "statistics differ from the reference's bits"
    for q in f["requests"].reshape(-1, 8):
        op, count, out = int(q[0]), int(q[3]), int(q[7])
        if op in (0, 7):  # exact quantile of the same rows
            assert _bits(values[out]) == _bits(f["exact_quantiles"][out]), (name, op)
        else:
            width = count if op == 4 else count + 2 if op == 5 else 1
            assert np.array_equal(_bits(values[out:out + width]), _bits(f["values"][out:out + width])), (name, op)


@pytest.mark.parametrize("name", ["engine_plain", "engine_csa"])
def test_restatement_reproduces_golden_engine(name):
    f = _load(name)
    nP = int(f["num_paths"])
    z = np.random.default_rng(int(f["seed"])).standard_normal((len(f["times"]) - 1) * int(f["num_normals"]) * int(f["streams"]))
    e = restated.engine_run(f["model"], f["netting_set"], 0.95, z, int(f["streams"]), nP)
    assert np.array_equal(e.times, f["times"]) and np.array_equal(e.reporting, f["reporting"])
    for i, k in enumerate(("ev", "ee", "ene", "pfe", "dee", "dene")):
        assert np.abs(e.profile[k] - f["profile"][i]).max() <= 1e-12 * max(np.abs(f["profile"][i]).max(), 1e-300), k
    scale = np.abs(f["netted"]).max()
    assert np.abs(e.netted[:, e.reporting] - f["netted"]).max() <= 1e-12 * scale
    assert np.abs(e.collateral[:, e.reporting] - f["collateral"]).max() <= 1e-12 * scale
    assert abs(e.pathwise_cva_04 - float(f["pathwise_cva_04"])) <= 1e-12 * abs(float(f["pathwise_cva_04"]))


@pytest.mark.parametrize("name", [n for n in FUSED if n != "fused_swap_book"])
def test_compiler_reproduces_golden_tables(name):
    """zk_compile on the fixture's flat arrays gives the reference's tables (AMC policy coefficients aside: the
    reference fits them by regression at compile time)."""
    f = _load(name)
    p = gpu.compile_arrays(f["model"], f["netting_set"], f["options"])
    for k in ("header", "indices", "params", "steps", "requests"):
        assert np.array_equal(getattr(p, k), f[k]), k
    rt, pt = f["terms"].reshape(-1, 8), p.terms.reshape(-1, 8)
    kind = rt[:, 0].astype(np.int64) & 15
    fitted = (kind == 6) | (kind == 7)
    assert np.array_equal(rt[~fitted], pt[~fitted]) and np.array_equal(rt[fitted][:, :2], pt[fitted][:, :2])
    assert np.array_equal(p.times, f["times"]) and np.array_equal(p.reporting, f["reporting"])


def test_two_schedule_swaps_match_the_reference_decomposition():
    """The swap book compiles natively (one floating leg per two-schedule swap); the reference's fixture holds
    the three-swap decomposition.  Same scenario, same statistics up to single-precision rounding, which the
    decomposition's cancelling legs (notionals up to 1e7 against net values near 1e5) magnify to ~2e-4."""
    f = _load("fused_swap_book")
    p = gpu.compile_arrays(f["model"], f["netting_set"], f["options"])
    assert p.terms.size < f["terms"].size
    sums, values = restated.run_plan(p)
    a, b = sums.reshape(-1, 8).astype(np.float64), f["sums"].reshape(-1, 8).astype(np.float64)
    for k in range(8):
        scale = max(np.abs(b[:, k]).max(), 1e-6 * np.abs(b).max(), 1e-30)
        assert np.abs(a[:, k] - b[:, k]).max() <= 1e-3 * scale, k


def test_a_planted_mistake_is_caught():
    """The pins are sensitive: one wrong coefficient in one term (a bond's notional off by one ulp) changes the
    statistics' bits, and a wrong margin threshold changes them by much more."""
    f = dict(_load("fused_csa_views"))
    terms = f["terms"].copy().reshape(-1, 8)
    k = int(np.nonzero((terms[:, 0].astype(np.int64) & 15) == 0)[0][0])
    terms[k, 2] = np.nextafter(terms[k, 2], np.float32(np.inf))
    sums, _ = restated.run_fused(f["header"], f["indices"], f["params"], f["steps"], terms.reshape(-1), f["requests"],
                                 int(f["rows_total"]), int(f["num_outputs"]))
    assert not np.array_equal(_bits(sums), _bits(f["sums"]))
    params = f["params"].copy()
    params[8] *= 2.0  # counterparty threshold
    sums2, _ = restated.run_fused(f["header"], f["indices"], params, f["steps"], f["terms"], f["requests"],
                                  int(f["rows_total"]), int(f["num_outputs"]))
    assert np.abs(sums2 - f["sums"]).max() > 1e-3 * np.abs(f["sums"]).max()


def test_workgroup_order_matters_only_through_rounding():
    """Statistics reduce per 64-path workgroup, then across workgroups with compensation: a permutation of the
    paths would change the bits, so the path order is part of the contract (the GPU keeps it)."""
    f = _load("fused_plain")
    s1, _ = _run(f)
    s2, _ = _run(f)
    assert np.array_equal(_bits(s1), _bits(s2))


# ------------------------------------------------------------------ 3. the reference itself
OPTIONS = [S.Options(), S.Options(per_trade=True, im_quantile=0.99),
           S.Options(samples=12, histogram_time=2.0, gross=True, collateral_bands=True, trade_views=True),
           S.Options(factor_views=True, samples=5, bond_maturity=8.0), S.Options(pfe_quantile=0.975),
           S.Options(im_quantile=0.99, im_inner_paths=64, samples=2),
           S.Options(per_trade=True, im_quantile=0.95, im_inner_paths=40)]


@needs_ref
@pytest.mark.parametrize("csa", [False, True])
@pytest.mark.parametrize("oi", range(len(OPTIONS)))
def test_restatement_is_bitwise_the_reference(csa, oi):
    m, ns = gpu_setup(700, csa)  # 700: a last workgroup of 60 paths
    r = ref.compile_plan(S.encode_model(m), S.encode_netting_set(ns), S.encode_options(OPTIONS[oi]))
    s1, v1 = ref.run_fused(r)
    rows_r = ref.run_rows(r)
    s2, v2, rows_o = restated.run_fused(r.header, r.indices, r.params, r.steps, r.terms, r.requests, r.rows_total,
                                        r.num_outputs, rows=True)
    assert np.array_equal(_bits(s1), _bits(s2))
    assert np.array_equal(_bits(rows_r), _bits(rows_o))
    for q in r.requests.reshape(-1, 8):
        op, row, count, out = int(q[0]), int(q[1]), int(q[3]), int(q[7])
        if op in (0, 7):
            x = rows_r[row].astype(np.float64)
            exact = ref.quantile(np.maximum(x, 0.0) if op == 7 else x, float(q[4]))
            assert _bits(v2[out]) == _bits(np.float32(exact))
            assert abs(float(v1[out]) - exact) <= 1e-6 * max(np.abs(x).max(), 1e-30)  # the reference kernel's approximation
        else:
            width = count if op == 4 else count + 2 if op == 5 else 1
            assert np.array_equal(_bits(v1[out:out + width]), _bits(v2[out:out + width]))


SUMMARY_OPTIONS = [S.Options(), S.Options(per_trade=True, im_quantile=0.99),
                   S.Options(per_trade=True, im_quantile=0.99, im_inner_paths=64, im_audit_paths=64, im_audit_inner_paths=256),
                   S.Options(im_quantile=0.975, im_inner_paths=128, samples=2)]


@needs_ref
@pytest.mark.parametrize("csa", [False, True])
@pytest.mark.parametrize("oi", range(len(SUMMARY_OPTIONS)))
def test_summarise_is_the_reference_summarise(csa, oi):
    """summary.summarise on the reference's own read-back gives gpu::summarise's FusedResult bit for bit: the
    profile, the CVA inputs, the per-trade statistics, the margin proxy, the nested margin's views and its
    audit (run on the restated kernels, which are the reference's bits)."""
    from zlatko_b200.summary import summarise

    m, ns = gpu_setup(300, csa)
    o = SUMMARY_OPTIONS[oi]
    r = ref.compile_plan(S.encode_model(m), S.encode_netting_set(ns), S.encode_options(o))
    p = gpu.compile(m, ns, o)
    sums, values = ref.run_fused(r)
    want, views = ref.summarise(r, sums, values), ref.summarise_views(r, sums, values)
    got = summarise(p, sums, values, run=restated.run_plan)
    same = lambda a, b: np.array_equal(np.asarray(a, np.float64), np.asarray(b, np.float64), equal_nan=True)  # noqa: E731
    for k in ("ev", "ee", "ene", "pfe", "dee", "dene", "cva_inc", "mean_survival", "mean_deflator"):
        assert same(got[k], want[k]), k
    assert same(got["conditional_discounted_ee"], views["conditional_discounted_ee"])
    nR = len(p.reporting)
    absent = np.full(nR, np.nan)
    assert same(got.get("value_change_quantile", absent), views["value_change_quantile"])
    assert same(got.get("conditional_im_discounted", absent), views["conditional_im_discounted"])
    assert same(got.get("conditional_im_mean", absent), views["conditional_im_mean"])
    for b, name in enumerate(("conditional_im_band_05", "conditional_im_band_50", "conditional_im_band_95")):
        assert same(got["conditional_im_bands"][b] if "conditional_im_bands" in got else absent, views[name]), name
    for k in ("conditional_im_audit_ratio", "conditional_im_discounted_uncorrected"):
        assert same(got.get(k, absent), views[k]), k
    if o.im_audit_paths:
        assert np.any(got["conditional_im_audit_ratio"] != 1.0)
    assert len(got["trades"]) == len(views["trades"])
    for a, b in zip(got["trades"], views["trades"]):
        for k in b:
            assert same(a[k], b[k]), k


VIEW_OPTIONS = [S.Options(samples=12, histogram_time=2.0, gross=True, collateral_bands=True, trade_views=True,
                          pfe_quantile=0.975, per_trade=True, im_quantile=0.99),
                S.Options(factor_views=True, samples=5, bond_maturity=8.0, histogram_time=0.0, histogram_bins=7),
                S.Options(factor_views=True, band_levels=(0.1, 0.9), factor_band_levels=(0.5,), gross=True, histogram_time=30.0),
                S.Options(exercise_views=True, samples=4, trade_views=True, im_quantile=0.99, im_inner_paths=64)]


def _same_tree(got, want, path="result"):
    """Every array of the reference's FusedResult bit for bit (NaN included); an absent key stands for the
    reference's empty series."""
    if isinstance(want, dict):
        for k, w in want.items():
            _same_tree(got.get(k) if got is not None else None, w, f"{path}.{k}")
    elif isinstance(want, list):
        got = [] if got is None else got
        assert len(got) == len(want), (path, len(got), len(want))
        for i, (a, b) in enumerate(zip(got, want)):
            _same_tree(a, b, f"{path}[{i}]")
    elif want is None:
        assert got is None, path
    else:
        w = np.asarray(want, np.float64)
        g = np.zeros(0) if got is None else np.asarray(got, np.float64)
        if w.size == 0 and g.size == 0:
            return
        assert g.shape == w.shape, (path, g.shape, w.shape)
        assert np.array_equal(g, w, equal_nan=True), (path, np.abs(g - w).max())


@needs_ref
@pytest.mark.parametrize("oi", range(len(VIEW_OPTIONS)))
def test_summarise_views_are_the_reference_views(oi):
    """Every view of gpu::summarise's FusedResult (samples, bands, gross profile, histogram, per-trade views,
    exercise distributions, factor views, the margin series) from summary.summarise on the reference's
    read-back, bit for bit."""
    from zlatko_b200.summary import summarise

    m, ns = gpu_setup(320, oi != 1)
    if oi == 3:
        ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0, 4.0), physical=True, degree=2))
        ns.trades.append(bermudan(exercise=(2.0, 3.0), physical=False, position=-0.5, degree=3))
    o = VIEW_OPTIONS[oi]
    r = ref.compile_plan(S.encode_model(m), S.encode_netting_set(ns), S.encode_options(o))
    p = gpu.compile(m, ns, o)
    sums, values = ref.run_fused(r)
    want = ref.summarise_full(r, sums, values)
    got = summarise(p, sums, values, run=restated.run_plan)
    ms = want.pop("market_survival")  # the plan's curve: the reference's compile against this package's
    assert np.abs(got.pop("market_survival") - ms).max() <= 1e-15
    if o.trade_views or o.exercise_views or o.factor_views or o.gross or o.samples:
        assert any(want.get(k) for k in ("trade_views", "exercise", "exposure_samples")) or want["factors"] or want["gross_profile"]
    _same_tree(got, want)


@needs_ref
def test_amc_states_are_bitwise_the_reference():
    m, ns = gpu_setup(900, False)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0), degree=3))
    ns.trades.append(bermudan(exercise=(2.0, 3.0), degree=2, physical=False))
    r = ref.compile_plan(S.encode_model(m), S.encode_netting_set(ns), S.encode_options(S.Options()))
    p = gpu.Plan.from_arrays(r.header, r.indices, r.params, r.steps, r.terms, r.requests, r.rows_total, r.num_outputs,
                             r.times, r.reporting.astype(np.int64))
    for a, b in zip(ref.amc_states(r), restated.amc_states(p)):
        assert np.array_equal(_bits(a), _bits(b))


@needs_ref
@pytest.mark.parametrize("csa", [False, True])
def test_engine_is_the_reference_engine(csa):
    m, ns = gpu_setup(600, csa)
    if csa:
        ns.csa.mpr = 20.0 / 250.0
    p = gpu.compile(m, ns, S.Options())
    streams = (m.num_paths + 1) // 2
    z = np.random.default_rng(3).standard_normal((p.num_dates - 1) * int(p.header[5]) * streams)
    e1 = ref.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.9, z, streams)
    e2 = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.9, z, streams, m.num_paths)
    assert np.array_equal(e1.times, e2.times) and np.array_equal(e1.reporting, e2.reporting)
    for k in e1.profile:
        assert np.abs(e1.profile[k] - e2.profile[k]).max() <= 1e-12 * max(np.abs(e1.profile[k]).max(), 1e-300), k
    for a, b in ((e1.netted, e2.netted), (e1.collateral, e2.collateral), (e1.deflator, e2.deflator),
                 (e1.survival[0], e2.survival)):
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(a).max(), 1e-300)
    assert abs(e1.pathwise_cva_04 - e2.pathwise_cva_04) <= 1e-12 * abs(e1.pathwise_cva_04)


@needs_ref
def test_building_blocks_are_the_reference():
    rng = np.random.default_rng(8)
    v = rng.normal(size=(333, 17)) * 100
    d = np.exp(-rng.uniform(0, 0.1, size=v.shape))
    t = np.sort(rng.uniform(0, 5, 17))
    t[0] = 0.0
    for q in (0.0, 0.5, 0.95, 1.0):
        assert restated.quantile(v[:, 3], q) == ref.quantile(v[:, 3], q)
    a, b = restated.profile(v, d, t, 0.975, 2.0), ref.profile(v, d, t, 0.975, 2.0)
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    price = np.exp(rng.normal(size=v.shape) * 0.1)
    for kind, up in ((0, None), (1, price), (2, price)):
        c1 = restated.collateral(v, t, 5.0, 7.0, 2.0, 1.0, 0.3, kind, 0.1, up)
        c2 = ref.collateral(v, t, 5.0, 7.0, 2.0, 1.0, 0.3, kind, 0.1, up)
        assert np.array_equal(c1, c2), kind
    pil, haz = [1.0, 3.0, 7.0], [0.01, 0.02, 0.05]
    assert restated.unilateral_cva(t, np.abs(v[0]), pil, haz, 0.4) == ref.unilateral_cva(t, np.abs(v[0]), pil, haz, 0.4)
    assert restated.bilateral_cva(t, np.abs(v[0]), -np.abs(v[1]), (pil, haz), ([2.0], [0.01]), 0.4, 0.3) == \
        ref.bilateral_cva(t, np.abs(v[0]), -np.abs(v[1]), (pil, haz), ([2.0], [0.01]), 0.4, 0.3)


# ------------------------------------------------------------------ the Longstaff-Schwartz fit
def test_fit_restatement_reproduces_golden_bermudan_terms():
    """fitAmc restated (oracle/amc_oracle.c) on the fixture's tables with the fitted records cleared gives back the
    reference's fitted records bit for bit (degrees 2 and 3, the fixture's Bermudans)."""
    f = _load("fused_bermudan")
    terms = f["terms"].reshape(-1, 8).copy()
    kind = terms[:, 0].astype(np.int64) & 15
    fitted = (kind == 6) | (kind == 7)
    terms[fitted, 2:] = 0.0
    p = gpu.Plan.from_arrays(f["header"], f["indices"], f["params"], f["steps"], terms.reshape(-1), f["requests"],
                             int(f["rows_total"]), int(f["num_outputs"]), f["times"], f["reporting"])
    out = restated.fit_amc(p, [2, 3])
    assert np.array_equal(_bits(out), _bits(f["terms"]))


def test_regression_known_answers():
    """PolynomialRegression (tests/test_core.cpp:37-54 of the reference): a cubic on 50 points is recovered
    (prediction at 0.7 within 1e-8), and a degenerate regressor falls back to the sample mean."""
    x = np.array([-2.0 + 0.08 * i for i in range(50)])
    y = 1.0 - 2.0 * x + 0.5 * x ** 3
    t = restated.fit_regression(x, y, 3)
    assert t["ncoef"] == 4
    z = (0.7 - t["center"]) / t["scale"]
    pred = sum(c * z ** d for d, c in enumerate(t["coef"]))
    assert abs(pred - (1.0 - 1.4 + 0.5 * 0.343)) <= 1e-8
    flat = restated.fit_regression(np.zeros(10), np.arange(1.0, 11.0), 3)
    assert flat["ncoef"] == 1 and abs(flat["coef"][0] - 5.5) <= 1e-12


@needs_ref
@pytest.mark.parametrize("physical", [True, False])
def test_fit_restatement_is_the_reference_fit(physical):
    m, ns = gpu_setup(1700, physical)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0, 4.0), physical=physical, degree=3))
    ns.trades.append(bermudan(exercise=(2.0, 3.0), physical=not physical, position=-0.5, degree=1, pay=True))
    ns.trades.append(bermudan(exercise=(1.0,), physical=physical, degree=2))
    r = ref.compile_plan(S.encode_model(m), S.encode_netting_set(ns), S.encode_options(S.Options()))
    p = gpu.compile(m, ns)  # this package's tables: the records still unfitted
    out = restated.fit_amc(p, p.amc_degrees)
    assert np.array_equal(_bits(out), _bits(r.terms))


@needs_ref
@pytest.mark.parametrize("csa", [False, True])
def test_engine_bermudans_are_the_reference_engine(csa):
    m, ns = gpu_setup(1200, csa)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0, 4.0), physical=True, degree=2))
    ns.trades.append(bermudan(exercise=(2.0, 3.0), physical=False, position=-0.5, degree=3))
    p = gpu.compile(m, ns)
    streams = (m.num_paths + 1) // 2
    z = np.random.default_rng(4).standard_normal((p.num_dates - 1) * int(p.header[5]) * streams)
    e1 = ref.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams)
    e2 = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, m.num_paths)
    assert np.array_equal(e1.netted, e2.netted) and np.array_equal(e1.collateral, e2.collateral)
    for k in e1.profile:
        assert np.array_equal(e1.profile[k], e2.profile[k]), k


# ------------------------------------------------------------------ xVA and allocation against the reference
def _xva_inputs(seed=3, n=41):
    rng = np.random.default_rng(seed)
    t = np.concatenate([[0.0], np.cumsum(rng.uniform(0.05, 0.3, n - 1))])
    dee = np.abs(rng.normal(1e6, 3e5, n)) * np.exp(-0.02 * t)
    dene = -np.abs(rng.normal(8e5, 2e5, n)) * np.exp(-0.02 * t)
    dim = np.abs(rng.normal(4e5, 1e5, n)) * np.exp(-0.02 * t)
    cpty = ([1.0, 3.0, 7.0], [0.01, 0.015, 0.02])
    own = ([2.0, 5.0], [0.005, 0.008])
    return t, dee, dene, dim, cpty, own


@needs_ref
@pytest.mark.parametrize("with_im", [False, True])
def test_xva_is_the_reference_xva(with_im):
    from zlatko_b200 import xva as X

    t, dee, dene, dim, cpty, own = _xva_inputs()
    p = X.XvaParameters(funding_spread_borrow=0.012, funding_spread_lend=0.004, margin_funding_spread=0.009)
    got = X.xva({"times": t, "dee": dee, "dene": dene}, dim if with_im else None, cpty, 0.4, own, 0.35, p)
    want = ref.xva(t, dee, dene, dim if with_im else None, cpty, 0.4, own, 0.35, p.as_dict())
    for k, w in want.items():
        assert abs(got[k] - w) <= 1e-12 * max(abs(w), 1e-300), (k, got[k], w)
    assert (got["mva"] > 0) == with_im
    alloc = X.allocate_exposure_xva(t, [dee * 0.3, dee * 0.7], cpty, 0.4, own, p)
    wa = ref.allocate_exposure_xva(t, [dee * 0.3, dee * 0.7], cpty, 0.4, own, p.as_dict())
    for a, w in zip(alloc, wa):
        for j, k in enumerate(("cva", "fca", "kva")):
            assert abs(a[k] - w[j]) <= 1e-12 * abs(w[j])
    assert abs(sum(a["cva"] for a in alloc) - got["cva"]) <= 1e-12 * got["cva"]  # the allocation adds up


@needs_ref
def test_allocation_and_margin_proxy_are_the_reference():
    from zlatko_b200 import xva as X

    rng = np.random.default_rng(9)
    P, T, N = 500, 13, 4
    times = np.linspace(0.0, 3.0, T)
    tv = rng.normal(0.0, 1e5, (N, P, T))
    tv[:, :, 0] = 0.0
    netted = tv.sum(axis=0)
    defl = np.exp(-0.02 * times)[None, :] * rng.uniform(0.9, 1.1, (P, T))
    for d in (None, defl):
        got = X.marginal_exposure_contributions(tv, netted, d)
        want = ref.marginal_contributions(tv, netted, d)
        assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max()
        assert np.abs(got.sum(axis=0) - (np.maximum(netted, 0) * (1 if d is None else d)).mean(axis=0)).max() <= 1e-6
        gi, wi = X.incremental_exposure(netted, tv[0], d), ref.incremental_exposure(netted, tv[0], d)
        assert np.abs(gi - wi).max() <= 1e-9 * np.abs(wi).max()
    gm = X.initial_margin_profile(netted, times, defl, 0.99, 10 / 250)
    wm = ref.initial_margin_profile(netted, defl, times, 0.99, 10 / 250)
    assert gm[0] == 0.0 and np.abs(gm - wm).max() <= 1e-12 * np.abs(wm).max()
