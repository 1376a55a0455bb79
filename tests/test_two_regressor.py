"""The two-regressor Longstaff-Schwartz basis (this library's extension; the reference regresses on the short rate
alone): the oracle's regression, the plan compiler's records and the FP64 engine's use of them, on the CPU.

The basis is the graded monomials of total degree <= 3 in the standardised short rate z and co-terminal swap rate w.
No reference code pins it, so these tests pin the oracle by construction: an exact polynomial is recovered, the
degree falls back as documented, the compiled records carry each regression's co-terminal swap, and the engine's
Bermudan with the richer basis stays within Monte Carlo noise of the one-regressor policy it extends.
"""
import numpy as np
import pytest

from oracle import restated
from setups import bermudan, gpu_setup
from zlatko_b200 import gpu
from zlatko_b200 import spec as S


def _graded(z, w):
    return np.stack([np.ones_like(z), z, w, z * z, z * w, w * w, z ** 3, z * z * w, z * w * w, w ** 3], axis=1)


def test_reg2_recovers_a_cubic():
    rng = np.random.default_rng(3)
    x = rng.normal(0.02, 0.01, 4000)
    s = 0.8 * x + rng.normal(0.03, 0.004, 4000)  # correlated, as a swap rate is with the short rate
    coef = rng.normal(size=10)
    z, w = (x - x.mean()) / x.std(), (s - s.mean()) / s.std()
    y = _graded(z, w) @ coef
    r = restated.fit_regression2(x, s, y, 3)
    assert r["degree"] == 3
    # Exact but for the ridge: 1e-6 n on a standardised cubic Gram of condition ~2e4 biases the coefficients by
    # ~4e-4 and the predictions by ~4e-6 of their range.
    assert np.allclose(r["coef"], coef, rtol=0, atol=2e-3)
    assert np.allclose(restated.predict_regression2(r, x, s), y, rtol=0, atol=2e-5 * np.abs(y).max())


def test_reg2_mask_and_degree_fallback():
    rng = np.random.default_rng(4)
    x, s, y = rng.normal(size=50), rng.normal(size=50), rng.normal(size=50)
    mask = np.zeros(50, np.uint8)
    mask[:10] = 1  # 10 samples: degree 3 needs 20, degree 2 needs 12, degree 1 needs 6
    assert restated.fit_regression2(x, s, y, 3, mask)["degree"] == 1
    r = restated.fit_regression2(x, np.full(50, 0.03), y, 3)  # a degenerate swap rate: the mean
    assert r["degree"] == 0 and r["coef"][0] == pytest.approx(y.mean(), rel=1e-12)
    assert restated.fit_regression2(x, s, y, 3, np.zeros(50, np.uint8))["degree"] == -1


def _two_regressor_book(paths, basis):
    m, ns = gpu_setup(paths, False)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0, 4.0), physical=True, degree=3, basis=basis))
    ns.trades.append(bermudan(exercise=(2.0, 3.0), physical=False, position=-0.5, degree=2, pay=True, basis=basis))
    return m, ns


def test_compiled_records_carry_the_coterminal_swap():
    m, ns = _two_regressor_book(256, "rate_swap")
    p = gpu.compile(m, ns, S.Options(exercise_views=True))
    t = np.asarray(p.terms, np.float64).reshape(-1, 8)
    kind = t[:, 0].astype(np.int64) & 15
    times = np.asarray(p.times)
    ind = np.asarray(p.indices, np.int64)[: len(times) + 1]
    regs = np.flatnonzero((kind == 6) | (kind == 7))
    assert regs.size > 0
    for r in regs:
        assert kind[r + 1] == 15 and kind[r + 2] == 15 and (r + 3 >= t.shape[0] or kind[r + 3] != 15)
        u = r
        while kind[u - 1] in (13, 14):
            u -= 1
        run = kind[u:r]
        ann = run == 13
        assert ann.sum() >= 1 and (run == 14).sum() == 2 and np.all(run[: ann.sum()] == 13)  # annuity, then the float leg
        assert np.allclose(t[u:r][ann, 2], 1.0)  # annual periods: tau = 1
        assert t[r - 2, 2] == 1.0 and t[r - 1, 2] == -1.0  # +P(t, T_first) - P(t, T_last)
        j = int(np.searchsorted(ind, r, side="right") - 1)
        if kind[r] == 6:  # at an exercise date the co-terminal swap starts now: P(t, t) = 1
            assert t[r - 2, 3] == pytest.approx(1.0, abs=1e-12) and t[r - 2, 4] == pytest.approx(0.0, abs=1e-12)
        assert times[j] >= 0.0
    # The one-regressor plan of the same book has none of these records.
    k1 = np.asarray(gpu.compile(*_two_regressor_book(256, "rate"), S.Options(exercise_views=True)).terms).reshape(-1, 8)
    assert not np.isin(k1[:, 0].astype(np.int64) & 15, (13, 14, 15)).any()


def _engine(basis, paths=4000, seed=11):
    m, ns = _two_regressor_book(paths, basis)
    p = gpu.compile(m, ns, S.Options(samples=1))
    streams = (paths + 1) // 2
    z = np.random.default_rng(seed).standard_normal((p.num_dates - 1) * int(p.header[5]) * streams)
    return restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, paths)


def test_engine_two_regressor_policy_is_close_to_the_one_regressor_policy():
    a, b = _engine("rate"), _engine("rate_swap")
    for k in range(2):
        agree = float((a.exercise[k] == b.exercise[k]).mean())
        assert agree >= 0.9, (k, agree)
    ee_a, ee_b = a.profile["ee"], b.profile["ee"]
    assert np.abs(ee_a - ee_b).max() <= 0.05 * np.abs(ee_a).max()


def test_oracle_plan_fit_matches_the_engine_basis():
    """The oracle's plan-level fit (fit_amc2, FP32 states) and its FP32 kernel evaluation of the fitted records give a
    Bermudan value close to the FP64 engine's with the same basis (independent normals: Monte Carlo tolerance)."""
    m, ns = _two_regressor_book(4000, "rate_swap")
    p = gpu.compile(m, ns, S.Options(exercise_views=True))
    terms = restated.fit_amc2(p, S.bermudan_degrees(S.encode_netting_set(ns)))
    po = gpu.Plan.from_arrays(p.header, p.indices, p.params, p.steps, terms, p.requests, p.rows_total, p.num_outputs,
                              p.times, p.reporting)
    sums, _ = restated.run_plan(po)
    e = _engine("rate_swap")
    ee_o = sums.reshape(-1, p.stats_per_date)[:, 1].astype(np.float64)[np.asarray(p.reporting)]
    ee_e = e.profile["ee"]
    n = min(ee_o.size, ee_e.size)
    assert np.abs(ee_o[:n] - ee_e[:n]).max() <= 0.05 * np.abs(ee_e).max()
