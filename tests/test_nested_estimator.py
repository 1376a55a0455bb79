"""The adaptive nested Monte Carlo estimator (zlatko_b200.nested) against the reference's estimateAdaptive and
estimateUniform compiled into the test library: on the same outer sample and the same inner payoffs, the same
split, proxy, bins, audit, refinement decisions and estimates, bit for bit."""
import math

import numpy as np
import pytest

from oracle import ref
from zlatko_b200 import nested as N

needs_ref = pytest.mark.skipif(not ref.available(), reason="the reference is not built in this container")


def toy(n=1200, dims=2, seed=4):
    """Outer scenarios of a known conditional value V(x) = 3 x0 - x1^2 + 0.5 x0 x1 with heteroscedastic noise;
    inner payoffs V(x) + (0.5 + |x0|) z from the counter-based normals of the job's seed."""
    rng = np.random.default_rng(seed)
    F = rng.normal(0.0, 1.0, (n, dims))
    v = 3.0 * F[:, 0] - F[:, 1] ** 2 + 0.5 * F[:, 0] * F[:, 1]
    sd = 0.5 + np.abs(F[:, 0])
    y = v + sd * rng.normal(0.0, 1.0, n)
    w = np.exp(-0.05 * rng.uniform(0.0, 5.0, n))

    def simulate(scenario, seed, out):
        for q in range(len(out)):
            out[q] = v[scenario] + sd[scenario] * N.counter_normal(seed, q)

    return F, y, w, v, simulate


def test_counter_normals_and_seeds_are_the_reference():
    if not ref.available():
        pytest.skip("the reference is not built in this container")
    for seed in (0, 1, 20261122, 2 ** 63 + 12345):
        for m in (0, 1, 2, 7, 100):
            assert N.counter_normal(seed, m) == ref.counter_normal(seed, m)
        assert N.derive_seed(seed, 3, 5, 7) == ref.derive_seed(seed, 3, 5, 7)


@needs_ref
@pytest.mark.parametrize("case", range(3))
def test_estimate_adaptive_is_the_reference(case):
    F, y, w, v, simulate = toy(seed=4 + case)
    o = N.AdaptiveOptions(inner_budget=60_000, max_rounds=12, seed=20261122 + case, hermite_degree=3 - case % 2,
                          max_scenarios_per_round=300 if case == 2 else 2000)
    size = float(np.mean(w * np.abs(y)))
    stats = [N.PositivePart(0.01, 1e-3 * size, "EE*"), N.Quantile(0.95, True, 2.0, "PFE")]
    got = N.estimate_adaptive(F, y, w, N.per_scenario(simulate), stats, o)
    want = ref.estimate_adaptive(F, y, w, simulate, 0.01, 1e-3 * size, 0.95, o)
    for k in ("estimate", "baseline", "regression", "proxy", "value"):
        assert np.array_equal(np.asarray(getattr(got, k)), want[k]), k
    for k in ("training", "evaluation", "inner"):
        assert np.array_equal(np.asarray(getattr(got, k), np.float64), want[k]), k
    for k in ("inner_paths", "audit_inner_paths", "refined_scenarios", "audited_scenarios", "rounds", "unresolved",
              "proxy_degree", "proxy_basis", "stop"):
        assert getattr(got, k) == want[k], k
    for b, wb in zip(got.bins, want["bins"]):
        assert np.array_equal(np.array([b["lower_probability"], b["upper_probability"], b["scenarios"], b["refined"],
                                        b["residual_std_dev"], b["bias_shift"], b["bias_rms"]]), wb)
    assert got.inner_paths > 0 and got.rounds > 0
    # The estimate is close to the exact statistic of the known conditional values.
    ev = np.asarray(got.evaluation)
    exact = stats[0].plug_in(v[ev], w[ev])
    assert abs(got.estimate[0] - exact) <= 0.05 * abs(exact)


@needs_ref
def test_estimate_adaptive_with_many_features_is_the_reference():
    """Ten features, one of them constant (dropped from the basis): 220 basis functions at degree 3, so the
    proxy's Gram, sandwich and predictions run on several host threads and must keep the reference's bits."""
    F, y, w, v, simulate = toy(n=2400, dims=10, seed=11)
    F[:, 7] = 0.25
    o = N.AdaptiveOptions(inner_budget=30_000, max_rounds=6, seed=7, hermite_degree=3)
    size = float(np.mean(w * np.abs(y)))
    stats = [N.PositivePart(0.01, 1e-3 * size, "EE*"), N.Quantile(0.95, True, 2.0, "PFE")]
    got = N.estimate_adaptive(F, y, w, N.per_scenario(simulate), stats, o)
    want = ref.estimate_adaptive(F, y, w, simulate, 0.01, 1e-3 * size, 0.95, o)
    assert got.proxy_basis == want["proxy_basis"] == 220 and got.proxy_degree == 3
    for k in ("estimate", "baseline", "regression", "proxy", "value"):
        assert np.array_equal(np.asarray(getattr(got, k)), want[k]), k
    assert got.inner_paths == want["inner_paths"]


def test_proxy_errors_are_the_reference_messages():
    F = np.random.default_rng(0).normal(size=(10, 2))
    with pytest.raises(ValueError, match="at least two training rows"):
        N.HermiteProxy(3).fit(F, F[:, 0], [3])
    with pytest.raises(RuntimeError, match="predict before fit"):
        N.HermiteProxy(3).predict(F, [0])
    p = N.HermiteProxy(3)
    p.fit(F, F[:, 0] + F[:, 1] ** 2, range(10))
    assert (p.degree(), p.num_basis()) == (1, 3)  # degree 2 has 6 terms > 10 / 2
    with pytest.raises(ValueError, match="do not match"):
        p.predict(F[:, :1], [0])
    with pytest.raises(ValueError, match="beyond the features"):
        p.predict(F, [0, 10])
    v, s = p.predict(F, [])
    assert v.size == s.size == 0


@needs_ref
def test_estimate_uniform_is_the_reference():
    F, y, w, v, simulate = toy()
    sc = list(range(0, 1200, 7))
    got = N.estimate_uniform(w, N.per_scenario(simulate), sc, 40, [N.PositivePart(0.01, 0.0), N.Quantile(0.9, True)], 99)
    want = ref.estimate_uniform(w, len(y), simulate, sc, 40, 0.01, 0.0, 0.9, 99)
    assert np.array_equal(np.array(got.estimate), want[:2])
    assert np.array_equal(np.array(got.value), want[2:])


def test_options_are_validated_like_the_reference():
    for kw in ({"training_fraction": 1.0}, {"inner_batch": 0}, {"min_inner_for_variance": 1},
               {"max_inner_per_scenario": 16}, {"bin_probabilities": (0.5, 0.4)}):
        with pytest.raises(ValueError):
            N.AdaptiveOptions(**kw).validate()
    with pytest.raises(ValueError):
        N.PositivePart(0.0, 0.0)
    with pytest.raises(ValueError):
        N.Quantile(1.0)


@needs_ref
def test_outer_normals_are_the_reference_normal_generator():
    from oracle import restated

    for seed in (42, 7, 20261203):
        assert np.array_equal(restated.normal_stream(seed, 3001), ref.normal_stream(seed, 3001))
