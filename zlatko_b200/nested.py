"""Adaptive nested Monte Carlo: a least-squares proxy on the outer paths, a stratified audit of its bias, and inner
simulations only where a statistic needs them.

Restates src/nested/adaptive_nested.cpp (the estimator: HermiteProxy, ScenarioEstimates, the PositivePart and
Quantile statistics, estimateAdaptive, estimateUniform) in the reference's arithmetic order, so that on the same
outer sample and the same inner payoffs it reaches the same decisions and estimates.  The estimator is host
control logic; its inner simulations are the expensive part and run as batches: every round hands all its jobs
(scenario, seed, paths) to the inner simulator at once, so a GPU simulator (nested_exposure.GpuInner) runs a round
in one kernel launch where the reference calls a per-scenario callback on a thread pool.
"""
from __future__ import annotations

import bisect
import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import _native
from .summary import exact_quantile

M64 = 0xFFFFFFFFFFFFFFFF
GOLDEN = 0x9E3779B97F4A7C15
MIN_GAIN = 0.05                 # refining a scenario that removes less of its error variance is skipped
ADAPTIVE_TAG = 0x6164617074697665
UNIFORM_TAG = 0x756E69666F726D00
SPLIT_TAG = 0x73706C6974000000

# An inner simulator takes a round's jobs [(scenario, seed, paths)] and returns one payoff array per job.
InnerBatches = Callable[[List[Tuple[int, int, int]]], List[np.ndarray]]


def split_mix(z: int) -> int:
    """SplitMix64 finaliser (adaptive_nested.cpp:23-28)."""
    z = (z + GOLDEN) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def derive_seed(seed: int, a: int, b: int = 0, c: int = 0) -> int:
    """deriveSeed (adaptive_nested.cpp:120-125)."""
    x = split_mix((seed + GOLDEN) & M64)
    x = split_mix(x ^ (a & M64))
    x = split_mix(x ^ ((b * 0xD1B54A32D192ED03) & M64))
    return split_mix(x ^ ((c * 0x8CB92BA72F3D8DD7) & M64))


def _split_mix_u64(z: np.ndarray) -> np.ndarray:
    """split_mix of every element of a uint64 array (numpy's uint64 arithmetic wraps modulo 2^64)."""
    z = z + np.uint64(GOLDEN)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def derive_seeds(seed: int, a: np.ndarray, b: np.ndarray, c: int) -> np.ndarray:
    """derive_seed(seed, a[k], b[k], c) for every k at once."""
    x = np.full(len(a), split_mix((seed + GOLDEN) & M64), np.uint64)
    x = _split_mix_u64(x ^ np.asarray(a, np.uint64))
    x = _split_mix_u64(x ^ (np.asarray(b, np.uint64) * np.uint64(0xD1B54A32D192ED03)))
    return _split_mix_u64(x ^ np.uint64((c * 0x8CB92BA72F3D8DD7) & M64))


def shuffle(v: List[int], seed: int) -> None:
    """Deterministic Fisher-Yates shuffle (adaptive_nested.cpp:31-38)."""
    s = seed
    for i in range(len(v), 1, -1):
        s = split_mix(s)
        j = s % i
        v[i - 1], v[j] = v[j], v[i - 1]


def counter_normal(seed: int, m: int) -> float:
    """Normal m (0-based) of CounterNormals(seed) (adaptive_nested.cpp:127-141): pair m // 2 of the SplitMix64
    stream, the cosine half first.  Counter-based, so any normal is reached directly."""
    state = (seed + (m // 2 + 1) * GOLDEN) & M64
    h1 = split_mix(state)
    h2 = split_mix(h1 ^ 0x68E31DA4B5297A4D)
    u1 = (float(h1 >> 11) + 0.5) * 2.0 ** -53
    u2 = float(h2 >> 11) * 2.0 ** -53
    r, a = math.sqrt(-2.0 * math.log(u1)), 6.283185307179586 * u2
    return r * math.cos(a) if m % 2 == 0 else r * math.sin(a)


def normal_cdf(x: float) -> float:
    """ccr::normalCdf (include/ccr/core/math.hpp:15)."""
    return 0.5 * math.erfc(-x / math.sqrt(2.0))


def _seq_sum(a) -> float:
    """A left-to-right sum from 0.0 (the reference's loops), not numpy's pairwise one: np.add.accumulate adds in
    order; the final + 0.0 turns the -0.0 of an all-negative-zero input into the loop's +0.0."""
    a = np.asarray(a, np.float64).ravel()
    return float(np.add.accumulate(a)[-1]) + 0.0 if a.size else 0.0


class HermiteProxy:
    """Least-squares proxy of V in probabilists' Hermite polynomials of the standardised features, all products
    up to a total degree, with the HC0 sandwich variance of every prediction (adaptive_nested.cpp:145-277).
    Fit and prediction are native host code (zk_hermite_fit / zk_hermite_predict) in the reference's arithmetic
    order, threaded over independent entries and rows; there is no Python fallback."""

    def __init__(self, degree: int = 3, ridge: float = 1e-10):
        self.degree_, self.ridge = degree, ridge
        self._h = None
        self._info = (0, 0)

    def __del__(self):
        if getattr(self, "_h", None) is not None:
            _native.lib().zk_hermite_destroy(self._h)
            self._h = None

    def fit(self, features: np.ndarray, y: Sequence[float], rows: Sequence[int]) -> None:
        F = np.ascontiguousarray(features, np.float64)
        if F.ndim != 2:
            raise ValueError("HermiteProxy: features must be [rows][dims]")
        yy = np.ascontiguousarray(y, np.float64)
        if F.shape[0] != yy.shape[0]:
            raise ValueError("HermiteProxy: features and targets differ in length")
        rr = np.ascontiguousarray(rows, np.uint64)
        L = _native.lib()
        h, err = C.c_void_p(), C.create_string_buffer(256)
        st = L.zk_hermite_fit(F.ctypes.data, F.shape[0], F.shape[1], yy.ctypes.data, rr.ctypes.data, rr.size,
                              int(self.degree_), float(self.ridge), C.byref(h), err, len(err))
        if st != 0:
            raise ValueError(err.value.decode() or f"HermiteProxy: fit failed ({st})")
        if self._h is not None:
            L.zk_hermite_destroy(self._h)
        self._h, self._dims = h, F.shape[1]
        info = (C.c_uint64 * 2)()
        L.zk_hermite_info(h, info)
        self._info = (int(info[0]), int(info[1]))

    def predict(self, features: np.ndarray, rows: Sequence[int]) -> Tuple[np.ndarray, np.ndarray]:
        """(value, estimation variance) of the feature rows `rows`."""
        if self._h is None:
            raise RuntimeError("HermiteProxy: predict before fit")
        F = np.ascontiguousarray(features, np.float64)
        if F.ndim != 2 or F.shape[1] != self._dims:
            raise ValueError("HermiteProxy: features do not match the fit")
        rr = np.ascontiguousarray(rows, np.uint64)
        value, var = np.empty(rr.size), np.empty(rr.size)
        st = _native.lib().zk_hermite_predict(self._h, F.ctypes.data, F.shape[0], F.shape[1], rr.ctypes.data, rr.size,
                                              value.ctypes.data, var.ctypes.data)
        if st != 0:
            raise ValueError("HermiteProxy: a row beyond the features")
        return value, var

    def degree(self) -> int:
        return self._info[0]

    def num_basis(self) -> int:
        return self._info[1]


_acc_sum = _seq_sum


def _binned_seq_sums(columns: Sequence[np.ndarray], bins: np.ndarray, nb: int) -> np.ndarray:
    """[k][b] = _seq_sum of columns[k] over the entries of bin b, in their order: every bin's entries are laid
    out in one row of a zero-padded matrix (stable by position), and each row is summed in order."""
    bins = np.asarray(bins, np.int64)
    out = np.zeros((len(columns), nb))
    if bins.size == 0:
        return out
    order = np.argsort(bins, kind="stable")
    counts = np.bincount(bins, minlength=nb)
    starts = np.cumsum(counts) - counts
    sb = bins[order]
    pos = np.arange(bins.size) - starts[sb]
    width = int(counts.max())
    for k, c in enumerate(columns):
        m = np.zeros((nb, width))
        m[sb, pos] = np.asarray(c, np.float64)[order]
        out[k] = _row_sums(m)
    return out


def _row_sums(a: np.ndarray) -> np.ndarray:
    """_seq_sum of every row of a 2-D array."""
    return np.add.accumulate(a, axis=1)[:, -1] + 0.0


def _merge_rows(count: np.ndarray, mean: np.ndarray, m2: np.ndarray, payoffs: np.ndarray):
    """Chan et al. merge of row k of payoffs into the running (count[k], mean[k], M2[k]) for every k, element by
    element in the reference's order (adaptive_nested.cpp:373-385)."""
    n = payoffs.shape[1]
    if n == 0:
        return count, mean, m2
    batch_mean = _row_sums(payoffs) / float(n)
    dev = payoffs - batch_mean[:, None]
    batch_m2 = _row_sums(dev * dev)
    na, nb = count.astype(np.float64), float(n)
    total = na + nb
    delta = batch_mean - mean
    return count + n, mean + delta * nb / total, m2 + (batch_m2 + delta * delta * (na * nb / total))


def _erfc(a: np.ndarray) -> np.ndarray:
    """erfc of every element by the C library's erfc (the one math.erfc calls), in one native call."""
    x = np.ascontiguousarray(a, np.float64)
    out = np.empty_like(x)
    if x.size and _native.lib().zk_erfc_array(x.ctypes.data, x.size, out.ctypes.data) != 0:
        raise RuntimeError("erfc failed")
    return out


class ScenarioEstimates:
    """What is known about every evaluation scenario: proxy value and uncertainty, bin, and inner samples in two
    folds (adaptive_nested.cpp:279-437).  The per-scenario quantities are computed for all scenarios at once with
    element-wise IEEE operations in the reference's order, so they carry the reference's bits."""

    def __init__(self, outer_payoff, weight, proxy_mean, proxy_variance, bins, residual_variance_by_bin,
                 min_inner_for_variance: int, max_inner_per_scenario: int):
        n = len(proxy_mean)
        if not (len(outer_payoff) == len(weight) == len(proxy_variance) == len(bins) == n):
            raise ValueError("ScenarioEstimates: inconsistent sizes")
        f = lambda v: np.array(v, np.float64)  # noqa: E731
        self.w, self.mu, self.pv = f(weight), f(proxy_mean), f(proxy_variance)
        self.bin = np.array(bins, np.int64)
        self.residual = f(residual_variance_by_bin)
        nb = len(self.residual)
        self.misspec, self.shift = np.zeros(nb), np.zeros(nb)
        self.min_inner, self.max_inner = min_inner_for_variance, max_inner_per_scenario
        self.count0, self.count1, self.batches = np.ones(n, np.int64), np.zeros(n, np.int64), np.zeros(n, np.int64)
        self.mean0, self.mean1 = f(outer_payoff), np.zeros(n)
        self.m20, self.m21 = np.zeros(n), np.zeros(n)
        # Derived arrays of the current state (pooled moments, blended estimates), dropped on every change: a
        # round asks for them many times between two changes.  Callers treat them as read-only.
        self._memo: dict = {}

    def _cached(self, key: str, make):
        v = self._memo.get(key)
        if v is None:
            v = self._memo[key] = make()
        return v

    def size(self) -> int:
        return len(self.mu)

    def num_bins(self) -> int:
        return len(self.residual)

    def proxy_mean(self) -> np.ndarray:
        return self._cached("proxy_mean", lambda: self.mu + self.shift[self.bin])

    def proxy_variance(self) -> np.ndarray:
        return self._cached("proxy_variance", lambda: self.pv + self.misspec[self.bin])

    def inner_paths(self) -> np.ndarray:
        return self.count0 + self.count1 - 1

    def pooled(self):
        return self._cached("pooled", self._pooled)

    def _pooled(self):
        n0, n1 = self.count0.astype(np.float64), self.count1.astype(np.float64)
        n = n0 + n1
        d = self.mean1 - self.mean0
        one = self.count1 == 0
        with np.errstate(invalid="ignore", divide="ignore"):
            mean = np.where(one, self.mean0, self.mean0 + d * n1 / n)
            m2 = np.where(one, self.m20, self.m20 + self.m21 + d * d * (n0 * n1 / n))
        return n, mean, m2

    def blend(self, sample_mean: np.ndarray, sample_variance: np.ndarray):
        pvar, proxy = self.proxy_variance(), self.proxy_mean()
        den = pvar + sample_variance
        pos = den > 0.0
        with np.errstate(invalid="ignore", divide="ignore"):
            value = np.where(pos, proxy + pvar / den * (sample_mean - proxy), proxy)
            var = np.where(pos, pvar * sample_variance / den, 0.0)
        return value, var

    def within_variance(self) -> np.ndarray:
        return self._cached("within", self._within_variance)

    def _within_variance(self) -> np.ndarray:
        n, _, m2 = self.pooled()
        with np.errstate(invalid="ignore", divide="ignore"):
            return np.where(n >= 1.0 + float(self.min_inner), m2 / (n - 1.0), self.residual[self.bin])

    def _current(self):
        n, mean, _ = self.pooled()
        return self._cached("current", lambda: self.blend(mean, self.within_variance() / n))

    def estimate(self) -> np.ndarray:
        return self._current()[0]

    def std_error(self) -> np.ndarray:
        return self._cached("std_error", lambda: np.sqrt(self._current()[1]))

    def refinement_gain(self) -> np.ndarray:
        n, mean, _ = self.pooled()
        within = self.within_variance()
        current = self._current()[1]
        used = self.inner_paths().astype(np.float64)
        remaining = np.maximum(0.0, float(self.max_inner) - used)
        best = self.blend(mean, within / (n + remaining))[1]
        with np.errstate(invalid="ignore", divide="ignore"):
            return np.where(current <= 0.0, 0.0, 1.0 - best / current)

    def selection_estimate(self) -> np.ndarray:
        value = self.blend(self.mean0, self.within_variance() / self.count0.astype(np.float64))[0]
        return np.where(self.count1 == 0, self.proxy_mean(), value)

    def value_estimate(self) -> np.ndarray:
        return np.where(self.count1 > 0, self.mean1, self.mean0)

    def value_variance(self) -> np.ndarray:
        return self.within_variance() / np.where(self.count1 > 0, self.count1, self.count0).astype(np.float64)

    def add_inner_batch(self, i: int, payoffs: np.ndarray) -> None:
        """ScenarioEstimates::addInnerBatch (adaptive_nested.cpp:390-400): the first half of the batch goes to the
        selection fold, the rest to the value fold, each merged as Chan et al."""
        self.add_inner_batches(np.array([i], np.int64), np.asarray(payoffs, np.float64)[None, :])

    def add_inner_batches(self, idx: np.ndarray, payoffs: np.ndarray) -> None:
        """add_inner_batch of scenario idx[k] with payoffs[k] for every k at once: distinct scenarios, batches
        of one length.  Every row's sums run in order, so the result is that of the one-by-one calls."""
        if payoffs.shape[1] == 0:
            return
        if not np.all(np.isfinite(payoffs)):
            raise RuntimeError("nested Monte Carlo: inner simulation returned a non-finite payoff")
        self._memo.clear()
        half = payoffs.shape[1] // 2
        for count, mean, m2, part in ((self.count0, self.mean0, self.m20, payoffs[:, :half]),
                                      (self.count1, self.mean1, self.m21, payoffs[:, half:])):
            c, m, q = _merge_rows(count[idx], mean[idx], m2[idx], part)
            count[idx], mean[idx], m2[idx] = c, m, q
        self.batches[idx] += 1

    def update_misspecification(self, min_scenarios_per_bin: int) -> None:
        nb = self.num_bins()
        n, mean, m2 = self.pooled()
        ok = np.nonzero(~(n < 1.0 + float(self.min_inner)))[0]
        s, sq, noise, cnt = [0.0] * nb, [0.0] * nb, [0.0] * nb, [0] * nb
        gsq = gnoise = 0.0
        if ok.size:
            # Per bin and overall, each sum runs over the scenarios in ascending order, as the reference's loop.
            d = mean[ok] - self.mu[ok]
            d2 = d * d
            sampling = m2[ok] / (n[ok] - 1.0) / n[ok] + self.pv[ok]
            bins = self.bin[ok]
            cnt = np.bincount(bins, minlength=nb).tolist()
            s, sq, noise = (v.tolist() for v in _binned_seq_sums((d, d2, sampling), bins, nb))
            gsq, gnoise = _seq_sum(d2), _seq_sum(sampling)
        gcount = int(ok.size)
        glob = max(0.0, (gsq - gnoise) / float(gcount)) if gcount > 0 else 0.0
        for b in range(nb):
            if cnt[b] >= min_scenarios_per_bin:
                c = float(cnt[b])
                self.shift[b] = s[b] / c
                self.misspec[b] = max(0.0, (sq[b] - c * self.shift[b] * self.shift[b] - noise[b]) / c)
            else:
                self.shift[b] = 0.0
                self.misspec[b] = glob
        self._memo.clear()  # the proxy's shift and variance changed


def _misclassification_probability(gap: np.ndarray, se: np.ndarray) -> np.ndarray:
    with np.errstate(invalid="ignore", divide="ignore"):
        x = -gap / se
    p = 0.5 * _erfc(-x / math.sqrt(2.0))
    return np.where(se > 0.0, p, 0.0)


def _mark_largest(contribution: np.ndarray, s: ScenarioEstimates, excess: float, urgency: np.ndarray) -> None:
    """The error-budget rule (adaptive_nested.cpp:85-106)."""
    gain = s.refinement_gain()
    reducible = contribution * gain
    order = np.argsort(-reducible, kind="stable")
    covered = 0.0
    for i in order.tolist():
        if covered >= excess or reducible[i] <= 0.0:
            break
        if gain[i] < MIN_GAIN:
            continue
        urgency[i] = max(urgency[i], 2.0)
        covered += reducible[i]


class PositivePart:
    """E[w max(V, 0)]: EE with w = 1, EE* with w = D(0, t) (adaptive_nested.cpp:439-488)."""

    def __init__(self, relative_tolerance: float = 0.01, absolute_tolerance: float = 0.0, label: str = "EE"):
        if not (relative_tolerance >= 0.0) or not (absolute_tolerance >= 0.0) or relative_tolerance + absolute_tolerance == 0.0:
            raise ValueError("PositivePart: tolerances must be non-negative and not both zero")
        self.rel, self.abs, self.label = relative_tolerance, absolute_tolerance, label

    def name(self) -> str:
        return self.label

    def evaluate(self, s: ScenarioEstimates) -> float:
        if not s.size():
            return 0.0
        sel = s.selection_estimate() > 0.0
        return _acc_sum((s.w * s.value_estimate())[sel]) / float(s.size())

    def plug_in(self, values, weights) -> float:
        v = np.asarray(values, np.float64)
        if not v.size:
            return 0.0
        w = np.ones_like(v) if weights is None or len(weights) == 0 else np.asarray(weights, np.float64)
        return _acc_sum(w * np.maximum(v, 0.0)) / float(v.size)

    def urgency(self, s: ScenarioEstimates, urgency: np.ndarray) -> None:
        n = s.size()
        if n == 0:
            return
        half = 0.5 * max(self.abs, self.rel * abs(self.evaluate(s)))
        if not (half > 0.0):
            return
        nn = float(n)
        sel = s.selection_estimate() > 0.0
        vv = s.value_variance()
        noise = _acc_sum((s.w * s.w * vv)[sel])
        counted = int(np.count_nonzero(sel))
        if counted > 0 and math.sqrt(noise) / nn > half:
            share = half * half * nn * nn / float(counted)
            cand = s.w * s.w * vv / share
            np.maximum(urgency, np.where(sel, cand, urgency), out=urgency)
        gap = np.abs(s.estimate())
        contribution = s.w * (gap * _misclassification_probability(gap, s.std_error())) / nn
        total = _acc_sum(contribution)
        if total > half:
            _mark_largest(contribution, s, total - half, urgency)


class Quantile:
    """The `level` quantile of V across scenarios, of max(V, 0) with positive_part (PFE) (adaptive_nested.cpp:490-523)."""

    def __init__(self, level: float, positive_part: bool = False, z_critical: float = 2.0, label: str = "quantile"):
        if not (0.0 < level < 1.0):
            raise ValueError("Quantile: level must be in (0, 1)")
        if not (z_critical > 0.0):
            raise ValueError("Quantile: zCritical must be positive")
        self.level, self.pos, self.z, self.label = level, positive_part, z_critical, label

    def name(self) -> str:
        return self.label

    def plug_in(self, values, weights=None) -> float:
        if len(values) == 0:
            return 0.0
        q = exact_quantile(values, self.level)
        return max(q, 0.0) if self.pos else q

    def evaluate(self, s: ScenarioEstimates) -> float:
        return self.plug_in(s.estimate())

    def urgency(self, s: ScenarioEstimates, urgency: np.ndarray) -> None:
        if s.size() == 0:
            return
        v = s.estimate()
        q = exact_quantile(v, self.level)
        if self.pos and q < 0.0:
            return
        threshold = normal_cdf(-self.z)
        p = _misclassification_probability(np.abs(v - q), s.std_error())
        np.maximum(urgency, s.refinement_gain() * p / threshold, out=urgency)


@dataclass
class AdaptiveOptions:
    """AdaptiveOptions (include/ccr/nested/adaptive_nested.hpp:205-227)."""

    training_fraction: float = 0.5
    hermite_degree: int = 3
    inner_batch: int = 64
    min_inner_for_variance: int = 32
    max_inner_per_scenario: int = 4096
    inner_budget: int = 2_000_000
    max_scenarios_per_round: int = 2000
    max_rounds: int = 50
    audit_per_bin: int = 16
    min_per_bin_for_misspecification: int = 8
    bin_probabilities: Sequence[float] = (0.005, 0.01, 0.025, 0.05, 0.1, 0.25, 0.5, 0.75, 0.9, 0.95, 0.975, 0.99, 0.995)
    refine_outside_training_range: bool = True
    seed: int = 20261122

    def validate(self) -> None:
        if not (0.0 < self.training_fraction < 1.0):
            raise ValueError("AdaptiveOptions: trainingFraction must be in (0, 1)")
        if self.inner_batch < 1:
            raise ValueError("AdaptiveOptions: innerBatch must be at least 1")
        if self.min_inner_for_variance < 2:
            raise ValueError("AdaptiveOptions: minInnerForVariance must be at least 2")
        if self.max_inner_per_scenario < max(self.inner_batch, self.min_inner_for_variance):
            raise ValueError("AdaptiveOptions: maxInnerPerScenario must be at least innerBatch and minInnerForVariance")
        if self.max_scenarios_per_round < 1:
            raise ValueError("AdaptiveOptions: maxScenariosPerRound must be at least 1")
        if self.min_per_bin_for_misspecification < 1:
            raise ValueError("AdaptiveOptions: minPerBinForMisspecification must be at least 1")
        for k, p in enumerate(self.bin_probabilities):
            if not (0.0 < p < 1.0) or (k > 0 and not p > self.bin_probabilities[k - 1]):
                raise ValueError("AdaptiveOptions: binProbabilities must be strictly increasing in (0, 1)")


STOP_REASONS = ("converged", "scenario caps", "budget", "max rounds")


@dataclass
class AdaptiveResult:
    names: List[str] = field(default_factory=list)
    estimate: List[float] = field(default_factory=list)
    baseline: List[float] = field(default_factory=list)
    regression: List[float] = field(default_factory=list)
    training: List[int] = field(default_factory=list)
    evaluation: List[int] = field(default_factory=list)
    proxy: List[float] = field(default_factory=list)
    value: List[float] = field(default_factory=list)
    inner: List[int] = field(default_factory=list)
    inner_paths: int = 0
    audit_inner_paths: int = 0
    refined_scenarios: int = 0
    audited_scenarios: int = 0
    rounds: int = 0
    unresolved: int = 0
    proxy_degree: int = 0
    proxy_basis: int = 0
    stop: str = "converged"
    bins: List[dict] = field(default_factory=list)


def _quantile_index(n: int, p: float) -> int:
    k = math.ceil(float(n) * p - 1e-9) - 1.0
    return int(min(max(k, 0.0), float(n - 1)))


def _run_batch(s: ScenarioEstimates, evaluation: List[int], chosen: List[int], batch: int, max_inner: int, budget: int,
               seed: int, inner: InnerBatches) -> int:
    """One inner batch for each chosen scenario that fits in the budget (adaptive_nested.cpp:541-573), all of the
    round's jobs handed to the simulator at once."""
    picked, sizes, total = [], [], 0
    inner_paths = s.inner_paths()
    for i in chosen:
        used = int(inner_paths[i])
        m = 0 if used >= max_inner else min(batch, max_inner - used)
        if m == 0:
            continue
        if total + m > budget:
            break
        picked.append(i)
        sizes.append(m)
        total += m
    if picked:
        idx = np.asarray(picked, np.int64)
        ev = np.asarray(evaluation, np.int64)[idx]
        seeds = derive_seeds(seed, ev, s.batches[idx], ADAPTIVE_TAG)
        outs = inner([(int(e), int(sd), m) for e, sd, m in zip(ev.tolist(), seeds.tolist(), sizes)])
        # The batches of one length go in together (a scenario appears once per round).
        sz = np.asarray(sizes, np.int64)
        for m in np.unique(sz).tolist():
            ks = np.nonzero(sz == m)[0]
            rows = np.stack([np.asarray(outs[k], np.float64)[:m] for k in ks.tolist()])
            s.add_inner_batches(idx[ks], rows)
    return total


def _candidates(s: ScenarioEstimates, statistics, outside: List[bool], o: AdaptiveOptions) -> Tuple[List[int], int]:
    """The scenarios to refine this round (adaptive_nested.cpp:578-625)."""
    n = s.size()
    queues, wanted, capped = [], np.zeros(n, bool), 0
    inner_paths = s.inner_paths()
    at_cap = inner_paths >= o.max_inner_per_scenario
    for st in statistics:
        urgency = np.zeros(n)
        st.urgency(s, urgency)
        asked = urgency > 1.0  # also skips NaN
        capped += int(np.count_nonzero(asked & at_cap & ~wanted))
        wanted |= asked & at_cap
        idx = np.nonzero(asked & ~at_cap)[0]
        order = np.argsort(-urgency[idx], kind="stable")  # stable, descending
        queues.append(idx[order])
    out: List[int] = []
    taken = np.zeros(n, bool)
    if o.refine_outside_training_range and o.max_scenarios_per_round > 0:
        first = np.nonzero(np.asarray(outside, bool) & (inner_paths < o.min_inner_for_variance))[0]
        first = first[:o.max_scenarios_per_round]
        out = first.tolist()
        taken[first] = True
    # Round robin over the queues (depth by depth, queue by queue), each scenario once, until the round is full.
    room = o.max_scenarios_per_round - len(out)
    if room > 0 and any(len(q) for q in queues):
        depth = max(len(q) for q in queues)
        grid = np.full((depth, len(queues)), -1, np.int64)
        for k, q in enumerate(queues):
            grid[:len(q), k] = q
        flat = grid.ravel()
        flat = flat[flat >= 0]
        flat = flat[~taken[flat]]
        _, first = np.unique(flat, return_index=True)
        out += flat[np.sort(first)][:room].tolist()
    return out, capped


def estimate_adaptive(features: np.ndarray, payoff: Sequence[float], weight: Optional[Sequence[float]], inner: InnerBatches,
                      statistics: Sequence, o: AdaptiveOptions) -> AdaptiveResult:
    """estimateAdaptive (adaptive_nested.cpp:629-767): features [n][dims] of the outer scenarios' states, their own
    discounted payoffs, optional weights, the inner simulator and the statistics refined jointly."""
    o.validate()
    F = np.asarray(features, np.float64)
    n = len(payoff)
    if F.shape[0] != n:
        raise ValueError("estimateAdaptive: features and payoffs differ in length")
    if weight is not None and len(weight) and len(weight) != n:
        raise ValueError("estimateAdaptive: weights differ in length")
    if not statistics:
        raise ValueError("estimateAdaptive: no statistic")
    n_train = int(math.floor(float(n) * o.training_fraction + 0.5))
    if n_train < 2 or n - n_train < 1:
        raise ValueError("estimateAdaptive: too few outer scenarios for the split")
    order = list(range(n))
    shuffle(order, derive_seed(o.seed, SPLIT_TAG))
    r = AdaptiveResult()
    r.training = sorted(order[:n_train])
    r.evaluation = sorted(order[n_train:])
    n_eval = len(r.evaluation)

    proxy = HermiteProxy(o.hermite_degree)
    proxy.fit(F, payoff, r.training)
    r.proxy_degree, r.proxy_basis = proxy.degree(), proxy.num_basis()
    mu_a, var_a = proxy.predict(F, r.evaluation)
    mu, est_var = [float(v) for v in mu_a], [float(v) for v in var_a]
    w_all = None if weight is None or len(weight) == 0 else [float(v) for v in weight]
    wts = [1.0 if w_all is None else w_all[i] for i in r.evaluation]
    pay = [float(payoff[i]) for i in r.evaluation]

    srt = sorted(mu)
    thresholds = [srt[_quantile_index(n_eval, p)] for p in o.bin_probabilities]
    nb = len(thresholds) + 1
    bins = [bisect.bisect_left(thresholds, v) for v in mu]
    rsum, rcount, rtotal = [0.0] * nb, [0] * nb, 0.0
    fitted_t, _ = proxy.predict(F, r.training)
    for k, i in enumerate(r.training):
        fitted = float(fitted_t[k])
        e2 = (float(payoff[i]) - fitted) * (float(payoff[i]) - fitted)
        b = bisect.bisect_left(thresholds, fitted)
        rsum[b] += e2
        rcount[b] += 1
        rtotal += e2
    rglobal = rtotal / float(n_train)
    rvar = [rsum[b] / float(rcount[b]) if rcount[b] >= 2 else rglobal for b in range(nb)]

    s = ScenarioEstimates(pay, wts, mu, est_var, bins, rvar, o.min_inner_for_variance, o.max_inner_per_scenario)
    for st in statistics:
        r.names.append(st.name())
        r.baseline.append(st.evaluate(s))
        r.regression.append(st.plug_in(mu, wts))
    r.proxy = mu

    # The training range of every feature (min and max are exact in any order); a scenario is outside it when
    # any of its features is.
    lo, hi = F[r.training].min(axis=0), F[r.training].max(axis=0)
    E = F[r.evaluation]
    outside = np.any((E < lo) | (E > hi), axis=1).tolist()

    audit_batch = max(o.inner_batch, o.min_inner_for_variance)
    audit_per_bin = min(o.audit_per_bin, max(2, o.inner_budget // 5 // (nb * audit_batch)))
    audit: List[int] = []
    if o.audit_per_bin > 0:
        members: List[List[int]] = [[] for _ in range(nb)]
        for k in range(n_eval):
            members[bins[k]].append(k)
        for b in range(nb):
            shuffle(members[b], derive_seed(o.seed, SPLIT_TAG, b + 1))
            audit += members[b][:min(audit_per_bin, len(members[b]))]
    used = _run_batch(s, r.evaluation, audit, audit_batch, o.max_inner_per_scenario, o.inner_budget, o.seed, inner)
    r.audit_inner_paths = used
    s.update_misspecification(o.min_per_bin_for_misspecification)

    while True:
        if r.rounds >= o.max_rounds:
            r.stop = "max rounds"
            break
        chosen, capped = _candidates(s, statistics, outside, o)
        if not chosen:
            r.stop = "scenario caps" if capped > 0 else "converged"
            break
        spent = _run_batch(s, r.evaluation, chosen, o.inner_batch, o.max_inner_per_scenario, o.inner_budget - used, o.seed, inner)
        if spent == 0:
            r.stop = "budget"
            break
        used += spent
        r.rounds += 1
        s.update_misspecification(o.min_per_bin_for_misspecification)
    chosen, capped = _candidates(s, statistics, outside, o)
    r.unresolved = len(chosen) + capped

    for st in statistics:
        r.estimate.append(st.evaluate(s))
    r.inner_paths = used
    per_bin, refined_bin = [0] * nb, [0] * nb
    r.value = s.estimate().tolist()
    r.inner = [int(v) for v in s.inner_paths()]
    for k in range(n_eval):
        per_bin[bins[k]] += 1
        if r.inner[k] > 0:
            r.refined_scenarios += 1
            refined_bin[bins[k]] += 1
    r.audited_scenarios = sum(1 for k in audit if r.inner[k] > 0)
    for b in range(nb):
        r.bins.append({"lower_probability": 0.0 if b == 0 else o.bin_probabilities[b - 1],
                       "upper_probability": 1.0 if b + 1 == nb else o.bin_probabilities[b],
                       "scenarios": per_bin[b], "refined": refined_bin[b], "residual_std_dev": math.sqrt(float(s.residual[b])),
                       "bias_shift": float(s.shift[b]), "bias_rms": math.sqrt(float(s.misspec[b]))})
    return r


@dataclass
class UniformResult:
    estimate: List[float]
    value: List[float]
    inner_paths: int


def estimate_uniform(weight: Optional[Sequence[float]], inner: InnerBatches, scenarios: Sequence[int], inner_per_scenario: int,
                     statistics: Sequence, seed: int) -> UniformResult:
    """estimateUniform (adaptive_nested.cpp:769-790): the classical nest with the same inner paths per scenario."""
    if inner_per_scenario < 1:
        raise ValueError("estimateUniform: at least one inner path per scenario")
    sc_ = np.asarray(scenarios, np.int64)
    seeds = derive_seeds(seed, sc_, np.zeros(sc_.size, np.int64), UNIFORM_TAG).tolist()
    outs = inner([(int(sc), sd, inner_per_scenario) for sc, sd in zip(sc_.tolist(), seeds)])
    value = [_seq_sum(np.asarray(o, np.float64)[:inner_per_scenario]) / float(inner_per_scenario) for o in outs]
    w = [1.0] * len(scenarios)
    if weight is not None and len(weight):
        w = [float(weight[sc]) for sc in scenarios]
    return UniformResult([st.plug_in(value, w) for st in statistics], value, len(scenarios) * inner_per_scenario)


def per_scenario(simulate: Callable[[int, int, np.ndarray], None]) -> InnerBatches:
    """Adapts a per-scenario simulator simulate(scenario, seed, out) -- the reference's InnerSimulator shape -- to
    the batch interface."""
    def run(jobs):
        outs = []
        for sc, seed, m in jobs:
            out = np.zeros(m)
            simulate(sc, seed, out)
            outs.append(out)
        return outs
    return run
