"""Exposure by adaptive nested Monte Carlo, with the inner simulations on the GPU.

Restates src/nested/nested_exposure.cpp: on every reporting date the conditional value of the netting set is
estimated from the outer paths' own discounted cash flows after the date (one-sample estimates), a least-squares
proxy on their Markov state, and inner simulations restarted from a path's state where a statistic needs them
(zlatko_b200.nested, the reference's estimator).  The supported trades are the reference's: swaps (one schedule),
asset forwards and European options; the closed form of each on the outer paths is the exact statistic the four
estimates (exact, regression, uniform nest, adaptive nest) are compared with.

B200 placement: the outer simulation is the FP64 risk-factor kernel (zk_factor_paths_f64) and the closed forms the
FP64 fused kernel (zk_run_plan_f64); every refinement round's inner simulations -- the expensive part, run by the
reference one scenario at a time on CPU threads -- are one launch of the inner-path kernel (zk_nest_run), one
thread per inner path, on the reference's counter-based normals.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field, replace
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import gpu
from . import nested as N
from . import spec as S
from ._native import check, lib

EPS = 1e-10  # the trades' own tolerance for "on or before t" (nested_exposure.cpp:19)


@dataclass
class NestedExposureOptions:
    """NestedExposureOptions (include/ccr/nested/nested_exposure.hpp:36-40)."""

    pfe_quantile: float = 0.95
    adaptive: N.AdaptiveOptions = field(default_factory=N.AdaptiveOptions)
    uniform: bool = True


@dataclass
class CashFlows:
    periods: np.ndarray        # [nPer][6]: ts, te, tau, amount, fixed rate, slot (the swap)
    terminals: np.ndarray      # [nTerm][6]: asset, option, call, notional, strike, maturity
    trades: List              # the supported trades
    unsupported: List[int]    # indices of the trades left out
    slots: int

    def event_times(self) -> List[float]:
        t = [v for p in self.periods for v in (p[0], p[1])]
        return t + [float(f[5]) for f in self.terminals]

    def last_payment(self) -> float:
        last = 0.0
        for p in self.periods:
            last = max(last, float(p[1]))
        for f in self.terminals:
            last = max(last, float(f[5]))
        return last


def collect(netting_set: S.NettingSet) -> CashFlows:
    """The netting set's cash flows (nested_exposure.cpp:59-82)."""
    periods, terminals, trades, unsupported, swaps = [], [], [], [], 0
    for k, t in enumerate(netting_set.trades):
        if type(t) is S.Swap:
            s = list(t.schedule)
            sign = 1.0 if t.pay_fixed else -1.0
            for i in range(1, len(s)):
                periods.append((s[i - 1], s[i], s[i] - s[i - 1], sign * t.notional, t.fixed_rate, float(swaps)))
            swaps += 1
            trades.append(t)
        elif isinstance(t, S.Forward):
            terminals.append((float(t.asset), 0.0, 1.0, t.notional, t.strike, t.maturity))
            trades.append(t)
        elif isinstance(t, S.Option):
            terminals.append((float(t.asset), 1.0, 1.0 if t.call else 0.0, t.notional, t.strike, t.expiry))
            trades.append(t)
        else:
            unsupported.append(k)
    return CashFlows(np.array(periods, np.float64).reshape(-1, 6), np.array(terminals, np.float64).reshape(-1, 6), trades,
                     unsupported, swaps)


def time_grid(times) -> List[float]:
    """TimeGrid(times) (src/core/time_grid.cpp:13-21): non-negative, with 0, sorted, 1e-9 apart."""
    t = sorted([float(v) for v in times if v >= 0.0 and math.isfinite(v)] + [0.0])
    out: List[float] = []
    for v in t:
        if not out or v - out[-1] > 1e-9:
            out.append(v)
    return out


def _find(grid: Sequence[float], t: float, tol: float) -> int:
    i = int(np.searchsorted(grid, t, side="right")) - 1
    i = max(i, 0)
    if abs(grid[i] - t) <= tol:
        return i
    if i + 1 < len(grid) and abs(grid[i + 1] - t) <= tol:
        return i + 1
    raise ValueError(f"nested exposure: date {t} not on the simulation grid")


class GpuInner:
    """The inner paths of one reporting date on the GPU (zk_nest_*), as a batch simulator for nested.py."""

    def __init__(self, ctx: gpu.Context, model_flat: np.ndarray, cf: CashFlows, t: float, x: np.ndarray, spot: np.ndarray,
                 known: np.ndarray):
        self.ctx = ctx
        h = C.c_void_p()
        per = np.ascontiguousarray(cf.periods, np.float64)
        term = np.ascontiguousarray(cf.terminals, np.float64)
        xs = np.ascontiguousarray(x, np.float64)
        sp = np.ascontiguousarray(spot, np.float64)
        kn = np.ascontiguousarray(known, np.float64)
        check(lib().zk_nest_create(ctx.handle, model_flat.ctypes.data, model_flat.size, per.ctypes.data if per.size else None,
                                   len(per), term.ctypes.data if term.size else None, len(term), float(t), xs.ctypes.data,
                                   sp.ctypes.data if sp.size else None, kn.ctypes.data if kn.size else None, cf.slots,
                                   len(xs), C.byref(h)), ctx.handle)
        self.handle = h
        self.launches = 0

    def events(self) -> int:
        e = C.c_uint64()
        check(lib().zk_nest_events(self.handle, C.byref(e)), self.ctx.handle)
        return int(e.value)

    def __call__(self, jobs):
        sc = np.array([j[0] for j in jobs], np.uint64)
        seeds = np.array([j[1] for j in jobs], np.uint64)
        paths = np.array([j[2] for j in jobs], np.uint64)
        out = np.zeros(int(paths.sum()))
        check(lib().zk_nest_run(self.handle, sc.ctypes.data, seeds.ctypes.data, paths.ctypes.data, len(jobs), out.ctypes.data),
              self.ctx.handle)
        self.launches += 1
        starts = np.concatenate([[0], np.cumsum(paths)]).astype(np.int64)
        return [out[starts[k]:starts[k + 1]] for k in range(len(jobs))]

    def close(self) -> None:
        if self.handle:
            lib().zk_nest_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def zero_bonds(model_flat: np.ndarray, ts_te: np.ndarray) -> np.ndarray:
    """[n][3] = ratio, c, B of P(ts, te | x) = ratio exp(c - B x) (zk_zero_bond_coefficients)."""
    pairs = np.ascontiguousarray(ts_te, np.float64).reshape(-1, 2)
    out = np.zeros((len(pairs), 3))
    if len(pairs):
        check(lib().zk_zero_bond_coefficients(model_flat.ctypes.data, model_flat.size, pairs.ctypes.data, len(pairs),
                                              out.ctypes.data))
    return out


def fixing(coef: np.ndarray, tau: float, x: np.ndarray) -> np.ndarray:
    """(1 / P(ts, te | x) - 1) / tau (nested_exposure.cpp:119-121)."""
    bond = coef[0] * np.exp(coef[1] - coef[2] * x)
    return (1.0 / bond - 1.0) / tau


def outer_plan(model: S.Model, netting_set: S.NettingSet, reporting: Sequence[float]) -> gpu.Plan:
    """The plan of the outer simulation and the closed forms: the supported trades on the reporting dates merged
    with every fixing and payment date (nested_exposure.cpp:133-134), exactly that grid."""
    cf = collect(netting_set)
    grid = time_grid(list(time_grid(reporting)) + cf.event_times())
    m = replace(model, base_grid=[t for t in grid if t > 0.0])
    plan = gpu.compile(m, S.NettingSet(list(cf.trades), None), S.Options(samples=1, extra_dates=tuple(grid)))
    if len(plan.times) != len(grid) or np.abs(np.asarray(plan.times) - np.asarray(grid)).max() > 1e-12:
        raise ValueError("nested exposure: the simulation grid does not match the reporting and event dates")
    return plan


@dataclass
class NestedExposureResult:
    points: List[Dict] = field(default_factory=list)
    outer_paths: int = 0
    unsupported: List[int] = field(default_factory=list)
    exact: Dict[str, List[float]] = field(default_factory=dict)
    regression: Dict[str, List[float]] = field(default_factory=dict)
    uniform: Dict[str, List[float]] = field(default_factory=dict)
    adaptive: Dict[str, List[float]] = field(default_factory=dict)
    inner_paths: int = 0
    inner_launches: int = 0


def nested_exposure(ctx: gpu.Context, model: S.Model, netting_set: S.NettingSet, reporting: Sequence[float],
                    options: Optional[NestedExposureOptions] = None, normals: Optional[np.ndarray] = None,
                    streams: int = 0) -> NestedExposureResult:
    """nestedExposure (src/nested/nested_exposure.cpp:124-322) on the reporting dates `reporting` (dates after
    the simulation's horizon dropped): the outer simulation on the reporting dates merged with every fixing and
    payment date, on the model's paths and seed, or on injected normals [step][normal][stream] (the layout of
    zk_run_plan_f64)."""
    options = options or NestedExposureOptions()
    options.adaptive.validate()
    cf = collect(netting_set)
    if not cf.trades:
        raise ValueError("nestedExposure: no supported trade (swaps, asset forwards, European options)")
    if cf.slots > 64:
        raise ValueError("nested exposure: at most 64 swaps")
    rep = time_grid(reporting)
    plan = outer_plan(model, netting_set, reporting)
    grid = list(plan.times)
    cube = ctx.factor_paths_f64(plan, normals, streams)
    _, _, rows = ctx.run_f64(plan, normals, streams, rows=True)
    nP, nA = plan.num_paths, len(model.assets)
    xs, D, Ss = cube[0], cube[1], cube[2:2 + nA]
    rowV = int(plan.header[21])
    plan_rep = np.asarray(plan.times)[plan.reporting.astype(np.int64)]
    mflat = S.encode_model(model)
    bonds = zero_bonds(mflat, cf.periods[:, :2]) if len(cf.periods) else np.zeros((0, 3))
    fix_at = [_find(grid, p[0], 1e-8) for p in cf.periods]
    pay_at = [_find(grid, p[1], 1e-8) for p in cf.periods]
    term_at = [_find(grid, f[5], 1e-8) for f in cf.terminals]

    res = NestedExposureResult(outer_paths=nP, unsupported=cf.unsupported)
    for prof in (res.exact, res.regression, res.uniform, res.adaptive):
        prof.update({"times": [], "dee": [], "pfe": []})
    for r, t in enumerate(rep):
        k = _find(grid, t, 1e-8)
        point = {"time": t, "ee_exact": 0.0, "ee_regression": 0.0, "ee_uniform": 0.0, "ee_adaptive": 0.0, "pfe_exact": 0.0,
                 "pfe_regression": 0.0, "pfe_uniform": 0.0, "pfe_adaptive": 0.0, "evaluated": 0, "inner_paths": 0,
                 "audit_inner_paths": 0, "refined": 0, "rounds": 0, "uniform_inner_per_scenario": 0, "max_bias_rms": 0.0,
                 "proxy_basis": 0, "stop": "converged", "live": cf.last_payment() > t + EPS}
        if point["live"]:
            live_assets = sorted({int(f[0]) for f in cf.terminals if f[5] > t + EPS})
            running = [i for i, p in enumerate(cf.periods) if p[0] < t - EPS and p[1] > t + EPS]
            known = {i: fixing(bonds[i], cf.periods[i][2], xs[fix_at[i]]) for i in running}
            cols = [xs[k]] + [np.log(Ss[a][k]) for a in live_assets] + [known[i] for i in running]
            features = np.stack(cols, axis=1)
            dk = D[k]
            y = np.zeros(nP)
            for i, p in enumerate(cf.periods):
                if p[1] <= t + EPS:
                    continue
                L = fixing(bonds[i], p[2], xs[fix_at[i]])
                y = y + p[3] * (L - p[4]) * p[2] * D[pay_at[i]] / dk
            for f, fl in enumerate(cf.terminals):
                if fl[5] <= t + EPS:
                    continue
                s = Ss[int(fl[0])][term_at[f]]
                pay = fl[3] * (np.maximum(s - fl[4] if fl[2] else fl[4] - s, 0.0) if fl[1] else s - fl[4])
                y = y + pay * D[term_at[f]] / dk
            weight = D[k].copy()
            rep_idx = int(np.argmin(np.abs(plan_rep - t)))
            if abs(plan_rep[rep_idx] - t) > 1e-8:
                raise ValueError("nested exposure: a reporting date is not a reporting date of the closed-form plan")
            exact = rows[rowV + rep_idx]
            size = N._seq_sum(weight * np.abs(y)) / float(nP)
            ee = N.PositivePart(0.01, 1e-3 * size, "EE*")
            pfe = N.Quantile(options.pfe_quantile, True, 2.0, "PFE")
            stats = [ee, pfe]
            constant = bool(np.all(features == features[0:1]))
            if constant:
                v, w0 = N._seq_sum(y) / float(nP), float(weight[0])
                point.update(ee_exact=w0 * max(exact[0], 0.0), pfe_exact=max(exact[0], 0.0), evaluated=nP)
                for key in ("regression", "uniform", "adaptive"):
                    point[f"ee_{key}"] = w0 * max(v, 0.0)
                    point[f"pfe_{key}"] = max(v, 0.0)
            else:
                slots = np.zeros((nP, max(cf.slots, 0)))
                for i in running:
                    slots[:, int(cf.periods[i][5])] = known[i]
                spot0 = np.stack([Ss[a][k] for a in range(nA)], axis=1) if nA else np.zeros((nP, 0))
                inner = GpuInner(ctx, mflat, cf, t, xs[k], spot0, slots)
                try:
                    o = replace(options.adaptive, seed=N.derive_seed(options.adaptive.seed, r))
                    a = N.estimate_adaptive(features, y, weight, inner, stats, o)
                    ev = np.asarray(a.evaluation, np.int64)
                    point.update(ee_exact=ee.plug_in(exact[ev], weight[ev]), pfe_exact=pfe.plug_in(exact[ev]),
                                 ee_regression=a.regression[0], pfe_regression=a.regression[1], ee_adaptive=a.estimate[0],
                                 pfe_adaptive=a.estimate[1], evaluated=len(ev), inner_paths=a.inner_paths,
                                 audit_inner_paths=a.audit_inner_paths, refined=a.refined_scenarios, rounds=a.rounds,
                                 stop=a.stop, proxy_basis=a.proxy_basis,
                                 max_bias_rms=max([b["bias_rms"] for b in a.bins] + [0.0]))
                    if options.uniform:
                        per_scenario = max(2, int(math.floor(float(a.inner_paths) / float(len(ev)) + 0.5)))
                        u = N.estimate_uniform(weight, inner, a.evaluation, per_scenario, stats, o.seed)
                        point.update(ee_uniform=u.estimate[0], pfe_uniform=u.estimate[1], uniform_inner_per_scenario=per_scenario)
                    res.inner_launches += inner.launches
                finally:
                    inner.close()
        res.inner_paths += point["inner_paths"]
        for key, prof in (("exact", res.exact), ("regression", res.regression), ("uniform", res.uniform), ("adaptive", res.adaptive)):
            prof["times"].append(t)
            prof["dee"].append(point[f"ee_{key}"])
            prof["pfe"].append(point[f"pfe_{key}"])
        res.points.append(point)
    return res
