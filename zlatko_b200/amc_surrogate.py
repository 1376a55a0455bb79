"""The AMC continuation value of Bermudan swaptions by the learned surrogate, beside the Longstaff-Schwartz
regression it would replace.

Under a fitted exercise policy the continuation of a Bermudan on date t_j (the mark-to-market of an option not
yet exercised) is the conditional expectation of y_j = D(t_e) V_e / D(t_j), where e is the first exercise after
t_j at which the policy exercises on the path and V_e the exercise value (the underlying swap's value there).
The reference estimates it per date by a polynomial regression in the short-rate state (fitAmc,
src/gpu/fused_exposure.cpp:145-154; evaluated by amcPoly, src/gpu/fused_kernels.cpp:78-81, as
pos * max(poly(x), 0)).  Here one perceptron for every date and every Bermudan of a book learns it from the
realised values the plain method itself generates: the AMC pass of the fused kernels (zk_amc_states: the state
x, the deflator D and the exercise values on every path) under the policy the Longstaff-Schwartz fit chose
(zk_fit_amc).  The policy still decides exercise; only the continuation values change.

Inputs (16): x, the co-terminal swap rate of the next exercise and its annuity, the intrinsic value of the
underlying from that exercise, t, the times to the next exercise and to the final maturity, the strike, the
pay / receive sign, the number of exercises left; the rest zero.  Target: y_j per unit notional.

Held-out paths (another seed) compare the two estimators by their mean squared error against the realised
values: both estimate the same conditional expectation and the noise is common to both, so the difference of the
two errors is the difference of their squared biases -- what the network gains over the regression.
"""
from __future__ import annotations

from dataclasses import dataclass, replace
from typing import Dict, List, Sequence

import numpy as np

from . import gpu
from . import spec as S
from .nested_exposure import zero_bonds

KIND_DECIDE, KIND_CONTINUE = 6, 7


@dataclass
class BermudanLayout:
    """Where the policy and continuation records of one Bermudan of a plan sit."""
    trade: S.Bermudan
    exercise_dates: List[int]        # plan date index of each exercise
    decide: List[np.ndarray]         # the policy record (8 floats) of each exercise
    cont: Dict[int, np.ndarray]      # date index -> continuation record
    ev_row: int                      # first row of its exercise values in zk_amc_states' output


def _poly(rec: np.ndarray, x: np.ndarray) -> np.ndarray:
    """amcPoly: ((c3 z + c2) z + c1) z + c0 with z = (x - center) / scale, in double."""
    r = rec.astype(np.float64)
    z = (x - r[2]) * r[3]
    return ((r[7] * z + r[6]) * z + r[5]) * z + r[4]


def layout(plan: gpu.Plan, ns: S.NettingSet) -> List[BermudanLayout]:
    berms = [t for t in ns.trades if isinstance(t, S.Bermudan)]
    out = [BermudanLayout(t, [], [None] * len(t.exercise), {}, 0) for t in berms]
    terms, idx = plan.terms.reshape(-1, 8), plan.indices
    for j in range(plan.num_dates):
        for u in range(int(idx[j]), int(idx[j + 1])):
            code = int(terms[u, 0])
            kind, b, e = code & 15, (code >> 8) & 15, code >> 12
            if kind == KIND_DECIDE:
                out[b].decide[e] = terms[u].copy()
                out[b].exercise_dates.append(j)
            elif kind == KIND_CONTINUE:
                out[b].cont[j] = terms[u].copy()
    row = 0
    for L in out:
        L.ev_row = row
        row += len(L.trade.exercise)
    return out


@dataclass
class AmcPaths:
    """The AMC pass of one plan: x and D [date][path], exercise values [row][path], times, layouts."""
    plan: gpu.Plan
    x: np.ndarray
    D: np.ndarray
    ev: np.ndarray
    layouts: List[BermudanLayout]


def amc_paths(ctx: gpu.Context, fitted: gpu.Plan, ns: S.NettingSet) -> AmcPaths:
    L = layout(fitted, ns)
    rows = sum(len(b.trade.exercise) for b in L)
    x, D, ev = ctx.amc_states(fitted, rows)
    return AmcPaths(fitted, x.astype(np.float64), D.astype(np.float64), ev.astype(np.float64), L)


def realised(a: AmcPaths, b: int):
    """For Bermudan b: per date j with an exercise ahead, y_j [path] of the policy applied from the next exercise
    on (the target of the continuation regression), and the regression's own estimate pos-free poly_j(x)."""
    B = a.layouts[b]
    nE = len(B.exercise_dates)
    dec = np.zeros((nE, a.x.shape[1]), bool)
    val = np.zeros((nE, a.x.shape[1]))
    for e, j in enumerate(B.exercise_dates):
        v = a.ev[B.ev_row + e]
        dec[e] = (v > 0.0) & (v > _poly(B.decide[e], a.x[j]))
        val[e] = a.D[j] * v
    out = {}
    for j, rec in B.cont.items():
        t = a.plan.times[j]
        nxt = int(np.searchsorted(np.asarray(B.trade.exercise), t + 1e-10, side="left"))
        y = np.zeros(a.x.shape[1])
        taken = np.zeros(a.x.shape[1], bool)
        for e in range(nxt, nE):
            hit = dec[e] & ~taken
            y[hit] = val[e][hit]
            taken |= hit
        out[j] = (y / a.D[j], _poly(rec, a.x[j]))
    return out


def features(model_flat: np.ndarray, trade: S.Bermudan, t: float, x: np.ndarray) -> np.ndarray:
    """[paths][16] inputs of the continuation network on date t."""
    sch = np.asarray(trade.swap.schedule, np.float64)
    ex = np.asarray(trade.exercise, np.float64)
    nxt = int(np.searchsorted(ex, t + 1e-10, side="left"))
    te = ex[min(nxt, len(ex) - 1)]
    starts = [k for k in range(len(sch) - 1) if sch[k] >= te - 1e-10]
    pairs = [(t, te)] + [(t, sch[k + 1]) for k in starts]
    c = zero_bonds(model_flat, np.array(pairs))
    bond = c[:, 0:1] * np.exp(c[:, 1:2] - c[:, 2:3] * x[None, :])  # [1 + periods][paths]
    taus = np.array([sch[k + 1] - sch[k] for k in starts])
    annuity = (taus[:, None] * bond[1:]).sum(0)
    rate = (bond[0] - bond[-1]) / np.maximum(annuity, 1e-12)
    sign = 1.0 if trade.swap.pay_fixed else -1.0
    k = trade.swap.fixed_rate
    f = np.zeros((x.size, 16), np.float32)
    f[:, 0] = x
    f[:, 1] = rate
    f[:, 2] = annuity
    f[:, 3] = sign * (rate - k) * annuity
    f[:, 4] = t
    f[:, 5] = te - t
    f[:, 6] = sch[-1] - t
    f[:, 7] = k
    f[:, 8] = sign
    f[:, 9] = len(ex) - nxt
    return f


def rows_of(a: AmcPaths, ns: S.NettingSet, model_flat: np.ndarray, max_paths: int = 0):
    """(X, y, poly) over every Bermudan and date with an exercise ahead, on the first max_paths paths (all when 0):
    inputs, realised values per unit notional and the regression's estimate per unit notional."""
    X, Y, P = [], [], []
    n = a.x.shape[1] if max_paths <= 0 else min(max_paths, a.x.shape[1])
    for b, B in enumerate(a.layouts):
        notional = B.trade.swap.notional
        for j, (y, poly) in realised(a, b).items():
            X.append(features(model_flat, B.trade, float(a.plan.times[j]), a.x[j, :n]))
            Y.append(y[:n] / notional)
            P.append(poly[:n] / notional)
    return np.concatenate(X), np.concatenate(Y).astype(np.float32), np.concatenate(P)


def book_rows(ctx: gpu.Context, model: S.Model, books: Sequence[S.NettingSet], max_paths: int = 0, fitted=None):
    """rows_of over a book: fits the Longstaff-Schwartz policy of each netting set on the GPU (unless `fitted`
    plans are given), runs its AMC pass and collects the rows.  Returns (X, y, poly, fitted plans)."""
    mflat = S.encode_model(model)
    Xs, Ys, Ps, plans = [], [], [], []
    for i, ns in enumerate(books):
        p = fitted[i] if fitted is not None else ctx.fit_amc(gpu.compile(model, ns, S.Options()))
        if fitted is not None and p.num_paths != model.num_paths:  # the policy fitted elsewhere, on these paths
            h = p.header.copy()
            h[0], h[15] = model.num_paths, (model.num_paths + 63) // 64
            p = gpu.Plan.from_arrays(h, p.indices, p.params, p.steps, p.terms, p.requests, p.rows_total, p.num_outputs,
                                     p.times, p.reporting)
        a = amc_paths(ctx, p, ns)
        X, y, poly = rows_of(a, ns, mflat, max_paths)
        Xs.append(X), Ys.append(y), Ps.append(poly), plans.append(p)
    return np.concatenate(Xs), np.concatenate(Ys), np.concatenate(Ps), plans


def held_out(model: S.Model, paths: int, seed: int) -> S.Model:
    return replace(model, num_paths=paths, seed=seed)


def compare(ctx: gpu.Context, sur, model: S.Model, books: Sequence[S.NettingSet], fitted, paths: int, seed: int) -> Dict:
    """Mean squared errors of the network and of the regression against the realised values on held-out paths
    (the same policy, another seed), per unit notional."""
    X, y, poly, _ = book_rows(ctx, held_out(model, paths, seed), books, fitted=fitted)
    pred = sur.predict(X).astype(np.float64)
    y = y.astype(np.float64)
    mse_nn, mse_ls = float(np.mean((pred - y) ** 2)), float(np.mean((poly - y) ** 2))
    return {"rows": int(len(y)), "mse_network": mse_nn, "mse_regression": mse_ls,
            "gain": (mse_ls - mse_nn) / mse_ls if mse_ls > 0 else 0.0,
            "mean_realised": float(y.mean()), "mean_network": float(pred.mean()), "mean_regression": float(poly.mean())}
