"""A book revalued by the learned surrogate, audited and corrected by the plain pricer.

The flow (the learned part of the exposure path; the reference has no counterpart):

1. train: the plain pricer (the fused kernels, zk_run_plan_rows with per-trade views) revalues every trade of
   the book on a few hundred paths; the features of each (trade, reporting date, path) are built on the GPU
   (zk_surrogate_features) from the simulated factors and the trade's terms, and the perceptron is trained on
   the values per unit notional (zk_surrogate_train);
2. revalue: zk_surrogate_book builds the features of every (trade, date, path), evaluates the perceptron on
   the tensor cores, nets per netting set and reduces EE and EE* per netting set and date, all on the GPU;
3. audit: the plain pricer revalues every netting set on the first 1% of the paths; a netting set whose
   surrogate EPE on those paths is off by more than 0.5% of the plain EPE falls back to the plain pricer on all
   paths;
4. CVA of each netting set from its EE* and the counterparty's market hazard curve (unilateral, LGD 0.6).

Uncollateralised, the surrogate revalues the reporting dates.  With the netting sets' cash CSAs (make_book with
csa=True) it revalues every simulation date, the margin-call dates t - MPR included, and zk_surrogate_book applies
the collateral rule (collateral.cpp:10-47) to each path's netted values before the exposure statistics.  Features: x, ln S of the trade's FX factor, t, time to
maturity, trade kind (one-hot), strike or fixed rate, call / pay sign, the Hull-White state at the reset of the
running floating period and that period's position (elapsed, remaining, length), the FX factor index, and the zero
bonds P(t, maturity | x) and P(t, end of the running period | x) (two exponentials per row, against the network's
~70 kflop).
"""
from __future__ import annotations

from dataclasses import dataclass, replace
from typing import List, Sequence

import numpy as np

from . import gpu
from . import spec as S
from ._native import check, lib
from .summary import unilateral_cva

TRADE_DTYPE = np.dtype([("netting_set", np.uint32), ("kind", np.uint32), ("asset", np.uint32), ("sign", np.int32),
                        ("notional", np.float32), ("strike", np.float32), ("maturity", np.float32), ("pad", np.float32)])
AUDIT_TOLERANCE = 0.005  # of the netting set's EPE on the audit paths
LGD = 0.6


@dataclass
class Book:
    model: S.Model
    netting_sets: List[S.NettingSet]   # uncollateralised
    trades: np.ndarray                 # TRADE_DTYPE, trade order = netting sets in order, trades in order
    specs: list                        # the spec object of each trade
    times: np.ndarray                  # reporting dates
    resets: np.ndarray                 # [nTr][nR] int32
    periods: np.ndarray                # [nTr][nR][2] float32
    bonds: np.ndarray                  # [nTr][nR][4] float32: (ln A, B) to maturity and to the running period's end
    report: np.ndarray = None          # indices of the reporting dates in `times` (all of them without a CSA)
    csa: np.ndarray = None             # [numNs][4] float32 (hc, ho or -1, mta or -1 without CSA, ia), None: no CSA
    call_index: np.ndarray = None      # [nR] uint32: margin-call date of each date (with csa)
    factor_model: S.Model = None       # the model whose factor views cover `times`

    @property
    def report_times(self) -> np.ndarray:
        return self.times[self.report].astype(np.float64)


def uncollateralised(books: Sequence[S.NettingSet]) -> List[S.NettingSet]:
    return [S.NettingSet(list(b.trades), None) for b in books]


def _float_schedule(t) -> np.ndarray:
    if isinstance(t, S.Swap2):
        return np.asarray(t.float_schedule, np.float64)
    if isinstance(t, S.Swap):
        return np.asarray(t.schedule, np.float64)
    return np.zeros(0)


def make_book(model: S.Model, books: Sequence[S.NettingSet], csa: bool = False) -> Book:
    """The surrogate's view of a book.  Without csa, the netting sets uncollateralised on their reporting dates.  With
    csa, their cash CSAs kept: the surrogate then revalues every simulation date, the margin-call dates t - MPR
    included, so that the collateral rule can look back to them."""
    nets = list(books) if csa else uncollateralised(books)
    report = call_index = csa_arr = None
    factor_model = model
    if csa:
        plans = [gpu.compile(model, ns, S.Options()) for ns in nets]
        p0 = plans[0]
        if any(not np.array_equal(p.times, p0.times) for p in plans):
            raise ValueError("the surrogate's CSA book needs its netting sets on one simulation grid")
        times = np.asarray(p0.times)
        report = p0.reporting.astype(np.int64)
        call_index = p0.indices[p0.num_dates + 1:2 * p0.num_dates + 1].astype(np.uint32)
        csa_arr = np.full((len(nets), 4), -1.0, np.float32)
        for k, ns in enumerate(nets):
            c = ns.csa
            if c is None:
                continue
            if c.kind != 0:
                raise ValueError("the surrogate's collateral is cash")
            csa_arr[k] = (c.threshold_cpty, c.threshold_own if np.isfinite(c.threshold_own) else -1.0, c.mta, c.ia)
        factor_model = replace(model, base_grid=[float(t) for t in times[1:]])
    else:
        probe = gpu.compile(model, S.NettingSet([]), S.Options(factor_views=True))
        times = probe.times[probe.reporting.astype(np.int64)]
        report = np.arange(len(times))
    rows, specs = [], []
    for n, ns in enumerate(nets):
        for t in ns.trades:
            if isinstance(t, (S.Swap, S.Swap2)):
                sign = 1 if t.pay_fixed else -1
                mat = float((t.fixed_schedule if isinstance(t, S.Swap2) else t.schedule)[-1])
                rows.append((n, 0, 0, sign, t.notional, t.fixed_rate, mat, 0.0))
            elif isinstance(t, S.Forward):
                rows.append((n, 1, t.asset, 1, t.notional, t.strike, t.maturity, 0.0))
            elif isinstance(t, S.Option):
                rows.append((n, 2, t.asset, 1 if t.call else -1, t.notional, t.strike, t.expiry, 0.0))
            else:
                raise ValueError(f"the surrogate does not revalue {type(t).__name__}")
            specs.append(t)
    trades = np.array(rows, TRADE_DTYPE)
    nTr, nR = len(specs), len(times)
    resets = np.full((nTr, nR), -1, np.int32)
    periods = np.zeros((nTr, nR, 2), np.float32)
    for i, t in enumerate(specs):
        sch = _float_schedule(t)
        for k in range(1, len(sch)):
            ts, te = sch[k - 1], sch[k]
            live = (times >= ts - 1e-9) & (times < te - 1e-9)
            r = np.nonzero(np.abs(times - ts) < 1e-6)[0]
            if live.any() and len(r):
                resets[i, live] = r[0]
                periods[i, live] = (ts, te)
    return Book(model, nets, trades, specs, times.astype(np.float32), resets, periods, bond_features(model, trades, times, periods),
                report, csa_arr, call_index, factor_model)


def bond_features(model: S.Model, trades: np.ndarray, times: np.ndarray, periods: np.ndarray) -> np.ndarray:
    """[nTr][nR][4] = (ln A, B) of P(t, maturity | x) and of P(t, end of the running period | x) (the maturity where
    none runs) on every reporting date, from the Hull-White bond formula (hull_white.cpp:27-31): the network's
    features 14 and 15.  Past the end (t >= T) the bond is 1."""
    from .nested_exposure import zero_bonds

    nTr, nR = len(trades), len(times)
    t = np.broadcast_to(np.asarray(times, np.float64)[None, :], (nTr, nR))
    mat = np.broadcast_to(trades["maturity"].astype(np.float64)[:, None], (nTr, nR))
    nxt = np.where(periods[..., 1] > 0, periods[..., 1].astype(np.float64), mat)
    out = np.zeros((nTr, nR, 4), np.float32)
    for k, T in ((0, mat), (2, nxt)):
        live = T > t + 1e-9
        pairs = np.stack([t[live], T[live]], axis=1)
        c = zero_bonds(S.encode_model(model), pairs)
        out[..., k][live] = np.log(c[:, 0]) + c[:, 1]
        out[..., k + 1][live] = c[:, 2]
    return out


def factor_rows(ctx: gpu.Context, model: S.Model, paths: int) -> np.ndarray:
    """[2 + nA][nR][paths]: deflator, x and ln S of each FX factor on the reporting dates, from the plain
    kernels' factor views (the same scenario as every plan of the model)."""
    m = replace(model, num_paths=paths)
    p = gpu.compile(m, S.NettingSet([]), S.Options(factor_views=True))
    nR, nA = p.num_reporting, len(m.assets)
    _, _, rows = ctx.run(p, rows=True)
    out = np.zeros((2 + nA, nR, paths), np.float32)
    base = nR  # exposure rows first, then the deflator, x, a bond, then per asset level and deflated level
    out[0] = rows[base:base + nR]
    out[1] = rows[base + nR:base + 2 * nR]
    for a in range(nA):
        lvl = rows[base + (3 + 2 * a) * nR:base + (4 + 2 * a) * nR]
        out[2 + a] = np.log(np.maximum(lvl, 1e-30))
    return out


def plain_trade_values(ctx: gpu.Context, book: Book, paths: int) -> np.ndarray:
    """[nTr][nR][paths]: every trade revalued by the plain pricer (per-trade views of plans of <= 16 trades)."""
    m = replace(book.model, num_paths=paths)
    nR = len(book.times)
    out = np.zeros((len(book.specs), nR, paths), np.float32)
    at = 0
    for ns in book.netting_sets:
        for g0 in range(0, len(ns.trades), 16):
            group = ns.trades[g0:g0 + 16]
            p = gpu.compile(m, S.NettingSet(group, None), S.Options(trade_views=True))
            _, _, rows = ctx.run(p, rows=True)
            base = int(p.header[24])
            for i in range(len(group)):
                out[at + i] = rows[base + i * nR:base + (i + 1) * nR]
            at += len(group)
    return out


def features(ctx: gpu.Context, book: Book, factors: np.ndarray) -> np.ndarray:
    nA, nR, nP = factors.shape[0] - 2, factors.shape[1], factors.shape[2]
    nTr = len(book.specs)
    X = np.zeros((nTr, nR, nP, 16), np.float32)
    f = np.ascontiguousarray(factors, np.float32)
    check(lib().zk_surrogate_features(ctx.handle, f.ctypes.data, nA, nR, nP, book.times.ctypes.data, book.trades.ctypes.data,
                                      nTr, book.resets.ctypes.data, book.periods.ctypes.data, book.bonds.ctypes.data,
                                      X.ctypes.data), ctx.handle)
    return X


def training_set(ctx: gpu.Context, book: Book, paths: int, seed: int = 1):
    """Inputs and per-unit-notional targets of every (trade, reporting date, path) on `paths` paths, with the
    rows past each trade's maturity left out (their value is zero by construction).  The book must be the
    uncollateralised one (a network trained on it revalues the same trades in the CSA book)."""
    if book.csa is not None:
        raise ValueError("train on the uncollateralised book (make_book without csa)")
    fac = factor_rows(ctx, book.model, paths)
    X = features(ctx, book, fac)
    V = plain_trade_values(ctx, book, paths) / book.trades["notional"][:, None, None]
    live = book.times[None, :] < book.trades["maturity"][:, None] - 1e-6
    X, y = X[live].reshape(-1, 16), V[live].reshape(-1)
    # The rows come trade by trade; mini-batches must mix trades, dates and paths.
    order = np.random.default_rng(seed).permutation(len(y))
    return X[order], y[order]


def surrogate_exposure(sur, book: Book, factors: np.ndarray, paths_out: int = 0, all_dates: bool = False):
    """(EE, EE*) [numNs][nR] from zk_surrogate_book on the reporting dates, the netted values (with a CSA: value minus
    collateral) of the first paths_out paths, and the device milliseconds; all_dates keeps every revalued date."""
    nA, nR, nP = factors.shape[0] - 2, factors.shape[1], factors.shape[2]
    nNs = len(book.netting_sets)
    exp = np.zeros((nNs, nR, 2))
    net = np.zeros((nNs, nR, max(paths_out, 1)), np.float32)
    ms = np.zeros(2, np.float32)
    f = np.ascontiguousarray(factors, np.float32)
    csa = None if book.csa is None else np.ascontiguousarray(book.csa, np.float32)
    call = None if book.csa is None else np.ascontiguousarray(book.call_index, np.uint32)
    check(lib().zk_surrogate_book(sur.handle, f.ctypes.data, nA, nR, nP, book.times.ctypes.data, book.trades.ctypes.data,
                                  len(book.specs), book.resets.ctypes.data, book.periods.ctypes.data, book.bonds.ctypes.data,
                                  nNs, None if csa is None else csa.ctypes.data, None if call is None else call.ctypes.data,
                                  exp.ctypes.data,
                                  net.ctypes.data if paths_out else None, paths_out, ms.ctypes.data), sur.ctx.handle)
    r = np.arange(nR) if all_dates else book.report  # (EE, EE*) and the audit paths' values on the reporting dates
    return exp[:, r, 0], exp[:, r, 1], net[:, r, :paths_out], ms


def plain_exposure(ctx: gpu.Context, book: Book, paths: int, netting_sets=None):
    """(EE, EE*) [numNs][nR] of the plain pricer, from the fused kernels' statistics, and their device ms."""
    m = replace(book.model, num_paths=paths)
    idx = range(len(book.netting_sets)) if netting_sets is None else netting_sets
    plans = [gpu.compile(m, book.netting_sets[i], S.Options()) for i in idx]
    b = ctx.batch(plans)
    try:
        b.execute()
        out = b.read()
        ms = float(np.sum(b.timings()))
    finally:
        b.close()
    rep = [p.reporting.astype(np.int64) for p in plans]
    ee = np.array([s.reshape(-1, p.stats_per_date)[r, 1] for (s, _), p, r in zip(out, plans, rep)], np.float64)
    dee = np.array([s.reshape(-1, p.stats_per_date)[r, 3] for (s, _), p, r in zip(out, plans, rep)], np.float64)
    return ee, dee, ms


def cva(book: Book, dee: np.ndarray) -> np.ndarray:
    c = book.model.credits[0]
    t = book.report_times
    return np.array([unilateral_cva(t, d, c.pillars, c.hazards, 1.0 - LGD) for d in dee])


@dataclass
class AuditedRun:
    ee: np.ndarray
    dee: np.ndarray
    cva: np.ndarray
    fallback: List[int]
    audit_error: np.ndarray
    ms_surrogate: float
    ms_audit: float
    ms_fallback: float


def audited_exposure(ctx: gpu.Context, sur, book: Book, paths: int, audit_fraction: float = 0.01) -> AuditedRun:
    """Surrogate revaluation of the book on `paths` paths, audited by the plain pricer on the first
    audit_fraction of them; netting sets beyond AUDIT_TOLERANCE are revalued by the plain pricer."""
    fac = factor_rows(ctx, book.factor_model or book.model, paths)
    nAudit = max(128, int(round(paths * audit_fraction)))
    ee, dee, net_a, ms = surrogate_exposure(sur, book, fac, paths_out=nAudit)
    # Audit: the plain pricer's EPE on the audit paths against the surrogate's on the same paths.
    pe, _, ms_audit = plain_exposure(ctx, book, nAudit)
    se = np.maximum(net_a, 0.0).mean(axis=2)
    dt = np.diff(book.report_times, prepend=0.0)
    epe_p = (pe * dt).sum(1) / max(dt.sum(), 1e-12)
    epe_s = (se * dt).sum(1) / max(dt.sum(), 1e-12)
    err = np.abs(epe_s - epe_p) / np.maximum(epe_p, 1e-12)
    fallback = [int(i) for i in np.nonzero(err > AUDIT_TOLERANCE)[0]]
    ms_fb = 0.0
    if fallback:
        fe, fd, ms_fb = plain_exposure(ctx, book, paths, fallback)
        ee[fallback], dee[fallback] = fe, fd
    return AuditedRun(ee, dee, cva(book, dee), fallback, err, float(ms[0] + ms[1]), ms_audit, ms_fb)
