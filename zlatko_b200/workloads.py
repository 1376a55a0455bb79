"""Seeded synthetic workloads of the benchmark configurations (no public dataset exists for this path).

swap_portfolio: one uncollateralised netting set of 20 swaps under HW(0.03, 0.01) on a flat 2% curve,
    notionals U[1e6, 1e7], fixed rates U[1%, 4%], payer / receiver 50/50, maturities U[1y, 5y],
    annual fixed and semiannual floating legs, 10,000 paths on 60 monthly dates, PFE 97.5%,
    counterparty hazard 1% (CVA with LGD 0.6).
correlated_csa_book: 1,000 trades (600 swaps, 300 FX forwards, 100 FX options) in 100 netting sets of
    Zipf(1.2) sizes, each under a two-way CSA (threshold U[0, 5e6], MTA 1e5, MPR 10/250), 100,000
    paths on 120 monthly dates to 10y, HW(a, sigma) with a ~ U[0.01, 0.1], sigma ~ U[0.005, 0.015],
    2 lognormal FX rates (vol U[8%, 15%]) and one CIR++ intensity (kappa 0.5, theta 0.02, xi 0.08)
    joined by a correlation with off-diagonals U[-0.3, 0.5] projected to the nearest positive
    definite matrix.  The two foreign currencies have Hull-White short rates of their own on flat
    curves drawn U[0%, 4%] (the configuration's three currencies); with foreign_rates=False they
    are the reference's deterministic carry curves instead.

xva_batch: the large wrong-way-risk XVA batch -- 10,000 trades (60% swaps, 25% FX forwards, 10% FX options, 5%
    Bermudan swaptions) in 500 netting sets of Zipf(1.1) sizes spread over 8 portfolios, on the correlated book's
    three-currency model with the intensity correlated 0.3 with the domestic short rate, monthly to 10y; each
    netting set with and without its CSA.

Cash-flow and maturity dates are whole months, so every event date falls on the monthly grid.
Draws use numpy's PCG64 seeded with 20261203 (portfolio) and the simulation seed 42.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from . import spec as S

PORTFOLIO_SEED = 20261203
SIM_SEED = 42


def back_schedule(months: int, step: int) -> List[float]:
    """0 and every `step` months counted back from maturity (a short first period)."""
    dates = list(range(months, 0, -step))[::-1]
    return [0.0] + [d / 12.0 for d in dates]


def random_swap(rng: np.random.Generator, max_months: int) -> S.Swap2:
    notional = rng.uniform(1e6, 1e7)
    k = rng.uniform(0.01, 0.04)
    pay = bool(rng.random() < 0.5)
    months = int(round(rng.uniform(12, max_months)))
    return S.Swap2(notional, k, pay, back_schedule(months, 12), back_schedule(months, 6))


def nearest_correlation(c: np.ndarray, floor: float = 1e-6, iters: int = 200) -> np.ndarray:
    """Nearest correlation matrix by alternating projections (Higham 2002): symmetric positive definite
    (eigenvalues >= floor) with a unit diagonal."""
    y = c.copy()
    ds = np.zeros_like(c)
    for _ in range(iters):
        r = y - ds
        w, v = np.linalg.eigh((r + r.T) / 2)
        x = (v * np.maximum(w, floor)) @ v.T
        ds = x - r
        y = x.copy()
        np.fill_diagonal(y, 1.0)
    w, v = np.linalg.eigh((y + y.T) / 2)
    y = (v * np.maximum(w, floor)) @ v.T
    d = np.sqrt(np.diag(y))
    y = y / np.outer(d, d)
    np.fill_diagonal(y, 1.0)
    return (y + y.T) / 2


def zipf_sizes(total: int, groups: int, s: float) -> List[int]:
    w = np.arange(1, groups + 1, dtype=np.float64) ** (-s)
    raw = total * w / w.sum()
    sizes = np.maximum(1, np.floor(raw).astype(int))
    rest = total - sizes.sum()
    order = np.argsort(-(raw - np.floor(raw)))
    for k in range(abs(rest)):
        sizes[order[k % groups]] += 1 if rest > 0 else -1
    return [int(x) for x in sizes]


def swap_portfolio(paths: int = 10_000) -> Tuple[S.Model, S.NettingSet, S.Options]:
    rng = np.random.default_rng(PORTFOLIO_SEED)
    m = S.Model(curve=S.Curve.flat(0.02), hw_a=0.03, hw_sigma=0.01,
                credits=[S.Credit(1e-6, 0.0, 0.0, 0.0, [1.0], [0.01], substeps=1)],
                num_paths=paths, seed=SIM_SEED, antithetic=True, base_grid=[k / 12.0 for k in range(1, 61)])
    ns = S.NettingSet([random_swap(rng, 60) for _ in range(20)])
    return m, ns, S.Options(pfe_quantile=0.975)


def correlated_csa_book(paths: int = 100_000, netting_sets: int = 100, num_trades: int = 1000,
                        foreign_rates: bool = True) -> Tuple[S.Model, List[S.NettingSet], S.Options, int]:
    """Returns (model, netting sets, options, number of trades).  num_trades keeps the 60/30/10 mix of swaps,
    FX forwards and FX options.  With foreign_rates the two foreign currencies have Hull-White short rates of
    their own (a ~ U[0.01, 0.1], sigma ~ U[0.005, 0.015]) on their carry curves, and the full 6 x 6
    correlation joins domestic rate, foreign rates, FX and the intensity: the configuration's three-currency
    model.  Without, the reference's model family: deterministic foreign curves, the 4 x 4 block of the
    simulated factors.  The trades are the same either way."""
    rng = np.random.default_rng(PORTFOLIO_SEED + 1)
    a, sigma = rng.uniform(0.01, 0.1), rng.uniform(0.005, 0.015)
    fx = [S.Asset(spot, rng.uniform(0.08, 0.15), S.Curve.flat(rng.uniform(0.0, 0.04))) for spot in (1.1, 0.9)]
    credit = S.Credit(0.5, 0.02, 0.08, 0.02, [1.0], [0.01], substeps=8)
    c6 = np.eye(6)
    iu = np.triu_indices(6, 1)
    c6[iu] = rng.uniform(-0.3, 0.5, size=len(iu[0]))
    c6 = np.triu(c6) + np.triu(c6, 1).T
    c6 = nearest_correlation(c6)
    # c6 joins [domestic rate, foreign rate 1, foreign rate 2, FX 1, FX 2, intensity]; the model orders its
    # factors [rate, assets, credits, foreign rates].
    keep = [0, 3, 4, 5, 1, 2] if foreign_rates else [0, 3, 4, 5]
    corr = c6[np.ix_(keep, keep)]
    m = S.Model(curve=S.Curve.flat(0.02), hw_a=a, hw_sigma=sigma, assets=fx, credits=[credit], correlation=corr,
                num_paths=paths, seed=SIM_SEED, antithetic=True, base_grid=[k / 12.0 for k in range(1, 121)])
    n_swaps, n_fwds = round(0.6 * num_trades), round(0.3 * num_trades)
    n_opts = num_trades - n_swaps - n_fwds
    trades: list = [random_swap(rng, 120) for _ in range(n_swaps)]
    for _ in range(n_fwds):
        asset = int(rng.integers(0, 2))
        months = int(rng.integers(3, 61))
        spot = fx[asset].spot
        trades.append(S.Forward(asset, rng.choice([-1.0, 1.0]) * rng.uniform(1e6, 1e7), spot * rng.uniform(0.9, 1.1), months / 12.0))
    for _ in range(n_opts):
        asset = int(rng.integers(0, 2))
        months = int(rng.integers(3, 37))
        spot = fx[asset].spot
        trades.append(S.Option(asset, bool(rng.random() < 0.5), rng.choice([-1.0, 1.0]) * rng.uniform(1e6, 5e6),
                               spot * rng.uniform(0.9, 1.1), months / 12.0))
    order = rng.permutation(len(trades))
    sizes = zipf_sizes(len(trades), netting_sets, 1.2)
    books, at = [], 0
    for n in sizes:
        t = rng.uniform(0.0, 5e6)
        books.append(S.NettingSet([trades[i] for i in order[at:at + n]], S.Csa(t, t, 1e5, 0.0, 10.0 / 250.0)))
        at += n
    foreign = [(rng.uniform(0.01, 0.1), rng.uniform(0.005, 0.015)) for _ in fx]  # drawn last: the trades do not move
    if foreign_rates:
        for asset, (fa, fs) in zip(fx, foreign):
            asset.rate_a, asset.rate_sigma = fa, fs
    return m, books, S.Options(pfe_quantile=0.975), len(trades)


def bermudan_book(paths: int = 200_000, bermudans: int = 200, basis: str = "rate") -> Tuple[S.Model, List[S.NettingSet], int]:
    """The AMC workload: `bermudans` Bermudan swaptions under Hull-White (a = 0.03, sigma = 0.01) on a flat 2%
    curve, each on a 10y annual swap with annual exercise from year 1 to year 9, strike at the at-the-money rate
    +- 100bp (uniform), notional 1e7, payer / receiver 50/50, degree-3 regressions -- in the short-rate state
    (basis "rate", the reference's) or in the short rate and the co-terminal swap rate (basis "rate_swap", the
    10-function two-regressor basis); four per netting set, uncollateralised; quarterly dates to 10y (40 exposure
    dates).  Returns (model, netting sets, number of Bermudans)."""
    rng = np.random.default_rng(PORTFOLIO_SEED + 2)
    m = S.Model(curve=S.Curve.flat(0.02), hw_a=0.03, hw_sigma=0.01, num_paths=paths, seed=SIM_SEED, antithetic=True,
                base_grid=[k / 4.0 for k in range(1, 41)])
    atm = float(np.expm1(0.02))  # annual par rate of the flat continuously compounded 2% curve
    trades = []
    for _ in range(bermudans):
        k = atm + rng.uniform(-0.01, 0.01)
        pay = bool(rng.random() < 0.5)
        trades.append(S.Bermudan(S.Swap(1e7, k, pay, S.vanilla_schedule(0.0, 10.0, 1)), [float(e) for e in range(1, 10)],
                                 physical=True, position=1.0, degree=3, basis=basis))
    books = [S.NettingSet(trades[i:i + 4], None) for i in range(0, bermudans, 4)]
    return m, books, bermudans


def nested_netting_set(seed: int = PORTFOLIO_SEED + 7, swaps: int = 20, forwards: int = 8, options: int = 4) -> S.NettingSet:
    """A netting set of the trades the nested exposure supports (src/nested/nested_exposure.cpp:59-82): one-schedule
    swaps (semiannual, 1-5y), FX forwards (3m-5y) and FX options (3m-3y) on the correlated book's two FX factors."""
    rng = np.random.default_rng(seed)
    trades: list = []
    for _ in range(swaps):
        months = int(rng.integers(12, 61)) // 6 * 6
        sched = [k / 12.0 for k in range(0, months + 1, 6)]
        trades.append(S.Swap(rng.uniform(1e6, 1e7), rng.uniform(0.01, 0.04), bool(rng.random() < 0.5), sched))
    for _ in range(forwards):
        asset = int(rng.integers(0, 2))
        trades.append(S.Forward(asset, rng.choice([-1.0, 1.0]) * rng.uniform(1e6, 5e6), (1.1, 0.9)[asset] * rng.uniform(0.9, 1.1),
                                int(rng.integers(3, 61)) / 12.0))
    for _ in range(options):
        asset = int(rng.integers(0, 2))
        trades.append(S.Option(asset, bool(rng.random() < 0.5), rng.choice([-1.0, 1.0]) * rng.uniform(1e6, 3e6),
                               (1.1, 0.9)[asset] * rng.uniform(0.9, 1.1), int(rng.integers(3, 37)) / 12.0))
    return S.NettingSet(trades, None)


def xva_batch(paths: int = 1_000_000, num_trades: int = 10_000, netting_sets: int = 500, portfolios: int = 8,
              rate_intensity_correlation: float = 0.3):
    """Returns (model, collateralised netting sets, uncollateralised netting sets, portfolio of each netting set,
    number of trades).  The model is the correlated book's (three Hull-White currencies, two FX rates, CIR++)
    with the correlation of the domestic rate and the intensity set to 0.3 and the matrix projected to the nearest
    correlation matrix.  Swaps, forwards and options are drawn as in the correlated book, Bermudans as in the AMC
    book (10y annual swaps, exercise annually from 1y, strike ATM +- 100bp); netting set sizes Zipf(1.1); CSA
    threshold U[0, 5e6], MTA 1e5, MPR 10 business days; netting set k belongs to portfolio k mod 8."""
    m, _, _, _ = correlated_csa_book(paths)
    c = np.asarray(m.correlation, dtype=np.float64).copy()
    credit = 1 + len(m.assets)  # factor order [rate, assets, credits, foreign rates]
    c[0, credit] = c[credit, 0] = rate_intensity_correlation
    m.correlation = nearest_correlation(c)
    rng = np.random.default_rng(PORTFOLIO_SEED + 4)
    n_swaps, n_fwds, n_opts = round(0.6 * num_trades), round(0.25 * num_trades), round(0.1 * num_trades)
    n_berm = num_trades - n_swaps - n_fwds - n_opts
    fx = m.assets
    trades: list = [random_swap(rng, 120) for _ in range(n_swaps)]
    for _ in range(n_fwds):
        a = int(rng.integers(0, 2))
        trades.append(S.Forward(a, rng.choice([-1.0, 1.0]) * rng.uniform(1e6, 1e7), fx[a].spot * rng.uniform(0.9, 1.1),
                                int(rng.integers(3, 61)) / 12.0))
    for _ in range(n_opts):
        a = int(rng.integers(0, 2))
        trades.append(S.Option(a, bool(rng.random() < 0.5), rng.choice([-1.0, 1.0]) * rng.uniform(1e6, 5e6),
                               fx[a].spot * rng.uniform(0.9, 1.1), int(rng.integers(3, 37)) / 12.0))
    atm = float(np.expm1(0.02))
    for _ in range(n_berm):
        k = atm + rng.uniform(-0.01, 0.01)
        trades.append(S.Bermudan(S.Swap(1e7, k, bool(rng.random() < 0.5), S.vanilla_schedule(0.0, 10.0, 1)),
                                 [float(e) for e in range(1, 10)], physical=True, position=1.0, degree=3))
    order = rng.permutation(len(trades))
    sizes = zipf_sizes(len(trades), netting_sets, 1.1)
    csa_books, plain_books, at = [], [], 0
    for n in sizes:
        t = rng.uniform(0.0, 5e6)
        chosen = [trades[i] for i in order[at:at + n]]
        csa_books.append(S.NettingSet(chosen, S.Csa(t, t, 1e5, 0.0, 10.0 / 250.0)))
        plain_books.append(S.NettingSet(list(chosen), None))
        at += n
    portfolio = [k % portfolios for k in range(netting_sets)]
    return m, csa_books, plain_books, portfolio, len(trades)
