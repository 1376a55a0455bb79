"""Netting sets and models used across the tests.

``gpu_setup`` is the set-up of the reference's own GPU tests (tests/test_gpu.cpp:27-55): a rising
curve, HW(0.05, 0.01), one FX asset, one CIR++ credit with 4 sub-steps, a 5y payer swap, an FX
forward and a short FX call, optionally under a two-way CSA.
"""
from __future__ import annotations

import numpy as np

from zlatko_b200 import spec as S


def standard_exposure_grid(horizon: float):
    """TimeGrid::standardExposureGrid (src/core/time_grid.cpp:28-37): weekly to 3m, monthly to 1y, then quarterly."""
    t = [w * 7.0 / 365.0 for w in range(1, 14)] + [m / 12.0 for m in range(4, 13)]
    q = 1.25
    while q < horizon + 1e-9:
        t.append(q)
        q += 0.25
    t = [x for x in t if x <= horizon]
    t.append(horizon)
    return t


def gpu_model(paths: int, seed: int = 7) -> S.Model:
    return S.Model(curve=S.Curve([1.0, 10.0], [0.02, 0.03]), hw_a=0.05, hw_sigma=0.01,
                   assets=[S.Asset(1.1, 0.12, S.Curve.flat(0.01))],
                   credits=[S.Credit(0.4, 0.02, 0.1, 0.02, [1.0], [0.02], substeps=4)],
                   correlation=np.array([[1.0, 0.2, 0.0], [0.2, 1.0, 0.0], [0.0, 0.0, 1.0]]),
                   num_paths=paths, seed=seed, antithetic=True, base_grid=standard_exposure_grid(5.0))


def gpu_netting_set(csa: bool) -> S.NettingSet:
    trades = [S.Swap(1e6, 0.028, True, S.vanilla_schedule(0.0, 5.0, 2)), S.Forward(0, 5e5, 1.12, 3.0),
              S.Option(0, True, -4e5, 1.15, 2.0)]
    return S.NettingSet(trades, S.Csa(2e4, 2e4, 5e3) if csa else None)


def gpu_setup(paths: int, csa: bool):
    return gpu_model(paths), gpu_netting_set(csa)


def bermudan(notional=1e6, fixed=0.03, pay=False, start=1.0, tenor=4.0, exercise=(1.0, 2.0, 3.0), physical=True,
             position=1.0, degree=3, basis="rate") -> S.Bermudan:
    return S.Bermudan(S.Swap(notional, fixed, pay, S.vanilla_schedule(start, tenor, 1)), list(exercise), physical, position, degree,
                      basis)


def swap_book(n: int, seed: int = 20261203, horizon_months: int = 60, csa=None) -> S.NettingSet:
    """n swaps with N ~ U[1e6, 1e7], K ~ U[1%, 4%], payer / receiver 50/50, maturity U[1y, 5y] rounded to whole
    months, annual fixed and semiannual floating legs (schedules built back from the maturity)."""
    rng = np.random.default_rng(seed)
    trades = []
    for _ in range(n):
        notional = rng.uniform(1e6, 1e7)
        k = rng.uniform(0.01, 0.04)
        pay = bool(rng.random() < 0.5)
        months = int(round(rng.uniform(12, horizon_months)))
        trades.append(S.Swap2(notional, k, pay, back_schedule(months, 12), back_schedule(months, 6)))
    return S.NettingSet(trades, csa)


def back_schedule(months: int, step: int):
    """Dates from 0 to `months` months, every `step` months counted back from the end (a short first period)."""
    dates = list(range(months, 0, -step))[::-1]
    return [0.0] + [d / 12.0 for d in dates]
