"""Flat encodings of a market model, a netting set and the fused-pipeline options.

The reference builds a netting set from C++ objects (``ExposureEngine``, ``NettingSet``,
``gpu::FusedOptions``; include/ccr/gpu/fused_exposure.hpp:293-329 and
include/ccr/exposure/exposure_engine.hpp:19-66).  Across a C ABI those objects travel as three
float64 arrays with the layouts below; the plan compiler of this package
(``zk_compile``) and the reference wrapper used by the tests decode the same arrays.

Model block::

    7001, nCurve, (t, r) * nCurve, hwA, hwSigma,
    nAssets, per asset (spot, vol, nCarry, (t, r) * nCarry),
    nCredits, per credit (kappa, theta, xi, y0, substeps, nHaz, (pillar, hazard) * nHaz),
    F, F * F correlation (row-major; F = 0 means identity),
    numPaths, seed, antithetic, nBase, base grid times,
    [7011, nForeign, (a, sigma) * nForeign]   only when assets carry a stochastic foreign rate (an extension)

    The factors are ordered [domestic rate, assets, credits, foreign rates]; foreign rate f belongs to asset f,
    so the assets with a stochastic foreign rate come first.

Netting-set block::

    7002, nTrades, per trade (type, fields), hasCsa, [csa fields]
    type 0 swap:      notional, fixedRate, payFixed, nSched, schedule
    type 1 forward:   asset, notional, strike, maturity
    type 2 option:    asset, isCall, notional, strike, expiry
    type 3 bermudan:  notional, fixedRate, payFixed, nSched, schedule, nEx, exercise, physical, position, degree
    type 4 swap with separate legs (an extension; see Swap2): notional, fixedRate, payFixed,
                      nFixed, fixed schedule, nFloat, float schedule
    csa: thresholdCounterparty, thresholdOwn (< 0: none), mta, ia, mpr, type (0 cash, 1 bond, 2 asset),
         haircut, bondMaturity, assetIndex

Options block::

    7003, pfeQuantile, counterparty, perTrade, imQuantile, imInnerPaths, imMarginPeriod,
    imAuditPaths, imAuditInnerPaths, samples, histogramTime, histogramBins, gross,
    collateralBands, tradeViews, exerciseViews, factorViews, bondMaturity,
    nExtra, extraDates, nBand, bandLevels, nFactorBand, factorBandLevels
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Union

import numpy as np

MODEL_MAGIC = 7001.0
FOREIGN_MAGIC = 7011.0
NETTING_MAGIC = 7002.0
OPTIONS_MAGIC = 7003.0


@dataclass
class Curve:
    """Continuously compounded zero curve, linear in the zero rate with flat ends
    (src/market/yield_curve.cpp:20-27)."""

    times: Sequence[float]
    rates: Sequence[float]

    @staticmethod
    def flat(rate: float) -> "Curve":
        return Curve([1.0], [rate])


@dataclass
class Asset:
    """Lognormal FX / equity factor (include/ccr/models/lognormal_asset.hpp:17-41).  The reference's foreign (carry)
    curve is deterministic; with rate_a > 0 the foreign currency's short rate is a Hull-White factor of its own
    (mean reversion rate_a, volatility rate_sigma) fitted to the carry curve: an extension with no counterpart in
    the reference."""

    spot: float
    vol: float
    carry: Curve
    rate_a: float = 0.0
    rate_sigma: float = 0.0

    @property
    def stochastic_rate(self) -> bool:
        return self.rate_a > 0.0


@dataclass
class Credit:
    """CIR++ intensity on a piecewise-flat market hazard curve
    (include/ccr/models/cir_intensity.hpp:22-53, src/market/credit_curve.cpp:23-41)."""

    kappa: float
    theta: float
    xi: float
    y0: float
    pillars: Sequence[float]
    hazards: Sequence[float]
    substeps: int = 8


@dataclass
class Model:
    curve: Curve
    hw_a: float
    hw_sigma: float
    assets: List[Asset] = field(default_factory=list)
    credits: List[Credit] = field(default_factory=list)
    correlation: Optional[np.ndarray] = None
    num_paths: int = 1000
    seed: int = 42
    antithetic: bool = True
    base_grid: Sequence[float] = (0.0,)

    @property
    def num_foreign(self) -> int:
        """Assets with a stochastic foreign rate (they come first)."""
        n = 0
        while n < len(self.assets) and self.assets[n].stochastic_rate:
            n += 1
        if any(a.stochastic_rate for a in self.assets[n:]):
            raise ValueError("the assets with a stochastic foreign rate must come first")
        return n

    @property
    def num_factors(self) -> int:
        return 1 + len(self.assets) + len(self.credits) + self.num_foreign


@dataclass
class Swap:
    """Fixed-vs-floating swap on one schedule for both legs
    (include/ccr/instruments/interest_rate_swap.hpp:10-57)."""

    notional: float
    fixed_rate: float
    pay_fixed: bool
    schedule: Sequence[float]


@dataclass
class Swap2:
    """Swap whose fixed and floating legs have their own schedules (annual fixed against
    semiannual floating, say).  Its value is linear in the legs, so it equals three one-schedule
    swaps: float(K=0, float schedule) + [swap(K, fixed schedule) - swap(0, fixed schedule)]."""

    notional: float
    fixed_rate: float
    pay_fixed: bool
    fixed_schedule: Sequence[float]
    float_schedule: Sequence[float]


@dataclass
class Forward:
    asset: int
    notional: float
    strike: float
    maturity: float


@dataclass
class Option:
    asset: int
    call: bool
    notional: float
    strike: float
    expiry: float


@dataclass
class Bermudan:
    """basis: "rate", the reference's Longstaff-Schwartz regression on the short-rate state; "rate_swap", this
    library's two-regressor basis -- the graded monomials of total degree <= `degree` in the short rate and the
    co-terminal swap rate (the swap from the next exercise date to maturity), an extension with no reference
    counterpart (encoded as degree + 10)."""
    swap: Swap
    exercise: Sequence[float]
    physical: bool = True
    position: float = 1.0
    degree: int = 3
    basis: str = "rate"


Trade = Union[Swap, Swap2, Forward, Option, Bermudan]


@dataclass
class Csa:
    """Collateral agreement (include/ccr/exposure/collateral.hpp:14-41)."""

    threshold_cpty: float = 0.0
    threshold_own: float = float("inf")
    mta: float = 0.0
    ia: float = 0.0
    mpr: float = 10.0 / 250.0
    kind: int = 0  # 0 cash, 1 bond, 2 asset
    haircut: float = 0.0
    bond_maturity: float = 0.0
    asset_index: int = 0


@dataclass
class NettingSet:
    trades: List[Trade] = field(default_factory=list)
    csa: Optional[Csa] = None


@dataclass
class Options:
    """The fused-pipeline options (include/ccr/gpu/fused_exposure.hpp:293-329)."""

    pfe_quantile: float = 0.95
    counterparty: int = 0
    per_trade: bool = False
    im_quantile: float = 0.0
    im_inner_paths: int = 0
    im_margin_period: float = 10.0 / 250.0
    im_audit_paths: int = 0
    im_audit_inner_paths: int = 1024
    samples: int = 0
    histogram_time: float = -1.0
    histogram_bins: int = 40
    gross: bool = False
    collateral_bands: bool = False
    trade_views: bool = False
    exercise_views: bool = False
    factor_views: bool = False
    bond_maturity: float = 0.0
    extra_dates: Sequence[float] = ()
    band_levels: Sequence[float] = (0.05, 0.5, 0.95)
    factor_band_levels: Sequence[float] = (0.05, 0.25, 0.5, 0.75, 0.95)


def _curve(out: list, c: Curve) -> None:
    assert len(c.times) == len(c.rates) and len(c.times) > 0
    out.append(float(len(c.times)))
    for t, r in zip(c.times, c.rates):
        out += [float(t), float(r)]


def encode_model(m: Model) -> np.ndarray:
    out: list = [MODEL_MAGIC]
    _curve(out, m.curve)
    out += [float(m.hw_a), float(m.hw_sigma), float(len(m.assets))]
    for a in m.assets:
        out += [float(a.spot), float(a.vol)]
        _curve(out, a.carry)
    out.append(float(len(m.credits)))
    for c in m.credits:
        out += [float(c.kappa), float(c.theta), float(c.xi), float(c.y0), float(c.substeps), float(len(c.pillars))]
        for p, h in zip(c.pillars, c.hazards):
            out += [float(p), float(h)]
    if m.correlation is None:
        out.append(0.0)
    else:
        corr = np.asarray(m.correlation, dtype=np.float64)
        f = m.num_factors
        assert corr.shape == (f, f), f"correlation must be {f}x{f}"
        out.append(float(f))
        out += [float(v) for v in corr.reshape(-1)]
    out += [float(m.num_paths), float(m.seed), 1.0 if m.antithetic else 0.0, float(len(m.base_grid))]
    out += [float(t) for t in m.base_grid]
    nf = m.num_foreign
    if nf:
        out += [FOREIGN_MAGIC, float(nf)]
        for a in m.assets[:nf]:
            out += [float(a.rate_a), float(a.rate_sigma)]
    return np.asarray(out, dtype=np.float64)


def _schedule(out: list, s: Sequence[float]) -> None:
    out.append(float(len(s)))
    out += [float(t) for t in s]


def encode_netting_set(ns: NettingSet) -> np.ndarray:
    out: list = [NETTING_MAGIC, float(len(ns.trades))]
    for t in ns.trades:
        if isinstance(t, Swap):
            out += [0.0, float(t.notional), float(t.fixed_rate), 1.0 if t.pay_fixed else 0.0]
            _schedule(out, t.schedule)
        elif isinstance(t, Forward):
            out += [1.0, float(t.asset), float(t.notional), float(t.strike), float(t.maturity)]
        elif isinstance(t, Option):
            out += [2.0, float(t.asset), 1.0 if t.call else 0.0, float(t.notional), float(t.strike), float(t.expiry)]
        elif isinstance(t, Bermudan):
            s = t.swap
            out += [3.0, float(s.notional), float(s.fixed_rate), 1.0 if s.pay_fixed else 0.0]
            _schedule(out, s.schedule)
            _schedule(out, t.exercise)
            if t.basis not in ("rate", "rate_swap"):
                raise ValueError(f"Bermudan basis {t.basis!r}: 'rate' or 'rate_swap'")
            out += [1.0 if t.physical else 0.0, float(t.position), float(t.degree + (10 if t.basis == "rate_swap" else 0))]
        elif isinstance(t, Swap2):
            out += [4.0, float(t.notional), float(t.fixed_rate), 1.0 if t.pay_fixed else 0.0]
            _schedule(out, t.fixed_schedule)
            _schedule(out, t.float_schedule)
        else:  # pragma: no cover - programming error
            raise TypeError(f"unknown trade {t!r}")
    if ns.csa is None:
        out.append(0.0)
    else:
        c = ns.csa
        own = -1.0 if not np.isfinite(c.threshold_own) else float(c.threshold_own)
        out += [1.0, float(c.threshold_cpty), own, float(c.mta), float(c.ia), float(c.mpr), float(c.kind),
                float(c.haircut), float(c.bond_maturity), float(c.asset_index)]
    return np.asarray(out, dtype=np.float64)


def bermudan_degrees(ns_array: np.ndarray) -> List[int]:
    """The regression degree of each Bermudan of an encoded netting set, in trade order (for either basis)."""
    a = np.asarray(ns_array, np.float64)
    i, out = 2, []
    for _ in range(int(a[1])):
        kind = int(a[i])
        if kind == 0:
            i += 4
            i += 1 + int(a[i])
        elif kind == 1:
            i += 5
        elif kind == 2:
            i += 6
        elif kind == 3:
            i += 4
            i += 1 + int(a[i])
            i += 1 + int(a[i])
            out.append(int(a[i + 2]) % 10)  # the two-regressor basis adds 10 (the plan's records carry it)
            i += 3
        elif kind == 4:
            i += 4
            i += 1 + int(a[i])
            i += 1 + int(a[i])
        else:
            raise ValueError(f"netting set: unknown trade type {kind}")
    return out


def encode_options(o: Options) -> np.ndarray:
    out = [OPTIONS_MAGIC, o.pfe_quantile, o.counterparty, float(o.per_trade), o.im_quantile, o.im_inner_paths,
           o.im_margin_period, o.im_audit_paths, o.im_audit_inner_paths, o.samples, o.histogram_time,
           o.histogram_bins, float(o.gross), float(o.collateral_bands), float(o.trade_views),
           float(o.exercise_views), float(o.factor_views), o.bond_maturity]
    for seq in (o.extra_dates, o.band_levels, o.factor_band_levels):
        out.append(float(len(seq)))
        out += [float(v) for v in seq]
    return np.asarray(out, dtype=np.float64)


def decode_options(a) -> Options:
    """The inverse of encode_options."""
    a = [float(v) for v in a]
    if not a or a[0] != OPTIONS_MAGIC:
        raise ValueError("options: bad magic")
    o = Options(pfe_quantile=a[1], counterparty=int(a[2]), per_trade=bool(a[3]), im_quantile=a[4], im_inner_paths=int(a[5]),
                im_margin_period=a[6], im_audit_paths=int(a[7]), im_audit_inner_paths=int(a[8]), samples=int(a[9]),
                histogram_time=a[10], histogram_bins=int(a[11]), gross=bool(a[12]), collateral_bands=bool(a[13]),
                trade_views=bool(a[14]), exercise_views=bool(a[15]), factor_views=bool(a[16]), bond_maturity=a[17])
    i = 18
    seqs = []
    for _ in range(3):
        n = int(a[i])
        seqs.append(tuple(a[i + 1:i + 1 + n]))
        i += 1 + n
    o.extra_dates, o.band_levels, o.factor_band_levels = seqs
    return o


def expand_swap2(t: Swap2) -> List[Swap]:
    """The three one-schedule swaps whose sum is a two-schedule swap (linear in the legs)."""
    return [Swap(t.notional, 0.0, t.pay_fixed, t.float_schedule),
            Swap(t.notional, t.fixed_rate, t.pay_fixed, t.fixed_schedule),
            Swap(t.notional, 0.0, not t.pay_fixed, t.fixed_schedule)]


def vanilla_schedule(start: float, tenor: float, per_year: int) -> List[float]:
    """InterestRateSwap::vanilla's schedule (src/instruments/interest_rate_swap.cpp:27-35)."""
    periods = int(round(tenor * per_year))
    s = [start + i / per_year for i in range(periods + 1)]
    s[-1] = start + tenor
    return s
