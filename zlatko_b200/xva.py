"""The valuation adjustments on top of the exposure profiles and their allocation to trades.

Restates src/xva/xva.cpp (CVA, DVA, FCA, FBA, MVA, KVA of a profile, the simulated initial-margin proxy and the
allocation of the EE*-linear adjustments) and src/exposure/allocation.cpp (marginal and incremental exposure from
path values).  These are host computations over per-date profiles: the GPU produces the profiles, the per-trade
Euler statistics and the conditional initial margin in the fused kernels (summary.summarise), and these functions
turn them into adjustments.  Integrals are summed with Kahan compensation; credit curves are (pillars, hazards)
pairs of piecewise-flat hazard rates.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .summary import _kahan, hazard_survival

Curve = Tuple[Sequence[float], Sequence[float]]


@dataclass
class XvaParameters:
    """XvaParameters (include/ccr/xva/xva.hpp:13-21)."""

    funding_spread_borrow: float = 0.0100  # paid to fund positive exposure
    funding_spread_lend: float = 0.0       # earned on the funding released by negative exposure
    margin_funding_spread: float = 0.0100  # paid to fund the initial margin posted (MVA)
    hurdle_rate: float = 0.10              # cost of capital (KVA)
    capital_ratio: float = 0.08
    risk_weight: float = 1.0
    alpha: float = 1.4                     # exposure-at-default multiplier

    def as_dict(self) -> Dict[str, float]:
        return dict(self.__dict__)


def _q(curve: Curve, t: float) -> float:
    return hazard_survival(curve[0], curve[1], t)


def _pd(curve: Curve, t1: float, t2: float) -> float:
    return _q(curve, t1) - _q(curve, t2)


def survival_weighted_integral(times, f, cpty: Curve, own: Curve) -> float:
    """Trapezoidal integral of f(t) Q_c(t) Q_own(t) dt with the survivals at the mid-points (xva.cpp:18-26)."""
    terms = []
    for i in range(1, len(times)):
        mid = 0.5 * (times[i - 1] + times[i])
        terms.append(0.5 * (f[i - 1] + f[i]) * (times[i] - times[i - 1]) * _q(cpty, mid) * _q(own, mid))
    return _kahan(terms)


def exposure_xva(times, dee, cpty: Curve, recovery_cpty: float, own: Curve, p: XvaParameters) -> Dict[str, float]:
    """CVA, FCA and KVA of a discounted EE profile (xva.cpp:30-42): the adjustments linear in EE*."""
    if len(times) != len(dee):
        raise ValueError("exposure_xva: size mismatch")
    cva = _kahan((1.0 - recovery_cpty) * 0.5 * (dee[i - 1] + dee[i]) * _q(own, 0.5 * (times[i - 1] + times[i])) *
                 _pd(cpty, times[i - 1], times[i]) for i in range(1, len(times)))
    weighted = survival_weighted_integral(times, dee, cpty, own)
    return {"cva": cva, "fca": p.funding_spread_borrow * weighted,
            "kva": p.hurdle_rate * p.capital_ratio * p.risk_weight * p.alpha * weighted}


def funding_benefit(times, dene, cpty: Curve, own: Curve, funding_spread_lend: float) -> float:
    """s_l times the integral of |ENE*| (xva.cpp:44-50)."""
    if len(times) != len(dene):
        raise ValueError("funding_benefit: size mismatch")
    return funding_spread_lend * survival_weighted_integral(times, [-v for v in dene], cpty, own)


def margin_valuation_adjustment(times, dim, cpty: Curve, own: Curve, margin_funding_spread: float) -> float:
    """s_m times the integral of the discounted initial margin (xva.cpp:52-57)."""
    if len(times) != len(dim):
        raise ValueError("margin_valuation_adjustment: size mismatch")
    return margin_funding_spread * survival_weighted_integral(times, dim, cpty, own)


def initial_margin_profile(values: np.ndarray, times, deflator: np.ndarray, quantile_level: float = 0.99,
                           margin_period: float = 10.0 / 250.0) -> np.ndarray:
    """The simulated initial-margin proxy (xva.cpp:59-76): per date the quantile of |V(t_k) - V(t_k-1)| over the
    paths, scaled by sqrt(margin period / dt) and discounted with the mean deflator; 0 at the first date.  values
    and deflator are [paths][dates]."""
    from .summary import exact_quantile

    v, d = np.asarray(values, np.float64), np.asarray(deflator, np.float64)
    if v.shape != d.shape or v.shape[1] != len(times):
        raise ValueError("initial_margin_profile: values, deflator and grid do not match")
    out = np.zeros(len(times))
    for k in range(1, len(times)):
        change = np.abs(v[:, k] - v[:, k - 1])
        scale = np.sqrt(margin_period / (times[k] - times[k - 1]))
        out[k] = exact_quantile(change, quantile_level) * scale * _kahan(d[:, k]) / v.shape[0]
    return out


def xva(profile: Dict[str, np.ndarray], dim: Optional[Sequence[float]], cpty: Curve, recovery_cpty: float, own: Curve,
        recovery_own: float, p: XvaParameters) -> Dict[str, float]:
    """Every adjustment of a profile (xva.cpp:78-95): profile holds times, dee (EE*) and dene (ENE*); dim is the
    discounted initial margin (None: no MVA), e.g. a summary's conditional_im_discounted.  Adds fva = fca - fba
    and total = cva - dva + fca - fba + mva + kva."""
    t, dee, dene = profile["times"], profile["dee"], profile["dene"]
    e = exposure_xva(t, dee, cpty, recovery_cpty, own, p)
    r = {"cva": e["cva"], "fca": e["fca"], "kva": e["kva"]}
    r["dva"] = _kahan((1.0 - recovery_own) * 0.5 * (-dene[i - 1] - dene[i]) * _q(cpty, 0.5 * (t[i - 1] + t[i])) *
                      _pd(own, t[i - 1], t[i]) for i in range(1, len(t)))
    r["fba"] = funding_benefit(t, dene, cpty, own, p.funding_spread_lend)
    r["mva"] = margin_valuation_adjustment(t, dim, cpty, own, p.margin_funding_spread) if dim is not None and len(dim) else 0.0
    r["fva"] = r["fca"] - r["fba"]
    r["total"] = r["cva"] - r["dva"] + r["fca"] - r["fba"] + r["mva"] + r["kva"]
    return r


def allocate_exposure_xva(times, contributions: Sequence[Sequence[float]], cpty: Curve, recovery_cpty: float, own: Curve,
                          p: XvaParameters) -> List[Dict[str, float]]:
    """CVA, FCA and KVA of each trade from its marginal discounted EE (xva.cpp:97-106).  With the Euler
    contributions of a summary's "trades" (marginal_discounted) they add up to the netting set's."""
    return [exposure_xva(times, c, cpty, recovery_cpty, own, p) for c in contributions]


def marginal_exposure_contributions(trade_values: np.ndarray, netted: np.ndarray,
                                    deflator: Optional[np.ndarray] = None) -> np.ndarray:
    """c_i(t) = E[w V_i 1{V > 0}] with w = 1 or the deflator (allocation.cpp:8-31): trade_values [trade][paths]
    [dates], netted and deflator [paths][dates]; returns [trade][dates]."""
    tv, nv = np.asarray(trade_values, np.float64), np.asarray(netted, np.float64)
    if tv.shape[1:] != nv.shape or (deflator is not None and np.shape(deflator) != nv.shape):
        raise ValueError("marginal_exposure_contributions: size mismatch")
    w = np.ones_like(nv) if deflator is None else np.asarray(deflator, np.float64)
    weight = np.where(nv > 0.0, w, 0.0)
    return np.einsum("ipt,pt->it", tv, weight) / nv.shape[0]


def incremental_exposure(netted: np.ndarray, new_trade: np.ndarray, deflator: Optional[np.ndarray] = None) -> np.ndarray:
    """EE(V + V_new) - EE(V), discounted with a deflator (allocation.cpp:33-45); [paths][dates] in, [dates] out."""
    nv, nt = np.asarray(netted, np.float64), np.asarray(new_trade, np.float64)
    if nv.shape != nt.shape:
        raise ValueError("incremental_exposure: size mismatch")
    w = np.ones_like(nv) if deflator is None else np.asarray(deflator, np.float64)
    return (w * (np.maximum(nv + nt, 0.0) - np.maximum(nv, 0.0))).sum(axis=0) / nv.shape[0]
