"""Host-side reductions after the kernels: the exposure profile of a read-back and the CVA integrals.

``summarise`` restates gpu::summarise (src/gpu/fused_exposure.cpp:816-867) for the netting-set
statistics; the CVA functions restate src/cva/cva.cpp:11-48 and the time averages
src/exposure/exposure_profile.cpp:51-60.  The integrals are summed with Kahan compensation.
"""
from __future__ import annotations

import math
from typing import Dict, Sequence

import numpy as np


def hazard_survival(pillars: Sequence[float], hazards: Sequence[float], t: float) -> float:
    """Survival of a piecewise-flat hazard curve (src/market/credit_curve.cpp:23-35)."""
    if t <= 0.0:
        return 1.0
    integral, prev = 0.0, 0.0
    for i, (p, h) in enumerate(zip(pillars, hazards)):
        end = t if i + 1 == len(pillars) else min(t, p)
        integral += h * (end - prev)
        if end >= t:
            break
        prev = end
    return math.exp(-integral)


def _kahan(values) -> float:
    s, c = 0.0, 0.0
    for v in values:
        y = float(v) - c
        t = s + y
        c = (t - s) - y
        s = t
    return s


def summarise(plan, sums: np.ndarray, values: np.ndarray) -> Dict[str, np.ndarray]:
    """Per reporting date: EV, EE, ENE, PFE, EE*, ENE*, pathwise-CVA increments, E[Q], E[D]."""
    nS = plan.stats_per_date
    if sums.size != plan.num_dates * nS or values.size < plan.num_outputs:
        raise ValueError("summarise: read-back does not match the plan")
    st = np.asarray(sums, np.float64).reshape(plan.num_dates, nS)
    rep = np.asarray(plan.reporting, np.int64)
    r = {"times": np.asarray(plan.times)[rep]}
    for k, name in enumerate(("ev", "ee", "ene", "dee", "dene", "cva_inc", "mean_survival", "mean_deflator")):
        r[name] = st[rep, k].copy()
    r["pfe"] = np.asarray(values[: len(rep)], np.float64).copy()  # the PFE requests come first
    if plan.market_survival is not None:
        r["market_survival"] = np.asarray(plan.market_survival)[rep]
    if int(plan.header[3]) == 0:
        r["cva_inc"][:] = np.nan
    return r


def pathwise_cva(result: Dict[str, np.ndarray], recovery: float) -> float:
    """FusedResult::pathwiseCva (src/gpu/fused_exposure.cpp:888-892)."""
    return (1.0 - recovery) * _kahan(result["cva_inc"])


def unilateral_cva(times, dee, pillars, hazards, recovery: float) -> float:
    """(1 - R) sum_i 1/2 (EE*_{i-1} + EE*_i) (Q(t_{i-1}) - Q(t_i)) (src/cva/cva.cpp:11-32)."""
    q = [hazard_survival(pillars, hazards, t) for t in times]
    terms = [(1.0 - recovery) * 0.5 * (dee[i - 1] + dee[i]) * (q[i - 1] - q[i]) for i in range(1, len(times))]
    return _kahan(terms)


def bilateral_cva(times, dee, dene, cpty, own, rc: float, ro: float):
    """First-to-default CVA and DVA (src/cva/cva.cpp:34-48); cpty / own are (pillars, hazards)."""
    cva, dva = [], []
    for i in range(1, len(times)):
        mid = 0.5 * (times[i - 1] + times[i])
        pdc = hazard_survival(*cpty, times[i - 1]) - hazard_survival(*cpty, times[i])
        pdo = hazard_survival(*own, times[i - 1]) - hazard_survival(*own, times[i])
        cva.append((1.0 - rc) * 0.5 * (dee[i - 1] + dee[i]) * hazard_survival(*own, mid) * pdc)
        dva.append((1.0 - ro) * 0.5 * (-dene[i - 1] - dene[i]) * hazard_survival(*cpty, mid) * pdo)
    return _kahan(cva), _kahan(dva)


def time_average(times, values, horizon: float) -> float:
    """Right-point time average on the grid (src/exposure/exposure_profile.cpp:51-60): EPE, effective EPE."""
    integral, end = [], 0.0
    for j in range(1, len(times)):
        if times[j] > horizon + 1e-10:
            break
        integral.append(values[j] * (times[j] - times[j - 1]))
        end = times[j]
    return _kahan(integral) / end if end > 0.0 else (values[0] if len(values) else 0.0)


def epe(result, horizon: float) -> float:
    return time_average(result["times"], result["ee"], horizon)


def effective_epe(result, horizon: float = 1.0) -> float:
    return time_average(result["times"], np.maximum.accumulate(result["ee"]), horizon)
