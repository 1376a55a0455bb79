"""Host-side reductions after the kernels: the exposure profile of a read-back and the CVA integrals.

``summarise`` restates gpu::summarise (src/gpu/fused_exposure.cpp:816-867) for the netting-set
statistics; the CVA functions restate src/cva/cva.cpp:11-48 and the time averages
src/exposure/exposure_profile.cpp:51-60.  The integrals are summed with Kahan compensation.
"""
from __future__ import annotations

import math
from dataclasses import replace
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


def exact_quantile(values, p: float) -> float:
    """ccr::quantile (include/ccr/core/math.hpp:39-47): the sorted values interpolated between the order
    statistics floor(h) and floor(h) + 1, h = p (n - 1)."""
    s = np.sort(np.asarray(values, np.float64))
    n = len(s)
    if n == 0:
        return math.nan
    h = p * (n - 1)
    lo = int(math.floor(h))
    hi = min(lo + 1, n - 1)
    return float(s[lo] + (h - lo) * (s[hi] - s[lo]))


def _kahan(values) -> float:
    s, c = 0.0, 0.0
    for v in values:
        y = float(v) - c
        t = s + y
        c = (t - s) - y
        s = t
    return s


NO_ROW = 0xFFFFFFFF
ROW_QUANTILE, ROW_MEAN, ROW_MEAN_PRODUCT = 0, 1, 6  # row-statistics operations (fused_exposure.hpp:64-75)
TRADE_FIELDS = ("marginal_discounted", "marginal", "incremental_discounted", "standalone_discounted", "standalone")
IM_BAND_LEVELS = (0.05, 0.5, 0.95)


def _outputs(plan):
    """(op, row, level) -> output offset of every row-statistics request of the plan."""
    out = {}
    for q in np.asarray(plan.requests, np.float32).reshape(-1, 8):
        out.setdefault((int(q[0]), int(q[1]), float(q[4])), int(q[7]))
    return out


def _per_date(plan, values, index, op, base, level=0.0):
    """The outputs of one view: request (op, base + r, level) for every reporting date r."""
    nR = len(plan.reporting)
    lv = float(np.float32(level))
    return np.array([float(values[index[(op, base + r, lv)]]) for r in range(nR)], np.float64)


PROFILE_FIELDS = ("times", "ev", "ee", "ene", "pfe", "dee", "dene")


class _Requests:
    """The plan's row-statistics requests in the order gpu::compile emits them (fused_exposure.cpp:505-609):
    each view takes the next requests and reads its outputs at their offsets."""

    def __init__(self, plan, values):
        self.q = np.asarray(plan.requests, np.float32).reshape(-1, 8)
        self.i = 0
        self.v = np.asarray(values, np.float64)
        self.nR = len(plan.reporting)

    def take(self, n: int = 1) -> np.ndarray:
        if self.i + n > len(self.q):
            raise ValueError("summarise: the plan's requests do not match its options")
        self.i += n
        return self.q[self.i - n:self.i]

    def per_date(self) -> int:
        return int(self.take(self.nR)[0, 7])

    def series(self, o: int) -> np.ndarray:
        return self.v[o:o + self.nR].copy()

    def samples(self, o: int, S: int) -> list:
        """Outputs [date][path] to [path][date]."""
        return list(self.v[o:o + self.nR * S].reshape(self.nR, S).T.copy())

    def profile(self, times) -> dict:
        o = [self.per_date() for _ in range(6)]  # mean, positive, negative, PFE, positive / negative deflated
        return {"times": np.asarray(times, np.float64), "ev": self.series(o[0]), "ee": self.series(o[1]),
                "ene": self.series(o[2]), "pfe": self.series(o[3]), "dee": self.series(o[4]), "dene": self.series(o[5])}


def _views(plan, values, o, times) -> dict:
    """addViews (src/gpu/fused_exposure.cpp:715-812): every view the options asked for, from the plan's
    requests in emission order."""
    H = plan.header
    Q = _Requests(plan, values)
    S, nR, nP = int(o.samples), len(times), plan.num_paths
    r: Dict = {"histogram_time": 0.0}
    Q.per_date()  # PFE (read by summarise directly)
    if o.im_quantile > 0.0:
        vc = Q.series(Q.per_date())
        vc[0] = 0.0
        r["value_change_quantile"] = vc
    collateral = int(H[22]) != NO_ROW
    if S > 0:
        r["exposure_samples"] = Q.samples(Q.per_date(), S)
        r["netted_samples"] = Q.samples(Q.per_date(), S)
        if collateral:
            r["collateral_samples"] = Q.samples(Q.per_date(), S)
    if int(H[29]) != NO_ROW:
        r["conditional_im_discounted"] = Q.series(Q.per_date())
        r["conditional_im_mean"] = Q.series(Q.per_date())
        r["conditional_im_bands"] = [Q.series(Q.per_date()) for _ in IM_BAND_LEVELS]
    if o.collateral_bands and collateral:
        r["collateral_bands"] = [Q.series(Q.per_date()) for _ in o.band_levels]
    if o.gross:
        r["gross_profile"] = Q.profile(times)
    if o.histogram_time >= 0.0:
        rank = 0
        for k in range(nR):
            if times[k] <= o.histogram_time + 1e-10:
                rank = k
        q = Q.take(1)[0]
        h, nB = int(q[7]), int(q[3])
        lo, hi = Q.v[h + nB], Q.v[h + nB + 1]
        r["histogram_time"] = float(times[rank])
        r["histogram_edges"] = np.array([lo + (hi - lo) * b / nB for b in range(nB + 1)])
        r["histogram_counts"] = Q.v[h:h + nB] / nP
    if o.trade_views:
        r["trade_views"] = []
        for _ in range(int(H[18])):
            t = {"profile": Q.profile(times)}
            t["samples"] = Q.samples(Q.per_date(), S) if S > 0 else []
            t["bands"] = [Q.series(Q.per_date()) for _ in o.band_levels]
            t["mean_deflated"] = Q.series(Q.per_date())
            r["trade_views"].append(t)
    if int(H[25]) != NO_ROW:
        r["exercise"] = []
        for _ in range(int(H[27])):
            q = Q.take(1)[0]
            h, nE = int(q[7]), int(q[3]) - 1
            e = {"distribution": np.append(Q.v[h + 1:h + 1 + nE], Q.v[h]) / nP}
            e["sample_index"] = Q.v[int(Q.take(1)[0, 7]):][:S].copy() if S > 0 else np.zeros(0)
            r["exercise"].append(e)
    if o.factor_views:
        nA, nC = int(H[2]), int(H[3])
        f = {"rate_samples": Q.samples(Q.per_date(), S) if S > 0 else []}
        f["rate_bands"] = [Q.series(Q.per_date()) for _ in o.factor_band_levels]
        f["rate_mean"], f["deflator_mean"], f["bond_mean"] = (Q.series(Q.per_date()) for _ in range(3))
        f["assets"] = []
        for _ in range(nA):
            a = {"samples": Q.samples(Q.per_date(), S) if S > 0 else []}
            a["bands"] = [Q.series(Q.per_date()) for _ in o.factor_band_levels]
            a["mean"], a["deflated_mean"] = Q.series(Q.per_date()), Q.series(Q.per_date())
            f["assets"].append(a)
        f["credits"] = []
        for _ in range(nC):
            c = {"intensity_samples": [], "survival_samples": []}
            if S > 0:
                c["intensity_samples"] = Q.samples(Q.per_date(), S)
                c["survival_samples"] = Q.samples(Q.per_date(), S)
            c["intensity_bands"] = [Q.series(Q.per_date()) for _ in o.factor_band_levels]
            c["survival_mean"] = Q.series(Q.per_date())
            f["credits"].append(c)
        n = 1 + nA + nC if plan.num_dates > 1 else 0  # first-step increments of x, ln S and y
        means = [float(np.float32(Q.v[int(q[7])])) for q in Q.take(n)]
        prods = np.array([Q.v[int(q[7])] for q in Q.take(n * n)]).reshape(n, n)
        corr = np.zeros((n, n))
        for i in range(n):
            for k in range(n):
                cov = prods[i, k] - means[i] * means[k]
                vi, vk = prods[i, i] - means[i] * means[i], prods[k, k] - means[k] * means[k]
                corr[i, k] = cov / np.sqrt(vi * vk) if vi > 0 and vk > 0 else (1.0 if i == k else 0.0)
        f["increment_correlation"] = corr
        r["factors"] = f
    if Q.i != len(Q.q):
        raise ValueError("summarise: the plan's requests do not match its options")
    return r


def summarise(plan, sums: np.ndarray, values: np.ndarray, run=None) -> Dict:
    """gpu::summarise (src/gpu/fused_exposure.cpp:816-867) on a read-back, per reporting date: EV, EE, ENE, PFE,
    EE*, ENE*, the pathwise-CVA increments, E[Q], E[D], the conditional EE* per default period and the
    per-trade statistics ("trades", one dict per trade group).  For a plan compiled here (plan.options) also
    every view its options asked for (addViews: path samples [path][date], bands, the gross profile, the
    histogram, per-trade views, Bermudan exercise distributions, factor views), under the names of
    FusedResult in snake case; for other plans the margin views the header locates.  The nested conditional
    initial margin: E[D IM], E[IM] and its 5 / 50 / 95% bands; with the plan's audit (im_audit_paths > 0) and a
    backend `run` (plan -> (sums, values)), scaled by the audit ratio (audit_conditional_im)."""
    nS = plan.stats_per_date
    if sums.size != plan.num_dates * nS or values.size < plan.num_outputs:
        raise ValueError("summarise: read-back does not match the plan")
    st = np.asarray(sums, np.float64).reshape(plan.num_dates, nS)
    rep = np.asarray(plan.reporting, np.int64)
    nR = len(rep)
    H = plan.header
    r = {"times": np.asarray(plan.times)[rep]}
    for k, name in enumerate(("ev", "ee", "ene", "dee", "dene", "cva_inc", "mean_survival", "mean_deflator")):
        r[name] = st[rep, k].copy()
    r["pfe"] = np.asarray(values[:nR], np.float64).copy()  # the PFE requests come first
    if plan.market_survival is not None:
        r["market_survival"] = np.asarray(plan.market_survival)[rep]
    r["trades"] = [{f: st[rep, 8 + 5 * i + k].copy() for k, f in enumerate(TRADE_FIELDS)} for i in range(int(H[18]))]
    if getattr(plan, "options", None) is not None:
        r.update(_views(plan, values, plan.options, r["times"]))
    else:
        index = _outputs(plan)
        if int(H[19]) != NO_ROW:  # the value-change rows of the initial-margin proxy, at the margin's quantile level
            lv = next(l for (op, row, l) in index if op == ROW_QUANTILE and row == int(H[19]))
            v = _per_date(plan, values, index, ROW_QUANTILE, int(H[19]), lv)
            v[0] = 0.0
            r["value_change_quantile"] = v
        im = int(H[29])
        if im != NO_ROW:
            r["conditional_im_discounted"] = _per_date(plan, values, index, ROW_MEAN_PRODUCT, im)
            r["conditional_im_mean"] = _per_date(plan, values, index, ROW_MEAN, im)
            r["conditional_im_bands"] = [_per_date(plan, values, index, ROW_QUANTILE, im, q) for q in IM_BAND_LEVELS]
    cdee = np.full(nR, np.nan)
    for k in range(1, nR):
        pd = r["mean_survival"][k - 1] - r["mean_survival"][k]
        if pd > 0:
            cdee[k] = r["cva_inc"][k] / pd
    r["conditional_discounted_ee"] = cdee
    if int(H[3]) == 0:
        r["cva_inc"][:] = np.nan
    if getattr(plan, "im_audit_paths", 0) > 0 and "conditional_im_discounted" in r and run is not None:
        ratio = audit_conditional_im(plan, run)
        r["conditional_im_audit_ratio"] = ratio
        r["conditional_im_discounted_uncorrected"] = r["conditional_im_discounted"].copy()
        r["conditional_im_discounted"] = r["conditional_im_discounted"] * ratio
        r["conditional_im_mean"] = r["conditional_im_mean"] * ratio
        r["conditional_im_bands"] = [b * ratio for b in r["conditional_im_bands"]]
    return r


def audit_conditional_im(plan, run) -> np.ndarray:
    """auditConditionalIm (src/gpu/fused_exposure.cpp:869-886): per reporting date, E[D IM] with the plan's
    im_audit_inner_paths inner paths over E[D IM] with its own inner paths, both on the plan's first
    im_audit_paths paths (the normals are keyed by path, date and inner index, so these are the same outer
    paths, and the first inner samples are the kernel's own); 1 where either is 0.  `run` is the backend."""
    if getattr(plan, "im_audit_paths", 0) == 0 or int(plan.header[30]) == 0 or int(plan.header[29]) == NO_ROW:
        return np.zeros(0)
    n = min(plan.num_paths, int(plan.im_audit_paths))
    h = plan.header.copy()
    h[0], h[15] = n, (n + 63) // 64

    def sub(header):
        p = replace(plan, header=header.copy(), im_audit_paths=0)
        return summarise(p, *run(p))["conditional_im_discounted"]

    base = sub(h)
    h[30] = int(plan.im_audit_inner_paths)
    audited = sub(h)
    ratio = np.ones(len(base))
    ok = (base > 0.0) & (audited > 0.0)
    ratio[ok] = audited[ok] / base[ok]
    return ratio


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
