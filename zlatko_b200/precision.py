"""The error of the single-precision path against the double-precision mode, output by output, beside the
Monte Carlo standard error of each output.

The production path runs in FP32 (simulation, closed-form revaluation, netting, collateral), as the reference's
fused kernels do.  The FP64 mode runs the same kernels in double precision on the same counter-based normals
(drawn in double instead of single precision), and it agrees with the reference's FP64 ExposureEngine to 1e-9 on
identical normals.  So the FP32-against-FP64 difference of every output is the error that reduced precision adds,
and the rule is that it stays below the Monte Carlo standard error of the output.

Outputs per netting set (src/gpu/fused_exposure.cpp:816-867, src/cva/cva.cpp): EE, ENE, PFE, EE*, ENE* on every
reporting date, the unilateral CVA, the first-to-default CVA and DVA against an own curve, and the pathwise CVA on
the simulated survival.  Standard errors per path: the sample standard deviation of each output's per-path
contribution over sqrt(paths), from the FP64 mode's path rows (path_standard_errors).
"""
from __future__ import annotations

from dataclasses import replace
from typing import Dict, List, Sequence

import numpy as np

from . import gpu
from . import spec as S
from .summary import bilateral_cva, pathwise_cva, summarise, unilateral_cva

SERIES = ("ee", "ene", "pfe", "dee", "dene")
# Entries whose standard error is below this fraction of the netting set's value scale are below what single
# precision resolves in a path's value (its rounding is 1e-6 .. 1e-5 of the scale): they count as entries without
# Monte Carlo error, checked relative to the scale (max_rel_err_without_mc_error).
RESOLUTION = 1e-5
SCALARS = ("cva", "cva_bilateral", "dva", "pathwise_cva")


def outputs(plan, sums, values, model: S.Model, own: S.Credit, recovery: float = 0.4, own_recovery: float = 0.4) -> Dict:
    """The profile series and the CVA / DVA numbers of one netting set's read-back."""
    r = summarise(plan, np.asarray(sums, np.float64), np.asarray(values, np.float64))
    out = {k: np.asarray(r[k], np.float64) for k in SERIES}
    cp = model.credits[0] if model.credits else None
    times = r["times"]
    if cp is not None:
        curve = (list(cp.pillars), list(cp.hazards))
        out["cva"] = unilateral_cva(times, r["dee"], *curve, recovery)
        out["cva_bilateral"], out["dva"] = bilateral_cva(times, r["dee"], r["dene"], curve, (list(own.pillars), list(own.hazards)),
                                                         recovery, own_recovery)
        out["pathwise_cva"] = pathwise_cva(r, recovery)
    return out


def _run32(ctx: gpu.Context, plans: Sequence[gpu.Plan]):
    return ctx.run_many(plans)


def _hazard_q(pillars, hazards, times):
    from .summary import hazard_survival
    return np.array([hazard_survival(pillars, hazards, t) for t in times])


def path_standard_errors(ctx: gpu.Context, model: S.Model, ns: S.NettingSet, options: S.Options, own: S.Credit,
                         deflators: Dict, recovery: float = 0.4, own_recovery: float = 0.4) -> Dict:
    """Monte Carlo standard errors of every output from the FP64 mode's per-path values: the netted value and the
    collateral on every reporting date (the plan with one path sample, which adds those rows and nothing to the
    statistics) and the deflator of every path (zk_factor_paths_f64).  SE = sd over the paths / sqrt(paths); for
    PFE(q) the order-statistic form (Q(q + d) - Q(q - d)) / 2 with d = sqrt(q (1 - q) / paths)."""
    p = gpu.compile(model, ns, replace(options, samples=max(1, options.samples)))
    _, _, rows = ctx.run_f64(p, rows=True)
    H, nR, nP = p.header, p.num_reporting, p.num_paths
    rep = np.asarray(p.reporting, np.int64)
    key = np.asarray(p.times).tobytes()
    if key not in deflators:
        deflators[key] = ctx.factor_paths_f64(p)[1]  # [date][path]
    D = deflators[key][rep]
    coll = rows[H[22]:H[22] + nR] if int(H[22]) != 0xFFFFFFFF else 0.0
    e = rows[H[21]:H[21] + nR] - coll
    ep, en = np.maximum(e, 0.0), np.minimum(e, 0.0)
    root = np.sqrt(nP)
    out = {"ee": ep.std(1) / root, "ene": en.std(1) / root, "dee": (D * ep).std(1) / root, "dene": (D * en).std(1) / root}
    q = float(options.pfe_quantile)
    d = np.sqrt(q * (1.0 - q) / nP)
    hi, lo = np.quantile(ep, min(q + d, 1.0), axis=1), np.quantile(ep, max(q - d, 0.0), axis=1)
    out["pfe"] = 0.5 * (hi - lo)
    times = np.asarray(p.times)[rep]
    if model.credits:
        cp = model.credits[0]
        qc = _hazard_q(cp.pillars, cp.hazards, times)
        qo = _hazard_q(own.pillars, own.hazards, times)
        mid = 0.5 * (times[1:] + times[:-1])
        sc_mid, so_mid = _hazard_q(cp.pillars, cp.hazards, mid), _hazard_q(own.pillars, own.hazards, mid)
        de, dn = D * ep, D * en
        avg_e, avg_n = 0.5 * (de[1:] + de[:-1]), 0.5 * (dn[1:] + dn[:-1])
        pdc, pdo = (qc[:-1] - qc[1:])[:, None], (qo[:-1] - qo[1:])[:, None]
        cva = (1.0 - recovery) * (avg_e * pdc).sum(0)
        cvab = (1.0 - recovery) * (avg_e * so_mid[:, None] * pdc).sum(0)
        dva = (1.0 - own_recovery) * (-avg_n * sc_mid[:, None] * pdo).sum(0)
        out.update({"cva": np.array([cva.std() / root]), "cva_bilateral": np.array([cvab.std() / root]),
                    "dva": np.array([dva.std() / root])})
    return out


def compare(ctx: gpu.Context, model: S.Model, books: Sequence[S.NettingSet], options: S.Options, own: S.Credit,
            batches: int = 8) -> Dict:
    """FP32 (zk_run_plans) against FP64 (zk_run_plan_f64) on every netting set of the book, beside each output's
    Monte Carlo standard error (path_standard_errors; batch means over `batches` independent seeds for the pathwise
    CVA, whose per-path survival the FP64 rows do not carry, and as a floor under the PFE's order-statistic SE, which
    collapses where a netting set's exposures cluster at the quantile).  Returns, per output, the largest
    |FP32 - FP64| / SE over netting sets and dates, the largest relative error |FP32 - FP64| / max|FP64|, the largest
    relative error on entries without Monte Carlo error (SE below RESOLUTION of the scale: date 0, dates past every
    trade, quantiles of tightly clustered exposures) and the netting set where the SE ratio peaks."""
    plans = [gpu.compile(model, b, options) for b in books]
    r32 = _run32(ctx, plans)
    o32, o64, ses = [], [], []
    deflators: Dict = {}
    for b, p, (s, v) in zip(books, plans, r32):
        o32.append(outputs(p, s, v, model, own))
        s64, v64 = ctx.run_f64(p)
        o64.append(outputs(p, s64, v64, model, own))
        ses.append(path_standard_errors(ctx, model, b, options, own, deflators))
    per = max(64, model.num_paths // batches // 64 * 64)
    est: List[List[Dict]] = []
    for k in range(batches):
        mk = replace(model, num_paths=per, seed=int(model.seed) + 7919 * (k + 1))
        pk = [gpu.compile(mk, b, options) for b in books]
        est.append([outputs(p, s, v, mk, own) for p, (s, v) in zip(pk, _run32(ctx, pk))])
    scale_paths = np.sqrt(per / model.num_paths)
    # The scale of a netting set's values, for entries without Monte Carlo error (a series that is exactly zero in
    # FP64, such as the ENE of a set whose exposure is never negative, has no scale of its own).
    vscale = [max(np.abs(o["ee"]).max(), np.abs(o["ene"]).max(), 1.0) for o in o64]
    report: Dict[str, Dict] = {}
    for key in SERIES + SCALARS:
        worst, worst_ns, rel, rel_det = 0.0, -1, 0.0, 0.0
        for i in range(len(plans)):
            if key not in o64[i]:
                continue
            a, b = np.atleast_1d(o32[i][key]), np.atleast_1d(o64[i][key])
            if key in ses[i]:
                se = np.atleast_1d(ses[i][key])
                if key == "pfe":  # the order-statistic form collapses where exposures cluster: not below batch means
                    se_b = np.std(np.array([np.atleast_1d(e[i][key]) for e in est]), axis=0, ddof=1) * scale_paths
                    se = np.where(se > 0.0, np.maximum(se, se_b), se)
            else:
                se = np.std(np.array([np.atleast_1d(e[i][key]) for e in est]), axis=0, ddof=1) * scale_paths
            err = np.abs(a - b)
            scale = max(np.abs(b).max(), vscale[i])
            live = se > RESOLUTION * scale
            if np.any(live):
                ratio = float(np.max(err[live] / se[live]))
                if ratio > worst:
                    worst, worst_ns = ratio, i
            if np.any(~live):
                rel_det = max(rel_det, float(err[~live].max() / scale))
            rel = max(rel, float(err.max() / scale))
        report[key] = {"max_err_over_se": worst, "max_rel_err": rel, "max_rel_err_without_mc_error": rel_det,
                       "netting_set": worst_ns}
    return {"outputs": report, "paths": model.num_paths, "netting_sets": len(plans),
            "se": "per path from the FP64 rows (batch means over %d seeds for the pathwise CVA)" % batches}
