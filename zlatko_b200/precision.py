"""The error of the single-precision path against the double-precision mode, output by output, beside the
Monte Carlo standard error of each output.

The production path runs in FP32 (simulation, closed-form revaluation, netting, collateral), as the reference's
fused kernels do.  The FP64 mode runs the same kernels in double precision on the same counter-based normals
(drawn in double instead of single precision), and it agrees with the reference's FP64 ExposureEngine to 1e-9 on
identical normals.  So the FP32-against-FP64 difference of every output is the error that reduced precision adds,
and the rule is that it stays below the Monte Carlo standard error of the output.

Outputs per netting set (src/gpu/fused_exposure.cpp:816-867, src/cva/cva.cpp): EE, ENE, PFE, EE*, ENE* on every
reporting date, the unilateral CVA, the first-to-default CVA and DVA against an own curve, and the pathwise CVA on
the simulated survival.  Standard errors by batch means: the same book on `batches` independent seeds of
P / batches paths each, SE = sd(batch estimates) / sqrt(batches), date by date.
"""
from __future__ import annotations

from dataclasses import replace
from typing import Dict, List, Sequence

import numpy as np

from . import gpu
from . import spec as S
from .summary import bilateral_cva, pathwise_cva, summarise, unilateral_cva

SERIES = ("ee", "ene", "pfe", "dee", "dene")
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


def compare(ctx: gpu.Context, model: S.Model, books: Sequence[S.NettingSet], options: S.Options, own: S.Credit,
            batches: int = 8) -> Dict:
    """FP32 (zk_run_plans) against FP64 (zk_run_plan_f64) on every netting set of the book, with the batch-means
    standard error.  Returns, per output, the largest |FP32 - FP64| / SE over netting sets and dates, the largest
    relative error |FP32 - FP64| / max|FP64| and the netting set where the SE ratio peaks."""
    plans = [gpu.compile(model, b, options) for b in books]
    r32 = _run32(ctx, plans)
    o32, o64 = [], []
    for p, (s, v) in zip(plans, r32):
        o32.append(outputs(p, s, v, model, own))
        s64, v64 = ctx.run_f64(p)
        o64.append(outputs(p, s64, v64, model, own))
    per = max(64, model.num_paths // batches // 64 * 64)
    est: List[List[Dict]] = []
    for k in range(batches):
        mk = replace(model, num_paths=per, seed=int(model.seed) + 7919 * (k + 1))
        pk = [gpu.compile(mk, b, options) for b in books]
        est.append([outputs(p, s, v, mk, own) for p, (s, v) in zip(pk, _run32(ctx, pk))])
    scale_paths = np.sqrt(per / model.num_paths)  # SE at the full path count from the batches' spread
    report: Dict[str, Dict] = {}
    for key in SERIES + SCALARS:
        worst, worst_ns, rel = 0.0, -1, 0.0
        for i in range(len(plans)):
            if key not in o64[i]:
                continue
            a, b = np.atleast_1d(o32[i][key]), np.atleast_1d(o64[i][key])
            spread = np.std(np.array([np.atleast_1d(e[i][key]) for e in est]), axis=0, ddof=1)
            se = spread * scale_paths
            err = np.abs(a - b)
            # Dates with no spread (exposure exactly zero, date 0) carry no Monte Carlo error and no FP error.
            live = se > 0
            if np.any(err[~live] > 1e-6 * max(np.abs(b).max(), 1e-30)):
                ratio = np.inf
            else:
                ratio = float(np.max(err[live] / se[live])) if np.any(live) else 0.0
            if ratio > worst:
                worst, worst_ns = ratio, i
            rel = max(rel, float(err.max() / max(np.abs(b).max(), 1e-30)))
        report[key] = {"max_err_over_se": worst, "max_rel_err": rel, "netting_set": worst_ns}
    return {"outputs": report, "paths": model.num_paths, "netting_sets": len(plans), "se_batches": batches,
            "se_paths_per_batch": per}
