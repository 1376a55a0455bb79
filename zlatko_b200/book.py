"""A book of netting sets on one set of scenarios, and the adjustments on top of it.

Restates the portfolio scope of the reference's analyses (src/app/analyses.cpp:1604-1830): every netting set of
the book draws the same scenarios.  They share the reporting dates (the union of all their reporting grids) and
the simulation dates (FusedOptions::extraDates: the union of every plan's grid), and each simulates only its own
counterparty's intensity, last in the factor order, so the rate and FX paths are pathwise identical across the
book (the normals are keyed by path, date and factor index).  Exposures, CVA, DVA, FVA, MVA and KVA of different
netting sets then add up exactly; quantiles (PFE) do not and stay per netting set.

On the GPU the whole book is one batch (zk_batch_*, or zk_run_plans): the netting sets of one counterparty share
one risk-factor simulation, and every plan is revalued by the fused kernels.  The combine steps (summaries, sums,
xVA, allocation) are host code over the per-date profiles.
"""
from __future__ import annotations

from dataclasses import dataclass, replace
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import gpu
from . import spec as S
from . import xva as X
from .summary import summarise

ADDITIVE = ("ev", "ee", "ene", "dee", "dene")  # sumProfiles (analyses.cpp:1770-1786): no PFE


def single_credit(model: S.Model, c: int) -> S.Model:
    """The model with only credit c simulated, last in the factor order, and the matching block of the
    correlation matrix (singleCredit, analyses.cpp:1642-1667)."""
    if not model.credits:
        return model
    nA = len(model.assets)
    corr = None
    if model.correlation is not None:
        full = np.asarray(model.correlation, np.float64)
        if full.shape != (1 + nA + len(model.credits),) * 2:
            raise ValueError("correlation matrix has wrong dimension")
        keep = list(range(nA + 1)) + [1 + nA + c]
        corr = full[np.ix_(keep, keep)]
    return replace(model, credits=[model.credits[c]], correlation=corr)


def _union(times: Sequence[np.ndarray]) -> List[float]:
    out: List[float] = []
    for t in sorted(float(v) for ts in times for v in ts):
        if not out or t > out[-1] + 1e-9:
            out.append(t)
    return out


def compile_book(model: S.Model, netting_sets: Sequence[S.NettingSet], counterparties: Sequence[int],
                 options: S.Options, fit: Optional[gpu.Context] = None) -> List[gpu.Plan]:
    """The plans of a book on common scenarios (bookParts and compileBook, analyses.cpp:1669-1768): the reporting
    grid of every netting set is the union of all of theirs, and every plan simulates the union of all simulation
    dates.  counterparties[i] is the credit (index into model.credits) of netting set i; `fit` fits the AMC
    regressions of Bermudans on the GPU (gpu.compile)."""
    if not netting_sets:
        raise ValueError("the portfolio has no netting sets")
    if len(counterparties) != len(netting_sets):
        raise ValueError("one counterparty per netting set")
    models = [single_credit(model, c) for c in counterparties]
    for i, ns in enumerate(netting_sets):
        if not ns.trades:
            raise ValueError(f"netting set {i + 1} has no trades")
    opts = replace(options, counterparty=0)
    first = [gpu.compile(m, ns, opts) for m, ns in zip(models, netting_sets)]
    reporting = [p.times[p.reporting.astype(np.int64)] for p in first]
    base = [t for t in _union(reporting) if t > 0.0]
    models = [replace(m, base_grid=base) for m in models]
    second = [gpu.compile(m, ns, opts) for m, ns in zip(models, netting_sets)]
    dates = _union([p.times for p in second])
    opts = replace(opts, extra_dates=tuple(dates))
    return [gpu.compile(m, ns, opts, fit=fit) for m, ns in zip(models, netting_sets)]


@dataclass
class BookResult:
    summaries: List[Dict]            # summary.summarise of each netting set
    total: Dict[str, np.ndarray]     # the additive profile quantities summed over the book
    xva: List[Dict[str, float]]      # per netting set (xva.xva; MVA from the nested initial margin when computed)
    xva_total: Dict[str, float]      # each adjustment summed over the book
    allocation: List[List[Dict[str, float]]]  # per netting set, per trade: CVA, FCA, KVA (per-trade plans only)


def run_book(plans: Sequence[gpu.Plan], model: S.Model, counterparties: Sequence[int], own: X.Curve,
             recovery_cpty: float = 0.4, recovery_own: float = 0.4, params: Optional[X.XvaParameters] = None,
             run: Optional[Callable] = None, ctx: Optional[gpu.Context] = None) -> BookResult:
    """Runs a compiled book and combines it (bookResult, analyses.cpp:1811-1830): `ctx` runs every plan in one
    zk_run_plans call on the GPU; `run` (plan -> (sums, values)) is any other backend.  The xVA of netting set i
    uses the market hazard curve of its counterparty and `own`."""
    params = params or X.XvaParameters()
    if ctx is not None:
        outs = ctx.run_many(plans)
        backend = ctx.run
    elif run is not None:
        outs = [run(p) for p in plans]
        backend = run
    else:
        raise ValueError("run_book needs a context or a backend")
    sums = [summarise(p, s, v, run=backend) for p, (s, v) in zip(plans, outs)]
    times = sums[0]["times"]
    for r in sums[1:]:
        if not np.array_equal(r["times"], times):
            raise ValueError("the book's plans do not share their reporting dates (compile_book)")
    total = {"times": times.copy()}
    for k in ADDITIVE:
        total[k] = np.sum([r[k] for r in sums], axis=0)
    xs, alloc = [], []
    for r, c in zip(sums, counterparties):
        cr = model.credits[c]
        curve = (cr.pillars, cr.hazards)
        dim = r.get("conditional_im_discounted")
        xs.append(X.xva(r, dim, curve, recovery_cpty, own, recovery_own, params))
        alloc.append(X.allocate_exposure_xva(r["times"], [t["marginal_discounted"] for t in r["trades"]], curve,
                                             recovery_cpty, own, params))
    xva_total = {k: float(sum(x[k] for x in xs)) for k in xs[0]}
    return BookResult(sums, total, xs, xva_total, alloc)
