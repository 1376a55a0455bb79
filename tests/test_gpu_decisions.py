"""Decisions of the single-precision path against the double-precision ones, decision by decision.

The FP64 mode decides every margin call and exercise as the FP64 engine does (test_gpu_parity, test_gpu_amc,
test_gpu_workloads).  The FP32 path evaluates the same rules on values that carry single-precision rounding, so a
decision can only come out the other way where the FP64 margin of the rule -- |required - held| - MTA for a
margin call (src/exposure/collateral.cpp:42), min(V_e, V_e - continuation) for an exercise
(src/instruments/bermudan_swaption.cpp:87) -- lies within that rounding of zero.  These tests check exactly that:
every decision that differs has its FP64 margin inside a band fixed in advance (a few single-precision units of
the netting set's value scale), so the rules themselves are the same decision for decision, and the count of such
decisions is small.  A rule that differed would show decisions apart far outside the band.
"""
import numpy as np
import pytest

from oracle import restated
from setups import gpu_setup
from test_gpu_parity import injected_normals
from zlatko_b200 import gpu, workloads
from zlatko_b200 import spec as S
from zlatko_b200.nested_exposure import zero_bonds

pytestmark = pytest.mark.gpu

BAND = 2e-5  # of the netting set's largest |value|: ~170 single-precision units


def _collateral_case(ctx, m, ns, seed):
    p = gpu.compile(m, ns, S.Options(samples=1, pfe_quantile=0.975))
    z, streams = injected_normals(p, seed)
    _, _, rows = ctx.run_injected(p, z, streams, rows=True)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.975, z, streams, m.num_paths)
    H, rep, nT = p.header, e.reporting, p.num_dates
    c32 = rows[H[22]:H[22] + len(rep)].T.astype(np.float64)
    c64 = e.collateral[:, rep]
    csa = ns.csa
    scale = np.abs(e.netted).max()
    apart = np.abs(c32 - c64) > 0.1 * csa.mta  # a call made on one side only moves the collateral by about MTA
    paths = np.nonzero(apart.any(axis=1))[0]
    # The FP64 margin of every call: |required(V at the call date) - held before| - MTA.
    call = p.indices[nT + 1:2 * nT + 1].astype(np.int64)
    v = e.netted[:, call]
    hc, ho = csa.threshold_cpty, csa.threshold_own
    req = np.where(v > hc, v - hc, 0.0) - (np.where(-v > ho, -v - ho, 0.0) if np.isfinite(ho) else 0.0)
    held = np.concatenate([np.zeros((m.num_paths, 1)), e.collateral[:, :-1] - csa.ia], axis=1)
    margin = np.abs(req - held) - csa.mta
    margin[:, 0] = np.inf  # the first date always calls
    for q in paths:
        first = rep[np.nonzero(apart[q])[0][0]]
        assert np.abs(margin[q, 1:first + 1]).min() <= BAND * scale, (q, np.abs(margin[q, 1:first + 1]).min() / scale)
    return len(paths), m.num_paths


def test_fp32_margin_calls_differ_only_inside_the_rounding_band(ctx):
    m, ns = gpu_setup(8000, True)
    cases = [_collateral_case(ctx, m, ns, 3)]
    mb, books, _, _ = workloads.correlated_csa_book(2048)
    order = sorted(range(len(books)), key=lambda i: len(books[i].trades))
    for i in (order[len(order) // 2], order[-3]):
        cases.append(_collateral_case(ctx, mb, books[i], 5 + i))
    apart = sum(c[0] for c in cases)
    total = sum(c[1] for c in cases)
    assert apart <= 0.01 * total, (apart, total)


def test_fp32_exercise_decisions_differ_only_inside_the_rounding_band(ctx):
    """The FP32 kernels run the policy the FP64 fit chose (its records rounded to single precision) on the same
    counter-based normals as the FP64 mode; exercise decisions differ only where the FP64 exercise margin is
    within the band of zero."""
    m, books, _ = workloads.bermudan_book(8000)
    ns = books[0]
    p = gpu.compile(m, ns, S.Options(exercise_views=True))
    f = ctx.fit_amc_f64(p)
    _, _, r64 = ctx.run_f64(f, rows=True)
    p32 = gpu.Plan.from_arrays(p.header, p.indices, p.params, p.steps, f.tables64["terms"].astype(np.float32), p.requests,
                               p.rows_total, p.num_outputs, p.times, p.reporting)
    _, _, r32 = ctx.run(p32, rows=True)
    ex = int(p.header[25])
    x64 = ctx.factor_paths_f64(p)[0]
    mflat = S.encode_model(m)
    terms = f.tables64["terms"].reshape(-1, 8)
    apart_total = 0
    for b, tr in enumerate(ns.trades):
        e64, e32 = r64[ex + b], r32[ex + b].astype(np.float64)
        apart = np.nonzero(e64 != e32)[0]
        apart_total += len(apart)
        if not len(apart):
            continue
        sch = np.asarray(tr.swap.schedule)
        sign = 1.0 if tr.swap.pay_fixed else -1.0
        n, k = tr.swap.notional, tr.swap.fixed_rate
        margins = []
        for ei, te in enumerate(tr.exercise):
            j = int(np.argmin(np.abs(p.times - te)))
            x = x64[j]
            ev = np.zeros_like(x)
            for i in range(1, len(sch)):
                if sch[i - 1] < te - 1e-10:
                    continue
                c = zero_bonds(mflat, np.array([(te, sch[i - 1]), (te, sch[i])]))
                bond = c[:, 0:1] * np.exp(c[:, 1:2] - c[:, 2:3] * x[None, :])
                ev += sign * n * (bond[0] - (1.0 + k * (sch[i] - sch[i - 1])) * bond[1])
            rec = next(terms[u] for u in range(int(p.indices[j]), int(p.indices[j + 1]))
                       if int(terms[u, 0]) & 15 == 6 and (int(terms[u, 0]) >> 8) & 15 == b and int(terms[u, 0]) >> 12 == ei)
            zz = (x - rec[2]) * rec[3]
            cont = ((rec[7] * zz + rec[6]) * zz + rec[5]) * zz + rec[4]
            margins.append(np.minimum(ev, ev - cont))
        margins = np.array(margins)
        for q in apart:
            first = int(min(v for v in (e64[q], e32[q]) if v >= 0))  # the first exercise where the two part
            assert np.abs(margins[:first + 1, q]).min() <= BAND * n, (b, q, np.abs(margins[:first + 1, q]).min() / n)
    assert apart_total <= 0.002 * m.num_paths * len(ns.trades), apart_total
