"""GPU parity of the Longstaff-Schwartz fit (zk_fit_amc, zk_fit_amc_f64) against the oracle.

FP32 mode: the GPU fits on its own AMC pass, the oracle (fitAmc restated, pinned bit for bit to the reference's
compile) on the CPU kernels' pass.  The states differ in the last bits of single-precision transcendentals, which
moves a path with an exercise value within rounding of zero in or out of the in-the-money set of a policy
regression: one path of n shifts the fitted records by O(1/n) (~3e-4 at 6,000 paths), and the exercise
decisions differ on the few paths this puts on the other side of the boundary.

FP64 mode: on identical normals, the GPU's FP64 state pass, fit (FP64 Cholesky) and revaluation against the
FP64 engine (Longstaff-Schwartz of BermudanSwaption, restated and pinned bit for bit to the reference): every
exercise decision identical, path for path, and the exposure profile within 1e-9.
"""
import dataclasses

import numpy as np
import pytest

from oracle import restated
from setups import bermudan, gpu_setup
from zlatko_b200 import gpu
from zlatko_b200 import spec as S

pytestmark = pytest.mark.gpu


def book(paths, csa=False):
    m, ns = gpu_setup(paths, csa)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0, 4.0), physical=True, degree=3))
    ns.trades.append(bermudan(exercise=(2.0, 3.0), physical=False, position=-0.5, degree=2, pay=True))
    ns.trades.append(bermudan(exercise=(1.0, 3.0), physical=True, degree=1))
    return m, ns


def records(terms):
    t = np.asarray(terms).reshape(-1, 8)
    kind = t[:, 0].astype(np.int64) & 15
    return t[(kind == 6) | (kind == 7)].astype(np.float64)


@pytest.mark.parametrize("paths", [6000, 70000])  # 70,000 paths: clusters of 8 CTAs per Bermudan
def test_fit_matches_the_oracle_fit(ctx, paths):
    m, ns = book(paths)
    p = gpu.compile(m, ns, S.Options(exercise_views=True))
    g = ctx.fit_amc(p)
    o = restated.fit_amc(p, p.amc_degrees)
    a, b = records(g.terms), records(o)
    assert np.array_equal(a[:, :2], b[:, :2])  # codes and positions untouched
    tol = 3e-3 if paths < 20000 else 1e-3
    for col in range(2, 8):
        scale = np.maximum(np.abs(b[:, col]), 1e-2 * np.abs(b[:, col]).max() + 1e-30)
        err = np.abs(a[:, col] - b[:, col]) / scale
        assert err.max() <= tol, (col, float(err.max()))
    # Exercise decisions: the GPU-fitted plan on the GPU against the oracle-fitted plan on the oracle, on the
    # same counter-based normals.
    po = gpu.Plan.from_arrays(p.header, p.indices, p.params, p.steps, o, p.requests, p.rows_total, p.num_outputs,
                              p.times, p.reporting)
    _, _, rows_g = ctx.run(g, rows=True)
    _, _, rows_o = restated.run_plan(po, rows=True)
    ex = int(p.header[25])
    mism = int((rows_g[ex:ex + 3] != rows_o[ex:ex + 3]).sum())
    assert mism <= 3e-3 * paths * 3, f"{mism} of {3 * paths} exercise decisions differ"


def normals(plan, seed):
    streams = (plan.num_paths + 1) // 2
    return np.random.default_rng(seed).standard_normal((plan.num_dates - 1) * int(plan.header[5]) * streams), streams


@pytest.mark.parametrize("csa", [False, True])
def test_fp64_decisions_match_the_engine(ctx, csa):
    m, ns = book(3000, csa)
    p = gpu.compile(m, ns, S.Options(exercise_views=True, samples=1))
    z, streams = normals(p, 7)
    f = ctx.fit_amc_f64(p, z, streams)
    sums, vals, rows = ctx.run_f64(f, z, streams, rows=True)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, m.num_paths)
    ex = int(p.header[25])
    for b in range(3):
        assert np.array_equal(rows[ex + b], e.exercise[b]), f"Bermudan {b}: exercise decisions differ"
    from zlatko_b200.summary import summarise

    res = summarise(f, sums, vals)
    for k in ("ev", "ee", "ene", "pfe", "dee", "dene"):
        scale = max(np.abs(e.profile[k]).max(), 1e-12)
        assert np.abs(res[k] - e.profile[k]).max() <= 1e-9 * scale, k
    rep = e.reporting
    H = p.header
    scale = np.abs(e.netted).max()
    assert np.abs(rows[H[21]:H[21] + len(rep)].T - e.netted[:, rep]).max() <= 1e-9 * scale


def test_fit_rejects_bad_arguments(ctx):
    from zlatko_b200._native import ZkError

    m, ns = book(500)
    p = gpu.compile(m, ns)
    bad = dataclasses.replace(p, amc_degrees=[3, 2])
    with pytest.raises(ZkError, match="INVALID_ARGUMENT"):
        ctx.fit_amc(bad)
    bad = dataclasses.replace(p, amc_degrees=[3, 2, 4])
    with pytest.raises(ZkError, match="INVALID_ARGUMENT"):
        ctx.fit_amc(bad)
    assert np.isfinite(ctx.run(ctx.fit_amc(p))[0]).all()  # the context stays usable
