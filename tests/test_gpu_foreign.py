"""Stochastic foreign rates on the GPU (config[1]'s three Hull-White currencies, an extension of the reference's
model): the FP64 kernels against the restated FP64 engine on identical normals at 1e-9 -- profiles, per-path netted
values, every margin call -- and the FP32 kernels against the FP64 mode on the same counter-based normals."""
import numpy as np
import pytest

from oracle import restated
from test_foreign_rates import model
from test_gpu_parity import injected_normals
from zlatko_b200 import gpu
from zlatko_b200 import spec as S
from zlatko_b200.summary import summarise

pytestmark = pytest.mark.gpu


def netting_set(csa=True):
    trades = [S.Swap(1e6, 0.025, True, S.vanilla_schedule(0.0, 4.0, 2)), S.Forward(0, 8e5, 1.15, 3.0),
              S.Forward(0, -5e5, 1.25, 4.5), S.Option(0, True, -4e5, 1.2, 2.0), S.Option(0, False, 6e5, 1.1, 3.5)]
    return S.NettingSet(trades, S.Csa(3e4, 3e4, 5e3, 0.0, 10.0 / 250.0) if csa else None)


@pytest.mark.parametrize("csa", [False, True])
def test_fp64_matches_the_engine_with_foreign_rates(ctx, csa):
    m, ns = model(3000), netting_set(csa)
    p = gpu.compile(m, ns, S.Options(samples=1, pfe_quantile=0.975))
    assert int(p.header[10]) == 8
    z, streams = injected_normals(p, 17)
    sums, vals, rows = ctx.run_f64(p, z, streams, rows=True)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.975, z, streams, m.num_paths)
    res = summarise(p, sums, vals)
    for k in ("ev", "ee", "ene", "pfe", "dee", "dene"):
        scale = max(np.abs(e.profile[k]).max(), 1e-12)
        assert np.abs(res[k] - e.profile[k]).max() <= 1e-9 * scale, k
    H, rep = p.header, e.reporting
    scale = np.abs(e.netted).max()
    assert np.abs(rows[H[21]:H[21] + len(rep)].T - e.netted[:, rep]).max() <= 1e-9 * scale
    if csa:
        assert np.abs(rows[H[22]:H[22] + len(rep)].T - e.collateral[:, rep]).max() <= 1e-9 * scale


def test_fp32_against_fp64_with_foreign_rates(ctx):
    m, ns = model(16384), netting_set(True)
    p = gpu.compile(m, ns, S.Options(pfe_quantile=0.975))
    s32, v32 = ctx.run(p)
    s64, v64 = ctx.run_f64(p)
    a, b = summarise(p, s32, v32), summarise(p, s64, v64)
    for k in ("ee", "ene", "dee", "dene", "pfe"):
        assert np.abs(a[k] - b[k]).max() <= 2e-4 * np.abs(b[k]).max(), k


def test_foreign_and_reference_models_share_a_call(ctx):
    """Plans of the three-currency model and of the reference's model in one zk_run_plans call: separate launch
    groups (different scenarios), each result the same bits as its plan run alone."""
    m3 = model(2000)
    m1 = S.Model(**{**m3.__dict__, "assets": [S.Asset(1.2, 0.2, S.Curve.flat(0.035))],
                    "correlation": m3.correlation[:2, :2].copy()})
    plans = [gpu.compile(m3, netting_set(True), S.Options()), gpu.compile(m1, netting_set(True), S.Options()),
             gpu.compile(m3, netting_set(False), S.Options())]
    many = ctx.run_many(plans)
    for p, (s, v) in zip(plans, many):
        s1, v1 = ctx.run(p)
        assert np.array_equal(s, s1) and np.array_equal(v, v1)
    assert not np.allclose(many[0][0], many[1][0])  # the foreign rate moves the exposure
