"""The nested exposure with its inner simulations on the GPU (zlatko_b200.nested_exposure) against the reference's
nestedExposure (tests/golden/nested_exposure.npz, made by the reference on its own outer simulation): the same
outer normals (the reference's NormalGenerator, restated by the oracle and pinned to it on the CPU), the FP64
outer simulation and closed forms of the fused kernels, the reference's estimator (pinned bit for bit), and the
inner paths of the GPU kernel on the reference's counter-based normals.  The outer states agree with the
reference's to rounding (1e-13), so every refinement decision and inner-path count is the same and the estimates
agree to 1e-7."""
import os

import numpy as np
import pytest

from oracle import restated
from setups import gpu_setup
from zlatko_b200 import nested as N
from zlatko_b200 import nested_exposure as E
from zlatko_b200 import spec as S

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("time", "ee_exact", "pfe_exact", "ee_regression", "pfe_regression", "ee_uniform", "pfe_uniform", "ee_adaptive",
          "pfe_adaptive", "evaluated", "inner_paths", "audit_inner_paths", "refined", "rounds", "uniform_inner_per_scenario",
          "live")


def reference_normals(plan, seed):
    """The reference's outer normals in the injected layout [step][normal][stream]: generate() draws path by path
    (antithetic pairs share a draw), step by step, normal by normal (scenario_generator.cpp:89-101)."""
    nP, nT, nN = plan.num_paths, plan.num_dates, int(plan.header[5])
    streams = (nP + 1) // 2 if int(plan.header[7]) else nP
    z = restated.normal_stream(seed, streams * (nT - 1) * nN).reshape(streams, nT - 1, nN)
    return np.ascontiguousarray(z.transpose(1, 2, 0)).ravel(), streams


def test_nested_exposure_matches_the_reference(ctx):
    f = np.load(os.path.join(GOLDEN, "nested_exposure.npz"))
    m, ns = gpu_setup(400, False)
    assert np.array_equal(S.encode_model(m), f["model"]) and np.array_equal(S.encode_netting_set(ns), f["netting_set"])
    o = N.AdaptiveOptions(inner_budget=150_000, max_rounds=20)
    reporting = list(f["reporting"])
    plan = E.outer_plan(m, ns, reporting)
    z, streams = reference_normals(plan, m.seed)
    res = E.nested_exposure(ctx, m, ns, reporting, E.NestedExposureOptions(float(f["pfe_quantile"]), o, True), normals=z,
                            streams=streams)
    want = f["points"]
    assert len(res.points) == len(want)
    for p, w in zip(res.points, want):
        w = dict(zip(FIELDS, w))
        for k in ("evaluated", "inner_paths", "audit_inner_paths", "refined", "rounds", "uniform_inner_per_scenario", "live"):
            assert float(p[k]) == w[k], (p["time"], k, p[k], w[k])
        for k in FIELDS[1:9]:
            assert abs(p[k] - w[k]) <= 1e-7 * max(abs(w[k]), 1.0), (p["time"], k, p[k], w[k])
    assert res.inner_paths > 0 and res.inner_launches > 0


def test_inner_paths_are_independent_of_the_batching(ctx):
    """A job's payoffs do not depend on the other jobs of the launch, nor on how its paths are split: inner path q
    starts at its own normal of the job's stream."""
    m, ns = gpu_setup(64, False)
    plan = E.outer_plan(m, ns, [1.0])
    cube = ctx.factor_paths_f64(plan)
    cf = E.collect(ns)
    k = int(np.argmin(np.abs(np.asarray(plan.times) - 1.0)))
    spot = np.stack([cube[2 + a][k] for a in range(len(m.assets))], axis=1)
    inner = E.GpuInner(ctx, S.encode_model(m), cf, 1.0, cube[0][k], spot, np.zeros((64, cf.slots)))
    try:
        assert inner.events() > 0
        a = inner([(3, 11, 40), (5, 12, 7), (3, 13, 40)])
        b = inner([(3, 13, 40)])
        c = inner([(5, 12, 7), (3, 11, 40)])
        assert np.array_equal(a[2], b[0]) and np.array_equal(a[0], c[1]) and np.array_equal(a[1], c[0])
        assert np.all(np.isfinite(a[0])) and np.std(a[0]) > 0
    finally:
        inner.close()
