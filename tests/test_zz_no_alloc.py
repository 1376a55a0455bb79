"""zk_run_plan_noalloc: the entry point for callers that cannot call cudaMalloc (a host that pools all
device memory itself, or a plug-in inside such a host).  It must give the same statistics as zk_run_plan,
call after call, with all of its device scratch in the library's fixed per-device array.

This file is collected last, so that a run stopping at the first failure has run every other test."""
import numpy as np
import pytest

from setups import gpu_setup
from zlatko_b200 import gpu
from zlatko_b200 import spec as S
from zlatko_b200._native import ZkError

pytestmark = pytest.mark.gpu

RTOL = 2e-4  # the tolerance of the parity tests (test_gpu_parity.py)


def _close(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    assert np.abs(a - b).max() <= RTOL * scale


def test_noalloc_matches_zk_run_plan_on_consecutive_calls(ctx):
    # Two different plans, one after the other: the second call must not see the first call's scratch.
    plans = [gpu.compile(*gpu_setup(4000, csa), S.Options(pfe_quantile=0.975)) for csa in (True, False)]
    for plan in plans:
        s_ref, v_ref = ctx.run(plan)
        s_na, v_na = gpu.run_plan_noalloc(plan, device=0)
        nS = plan.stats_per_date
        for k in range(nS):
            _close(s_na.reshape(-1, nS)[:, k], s_ref.reshape(-1, nS)[:, k])
        _close(v_na, v_ref)
    # The same plan twice in a row gives the same bits.
    a = gpu.run_plan_noalloc(plans[0], device=0)
    b = gpu.run_plan_noalloc(plans[0], device=0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_noalloc_rejects_plans_beyond_its_scratch(ctx):
    m, ns = gpu_setup(200_000, False)  # a factor cube far beyond the fixed array
    plan = gpu.compile(m, ns, S.Options())
    with pytest.raises(ZkError, match="scratch"):
        gpu.run_plan_noalloc(plan, device=0)
