"""Failure paths on the GPU, made on the host: a kernel launch that fails in the launcher, and a bounded loop in a
kernel (the row statistics' quantile search) that runs out of rounds.  Neither faults, traps or hangs the GPU:
the failed launch never reaches the device, and the capped search returns early and sets the error word the
host reads.  After each failure the same context must run the plan again and give the same bits."""
import numpy as np
import pytest

from setups import gpu_setup
from zlatko_b200 import gpu
from zlatko_b200 import spec as S
from zlatko_b200._native import ZkError

pytestmark = pytest.mark.gpu



@pytest.fixture(scope="module")
def plan():
    m, ns = gpu_setup(4000, True)
    return gpu.compile(m, ns, S.Options(pfe_quantile=0.975))


@pytest.mark.parametrize("launch", [1, 2, 3, 4])
def test_injected_launch_failure_leaves_the_context_usable(ctx, plan, launch):
    # Launches of one call: simulate, revalue, reduce, row statistics.  The k-th fails before reaching the GPU.
    s0, v0 = ctx.run(plan)
    ctx.inject(ctx.INJECT_FAIL_LAUNCH, launch)
    with pytest.raises(ZkError, match="injected failure of kernel launch") as e:
        ctx.run(plan)
    assert e.value.code == 5  # ZK_ERR_CUDA
    s1, v1 = ctx.run(plan)  # the injection fired once; the context runs the plan as before
    assert np.array_equal(s0, s1) and np.array_equal(v0, v1)


def test_row_statistics_round_cap_reports_an_error(ctx, plan):
    s0, v0 = ctx.run(plan)
    ctx.inject(ctx.INJECT_ROW_ROUNDS, 0)  # no narrowing round allowed: every quantile gives up at once
    try:
        with pytest.raises(ZkError, match="quantile search") as e:
            ctx.run(plan)
        assert e.value.code == 5  # ZK_ERR_CUDA
    finally:
        ctx.inject(ctx.INJECT_ROW_ROUNDS, 16)
    s1, v1 = ctx.run(plan)
    assert np.array_equal(s0, s1) and np.array_equal(v0, v1)


def test_injection_arguments_are_checked(ctx):
    with pytest.raises(ZkError):
        ctx.inject(ctx.INJECT_ROW_ROUNDS, 17)
    with pytest.raises(ZkError):
        ctx.inject(99, 1)
