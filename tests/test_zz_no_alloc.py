"""zk_run_plan_noalloc: the entry point for callers that cannot call cudaMalloc (a host that pools all
device memory itself, or a plug-in inside such a host).  It runs the kernels of zk_run_plan with all of its
device scratch in the library's fixed per-device array, so it must give zk_run_plan's bits, call after call,
on the legacy default stream and on a stream the caller created.

This file is collected last, so that a run stopping at the first failure has run every other test."""
import numpy as np
import pytest

from setups import gpu_setup
from zlatko_b200 import gpu
from zlatko_b200 import spec as S
from zlatko_b200._native import ZkError

pytestmark = pytest.mark.gpu


def _plans():
    plain, csa = (gpu.compile(*gpu_setup(4000, c), S.Options(pfe_quantile=0.975)) for c in (False, True))
    # The nested initial margin: the no-alloc path's launch sequence includes its inner Monte Carlo.
    im = gpu.compile(*gpu_setup(1500, True), S.Options(im_quantile=0.99, im_inner_paths=64))
    return [plain, csa, im]


def _same(a, b):
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_noalloc_gives_the_bits_of_zk_run_plan_on_consecutive_calls(ctx):
    # Different plans one after the other: a call must not see the previous call's scratch.
    for plan in _plans():
        _same(gpu.run_plan_noalloc(plan, device=0), ctx.run(plan))
    plan = _plans()[1]
    _same(gpu.run_plan_noalloc(plan, device=0), gpu.run_plan_noalloc(plan, device=0))


def test_noalloc_on_a_stream_the_caller_created(ctx):
    import torch

    s = torch.cuda.Stream()
    for plan in _plans():
        _same(gpu.run_plan_noalloc(plan, device=0, stream=s.cuda_stream), ctx.run(plan))
    assert torch.cuda.current_device() == 0


def test_noalloc_rejects_plans_beyond_its_scratch(ctx):
    m, ns = gpu_setup(200_000, False)  # a factor cube far beyond the fixed array
    plan = gpu.compile(m, ns, S.Options())
    with pytest.raises(ZkError, match="scratch"):
        gpu.run_plan_noalloc(plan, device=0)
