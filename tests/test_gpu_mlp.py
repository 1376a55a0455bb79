"""The surrogate's tensor-core kernels against plain FP32 / FP64 references (numpy on the bf16-rounded inputs)."""
import numpy as np
import pytest

from zlatko_b200.gpu import from_bf16_bits, to_bf16_bits

pytestmark = pytest.mark.gpu


def bf16(a):
    return from_bf16_bits(to_bf16_bits(a)).astype(np.float64)


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 128, 128), (384, 48, 16), (128, 16, 144), (512, 64, 208)])
def test_gemm_matches_fp64_of_the_bf16_inputs(ctx, M, N, K):
    rng = np.random.default_rng(M + N + K)
    a = rng.standard_normal((M, K)).astype(np.float32)
    b = rng.standard_normal((N, K)).astype(np.float32)
    bias = rng.standard_normal(N).astype(np.float32)
    ref = bf16(a) @ bf16(b).T + bias
    got = ctx.gemm_bf16(a, b, bias)
    assert np.abs(got - ref).max() <= 1e-5 * np.sqrt(K) * np.abs(ref).max() + 1e-6
    silu = ref / (1.0 + np.exp(-ref))
    got2 = ctx.gemm_bf16(a, b, bias, act=1)
    assert np.abs(got2 - ref).max() <= 1e-5 * np.sqrt(K) * np.abs(ref).max() + 1e-6  # C holds the pre-activation
    del silu


def test_gemm_rejects_bad_shapes(ctx):
    from zlatko_b200._native import ZkError

    with pytest.raises(ZkError, match="INVALID_ARGUMENT"):
        ctx.gemm_bf16(np.zeros((100, 16)), np.zeros((16, 16)))
