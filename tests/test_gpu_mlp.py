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


# ---------------------------------------------------------------- the surrogate perceptron
def data(n, seed):
    rng = np.random.default_rng(seed)
    sd = np.array([0.02, 0.1, 0.1, 0.01, 1.0, 3.0, 0.5, 1, 1, 1, 0.03, 5.0, 0.2, 1.0, 0.1, 1.0], np.float32)
    x = (rng.standard_normal((n, 16)) * sd + np.arange(16) * 0.1).astype(np.float32)
    z = (x - np.arange(16) * 0.1) / sd
    y = (np.sin(z[:, 0]) + 0.5 * z[:, 1] * z[:, 2] + np.tanh(z[:, 4] - z[:, 5]) + 0.1 * z[:, 11] ** 2).astype(np.float32)
    return x, y


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_surrogate_gradients_match_the_fp64_oracle(ctx):
    """Per parameter block: within 5e-3 (relative L2) of the oracle at the GPU's bf16 rounding points (what is
    left is FP32 against FP64 accumulation and the odd bf16 tie), within 5e-2 of the exact FP64 network."""
    from oracle import mlp_oracle as O
    from zlatko_b200.surrogate import LAYOUT, Surrogate

    with Surrogate(ctx, seed=3) as s:
        x, y = data(1000, 1)  # 1000 rows: a padded last tile of 128
        loss, g = s.gradients(x, y)
        p, sc = s.params()
        lo, go = O.loss_and_grads(p, sc, x, y, emulate=True)
        l64, g64 = O.loss_and_grads(p, sc, x, y, emulate=False)
        assert abs(loss - lo) <= 1e-4 * lo
        assert abs(loss - l64) <= 2e-2 * l64
        o = 0
        for name, shape in LAYOUT:
            k = int(np.prod(shape))
            assert rel(g[o:o + k], go[o:o + k]) <= 5e-3, name
            assert rel(g[o:o + k], g64[o:o + k]) <= 5e-2, name
            o += k


# Inference evaluates SiLU in packed bf16 arithmetic (h = z / 2 rounded to bf16, tanh.approx.bf16x2, a bf16 FMA)
# where training and the oracle use the exact function rounded once to bf16: about one more bf16 unit in the last
# place per activation, unbiased.  Modelled on random networks that is ~0.7% of the output's spread (RMS), 0.35%
# of its largest value at the 99th percentile; the bounds leave room for the approximate tanh.
INFER_Q99, INFER_MAX, INFER_BIAS = 1e-2, 3e-2, 1e-3


def check_inference(got, ref):
    err = (got - ref) / np.abs(ref).max()
    assert np.abs(err).max() <= INFER_MAX and np.quantile(np.abs(err), 0.99) <= INFER_Q99, (np.abs(err).max(), np.quantile(np.abs(err), 0.99))
    assert abs(err.mean()) <= INFER_BIAS, err.mean()


def test_surrogate_forward_matches_the_oracle(ctx):
    """Inference against the FP64 oracle at the GPU's bf16 rounding points, within the bf16 activation's error."""
    from oracle import mlp_oracle as O
    from zlatko_b200.surrogate import Surrogate

    with Surrogate(ctx, seed=5) as s:
        x, y = data(3000, 2)
        s.gradients(x, y)  # fixes the scaling from this set
        p, sc = s.params()
        got = s.predict(x)
        check_inference(got, O.predict(p, sc, x, emulate=True))


def test_surrogate_training_learns_a_smooth_function(ctx):
    from oracle import mlp_oracle as O
    from zlatko_b200.surrogate import Surrogate

    with Surrogate(ctx, seed=7) as s:
        x, y = data(65536, 3)
        losses = s.train(x, y, epochs=30, batch=4096, lr=2e-3)
        assert losses[-1] < 0.05 * losses[0], losses
        xt, yt = data(8192, 4)  # held-out rows
        pred = s.predict(xt)
        assert np.sqrt(np.mean((pred - yt) ** 2)) <= 0.15 * np.std(yt)
        p, sc = s.params()
        check_inference(pred, O.predict(p, sc, xt, emulate=True))
