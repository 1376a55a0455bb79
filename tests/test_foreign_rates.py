"""Stochastic foreign short rates: the extension of the reference's model (whose foreign curves are deterministic)
to config[1]'s three Hull-White currencies.  No reference code exists for it, so its parity is unpinned against the
reference; the restated FP64 engine (oracle/engine_oracle.c) is pinned here by the model's own no-arbitrage
identities, as the reference's model tests pin its factors (tests/test_models.cpp:23-36, :92-108):

- the deflated FX forward with strike 0, N S_t P_f(t, T | x_f), is a martingale: its mean is N S_0 P_f(0, T) on
  every date (this holds only with the quanto drift of x_f and the simulated foreign integral in the FX drift);
- the deflator's mean is the domestic discount curve.

The compiler: plans of the three-currency model carry 40-value step rows, the foreign terms, the extra normals,
and are refused where a kernel runs the reference's model only (the nested initial margin, the restated FP32
kernels)."""
import math

import numpy as np
import pytest

from oracle import restated
from zlatko_b200 import gpu
from zlatko_b200 import spec as S


def model(paths=20_000, rho_fx=0.4):
    fx = S.Asset(1.2, 0.2, S.Curve.flat(0.035), rate_a=0.06, rate_sigma=0.02)
    corr = np.array([[1.0, 0.1, 0.3],     # domestic rate, FX, foreign rate
                     [0.1, 1.0, rho_fx],
                     [0.3, rho_fx, 1.0]])
    return S.Model(curve=S.Curve.flat(0.02), hw_a=0.03, hw_sigma=0.01, assets=[fx], correlation=corr,
                   num_paths=paths, seed=3, antithetic=True, base_grid=[0.5 * k for k in range(1, 11)])


def normals(plan, seed=5):
    streams = (plan.num_paths + 1) // 2
    return np.random.default_rng(seed).standard_normal((plan.num_dates - 1) * int(plan.header[5]) * streams), streams


def test_spec_and_compiler_carry_the_foreign_rates():
    m = model(1000)
    assert m.num_foreign == 1 and m.num_factors == 3
    enc = S.encode_model(m)
    assert enc[-4] == S.FOREIGN_MAGIC and enc[-3] == 1.0 and enc[-2] == 0.06
    ns = S.NettingSet([S.Forward(0, 1e6, 1.1, 4.0), S.Option(0, True, 1e6, 1.2, 3.0)])
    p = gpu.compile(m, ns, S.Options())
    assert p.header[10] == 8 and p.steps.size == 32 * p.num_dates      # 24 + 8 values per date
    assert p.header[11] == 3 and p.header[5] == 3 + 1 + 1               # drivers, rate integral, foreign integral
    kinds = set((p.terms.reshape(-1, 8)[:, 0].astype(np.int64) & 15).tolist())
    assert {11, 12} <= kinds and 2 not in kinds and 4 not in kinds      # foreign forward / option, no carry terms
    with pytest.raises(ValueError, match="foreign"):
        gpu.compile(m, ns, S.Options(im_quantile=0.99, im_inner_paths=64))
    with pytest.raises(ValueError):
        restated.run_plan(p)  # the restated reference kernels run the reference's plans only
    bad = S.Model(**{**m.__dict__, "assets": [S.Asset(1.0, 0.1, S.Curve.flat(0.01)), m.assets[0]]})
    with pytest.raises(ValueError, match="first"):
        bad.num_foreign


@pytest.mark.parametrize("rho_fx", [0.6, -0.5])
def test_engine_fx_forward_is_a_martingale_with_the_quanto_drift(rho_fx):
    m = model(20_000, rho_fx)
    N, T = 1e6, 5.0
    ns = S.NettingSet([S.Forward(0, N, 1e-9, T)])
    p = gpu.compile(m, ns, S.Options())
    z, streams = normals(p)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, m.num_paths)
    fx = m.assets[0]
    target = N * fx.spot * math.exp(-0.035 * T)
    dv = e.deflator * e.netted  # [path][date]
    live = e.times < T - 1e-9
    mean, se = dv.mean(0)[live], dv.std(0)[live] / math.sqrt(m.num_paths)
    assert np.all(np.abs(mean - target) <= 4.0 * se + 1e-9 * target), (np.abs(mean - target) / se).max()
    # Without the quanto drift the forward would drift by about rho sigma_f sigma_S B_f per unit of time: the
    # test is sensitive to it (the drift's effect at T exceeds the bound by far).
    drift = abs(rho_fx) * fx.rate_sigma * fx.vol * (T - (1 - math.exp(-fx.rate_a * T)) / fx.rate_a) / fx.rate_a
    assert drift * target > 4.0 * se.max()


def test_engine_deflator_is_the_domestic_curve():
    m = model(20_000)
    ns = S.NettingSet([S.Forward(0, 1e6, 1.0, 5.0)])
    p = gpu.compile(m, ns, S.Options())
    z, streams = normals(p, 8)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, m.num_paths)
    mean, se = e.deflator.mean(0), e.deflator.std(0) / math.sqrt(m.num_paths)
    assert np.all(np.abs(mean - np.exp(-0.02 * e.times)) <= 4.0 * se + 1e-12)
