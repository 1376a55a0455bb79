"""The host plan compiler (zk_compile) against the reference's gpu::compile: identical tables."""
import numpy as np
import pytest

from oracle import ref
from setups import bermudan, gpu_model, gpu_netting_set, gpu_setup, swap_book
from zlatko_b200 import gpu
from zlatko_b200 import spec as S

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

OPTIONS = [S.Options(), S.Options(per_trade=True, im_quantile=0.99),
           S.Options(samples=12, histogram_time=2.0, gross=True, collateral_bands=True, trade_views=True),
           S.Options(factor_views=True, samples=5, bond_maturity=8.0), S.Options(pfe_quantile=0.975),
           S.Options(im_quantile=0.99, im_inner_paths=64, samples=2), S.Options(per_trade=True, im_quantile=0.95, im_inner_paths=40),
           S.Options(im_quantile=0.99, im_inner_paths=128, im_audit_paths=32, im_audit_inner_paths=512, im_margin_period=20 / 250)]


def _ref_plan(m, ns, o):
    return ref.compile_plan(S.encode_model(m), S.encode_netting_set(ns), S.encode_options(o))


def _same(r, p, skip_amc=False):
    for k in ("header", "indices", "params", "steps", "requests"):
        assert np.array_equal(getattr(r, k), getattr(p, k)), k
    rt, pt = r.terms.reshape(-1, 8), p.terms.reshape(-1, 8)
    assert rt.shape == pt.shape
    if skip_amc:  # decide / continue coefficients are fitted by the reference's compile
        kind = rt[:, 0].astype(np.int64) & 15
        fitted = (kind == 6) | (kind == 7)
        assert np.array_equal(rt[~fitted], pt[~fitted])
        assert np.array_equal(rt[fitted][:, :2], pt[fitted][:, :2])
    else:
        assert np.array_equal(rt, pt)
    assert r.rows_total == p.rows_total and r.num_outputs == p.num_outputs
    assert np.array_equal(r.times, p.times) and np.array_equal(r.reporting.astype(np.int64), p.reporting)


@pytest.mark.parametrize("csa", [False, True])
@pytest.mark.parametrize("oi", range(len(OPTIONS)))
def test_tables_identical_to_reference(csa, oi):
    m, ns = gpu_setup(1000, csa)
    _same(_ref_plan(m, ns, OPTIONS[oi]), gpu.compile(m, ns, OPTIONS[oi]))


@pytest.mark.parametrize("kind", [1, 2])
def test_securities_collateral_tables(kind):
    m, ns = gpu_setup(500, True)
    ns.csa.kind, ns.csa.haircut, ns.csa.bond_maturity, ns.csa.mpr = kind, 0.02 if kind == 1 else 0.15, 10.0, 20.0 / 250.0
    _same(_ref_plan(m, ns, S.Options()), gpu.compile(m, ns, S.Options()))


@pytest.mark.parametrize("physical", [True, False])
def test_bermudan_tables(physical):
    m, ns = gpu_setup(300, False)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0, 4.0), physical=physical, degree=2))
    ns.trades.append(bermudan(exercise=(2.0, 3.0), physical=physical, position=-0.5, degree=3))
    _same(_ref_plan(m, ns, S.Options(exercise_views=True, samples=4)), gpu.compile(m, ns, S.Options(exercise_views=True, samples=4)),
          skip_amc=True)


@pytest.mark.parametrize("csa", [False, True])
def test_two_schedule_swaps_value_like_the_reference_decomposition(csa):
    """A swap with annual fixed and semiannual floating legs compiles natively (one running coupon); the
    reference has one schedule per swap and represents it as float(K=0) + [swap(K) - swap(0)] on the fixed
    schedule.  The reference's own CPU kernels run both plans on the same normals: same statistics."""
    m = gpu_model(512)
    m.base_grid = [k / 12 for k in range(1, 61)]
    ns = swap_book(9, csa=S.Csa(1e5, 1e5, 1e4) if csa else None)
    o = S.Options(pfe_quantile=0.975)
    r = _ref_plan(m, ns, o)
    p = gpu.compile(m, ns, o)
    assert p.terms.size < r.terms.size  # fewer terms: one floating leg instead of three
    assert np.array_equal(r.times, p.times) and r.header[16] == p.header[16]
    mine = ref.plan_from_buffers(p.header, p.indices, p.params, p.steps, p.terms, p.requests, p.rows_total,
                                 p.num_outputs, p.times, p.reporting)
    s1, v1 = ref.run_fused(r)
    s2, v2 = ref.run_fused(mine)
    nS = int(p.header[16])
    a, b = s1.reshape(-1, nS).astype(np.float64), s2.reshape(-1, nS).astype(np.float64)
    for k in range(nS):
        scale = max(np.abs(a[:, k]).max(), 1e-6 * np.abs(a).max(), 1e-30)
        assert np.abs(a[:, k] - b[:, k]).max() <= 1e-4 * scale, k
    assert np.abs(v1 - v2).max() <= 1e-4 * np.abs(v1).max()


def test_beyond_32_swaps_reuses_slots():
    """The reference caps a netting set at 32 swaps; the compiler reuses a slot once a swap's coupons are paid."""
    m = gpu_model(100)
    m.base_grid = [k / 12 for k in range(1, 61)]
    ns = swap_book(40, seed=3)
    with pytest.raises(ValueError):
        _ref_plan(m, ns, S.Options())
    p = gpu.compile(m, ns, S.Options())
    t = p.terms.reshape(-1, 8)
    kind = t[:, 0].astype(np.int64) & 15
    slots = t[(kind == 1) | (kind == 3), 1]
    assert slots.max() < 32


def test_invalid_inputs_raise_like_the_reference():
    m, ns = gpu_setup(100, False)
    with pytest.raises(ValueError):
        gpu.compile(m, ns, S.Options(counterparty=3))
    with pytest.raises(ValueError):
        gpu.compile(m, ns, S.Options(im_quantile=1.5))
    # Nested initial margin (fused_exposure.cpp:233-247): 2 to 1024 inner paths, the quantile's order statistic
    # among the 16 largest samples, an audit with more inner paths than the kernel.
    for o in (S.Options(im_quantile=0.99, im_inner_paths=1), S.Options(im_quantile=0.99, im_inner_paths=2048),
              S.Options(im_quantile=0.5, im_inner_paths=64),
              S.Options(im_quantile=0.99, im_inner_paths=64, im_audit_paths=8, im_audit_inner_paths=64)):
        with pytest.raises(ValueError):
            gpu.compile(m, ns, o)
        with pytest.raises(ValueError):
            ref.compile_plan(S.encode_model(m), S.encode_netting_set(ns), S.encode_options(o))
    m.assets, m.correlation = m.assets * 5, None
    with pytest.raises(ValueError):
        gpu.compile(m, ns, S.Options())
