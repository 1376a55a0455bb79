"""The book of netting sets on common scenarios (zlatko_b200.book): compile_book's common grid, the combine
steps and the xVA on top, run on the oracle (the restated kernels) on the CPU.  The GPU run of the same book is
in test_gpu_parity.py."""
import numpy as np
import pytest

from oracle import restated
from setups import gpu_model, gpu_netting_set, swap_book
from zlatko_b200 import book as B
from zlatko_b200 import spec as S
from zlatko_b200 import xva as X

OWN = ([1.0, 5.0], [0.004, 0.006])


def two_credit_model(paths):
    m = gpu_model(paths)
    m.credits = [m.credits[0], S.Credit(0.6, 0.03, 0.12, 0.025, [2.0, 6.0], [0.015, 0.03], substeps=4)]
    m.correlation = np.array([[1.0, 0.2, 0.0, 0.1], [0.2, 1.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.3], [0.1, 0.0, 0.3, 1.0]])
    return m


def small_book():
    nets = [gpu_netting_set(True), swap_book(3, seed=11), gpu_netting_set(False), swap_book(2, seed=5, horizon_months=30)]
    return two_credit_model(256), nets, [0, 1, 1, 0]


def test_single_credit_keeps_the_rates_and_fx_block():
    m = two_credit_model(64)
    m1 = B.single_credit(m, 1)
    assert len(m1.credits) == 1 and m1.credits[0] is m.credits[1]
    assert np.array_equal(m1.correlation, m.correlation[np.ix_([0, 1, 3], [0, 1, 3])])


def test_book_shares_dates_and_adds_up():
    m, nets, cps = small_book()
    o = S.Options(per_trade=True)
    plans = B.compile_book(m, nets, cps, o)
    t0, r0 = plans[0].times, plans[0].reporting
    for p in plans[1:]:
        assert np.array_equal(p.times, t0) and np.array_equal(p.reporting, r0)
    res = B.run_book(plans, m, cps, OWN, run=restated.run_plan)
    for k in B.ADDITIVE:
        assert np.allclose(res.total[k], sum(r[k] for r in res.summaries), rtol=0, atol=0)
    # Netting sets of different counterparties on the same paths: rates and FX pathwise identical, so a plan's
    # mean deflator is the same for every netting set.
    for r in res.summaries[1:]:
        assert np.array_equal(r["mean_deflator"], res.summaries[0]["mean_deflator"])
    for ns, x, a in zip(nets, res.xva, res.allocation):
        assert len(a) == len(ns.trades)
        if ns.csa is None:  # the Euler allocation of an uncollateralised netting set adds up to its CVA
            assert abs(sum(t["cva"] for t in a) - x["cva"]) <= 1e-5 * abs(x["cva"])
    assert abs(res.xva_total["cva"] - sum(x["cva"] for x in res.xva)) <= 1e-9 * abs(res.xva_total["cva"])
    assert res.xva_total["cva"] > 0 and res.xva_total["dva"] > 0 and res.xva_total["mva"] == 0.0


def test_book_mva_from_the_nested_margin():
    m, nets, cps = small_book()
    m.num_paths = 128
    plans = B.compile_book(m, nets[:2], cps[:2], S.Options(im_quantile=0.99, im_inner_paths=32))
    res = B.run_book(plans, m, cps[:2], OWN, run=restated.run_plan)
    for r, x in zip(res.summaries, res.xva):
        want = X.margin_valuation_adjustment(r["times"], r["conditional_im_discounted"], (m.credits[0].pillars, m.credits[0].hazards)
                                             if x is res.xva[0] else (m.credits[1].pillars, m.credits[1].hazards), OWN,
                                             X.XvaParameters().margin_funding_spread)
        assert x["mva"] > 0 and abs(x["mva"] - want) <= 1e-12 * want


def test_book_rejects_bad_input():
    m, nets, cps = small_book()
    with pytest.raises(ValueError):
        B.compile_book(m, [], [], S.Options())
    with pytest.raises(ValueError):
        B.compile_book(m, nets, cps[:2], S.Options())
    with pytest.raises(ValueError):
        B.compile_book(m, [S.NettingSet([])], [0], S.Options())
