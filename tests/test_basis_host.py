"""The basis lowering of the tensor-core revalue kernel (csrc/basis_plan.cpp), on the host, without a GPU.

Along one path of factor values, the lowered group -- each basis column's function times its FP16 hi + lo
coefficients times the date's power-of-two scale, fixings through the group's shared slots -- against the plans'
terms summed one by one (both in double): the difference is the coefficients' FP16 hi/lo rounding, below 2^-21 of
the gross sum of the netting set's basis terms.  On the bench's books the ~1,500 linear terms and options per
(path, date) collapse to ~140 basis columns.  Plans with terms the kernel does not run are refused."""
import numpy as np
import pytest

from zlatko_b200 import gpu, workloads
from zlatko_b200 import spec as S


def _path(nT, seed=1):
    rng = np.random.default_rng(seed)
    x = np.cumsum(rng.normal(0.0, 0.004, nT))
    S_ = np.exp(np.cumsum(rng.normal(0.0, 0.03, (nT, 4)), axis=0)) * np.array([1.1, 0.9, 1.0, 1.0])
    xf = np.cumsum(rng.normal(0.0, 0.004, (nT, 2)), axis=0)
    return x, S_, xf


@pytest.mark.parametrize("foreign", [True, False])
def test_book_lowering_matches_the_terms(foreign):
    m, books, o, _ = workloads.correlated_csa_book(1000, 100, 2000, foreign_rates=foreign)
    plans = [gpu.compile(m, b, o) for b in books]
    nT = plans[0].num_dates
    for seed in (1, 2):
        r = gpu.basis_check(plans, *_path(nT, seed))
        assert r["rel_err"] <= 2.0 ** -21, r
    assert r["columns"] * 8 < r["linear_terms"]  # the basis is far smaller than the terms
    assert 0 < r["fixing_slots"] <= 64


def test_a_small_group_with_every_column_type():
    m, books, o, _ = workloads.correlated_csa_book(1000, 100, 2000, foreign_rates=True)
    trades = [S.Swap2(5e6, 0.03, True, workloads.back_schedule(60, 12), workloads.back_schedule(60, 6)),
              S.Forward(0, 2e6, 1.1, 2.0), S.Forward(1, -3e6, 0.9, 3.0), S.Option(0, True, 1e6, 1.15, 1.5),
              S.Option(1, False, -2e6, 0.85, 2.5)]
    plans = [gpu.compile(m, S.NettingSet(trades[:k], S.Csa(1e5, 1e5, 1e4, 0.0, 10.0 / 250.0)), o) for k in range(1, 6)]
    r = gpu.basis_check(plans, *_path(plans[0].num_dates, 3))
    assert r["rel_err"] <= 2.0 ** -21, r


def test_refuses_what_the_kernel_does_not_run():
    m, books, _ = workloads.bermudan_book(1000, 4)
    p = gpu.compile(m, books[0], S.Options())
    with pytest.raises(RuntimeError, match="does not lower"):
        gpu.basis_check([p], *_path(p.num_dates))
