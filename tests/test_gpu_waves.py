"""Memory-bounded books: with a row budget below the book's rows and partials, the netting sets run in waves that
reuse one device region (zk_context_set_row_budget).  Every output must be the same bits as the book in one wave,
through zk_run_plans and through a batch replaying its captured graph."""
import numpy as np
import pytest

from test_gpu_parity import check_sums
from zlatko_b200 import gpu, workloads

pytestmark = pytest.mark.gpu


def test_waves_give_the_bits_of_one_wave(ctx):
    m, books, o, _ = workloads.correlated_csa_book(4096, 20, 300)
    plans = [gpu.compile(m, b, o) for b in books]
    whole = ctx.run_many(plans)
    b = ctx.batch(plans)
    try:
        assert b.info().num_waves == 1
    finally:
        b.close()
    rows = sum(p.rows_total * p.num_paths * 4 for p in plans)
    try:
        ctx.set_row_budget(rows // 5)
        waved = ctx.run_many(plans)
        b = ctx.batch(plans)
        try:
            for _ in range(3):
                b.execute()  # autotunes, then replays the captured graph
            replay = b.read()
            info = b.info()
        finally:
            b.close()
    finally:
        ctx.set_row_budget(0)
    assert info.num_waves >= 4
    for (s0, v0), (s1, v1), (s2, v2) in zip(whole, waved, replay):
        assert np.array_equal(s0, s1) and np.array_equal(v0, v1)
        assert np.array_equal(s0, s2) and np.array_equal(v0, v2)


def test_xva_batch_in_waves_matches_each_netting_set_alone(ctx):
    """config[4]'s construction at a small size: netting sets with tens of Bermudans fitted on the GPU, in one batch
    run in waves; the largest netting sets give the bits of their own single runs."""
    from zlatko_b200 import spec as S

    m, cb, _, _, _ = workloads.xva_batch(2048, num_trades=2000, netting_sets=100)
    o = S.Options(pfe_quantile=0.975)
    plans = [gpu.compile(m, b, o) for b in cb]
    plans = [ctx.fit_amc(p) if int(p.header[27]) > 0 else p for p in plans]
    assert max(int(p.header[27]) for p in plans) > 4
    rows = sum(p.rows_total * p.num_paths * 4 for p in plans)
    try:
        ctx.set_row_budget(rows // 4)
        many = ctx.run_many(plans)
    finally:
        ctx.set_row_budget(0)
    order = sorted(range(len(plans)), key=lambda i: -int(plans[i].header[27]))
    for i in order[:3]:  # term by term in the batch as alone: the same bits
        s1, v1 = ctx.run(plans[i])
        assert np.array_equal(many[i][0], s1) and np.array_equal(many[i][1], v1), i
        assert np.isfinite(s1).all()
    # a netting set without Bermudans runs on the basis kernel in the batch (a group of the batch's eligible sets)
    # and term by term alone: the same results to single-precision rounding and the odd margin call
    i = order[-1]
    s1, v1 = ctx.run(plans[i])
    check_sums(plans[i], many[i][0], s1, 1e-3)
