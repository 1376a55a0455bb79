"""Memory-bounded books: with a row budget below the book's rows and partials, the netting sets run in waves that
reuse one device region (zk_context_set_row_budget).  Every output must be the same bits as the book in one wave,
through zk_run_plans and through a batch replaying its captured graph."""
import numpy as np
import pytest

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
