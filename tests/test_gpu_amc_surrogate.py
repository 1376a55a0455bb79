"""The AMC continuation value by the learned surrogate (zlatko_b200.amc_surrogate) against the Longstaff-Schwartz
regression it would replace, on held-out paths: the network is trained on the realised values of the plain
method's AMC pass under the fitted policy, one network for every date and Bermudan of the book.  The test
measures what the network gains: its mean squared error against the realised values below the regression's."""
import numpy as np
import pytest

from zlatko_b200 import amc_surrogate as AS
from zlatko_b200 import workloads
from zlatko_b200.surrogate import Surrogate

pytestmark = pytest.mark.gpu


def test_continuation_network_against_the_regression(ctx):
    m, books, _ = workloads.bermudan_book(16384)
    books = books[:4]  # 16 Bermudans
    X, y, poly, fitted = AS.book_rows(ctx, m, books)
    assert len(y) > 1_000_000 and np.isfinite(X).all()
    # In-sample the regression is the least-squares fit per date: the realised values are its targets.
    assert abs(np.mean(poly - y)) <= 0.02 * np.std(y)
    with Surrogate(ctx, seed=4) as s:
        for lr, ep in ((2e-3, 6), (5e-4, 4), (1e-4, 2)):
            s.train(X, y, epochs=ep, batch=8192, lr=lr)
        r = AS.compare(ctx, s, m, books, fitted, paths=16384, seed=4242)
    # Both estimate the same conditional expectation on paths neither has seen; the network's error is below the
    # regression's, and its mean is unbiased against the realised values.
    assert r["mse_network"] < r["mse_regression"], r
    assert abs(r["mean_network"] - r["mean_realised"]) <= 0.02 * np.sqrt(r["mse_regression"]) + 1e-3 * abs(r["mean_realised"]), r
