"""The surrogate revaluation of a book (zk_surrogate_features, zk_surrogate_book) and its audit by the plain
pricer: the features against their definition, the GPU netting against the per-trade predictions, and the
audited CVA against the plain pricer's."""
import numpy as np
import pytest

from zlatko_b200 import gpu
from zlatko_b200 import spec as S
from zlatko_b200 import surrogate_book as SB
from zlatko_b200 import workloads as W
from zlatko_b200.surrogate import Surrogate

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def book():
    m, books, _, _ = W.correlated_csa_book(2048, 10, 100, foreign_rates=False)
    return SB.make_book(m, books)


def expected_features(book, fac):
    """The feature definition of zk_surrogate_features, restated with numpy."""
    nA, nR, nP = fac.shape[0] - 2, fac.shape[1], fac.shape[2]
    T = book.trades
    X = np.zeros((len(T), nR, nP, 16), np.float32)
    t = book.times[None, :, None]
    X[..., 0] = fac[1][None]
    for i, tr in enumerate(T):
        if tr["kind"] != 0:
            X[i, ..., 1] = fac[2 + tr["asset"]]
    X[..., 2] = t
    X[..., 3] = np.maximum(T["maturity"][:, None, None] - t, 0.0)
    for k in range(3):
        X[..., 4 + k] = (T["kind"] == k)[:, None, None]
    X[..., 7] = T["strike"][:, None, None]
    X[..., 8] = T["sign"][:, None, None]
    live = book.resets >= 0
    for i in range(len(T)):
        for r in range(nR):
            k = book.resets[i, r]
            if k >= 0:
                X[i, r, :, 9] = fac[1][k]
                X[i, r, :, 10] = book.times[r] - book.periods[i, r, 0]
                X[i, r, :, 11] = book.periods[i, r, 1] - book.times[r]
    X[..., 12] = (book.periods[..., 1] - book.periods[..., 0])[..., None]
    X[..., 13] = T["asset"][:, None, None]
    x = fac[1][None]  # [1][nR][nP]
    X[..., 14] = np.exp(book.bonds[..., 0:1] - book.bonds[..., 1:2] * x)
    X[..., 15] = np.exp(book.bonds[..., 2:3] - book.bonds[..., 3:4] * x)
    del live
    return X


def test_features_follow_their_definition(ctx, book):
    fac = SB.factor_rows(ctx, book.model, 256)
    X = SB.features(ctx, book, fac)
    assert np.allclose(X, expected_features(book, fac), rtol=2e-6, atol=1e-6)


def test_book_netting_is_the_sum_of_trade_predictions(ctx, book):
    with Surrogate(ctx, seed=2) as s:
        X, y = SB.training_set(ctx, book, 128)
        s.train(X, y, epochs=1, batch=4096, lr=1e-3)
        fac = SB.factor_rows(ctx, book.model, 512)
        _, _, net, _ = SB.surrogate_exposure(s, book, fac, paths_out=32)
        F = SB.features(ctx, book, fac[:, :, :32].copy())
        pred = s.predict(F.reshape(-1, 16)).reshape(len(book.specs), len(book.times), 32)
        live = (book.times[None, :] < book.trades["maturity"][:, None] - 1e-6)[..., None]
        want = np.zeros_like(net)
        for i, tr in enumerate(book.trades):
            want[tr["netting_set"]] += tr["notional"] * pred[i] * live[i]
        assert np.abs(net - want).max() <= 1e-5 * np.abs(want).max()


def test_audited_surrogate_cva_within_half_a_percent(ctx, book):
    """Trained on 512 paths, applied to 2,048; netting sets whose audit misses by more than 0.5% of EPE go back to
    the plain pricer, so the book's CVA lands within 0.5% of the plain pricer's."""
    with Surrogate(ctx, seed=1) as s:
        X, y = SB.training_set(ctx, book, 512)
        for lr, ep in ((2e-3, 10), (5e-4, 6), (1e-4, 4)):
            losses = s.train(X, y, epochs=ep, batch=4096, lr=lr)
        assert losses[-1] < 0.01  # standardised mean squared error: R^2 above 0.99
        _, dee_p, _ = SB.plain_exposure(ctx, book, 2048)
        plain = SB.cva(book, dee_p).sum()
        run = SB.audited_exposure(ctx, s, book, 2048)
        assert abs(run.cva.sum() - plain) <= 0.005 * plain, (run.cva.sum(), plain, run.fallback)
        passed = [i for i in range(len(book.netting_sets)) if i not in run.fallback]
        assert all(run.audit_error[i] <= SB.AUDIT_TOLERANCE for i in passed)


def test_collateral_of_the_surrogate_book_is_the_csa_rule(ctx, book):
    """With the netting sets' cash CSAs the surrogate revalues every simulation date and the GPU applies the
    collateral rule per path: the result equals the oracle's collateral (collateral.cpp:10-47) applied to the same
    netted values on the host."""
    from oracle import restated

    m, books, _, _ = W.correlated_csa_book(2048, 10, 100, foreign_rates=False)
    cb = SB.make_book(m, books, csa=True)
    assert len(cb.times) > len(cb.report)  # the margin-call dates are revalued too
    with Surrogate(ctx, seed=2) as s:
        X, y = SB.training_set(ctx, book, 64)
        s.train(X, y, epochs=1, batch=4096, lr=1e-3)
        fac = SB.factor_rows(ctx, cb.factor_model, 256)
        _, _, e, _ = SB.surrogate_exposure(s, cb, fac, paths_out=64, all_dates=True)
        bare = SB.Book(**{**cb.__dict__, "csa": np.full_like(cb.csa, -1.0)})
        _, _, v, _ = SB.surrogate_exposure(s, bare, fac, paths_out=64, all_dates=True)
    t = np.asarray(gpu.compile(m, books[0], S.Options()).times, np.float64)  # the grid in double precision
    assert np.allclose(t, cb.times, atol=1e-6)
    for k, ns in enumerate(books):
        c = ns.csa
        coll = restated.collateral(v[k].T.astype(np.float64), t, c.threshold_cpty, c.threshold_own, c.mta, c.ia, c.mpr)
        want = v[k].T - coll
        scale = max(np.abs(v[k]).max(), 1.0)
        assert np.abs(e[k].T - want).max() <= 1e-5 * scale, k


def test_audited_surrogate_cva_with_csa(ctx, book):
    """The CSA book: the network trained on the uncollateralised trades, the audit and fallback against the plain
    pricer with the CSAs; the audited CVA within 0.5% of the plain pricer's."""
    m, books, _, _ = W.correlated_csa_book(2048, 10, 100, foreign_rates=False)
    cb = SB.make_book(m, books, csa=True)
    with Surrogate(ctx, seed=1) as s:
        X, y = SB.training_set(ctx, book, 256)
        for lr, ep in ((2e-3, 6), (5e-4, 3)):
            s.train(X, y, epochs=ep, batch=4096, lr=lr)
        _, dee_p, _ = SB.plain_exposure(ctx, cb, 2048)
        plain = SB.cva(cb, dee_p).sum()
        run = SB.audited_exposure(ctx, s, cb, 2048)
    assert abs(run.cva.sum() - plain) <= 0.005 * plain, (run.cva.sum(), plain, run.fallback)
    assert len(run.fallback) <= len(books)
