"""Netting sets with more than 4 Bermudan swaptions (the reference's kernel stops at 4 per netting set,
src/gpu/fused_exposure.cpp:161-189; config[4]'s largest netting sets hold about 90).  Beyond 4 the kernel keeps each
path's exercise indices in shared memory and the plan orders each Bermudan's exercise terms before its policy.

- FP64 mode against the FP64 engine on identical normals: every exercise decision of all 10 Bermudans identical,
  profiles and per-path netted values within 1e-9.
- FP32: the 10 Bermudans in one netting set against the same Bermudans in netting sets of at most 4 on the same
  scenario: the same fitted policies (each Bermudan is fitted on its own exercise values), the same exercise
  decisions path for path, and netted values that add up to rounding."""
import numpy as np
import pytest

from oracle import restated
from test_gpu_parity import injected_normals
from zlatko_b200 import gpu, workloads
from zlatko_b200 import spec as S
from zlatko_b200.summary import summarise

pytestmark = pytest.mark.gpu


def book(paths, n=10, csa=False):
    m, books, _ = workloads.bermudan_book(paths, n)
    trades = [t for b in books for t in b.trades][:n]
    trades[1] = S.Bermudan(trades[1].swap, trades[1].exercise, physical=False, position=-0.5, degree=2)
    return m, S.NettingSet(trades, S.Csa(1e5, 1e5, 1e4) if csa else None)


@pytest.mark.parametrize("csa", [False, True])
def test_fp64_many_bermudans_match_the_engine(ctx, csa):
    m, ns = book(2000, 10, csa)
    p = gpu.compile(m, ns, S.Options(exercise_views=True, samples=1))
    assert int(p.header[27]) == 10
    z, streams = injected_normals(p, 23)
    f = ctx.fit_amc_f64(p, z, streams)
    sums, vals, rows = ctx.run_f64(f, z, streams, rows=True)
    e = restated.engine_run(S.encode_model(m), S.encode_netting_set(ns), 0.95, z, streams, m.num_paths)
    ex = int(p.header[25])
    for b in range(10):
        assert np.array_equal(rows[ex + b], e.exercise[b]), f"Bermudan {b}: exercise decisions differ"
    res = summarise(f, sums, vals)
    for k in ("ev", "ee", "ene", "pfe", "dee", "dene"):
        scale = max(np.abs(e.profile[k]).max(), 1e-12)
        assert np.abs(res[k] - e.profile[k]).max() <= 1e-9 * scale, k
    H, rep = p.header, e.reporting
    scale = np.abs(e.netted).max()
    assert np.abs(rows[H[21]:H[21] + len(rep)].T - e.netted[:, rep]).max() <= 1e-9 * scale


def test_fp32_many_bermudans_equal_their_split_netting_sets(ctx):
    m, ns = book(8192, 10)
    o = S.Options(exercise_views=True, samples=1)
    whole = ctx.fit_amc(gpu.compile(m, ns, o))
    parts = [ctx.fit_amc(gpu.compile(m, S.NettingSet(ns.trades[k:k + 4], None), o)) for k in (0, 4, 8)]
    _, _, rw = ctx.run(whole, rows=True)
    got = [ctx.run(p, rows=True)[2] for p in parts]
    H = whole.header
    nR = whole.num_reporting
    for k, (p, r) in enumerate(zip(parts, got)):
        for b in range(int(p.header[27])):
            assert np.array_equal(rw[int(H[25]) + 4 * k + b], r[int(p.header[25]) + b]), (k, b)
    v_whole = rw[int(H[21]):int(H[21]) + nR].astype(np.float64)
    v_parts = sum(r[int(p.header[21]):int(p.header[21]) + nR].astype(np.float64) for p, r in zip(parts, got))
    assert np.abs(v_whole - v_parts).max() <= 1e-5 * np.abs(v_parts).max()
