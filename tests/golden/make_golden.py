"""Generates the golden fixtures of the exposure path from the reference itself.

Run in a container that has the reference's sources (``make -C oracle ref`` builds oracle/_ref/libccr_ref.so
from them): ``python tests/golden/make_golden.py [name ...]``.  Each fixture holds the flat model / netting-set / options
arrays, the tables the reference's gpu::compile produced for them, and what the reference computed:

  fused_*.npz   gpu::runFusedReference (the reference's FP32 CPU kernels): sums and values; plus, for every
                quantile request, ccr::quantile of the reference's own exposure row at the plan's level
                (the exact value the fused pipeline approximates);
  engine_*.npz  ExposureEngine::run (FP64) on injected normals drawn from numpy's PCG64 with a stored seed:
                the exposure profile, pathwise CVA, and netted / collateral values on the reporting dates;
  nested_*.npz  nested::nestedExposure on the reference's own outer normals (NormalGenerator, restated by
                oracle/restated.py:normal_stream): per reporting date the exact, regression, uniform and adaptive
                EE* and PFE with the inner-path counts.

The tests read these files on machines without the reference (tests/test_oracle_pins.py).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from setups import bermudan, gpu_setup, swap_book, gpu_model  # noqa: E402
from zlatko_b200 import spec as S  # noqa: E402


def fused_cases():
    m, ns = gpu_setup(512, False)
    yield "fused_plain", m, ns, S.Options(per_trade=True, im_quantile=0.99)
    m, ns = gpu_setup(512, True)
    yield "fused_csa_views", m, ns, S.Options(samples=12, histogram_time=2.0, gross=True, collateral_bands=True,
                                              trade_views=True, pfe_quantile=0.975)
    m, ns = gpu_setup(384, True)
    ns.csa.kind, ns.csa.haircut, ns.csa.bond_maturity, ns.csa.mpr = 1, 0.02, 10.0, 20.0 / 250.0
    yield "fused_bond_collateral", m, ns, S.Options()
    m, ns = gpu_setup(384, True)
    ns.csa.kind, ns.csa.haircut, ns.csa.mpr = 2, 0.15, 20.0 / 250.0
    yield "fused_asset_collateral", m, ns, S.Options(factor_views=True, samples=5, bond_maturity=8.0)
    m, ns = gpu_setup(448, False)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0, 4.0), physical=True, degree=2))
    ns.trades.append(bermudan(exercise=(2.0, 3.0), physical=False, position=-0.5, degree=3))
    yield "fused_bermudan", m, ns, S.Options(exercise_views=True, samples=4)
    m = gpu_model(300, seed=11)
    m.base_grid = [k / 12 for k in range(1, 61)]
    yield "fused_swap_book", m, swap_book(6, seed=5, csa=S.Csa(1e5, 1e5, 1e4)), S.Options(pfe_quantile=0.9)
    m, ns = gpu_setup(256, True)
    ns.trades.append(bermudan(exercise=(1.0, 2.0, 3.0), degree=2))
    yield "fused_nested_im", m, ns, S.Options(im_quantile=0.99, im_inner_paths=64, samples=2)


def engine_cases():
    for csa in (False, True):
        m, ns = gpu_setup(256, csa)
        yield f"engine_{'csa' if csa else 'plain'}", m, ns, 5 if csa else 6


def nested_cases():
    """nestedExposure of the reference (the adaptive nest, src/nested/) on its own outer simulation."""
    from zlatko_b200 import nested as N

    m, ns = gpu_setup(400, False)
    o = N.AdaptiveOptions(inner_budget=150_000, max_rounds=20)
    yield "nested_exposure", m, ns, [0.5, 1.0, 2.0, 3.5], 0.95, o


def main() -> None:
    only = set(sys.argv[1:])  # fixture names to (re)generate; all when none are given
    if not ref.available():
        raise SystemExit("oracle/_ref/libccr_ref.so is not built: run `make -C oracle ref` where the reference is")
    for name, m, ns, o in fused_cases():
        if only and name not in only:
            continue
        em, en, eo = S.encode_model(m), S.encode_netting_set(ns), S.encode_options(o)
        r = ref.compile_plan(em, en, eo)
        sums, values = ref.run_fused(r)
        rows = ref.run_rows(r)
        exact = np.zeros_like(values)
        for q in r.requests.reshape(-1, 8):
            op, row, out = int(q[0]), int(q[1]), int(q[7])
            if op in (0, 7):
                x = rows[row].astype(np.float64)
                exact[out] = np.float32(ref.quantile(np.maximum(x, 0.0) if op == 7 else x, float(q[4])))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), model=em, netting_set=en, options=eo, header=r.header,
                            indices=r.indices, params=r.params, steps=r.steps, terms=r.terms, requests=r.requests,
                            rows_total=r.rows_total, num_outputs=r.num_outputs, times=r.times,
                            reporting=r.reporting.astype(np.int64), sums=sums, values=values, exact_quantiles=exact)
        print(name, r.num_dates, "dates", r.stats_per_date, "stats", len(r.requests) // 8, "requests")
    for name, m, ns, reporting, q, o in nested_cases():
        if only and name not in only:
            continue
        em, en = S.encode_model(m), S.encode_netting_set(ns)
        pts = ref.nested_exposure(em, en, reporting, q, o, True)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), model=em, netting_set=en, reporting=np.array(reporting),
                            pfe_quantile=q, adaptive=ref._adaptive_opts(o), seed=o.seed,
                            points=np.array([[p[k] for k in ref.NESTED_POINT_FIELDS] for p in pts]))
        print(name, len(pts), "points")
    for name, m, ns, seed in engine_cases():
        if only and name not in only:
            continue
        em, en = S.encode_model(m), S.encode_netting_set(ns)
        from zlatko_b200 import gpu

        p = gpu.compile(m, ns, S.Options())
        streams = (m.num_paths + 1) // 2
        z = np.random.default_rng(seed).standard_normal((p.num_dates - 1) * int(p.header[5]) * streams)
        e = ref.engine_run(em, en, 0.95, z, streams)
        rep = e.reporting
        np.savez_compressed(os.path.join(HERE, name + ".npz"), model=em, netting_set=en, seed=seed, streams=streams,
                            num_paths=m.num_paths,
                            num_normals=int(p.header[5]), times=e.times, reporting=rep,
                            profile=np.stack([e.profile[k] for k in ("ev", "ee", "ene", "pfe", "dee", "dene")]),
                            netted=e.netted[:, rep], collateral=e.collateral[:, rep], pathwise_cva_04=e.pathwise_cva_04)
        print(name, len(e.times), "dates")


if __name__ == "__main__":
    main()
