"""Benchmark of the exposure hot path: scenario x trade revaluations per second.

Workload (default): the correlated CSA book at the size of the surrogate target -- 2,000 trades (1,200 swaps
with annual fixed and semiannual floating legs, 600 FX forwards, 200 FX options; the 60/30/10 mix of the
1,000-trade book scaled x2) in 100 collateralised netting sets of Zipf(1.2) sizes, 1,000,000 paths, 120 monthly
reporting dates to 10y (241 simulation dates with the margin-call dates t - MPR), HW1F + 2 lognormal FX + CIR++,
synthetic seeded data.  One step = the fused simulate -> revalue -> net -> collateralise -> reduce kernels over
every netting set, the reduction of the per-warp partials, and the row statistics (PFE 97.5% and means) of every
netting set and reporting date.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl zlatko|reference] [--paths P] [--trades N]

value   revaluations/s = paths x simulation dates x trades / device time of a step (CUDA events on the
        library's stream; inputs resident in HBM; L2 flushed between steps).  per_reporting_date counts the
        120 + 1 reporting dates only.
e2e     the same metric through the public C ABI (zk_run_plans): plan tables copied host -> device and
        statistics device -> host inside the timed region, wall clock of the blocking call.
--impl reference: the reference's own FP32 CPU kernels (gpu::runFusedReference, compiled from the reference
        sources into oracle/_ref) on the host cores, on plans its own gpu::compile builds, on a bounded sample
        of paths; this process never loads this library.
N > 1: replicas (the path runs on one GPU by design); every rank runs the workload, value = all ranks'
        revaluations / the slowest rank's time.
"""
from __future__ import annotations

import argparse
from dataclasses import replace
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "scenario x trade revaluations/s"
UNIT = "revals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="zlatko", choices=["zlatko", "reference"])
    ap.add_argument("--paths", type=int, default=1_000_000)
    ap.add_argument("--trades", type=int, default=2000)
    ap.add_argument("--netting-sets", type=int, default=100)
    ap.add_argument("--precision-paths", type=int, default=16_384, help="paths of the FP32-against-FP64 comparison")
    ap.add_argument("--no-precision", action="store_true", help="skip the FP32-against-FP64 comparison")
    ap.add_argument("--no-exact", action="store_true", help="skip the exact-decision leg")
    ap.add_argument("--exact-paths", type=int, default=65_536, help="paths of the exact-decision leg")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target duration of the CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--tile-paths", type=int, default=0, help="pin the tile shape (128/256/512) instead of the autotuned one")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate leg")
    ap.add_argument("--surrogate-paths", type=int, default=65_536)
    ap.add_argument("--surrogate-train-paths", type=int, default=512)
    ap.add_argument("--no-amc", action="store_true", help="skip the Bermudan (AMC) leg")
    ap.add_argument("--amc-paths", type=int, default=200_000)
    ap.add_argument("--no-amc-surrogate", action="store_true", help="skip the AMC continuation surrogate leg")
    ap.add_argument("--amc-sur-paths", type=int, default=100_000)
    ap.add_argument("--amc-sur-sets", type=int, default=4, help="netting sets (4 Bermudans each) of the AMC surrogate leg")
    ap.add_argument("--no-im", action="store_true", help="skip the nested initial-margin leg")
    ap.add_argument("--no-xva-batch", action="store_true", help="skip the large XVA batch leg")
    ap.add_argument("--xva-paths", type=int, default=1_000_000)
    ap.add_argument("--xva-steps", type=int, default=2)
    ap.add_argument("--no-nest", action="store_true", help="skip the adaptive nested-exposure leg")
    ap.add_argument("--nest-paths", type=int, default=4000)
    ap.add_argument("--im-paths", type=int, default=20_000)
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            with open(path) as f:
                d = json.load(f)
        except (OSError, ValueError):
            d = {}

        def find(node):  # "hbm_gbs" at the top, else the first numeric HBM GB/s entry anywhere
            if isinstance(node, dict):
                for k, v in node.items():
                    if "hbm" in str(k).lower() and "gb" in str(k).lower() and isinstance(v, (int, float)) and v > 0:
                        return float(v)
                for v in node.values():
                    r = find(v)
                    if r:
                        return r
            return None

        v = d.get("hbm_gbs") if isinstance(d, dict) else None
        v = float(v) if isinstance(v, (int, float)) and v > 0 else find(d)
        if v:
            return v, "measured"
    return 6650.0, "fallback"


def tensor_peak():
    """Dense BF16 / FP16 tensor TFLOP/s: the measured burst figure, else the fallback measured earlier on this pool."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = json.load(f).get("bf16_tflops")
        if isinstance(v, (int, float)) and v > 0:
            return float(v), "measured"
    except (OSError, ValueError, AttributeError):
        pass
    return 1590.0, "fallback"


def traffic_per_launch(paths: int, basis: bool = True):
    """DRAM bytes of one revalue launch from the committed ncu summary (the basis kernel's, or the term-by-term
    kernel's), scaled by paths."""
    path = os.path.join(ROOT, "profiles", "basis_book2000.txt" if basis else "revalue_book2000.txt")
    if not os.path.exists(path):
        return None
    ref_paths, ref_bytes = None, None
    for line in open(path):
        if line.startswith("capture_paths:"):
            ref_paths = float(line.split(":")[1])
        if line.startswith("dram_bytes_per_launch:"):
            ref_bytes = float(line.split(":")[1])
    if not ref_paths or not ref_bytes:
        return None
    return ref_bytes * paths / ref_paths


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def workload_name(trades: int, netting_sets: int, paths: int, foreign_rates: bool = True) -> str:
    n_swaps, n_fwds = round(0.6 * trades), round(0.3 * trades)
    model = ("3 Hull-White currencies (stochastic foreign rates) + 2 lognormal FX + CIR++, 6x6 correlation" if foreign_rates else
             "HW1F + 2 lognormal FX on deterministic foreign curves + CIR++ (the reference's model family)")
    return (f"correlated CSA book: {trades} trades ({n_swaps} IRS / {n_fwds} FX fwd / {trades - n_swaps - n_fwds} FX opt) in "
            f"{netting_sets} CSA netting sets Zipf(1.2), {model}, {paths} paths, 120 monthly reporting dates "
            "(241 simulation dates with the margin-call dates)")


def workload(paths: int, trades: int = 2000, netting_sets: int = 100, foreign_rates: bool = True):
    from zlatko_b200 import gpu, workloads

    m, books, opts, trades = workloads.correlated_csa_book(paths, netting_sets, trades, foreign_rates)
    t0 = time.perf_counter()
    plans = [gpu.compile(m, b, opts) for b in books]
    compile_s = time.perf_counter() - t0
    return m, books, opts, trades, plans, compile_s


def cpu_reference(plans, trades: int, target_s: float, steps: int = 1):
    """The reference's FP32 CPU kernels (gpu::runFusedReference, built from the reference's sources into
    oracle/_ref) on all host threads over a bounded sample of paths of every netting set's plan.  Where that
    library is absent, the plain-C restatement of the same kernels (oracle/fused_oracle.c, one thread).
    Returns (revals/s, sample paths, threads, seconds, per-step seconds, kind)."""
    from oracle import ref

    nT = plans[0].num_dates
    if ref.available():
        kind, threads = "reference", os.cpu_count() or 1

        def run(paths):
            rps = [ref.plan_from_buffers(p.header, p.indices, p.params, p.steps, p.terms, p.requests, p.rows_total,
                                         p.num_outputs, p.times, p.reporting, num_paths=paths) for p in plans]
            t0 = time.perf_counter()
            for rp in rps:
                ref.run_fused(rp, threads)
            return time.perf_counter() - t0
    else:
        from oracle import restated

        kind, threads = "port", 1

        def run(paths):
            heads = []
            for p in plans:
                h = p.header.copy()
                h[0], h[15] = paths, (paths + 63) // 64
                heads.append(h)
            t0 = time.perf_counter()
            for p, h in zip(plans, heads):
                restated.run_fused(h, p.indices, p.params, p.steps, p.terms, p.requests, p.rows_total, p.num_outputs)
            return time.perf_counter() - t0

    probe = 256 if kind == "reference" else 64
    dt = run(probe)
    paths = int(max(probe, min(64 * probe, probe * target_s / max(dt, 1e-3))) // 64 * 64)
    times = [run(paths) for _ in range(steps)]
    dt = float(np.median(times))
    return paths * nT * trades / dt, paths, threads, dt, times, kind


def replica_throughput(units: float, t_device: float, t_e2e: float, world: int, dist=None, device: str = "cpu"):
    """Whole-job throughput of `world` replicas: every rank processed `units`; the job takes the slowest rank's
    time (max over ranks of the device time and of the end-to-end time).  Returns (value, e2e, t_device, t_e2e)."""
    if dist is not None and world > 1:
        import torch

        t = torch.tensor([t_device, t_e2e], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_device, t_e2e = float(t[0]), float(t[1])
    total = units * world
    return total / t_device, total / t_e2e, t_device, t_e2e


def exact_leg(ctx, a):
    """The exact-decision check (zk_context_set_exact_decisions, guard 3e-7) on the bench's book (three-currency
    model, 2,000 trades in 100 netting sets with cash CSAs): the wall time of one zk_run_plans call (uploads and
    read-back included) without it (tensor-core basis kernel; term by term) and with it (term by term, then the
    flagged paths again in FP64 and FP32), and the share of paths it re-ran."""
    from zlatko_b200 import gpu, workloads

    m, books, opts, _ = workloads.correlated_csa_book(a.exact_paths, num_trades=a.trades, netting_sets=a.netting_sets)
    plans = [gpu.compile(m, b, opts) for b in books]

    def timed(guard, basis):
        ctx.set_exact_decisions(guard)
        ctx.set_basis(basis)
        ctx.run_many(plans)  # warm-up
        ctx.exact_stats()
        t0 = time.perf_counter()
        ctx.run_many(plans)
        return time.perf_counter() - t0, ctx.exact_stats()

    try:
        basis_s, _ = timed(0.0, ctx.BASIS_AUTO)
        term_s, _ = timed(0.0, ctx.BASIS_OFF)
        exact_s, (flagged, checked) = timed(3e-7, ctx.BASIS_AUTO)
    finally:
        ctx.set_exact_decisions(0.0)
        ctx.set_basis(ctx.BASIS_AUTO)
    return {"workload": f"the bench's book on {a.exact_paths} paths, zk_run_plans (host buffers)", "guard": 3e-7,
            "s_basis_kernel": basis_s, "s_term_kernel": term_s, "s_exact": exact_s,
            "paths_rerun_fp64": flagged, "paths_checked": checked,
            "share_rerun": flagged / checked if checked else None,
            "note": "decisions equal to the FP64 mode's (tests/test_gpu_exact_decisions.py)"}


def guarded(fn, *args):
    try:
        return fn(*args)
    except Exception as exc:  # pragma: no cover - reported in the JSON line instead of failing the bench
        return {"unavailable": f"{type(exc).__name__}: {exc}"}


def surrogate_leg(ctx, a):
    """CVA of the bench's book, with its cash CSAs, by the surrogate with its 1% plain-pricer audit and
    per-netting-set fallback, against the plain GPU pricer on the same paths: device time of each, the CVA difference
    and the fallbacks.  The surrogate revalues every simulation date (the margin-call dates included) and the GPU
    applies the collateral rule per path.  The network is trained on the per-trade values the plain pricer itself
    produces on --surrogate-train-paths paths (every live trade and reporting date: about 53M revaluations for this
    book at 512 paths, the 50M the surrogate configuration asks for); training is reported apart, it runs once per
    book."""
    from zlatko_b200 import surrogate_book as SB
    from zlatko_b200 import workloads
    from zlatko_b200.surrogate import Surrogate

    # The surrogate's features cover the reference's model family: deterministic foreign curves.
    m, books, _, trades = workloads.correlated_csa_book(a.surrogate_paths, a.netting_sets, a.trades, foreign_rates=False)
    train_book = SB.make_book(m, books)
    book = SB.make_book(m, books, csa=True)
    t0 = time.perf_counter()
    X, y = SB.training_set(ctx, train_book, a.surrogate_train_paths)
    rows_s = time.perf_counter() - t0
    with Surrogate(ctx, seed=1) as s:
        t0 = time.perf_counter()
        losses = []
        for lr, ep in ((2e-3, 2), (5e-4, 1), (1e-4, 1)):
            losses += list(s.train(X, y, epochs=ep, batch=8192, lr=lr))
        train_s = time.perf_counter() - t0
        _, dee_p, ms_plain = SB.plain_exposure(ctx, book, a.surrogate_paths)
        run = SB.audited_exposure(ctx, s, book, a.surrogate_paths)
    plain = float(SB.cva(book, dee_p).sum())
    ms_sur = run.ms_surrogate + run.ms_audit + run.ms_fallback
    revals = float(a.surrogate_paths) * len(book.times) * trades
    return {"workload": f"the bench's book with its cash CSAs: {trades} trades in {len(books)} netting sets, {a.surrogate_paths} "
                        f"paths, {len(book.times)} simulation dates (margin-call dates included), reference model family; "
                        f"trained on {a.surrogate_train_paths} paths",
            "cva_plain": plain, "cva_surrogate_audited": float(run.cva.sum()),
            "delta_cva_rel": float(run.cva.sum() / plain - 1.0),
            "ms_plain": ms_plain, "ms_surrogate": run.ms_surrogate, "ms_audit": run.ms_audit, "ms_fallback": run.ms_fallback,
            "speedup_vs_plain": ms_plain / ms_sur if ms_sur > 0 else None,
            "surrogate_revals_per_s": revals / (run.ms_surrogate / 1e3),
            "plain_revals_per_s": revals / (ms_plain / 1e3),
            "fallback_netting_sets": len(run.fallback), "netting_sets": len(books),
            "audit_error_median": float(np.median(run.audit_error)), "train_rows": int(len(y)),
            "training_rows_s": rows_s, "train_s": train_s, "train_loss": float(losses[-1])}


def amc_leg(ctx, a):
    """Bermudan swaption book: the Longstaff-Schwartz fit on the GPU (zk_fit_amc, with its AMC state pass) and the
    fused revaluation of the fitted plans."""
    from zlatko_b200 import gpu, workloads
    from zlatko_b200 import spec as S

    m, books, n = workloads.bermudan_book(a.amc_paths)
    plans = [gpu.compile(m, b, S.Options()) for b in books]
    ctx.fit_amc(plans[0])  # warm-up
    t0 = time.perf_counter()
    fitted = [ctx.fit_amc(p) for p in plans]
    fit_s = time.perf_counter() - t0
    b = ctx.batch(fitted)
    try:
        for _ in range(3):
            b.execute()
        b.execute()
        ms = float(np.sum(b.timings()))
    finally:
        b.close()
    nT = plans[0].num_dates
    revals = float(a.amc_paths) * nT * n
    line = {"workload": f"{n} Bermudan swaptions (10y, annual exercise 1y-9y, degree 3) in {len(books)} netting sets, "
                        f"{a.amc_paths} paths, {nT} dates",
            "fit_s": fit_s, "revalue_ms": ms, "revals_per_s": revals / (fit_s + ms / 1e3),
            "revalue_revals_per_s": revals / (ms / 1e3),
            "fit_unit": "Bermudan path-dates fitted/s", "fit_rate": revals / fit_s}
    # The same book with the two-regressor basis (short rate and co-terminal swap rate, 10 functions of degree <= 3).
    m2, books2, _ = workloads.bermudan_book(a.amc_paths, basis="rate_swap")
    plans2 = [gpu.compile(m2, b, S.Options()) for b in books2]
    ctx.fit_amc(plans2[0])  # warm-up
    t0 = time.perf_counter()
    fitted2 = [ctx.fit_amc(p) for p in plans2]
    fit2_s = time.perf_counter() - t0
    b2 = ctx.batch(fitted2)
    try:
        for _ in range(3):
            b2.execute()
        b2.execute()
        ms2 = float(np.sum(b2.timings()))
    finally:
        b2.close()
    line["two_regressor"] = {"basis": "1, z, w, z^2, z w, w^2, z^3, z^2 w, z w^2, w^3 (z short rate, w co-terminal swap rate)",
                             "fit_s": fit2_s, "revalue_ms": ms2, "revals_per_s": revals / (fit2_s + ms2 / 1e3),
                             "fit_rate": revals / fit2_s}
    from oracle import ref
    if not a.no_cpu and ref.available():
        # The reference's gpu::compile fits the same book with its CPU kernels (fitAmc on the SpinPool, all host
        # threads) on a bounded sample of paths: the fit's work is linear in the paths.
        sample = min(a.amc_paths, 10_000)
        ms_, bs_, _ = workloads.bermudan_book(sample)
        mflat, oflat = S.encode_model(ms_), S.encode_options(S.Options())
        t0 = time.perf_counter()
        for bk in bs_:
            ref.compile_plan(mflat, S.encode_netting_set(bk), oflat)
        cpu_s = time.perf_counter() - t0
        cpu_rate = float(sample) * nT * n / cpu_s
        line["cpu_baseline"] = {"value": cpu_rate, "unit": "Bermudan path-dates fitted/s", "cores": os.cpu_count() or 1,
                                "kind": "reference", "sample": f"all {len(bs_)} netting sets on {sample} paths "
                                                               f"(gpu::compile with fitAmc): {cpu_s:.2f} s"}
        line["fit_speedup_vs_cpu"] = line["fit_rate"] / cpu_rate
    return line


def amc_surrogate_leg(ctx, a):
    """The AMC continuation value of the Bermudan book by the learned surrogate against the Longstaff-Schwartz
    regression: one network for every date and Bermudan of the first netting sets, trained on the realised values of
    the AMC pass under the fitted policy, compared on held-out paths (another seed) by mean squared error against
    the realised values; and the network's inference rate on those rows."""
    from zlatko_b200 import amc_surrogate as AS
    from zlatko_b200 import workloads
    from zlatko_b200.surrogate import Surrogate

    m, books, _ = workloads.bermudan_book(a.amc_sur_paths)
    books = books[:a.amc_sur_sets]
    t0 = time.perf_counter()
    X, y, poly, fitted = AS.book_rows(ctx, m, books)
    rows_s = time.perf_counter() - t0
    import torch

    with Surrogate(ctx, seed=4) as s:
        t0 = time.perf_counter()
        losses = []
        for lr, ep in ((2e-3, 2), (5e-4, 1), (1e-4, 1)):
            losses += list(s.train(X, y, epochs=ep, batch=8192, lr=lr))
        train_s = time.perf_counter() - t0
        r = AS.compare(ctx, s, m, books, fitted, paths=a.amc_sur_paths // 4, seed=4242)
        Xh = X[: min(len(X), 8_000_000)]
        s.predict(Xh[:65536])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.predict(Xh)
        infer_s = time.perf_counter() - t0
    nb = sum(len(b.trades) for b in books)
    r.update({"workload": f"{nb} Bermudan swaptions of the AMC book, {a.amc_sur_paths} training paths, {len(y)} training rows "
                          f"(every date with an exercise ahead), held out on {a.amc_sur_paths // 4} paths of another seed",
              "train_rows": int(len(y)), "rows_s": rows_s, "train_s": train_s, "train_loss": float(losses[-1]),
              "infer_rows_per_s": len(Xh) / infer_s,
              "note": "infer_rows_per_s is the network's rate through zk_surrogate_predict from host buffers; the "
                      "regression's polynomial is evaluated inside the fused kernel at no measurable cost"})
    return r


def xva_batch_leg(ctx, a):
    """config[4]: the large wrong-way-risk XVA batch (10,000 trades with 5% Bermudans in 500 netting sets over 8
    portfolios, intensity correlated 0.3 with the domestic rate), every netting set with and without its CSA -- 1,000
    plans on one scenario -- as one batch replaying one captured graph, its rows and partials in waves within the
    row budget.  The Bermudans are fitted on the GPU (zk_fit_amc, on the CSA plan; the uncollateralised twin runs on
    the same grid and takes the same fitted records).  CVA (the counterparty curve) and DVA (own hazard 0.5%, LGD
    0.6) per portfolio, collateralised and not."""
    from zlatko_b200 import gpu, workloads
    from zlatko_b200 import spec as S
    from zlatko_b200.summary import bilateral_cva, summarise

    m, cb, pb, port, trades = workloads.xva_batch(a.xva_paths)
    o = S.Options(pfe_quantile=0.975)
    t0 = time.perf_counter()
    csa = [gpu.compile(m, b, o) for b in cb]
    grid = tuple(float(t) for t in csa[0].times)
    plain = [gpu.compile(m, b, replace(o, extra_dates=grid)) for b in pb]
    compile_s = time.perf_counter() - t0
    assert all(p.num_dates == csa[0].num_dates for p in csa + plain)
    t0 = time.perf_counter()
    bermudans = 0
    for i, p in enumerate(csa):
        if int(p.header[27]) > 0:
            bermudans += int(p.header[27])
            f = ctx.fit_amc(p)
            csa[i] = f
            q = plain[i]
            plain[i] = gpu.Plan.from_arrays(q.header, q.indices, q.params, q.steps, f.terms, q.requests, q.rows_total,
                                            q.num_outputs, q.times, q.reporting)
    fit_s = time.perf_counter() - t0
    # The tile shape: the autotuner's choice on the same batch at 65,536 paths, pinned on the full batch (tuning at
    # full size would take six executes of the whole batch).
    small = []
    for p in csa + plain:
        h = p.header.copy()
        h[0], h[15] = min(65536, a.xva_paths), (min(65536, a.xva_paths) + 63) // 64
        small.append(gpu.Plan.from_arrays(h, p.indices, p.params, p.steps, p.terms, p.requests, p.rows_total, p.num_outputs,
                                          p.times, p.reporting))
    tb = ctx.batch(small)
    try:
        tb.execute()
        tile = int(tb.info().tile_paths)
    finally:
        tb.close()
    b = ctx.batch(csa + plain)
    try:
        b.set_tile_paths(tile)
        b.execute()  # captures the graph
        ms = []
        for _ in range(a.xva_steps):
            b.execute()
            ms.append(float(np.sum(b.timings())))
        out = b.read()
        info = b.info()
    finally:
        b.close()
    own = ([1.0], [0.005])
    cp = m.credits[0]
    res = {"collateralised": [0.0] * 8, "uncollateralised": [0.0] * 8}
    dva = {"collateralised": [0.0] * 8, "uncollateralised": [0.0] * 8}
    for k, (p, (sums, vals)) in enumerate(zip(csa + plain, out)):
        r = summarise(p, sums, vals)
        c, d = bilateral_cva(r["times"], r["dee"], r["dene"], (list(cp.pillars), list(cp.hazards)), own, 0.4, 0.4)
        kind = "collateralised" if k < len(csa) else "uncollateralised"
        res[kind][port[k % len(csa)]] += c
        dva[kind][port[k % len(csa)]] += d
    nT = csa[0].num_dates
    revals = float(a.xva_paths) * nT * trades * 2
    step = float(np.median(ms))
    return {"workload": f"{trades} trades (60% IRS, 25% FX fwd, 10% FX opt, {bermudans} Bermudans) in {len(cb)} netting sets "
                        f"Zipf(1.1) over 8 portfolios, each with and without its CSA ({2 * len(cb)} plans), three-currency "
                        f"model with intensity-rate correlation 0.3, {a.xva_paths} paths, {nT} simulation dates",
            "revals_per_s": revals / (step / 1e3), "ms_per_step": step, "waves": int(info.num_waves), "tile_paths": tile,
            "kernels_per_execute": int(info.kernels_per_execute), "graph_replay": int(info.graph_replay),
            "largest_netting_set": {"trades": max(len(x.trades) for x in cb),
                                    "bermudans": max(sum(isinstance(t, S.Bermudan) for t in x.trades) for x in cb)},
            "compile_s": compile_s, "amc_fit_s": fit_s,
            "cva_by_portfolio": res, "dva_by_portfolio": dva,
            "note": "collateralised and uncollateralised EE / PFE of every netting set come out of the same batch; "
                    "the surrogate is not applied here (it revalues swaps, forwards and options without a CSA)"}


def inner_revaluations(plan, trades: int) -> float:
    """Inner path-date-trade revaluations of one run of a plan with the nested margin: every path, on every
    reporting date with a target, steps its inner paths to the target date and revalues the netting set there."""
    nT, nP, nInner = plan.num_dates, plan.num_paths, int(plan.header[30])
    I = plan.indices
    rep, tgt = I[2 * nT + 1:3 * nT + 1], I[3 * nT + 1:4 * nT + 1]
    dates = sum(int(tgt[j]) - j for j in range(nT) if rep[j] > 0 and tgt[j] != 0xFFFFFFFF)
    return float(nP) * nInner * dates * trades


def im_leg(ctx, a):
    """Nested conditional initial margin with the reference's XVA defaults (128 inner paths, the 99% quantile,
    a 10-day margin period) on the book's largest netting set: inner revaluations per second of the whole plan
    on the GPU and on the reference's CPU kernels (a path sample, all host threads), and the device time of the
    inner Monte Carlo (the plan's revalue phase with the margin minus without)."""
    from oracle import ref
    from zlatko_b200 import gpu, workloads
    from zlatko_b200 import spec as S

    m, books, _, _ = workloads.correlated_csa_book(a.im_paths, foreign_rates=False)  # the reference's nested-margin model
    ns = max(books, key=lambda b: len(b.trades))
    p_im, p0 = gpu.compile(m, ns, S.Options(im_quantile=0.99, im_inner_paths=128)), gpu.compile(m, ns, S.Options(im_quantile=0.99))

    def device_ms(p):
        b = ctx.batch([p])
        try:
            for _ in range(3):
                b.execute()  # the first execute autotunes the tile shape
            t = []
            for _ in range(5):
                b.execute()
                t.append(b.timings())
            return np.median(np.array(t), axis=0)
        finally:
            b.close()

    ms_im, ms0 = device_ms(p_im), device_ms(p0)
    trades = len(ns.trades)
    inner = inner_revaluations(p_im, trades)
    line = {"workload": f"largest CSA netting set of the correlated book ({trades} trades), {a.im_paths} paths, 128 inner paths, "
                        f"99% quantile, 10-day margin period, {p_im.num_dates} dates",
            "inner_revals_per_s": inner / (float(ms_im.sum()) / 1e3), "plan_ms": float(ms_im.sum()),
            "inner_mc_ms": float(ms_im[1] - ms0[1]), "plan_without_margin_ms": float(ms0.sum())}
    if not a.no_cpu:
        if ref.available():
            kind, threads = "reference", os.cpu_count() or 1

            def run(n):
                rp = ref.plan_from_buffers(p_im.header, p_im.indices, p_im.params, p_im.steps, p_im.terms, p_im.requests,
                                           p_im.rows_total, p_im.num_outputs, p_im.times, p_im.reporting, num_paths=n)
                t0 = time.perf_counter()
                ref.run_fused(rp, threads)
                return time.perf_counter() - t0
        else:
            from oracle import restated

            kind, threads = "port", 1

            def run(n):
                h = p_im.header.copy()
                h[0], h[15] = n, (n + 63) // 64
                t0 = time.perf_counter()
                restated.run_fused(h, p_im.indices, p_im.params, p_im.steps, p_im.terms, p_im.requests, p_im.rows_total,
                                   p_im.num_outputs)
                return time.perf_counter() - t0

        sample = 64
        dt = run(sample)
        sample = int(min(a.im_paths, max(64, sample * 5.0 / max(dt, 1e-3))) // 64 * 64)  # about 5 s of CPU work
        dt = run(sample)
        cpu = inner * sample / a.im_paths / dt
        line["cpu_baseline"] = {"value": cpu, "unit": "inner revaluations/s", "cores": threads, "kind": kind,
                                "sample": f"{sample} of {a.im_paths} paths of the same plan"}
        line["speedup_vs_cpu"] = line["inner_revals_per_s"] / cpu
    return line


def nest_leg(ctx, a):
    """Exposure by the adaptive nest (the reference's defaults: 2M inner paths per date, 50 rounds) of 32 trades on
    the correlated book's model, quarterly to 5y: the inner simulations on the GPU (one launch per round) and the
    reference's nestedExposure on all host threads.  The two arms draw their own outer scenarios (the GPU's
    counter-based normals, the reference's Mersenne twister), so they are compared by inner paths per second."""
    from oracle import ref
    from zlatko_b200 import nested_exposure as E
    from zlatko_b200 import spec as S
    from zlatko_b200 import workloads

    m, _, _, _ = workloads.correlated_csa_book(a.nest_paths, foreign_rates=False)  # the reference's nested model
    ns = workloads.nested_netting_set()
    reporting = [q / 4.0 for q in range(1, 21)]
    o = E.NestedExposureOptions()
    E.nested_exposure(ctx, replace(m, num_paths=512), ns, reporting[:2], o)  # warm-up
    t0 = time.perf_counter()
    res = E.nested_exposure(ctx, m, ns, reporting, o)
    gpu_s = time.perf_counter() - t0
    line = {"workload": f"{len(ns.trades)} trades (20 swaps, 8 FX forwards, 4 FX options), {a.nest_paths} outer paths, "
                        f"{len(reporting)} quarterly dates, adaptive nest with the reference's defaults",
            "wall_s": gpu_s, "inner_paths": res.inner_paths, "inner_launches": res.inner_launches,
            "inner_paths_per_s": res.inner_paths / gpu_s}
    if not a.no_cpu and ref.available():
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        pts = ref.nested_exposure(S.encode_model(m), S.encode_netting_set(ns), reporting, o.pfe_quantile, o.adaptive, True, threads)
        cpu_s = time.perf_counter() - t0
        inner = sum(p["inner_paths"] for p in pts)
        line["cpu_baseline"] = {"value": inner / cpu_s, "unit": "inner paths/s", "cores": threads, "kind": "reference",
                                "sample": f"the whole workload (nestedExposure, {threads} threads): {cpu_s:.2f} s, {int(inner)} inner paths"}
        line["speedup_vs_cpu"] = line["inner_paths_per_s"] / line["cpu_baseline"]["value"]
    return line


def replace_args(a, **kw):
    b = argparse.Namespace(**vars(a))
    for k, v in kw.items():
        setattr(b, k, v)
    return b


def precision_leg(ctx, a):
    """The error of the FP32 path against the FP64 mode for every output of every netting set (EE, ENE, PFE, EE*,
    ENE* per reporting date; CVA, first-to-default CVA and DVA with an own hazard of 0.5%, pathwise CVA), beside
    its Monte Carlo standard error (batch means over 8 independent seeds), on the bench's book at fewer paths."""
    from zlatko_b200 import precision, workloads
    from zlatko_b200 import spec as S

    m, books, opts, _ = workloads.correlated_csa_book(a.precision_paths, a.netting_sets, a.trades)
    own = S.Credit(1e-6, 0.0, 0.0, 0.0, [1.0], [0.005], substeps=1)
    t0 = time.perf_counter()
    r = precision.compare(ctx, m, books, opts, own)
    r["wall_s"] = time.perf_counter() - t0
    r["all_below_se"] = all(v["max_err_over_se"] < 1.0 for v in r["outputs"].values())
    r["note"] = ("max_err_over_se: largest |FP32 - FP64| / (Monte Carlo standard error, per path from the FP64 rows) over "
                 "netting sets and dates; entries without Monte Carlo error (date 0) are compared relative to the output's "
                 "scale instead")
    return r


def reference_arm(a) -> dict:
    """The reference's own path on the host cores: gpu::compile (src/gpu/fused_exposure.cpp:214) builds the plans
    and gpu::runFusedReference (src/gpu/fused_reference.cpp:628-630) runs them on all host threads, both from the
    reference's sources compiled into oracle/_ref.  The book comes from the pure-Python generator; this library's
    compiler and kernels are never loaded.  The reference's compile caps a netting set at 32 swaps
    (src/gpu/fused_exposure.cpp:161-189), and a two-schedule swap enters it as three one-schedule swaps, so the
    largest netting sets are left out: the rate is measured on the netting sets it accepts, per trade, on a sample
    of the paths of each step, and that is stated on the line."""
    from oracle import ref
    from zlatko_b200 import spec as S
    from zlatko_b200 import workloads

    if not ref.available():
        return {"impl": "reference", "unavailable": "the reference library oracle/_ref/libccr_ref.so was not built"}
    # The reference's own model family: its foreign curves are deterministic (it has no stochastic foreign rates).
    m, books, opts, trades = workloads.correlated_csa_book(a.paths, a.netting_sets, a.trades, foreign_rates=False)
    mflat, oflat = S.encode_model(m), S.encode_options(opts)
    plans, kept, left_out = [], 0, []
    for i, b in enumerate(books):
        try:
            plans.append(ref.compile_plan(mflat, S.encode_netting_set(b), oflat))
            kept += len(b.trades)
        except ValueError as exc:
            left_out.append({"netting_set": i, "trades": len(b.trades), "why": str(exc)[:120]})
    if not plans:
        return {"impl": "reference", "unavailable": "the reference's gpu::compile accepts none of the book's netting sets"}
    nT = plans[0].num_dates
    threads = os.cpu_count() or 1

    def run(paths):
        for p in plans:
            p.set_paths(paths)
        t0 = time.perf_counter()
        for p in plans:
            ref.run_fused(p, threads)
        return time.perf_counter() - t0

    per_step = max(2.0, a.cpu_seconds / max(a.steps, 1))
    probe = 256
    dt = run(probe)
    paths = int(max(probe, min(a.paths, probe * per_step / max(dt, 1e-3))) // 64 * 64)
    for _ in range(min(a.warmup, 1)):
        run(min(paths, 1024))
    times = [run(paths) for _ in range(a.steps)]
    dt = float(np.median(times))
    value = paths * nT * kept / dt
    sample = (f"{paths} of {a.paths} paths per step of the {len(plans)} netting sets ({kept} of {trades} trades) that the "
              f"reference's gpu::compile accepts; {len(left_out)} netting sets above its 32-swap cap left out; "
              f"gpu::runFusedReference on {threads} threads")
    return {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(trades, a.netting_sets, a.paths, foreign_rates=False), "paths_per_step": paths,
                       "simulation_dates": nT, "trades_timed": kept, "netting_sets_timed": len(plans),
                       "netting_sets_left_out": left_out},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if a.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(reference_arm(a)))
        return

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    device = torch.cuda.current_device()
    from zlatko_b200 import gpu
    from zlatko_b200._native import lib

    m, books, opts, trades, plans, compile_s = workload(a.paths, a.trades, a.netting_sets)
    nT, nP = plans[0].num_dates, plans[0].num_paths
    nR = len(plans[0].reporting)
    revals = float(nP) * nT * trades
    ctx = gpu.Context(device)
    batch = ctx.batch(plans)
    if a.tile_paths:
        batch.set_tile_paths(a.tile_paths)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    for _ in range(max(a.warmup, 3)):
        batch.execute()  # the first execute autotunes the tile shape
    batch.read()
    info = batch.info()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    step_ms, sim_ms, fused_ms, reduce_ms, rows_ms = [], [], [], [], []
    with ClockSampler(device) as clocks:
        torch.cuda.synchronize()
        for _ in range(a.steps):
            flush.zero_()  # L2 flush between steps (outside the step's events)
            torch.cuda.synchronize()
            batch.execute()
            ms = batch.timings()
            sim_ms.append(ms[0]), fused_ms.append(ms[1]), reduce_ms.append(ms[2]), rows_ms.append(ms[3])
            step_ms.append(float(ms.sum()))
        torch.cuda.synchronize()
        batch.close()  # its device arena goes back before the context allocates its own for the calls below
        # e2e through the public C ABI: host plan tables in, host statistics out.
        for _ in range(a.warmup):
            ctx.run_many(plans)
        e2e_s, phases = [], []
        for _ in range(a.steps):
            t0 = time.perf_counter()
            ctx.run_many(plans)
            e2e_s.append(time.perf_counter() - t0)
            phases.append(ctx.call_timings())
    value, e2e, t_step, t_e2e = replica_throughput(revals * a.steps, float(np.sum(step_ms)) / 1e3, float(np.sum(e2e_s)), world,
                                                   dist, "cuda")

    peak, peak_kind = peaks()
    fused_s = float(np.mean(fused_ms)) / 1e3
    nA, nC = int(plans[0].header[2]), int(plans[0].header[3])
    nF = (int(plans[0].header[10]) - 6) // 2
    cube_bytes = (2 + nA + nC + nF) * nT * nP * 4  # factor state read once (L2 serves the other netting sets)
    # statistics partials: one per 64 paths on the basis kernel, one per revalue warp term by term
    nb = int(info.num_basis_netting_sets)
    units = [-(-nP // 64) if k < nb else -(-nP // (32 * (int(info.tile_paths) // 128))) for k in range(len(plans))]
    alg_bytes = (sum(p.rows_total * nP * 4 + u * nT * p.stats_per_date * 4 for p, u in zip(plans, units)) + info.table_bytes +
                 cube_bytes + int(info.basis_bytes))
    # the basis kernel's products: per 128-path tile and column, C_hi Phi_hi + C_hi Phi_lo + C_lo Phi_hi over 128 rows
    tensor_flops = 2.0 * 3 * 128 * (-(-nP // 128) * 128) * float(info.basis_columns)
    tpeak, tpeak_kind = tensor_peak()
    ex2 = C_ex2 = None
    try:
        import ctypes as C

        g = C.c_double()
        if lib().zk_peak_ex2(device, C.byref(g)) == 0:
            C_ex2 = g.value * 1e9
    except Exception:
        C_ex2 = None
    exp_per_launch = float(info.exp_evaluations) * nP  # one ex2 per bond-like term and path
    row_bytes = float(sum(p.rows_total for p in plans)) * nP * 4
    h2d = info.table_bytes + sum(p.indices.size * 4 for p in plans) + int(info.basis_bytes)
    d2h = sum((p.sums_len() + p.values_len()) * 4 for p in plans)

    if rank == 0:
        cpu = None
        try:
            if a.no_cpu:
                raise RuntimeError("skipped (--no-cpu)")
            if world > 1:
                raise RuntimeError("measured with --gpus 1 only")
            r = reference_arm(replace_args(a, steps=1, warmup=0, cpu_seconds=a.cpu_seconds / 2))
            if "unavailable" in r:  # the reference library is absent: the plain-C restatement of its kernels, on the
                # book in the reference's model family (the restatement has no stochastic foreign rates)
                lplans = workload(a.paths, a.trades, a.netting_sets, foreign_rates=False)[4]
                cv, cpaths, cthreads, cdt, _, ckind = cpu_reference(lplans, trades, a.cpu_seconds / 2)
                cpu = {"value": cv, "unit": UNIT, "cores": cthreads, "kind": ckind,
                       "sample": f"{cpaths} of {nP} paths of all {len(plans)} netting sets (the plain-C restatement of "
                                 f"gpu::runFusedReference, {cthreads} threads)"}
            else:
                cpu = dict(r["cpu_baseline"])
        except Exception as exc:  # pragma: no cover
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {exc}"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": t_step / a.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(trades, len(plans), nP), "paths": nP, "simulation_dates": nT,
                       "reporting_dates": nR, "trades": trades, "netting_sets": len(plans),
                       "l2": "flushed between steps (256 MB write); the step's rows and partials exceed L2 anyway",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "per_reporting_date": {"value": value * nR / nT, "unit": "scenario x trade revaluations/s on reporting dates",
                                   "note": "paths x reporting dates x trades / device time; the other simulation dates "
                                           "are the margin-call dates t - MPR"},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "host_ms_median": {k: float(np.median([ph[k] for ph in phases])) for k in phases[0]} if phases else None},
            "gpu_launches": int(info.kernels_per_execute) * a.steps,
            "tile_paths": int(info.tile_paths),
            "kernel_ms": {"simulate": float(np.mean(sim_ms)), "revalue": float(np.mean(fused_ms)), "reduce": float(np.mean(reduce_ms)),
                          "row_stats": float(np.mean(rows_ms))},
            "roofline": {"bound": "hbm", "achieved": alg_bytes / fused_s / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg_bytes / fused_s / 1e9 / peak, "traffic": traffic_per_launch(nP, nb > 0),
                         "note": f"revalue step (the dominant kernel: {'basisRevalueKernel' if nb else 'revalueKernel'}); "
                                 f"peak of {peak_kind}; algorithmic bytes = factor cube read once + PFE rows written + "
                                 "per-unit partials + plan and basis tables"},
            "roofline_tensor": {"bound": "tensor", "achieved": tensor_flops / fused_s / 1e12, "peak": tpeak, "unit": "TFLOP/s",
                                "frac": tensor_flops / fused_s / 1e12 / tpeak,
                                "note": f"basisRevalueKernel's FP16 hi/lo products (3 MMAs per 16 columns) against the dense "
                                        f"BF16/FP16 peak of {tpeak_kind}; the kernel is bound by its CUDA-core work (the "
                                        "basis functions and the netting-set epilogue), not by the tensor pipe"},
            "basis": {"netting_sets": nb, "columns_per_date": float(info.basis_columns) / nT,
                      "terms_per_date": float(info.basis_terms) / nT,
                      "terms_per_column": float(info.basis_terms) / max(float(info.basis_columns), 1.0),
                      "table_bytes": int(info.basis_bytes)},
            "roofline_row_stats": {"bound": "hbm", "achieved": row_bytes / (float(np.mean(rows_ms)) / 1e3) / 1e9, "peak": peak,
                                   "unit": "GB/s", "frac": row_bytes / (float(np.mean(rows_ms)) / 1e3) / 1e9 / peak,
                                   "note": "row-statistics kernel: algorithmic bytes = every exposure row read once; the exact "
                                           "quantile reads a row up to three times (min/max of a sample, histogram, bracket)"},
            # the term-by-term kernel's SFU rate (one ex2 per bond-like term and path); with the basis kernel the
            # book's exponentials are the basis columns', far fewer, and this rate does not describe the kernel
            "roofline_mufu": ({"bound": "sfu", "achieved": exp_per_launch / fused_s / 1e9 if C_ex2 else None,
                               "peak": C_ex2 / 1e9 if C_ex2 else None, "unit": "G ex2/s",
                               "frac": exp_per_launch / fused_s / C_ex2 if C_ex2 else None} if nb == 0 else None),
            "clocks": clocks.summary(),
            "plan_compile_s": compile_s,
            "cpu_baseline": cpu,
        }
        if world > 1:  # the other ranks wait at the closing barrier: the legs run in the one-GPU line only
            a.no_precision = a.no_exact = a.no_surrogate = a.no_amc = a.no_amc_surrogate = True
            a.no_im = a.no_xva_batch = a.no_nest = True
            line["legs"] = "run with --gpus 1 only"
        if not a.no_precision:
            line["fp32_vs_fp64"] = guarded(precision_leg, ctx, a)
        if not a.no_exact:
            line["exact_decisions"] = guarded(exact_leg, ctx, a)
        if not a.no_surrogate:
            line["surrogate"] = guarded(surrogate_leg, ctx, a)
        if not a.no_amc:
            line["amc"] = guarded(amc_leg, ctx, a)
        if not a.no_amc_surrogate:
            line["amc_surrogate"] = guarded(amc_surrogate_leg, ctx, a)
        if not a.no_im:
            line["nested_im"] = guarded(im_leg, ctx, a)
        if not a.no_xva_batch:
            line["xva_batch"] = guarded(xva_batch_leg, ctx, a)
        if not a.no_nest:
            line["adaptive_nest"] = guarded(nest_leg, ctx, a)
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
