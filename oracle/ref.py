"""ORACLE / TEST INFRASTRUCTURE ONLY: ctypes access to oracle/_ref/libccr_ref.so.

That library is the reference (svr-net/zlatko) compiled unmodified from its own sources plus the
C-ABI wrapper oracle/ref_shim.cpp.  Only tests/, the smoke check and bench.py's CPU-baseline leg
may import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "libccr_ref.so")
_lib: Optional[C.CDLL] = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
INNER_FN = C.CFUNCTYPE(None, C.c_size_t, C.c_uint64, C.POINTER(C.c_double), C.c_size_t, C.c_void_p)
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def available() -> bool:
    return os.path.exists(_LIB_PATH)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{_LIB_PATH} is not built (run `make -C oracle`)")
        L = C.CDLL(_LIB_PATH)
        sz = C.c_size_t
        L.ref_plan_compile.restype = C.c_void_p
        L.ref_plan_compile.argtypes = [_dp, sz, _dp, sz, _dp, sz, C.c_char_p, sz]
        L.ref_plan_free.argtypes = [C.c_void_p]
        L.ref_plan_from_buffers.restype = C.c_void_p
        L.ref_plan_from_buffers.argtypes = [_up, _up, sz, _fp, _fp, sz, _fp, sz, _fp, sz, C.c_uint32, C.c_uint32, _dp, sz,
                                            _u64p, sz]
        L.ref_plan_sizes.argtypes = [C.c_void_p, _u64p]
        L.ref_plan_get.argtypes = [C.c_void_p, _up, _up, _fp, _fp, _fp, _fp, _dp, _u64p, _dp]
        L.ref_plan_set_terms.argtypes = [C.c_void_p, _fp, sz]
        L.ref_plan_set_paths.argtypes = [C.c_void_p, sz]
        L.ref_run_fused.restype = C.c_int
        L.ref_run_fused.argtypes = [C.c_void_p, C.c_int, _fp, _fp, C.c_char_p, sz]
        L.ref_run_rows.restype = C.c_int
        L.ref_run_rows.argtypes = [C.c_void_p, C.c_int, _fp, C.c_char_p, sz]
        L.ref_amc_states.restype = C.c_int
        L.ref_amc_states.argtypes = [C.c_void_p, C.c_int, _fp, _fp, _fp, C.c_char_p, sz]
        L.ref_amc_rows.restype = C.c_uint64
        L.ref_amc_rows.argtypes = [C.c_void_p]
        L.ref_summarise.restype = C.c_int
        L.ref_summarise.argtypes = [C.c_void_p, _fp, _fp, _dp, C.c_char_p, sz]
        L.ref_summarise_views.restype = C.c_int
        L.ref_summarise_views.argtypes = [C.c_void_p, _fp, _fp, _dp, sz, C.c_char_p, sz]
        L.ref_summarise_full.restype = C.c_int64
        L.ref_summarise_full.argtypes = [C.c_void_p, _fp, _fp, C.c_void_p, sz, C.c_char_p, sz]
        L.ref_engine_run.restype = C.c_void_p
        L.ref_engine_run.argtypes = [_dp, sz, _dp, sz, C.c_double, C.c_void_p, sz, C.c_char_p, sz]
        L.ref_engine_free.argtypes = [C.c_void_p]
        L.ref_engine_sizes.argtypes = [C.c_void_p, _u64p]
        L.ref_engine_get.argtypes = [C.c_void_p] + [C.c_void_p] * 9
        L.ref_engine_pathwise_cva.restype = C.c_double
        L.ref_engine_pathwise_cva.argtypes = [C.c_void_p, sz, C.c_double]
        L.ref_unilateral_cva.restype = C.c_double
        L.ref_unilateral_cva.argtypes = [_dp, _dp, sz, _dp, _dp, sz, C.c_double]
        L.ref_bilateral_cva.argtypes = [_dp, _dp, _dp, sz, _dp, _dp, sz, _dp, _dp, sz, C.c_double, C.c_double, _dp]
        vp = C.c_void_p
        L.ref_xva.restype = None
        L.ref_xva.argtypes = [_dp, _dp, _dp, sz, vp, _dp, _dp, sz, C.c_double, _dp, _dp, sz, C.c_double, _dp, _dp]
        L.ref_allocate_exposure_xva.restype = None
        L.ref_allocate_exposure_xva.argtypes = [_dp, sz, _dp, sz, _dp, _dp, sz, C.c_double, _dp, _dp, sz, _dp, _dp]
        L.ref_initial_margin_profile.restype = None
        L.ref_initial_margin_profile.argtypes = [_dp, _dp, sz, _dp, sz, C.c_double, C.c_double, _dp]
        L.ref_marginal_contributions.restype = None
        L.ref_marginal_contributions.argtypes = [_dp, sz, _dp, vp, sz, sz, _dp]
        L.ref_incremental_exposure.restype = None
        L.ref_incremental_exposure.argtypes = [_dp, _dp, vp, sz, sz, _dp]
        L.ref_estimate_adaptive.restype = C.c_int64
        L.ref_estimate_adaptive.argtypes = [_dp, sz, sz, _dp, vp, INNER_FN, vp, C.c_double, C.c_double, C.c_double, _dp, sz,
                                            C.c_uint64, vp, sz, C.c_char_p, sz]
        L.ref_estimate_uniform.restype = C.c_int
        L.ref_estimate_uniform.argtypes = [vp, sz, INNER_FN, vp, vp, sz, sz, C.c_double, C.c_double, C.c_double, C.c_uint64, _dp,
                                           C.c_char_p, sz]
        L.ref_normal_stream.restype = None
        L.ref_normal_stream.argtypes = [C.c_uint64, sz, _dp]
        L.ref_nested_exposure.restype = C.c_int64
        L.ref_nested_exposure.argtypes = [_dp, sz, _dp, sz, _dp, sz, C.c_double, _dp, sz, C.c_uint64, C.c_int, sz, vp, sz,
                                          C.c_char_p, sz]
        L.ref_counter_normal.restype = C.c_double
        L.ref_counter_normal.argtypes = [C.c_uint64, sz]
        L.ref_derive_seed.restype = C.c_uint64
        L.ref_derive_seed.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]
        L.ref_quantile.restype = C.c_double
        L.ref_quantile.argtypes = [_dp, sz, C.c_double]
        L.ref_profile.argtypes = [_dp, _dp, sz, _dp, sz, C.c_double, C.c_double, _dp]
        L.ref_collateral.restype = C.c_int
        L.ref_collateral.argtypes = [_dp, C.c_void_p, sz, _dp, sz] + [C.c_double] * 5 + [C.c_int, C.c_double, _dp, C.c_char_p, sz]
        L.ref_grid.restype = sz
        L.ref_grid.argtypes = [_dp, sz, _dp, sz, _dp, sz, C.c_int, _dp, sz]
        _lib = L
    return _lib


def _err() -> C.Array:
    return C.create_string_buffer(512)


@dataclass
class RefPlan:
    """A reference gpu::FusedPlan: its GPU buffers and the fields summarise() needs."""

    handle: int
    header: np.ndarray
    indices: np.ndarray
    params: np.ndarray
    steps: np.ndarray
    terms: np.ndarray
    requests: np.ndarray
    rows_total: int
    num_outputs: int
    times: np.ndarray
    reporting: np.ndarray
    market_survival: np.ndarray
    stats_per_date: int
    num_amc: int
    num_unsupported: int
    num_paths: int

    @property
    def num_dates(self) -> int:
        return len(self.times)

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            if self.handle and _lib is not None:
                _lib.ref_plan_free(self.handle)
        except Exception:
            pass

    def _refresh(self) -> None:
        s = np.zeros(14, dtype=np.uint64)
        lib().ref_plan_sizes(self.handle, s)
        n = [int(v) for v in s]
        self.header = np.zeros(n[0], np.uint32)
        self.indices = np.zeros(n[1], np.uint32)
        self.params = np.zeros(n[2], np.float32)
        self.steps = np.zeros(n[3], np.float32)
        self.terms = np.zeros(max(n[4], 1), np.float32)
        self.requests = np.zeros(max(n[5], 1), np.float32)
        self.times = np.zeros(n[8])
        self.reporting = np.zeros(n[9], np.uint64)
        self.market_survival = np.zeros(n[8])
        lib().ref_plan_get(self.handle, self.header, self.indices, self.params, self.steps, self.terms, self.requests,
                           self.times, self.reporting, self.market_survival)
        self.terms = self.terms[: n[4]]
        self.requests = self.requests[: n[5]]
        self.rows_total, self.num_outputs, self.stats_per_date = n[6], n[7], n[10]
        self.num_amc, self.num_unsupported, self.num_paths = n[11], n[12], n[13]

    def set_terms(self, terms: np.ndarray) -> None:
        t = np.ascontiguousarray(terms, dtype=np.float32)
        lib().ref_plan_set_terms(self.handle, t, t.size)
        self._refresh()

    def set_paths(self, n: int) -> None:
        lib().ref_plan_set_paths(self.handle, n)
        self._refresh()


def compile_plan(model: np.ndarray, ns: np.ndarray, opts: np.ndarray) -> RefPlan:
    """gpu::compile (src/gpu/fused_exposure.cpp:214) on the decoded spec."""
    e = _err()
    h = lib().ref_plan_compile(model, model.size, ns, ns.size, opts, opts.size, e, 512)
    if not h:
        raise ValueError(e.value.decode())
    p = RefPlan(h, *([None] * 15))  # type: ignore[arg-type]
    p._refresh()
    return p


def plan_from_buffers(header, indices, params, steps, terms, requests, rows_total, num_outputs, times, reporting,
                      num_paths: Optional[int] = None) -> RefPlan:
    """A reference FusedPlan holding the given buffers (e.g. a plan compiled by zlatko_b200), optionally with
    another number of paths (header words 0 and 15, as auditConditionalIm does)."""
    h = np.array(header, np.uint32)
    if num_paths is not None:
        h[0], h[15] = num_paths, (num_paths + 63) // 64
    f = lambda a: np.ascontiguousarray(a if len(a) else np.zeros(8), np.float32)
    idx = np.ascontiguousarray(indices, np.uint32)
    t, rq = f(terms), f(requests)
    tm = np.ascontiguousarray(times, np.float64)
    rep = np.ascontiguousarray(reporting, np.uint64)
    handle = lib().ref_plan_from_buffers(h, idx, idx.size, f(params), f(steps), len(steps), t, len(terms), rq, len(requests),
                                         int(rows_total), int(num_outputs), tm, tm.size, rep, rep.size)
    p = RefPlan(handle, *([None] * 15))  # type: ignore[arg-type]
    p._refresh()
    return p


def run_fused(plan: RefPlan, threads: int = 0):
    """gpu::runFusedReference: the reference's FP32 CPU kernels.  Returns (sums, values)."""
    sums = np.zeros(plan.num_dates * plan.stats_per_date, np.float32)
    values = np.zeros(max(1, plan.num_outputs), np.float32)
    e = _err()
    if lib().ref_run_fused(plan.handle, threads, sums, values, e, 512):
        raise ValueError(e.value.decode())
    return sums, values


def run_rows(plan: RefPlan, threads: int = 0) -> np.ndarray:
    """The exposure rows [row][path] the reference's fused kernel writes."""
    out = np.zeros(plan.rows_total * plan.num_paths, np.float32)
    e = _err()
    if lib().ref_run_rows(plan.handle, threads, out, e, 512):
        raise ValueError(e.value.decode())
    return out.reshape(plan.rows_total, plan.num_paths)


def amc_states(plan: RefPlan, threads: int = 0):
    """gpu::runAmcStates: x and deflator [date][path] and exercise values [row][path]."""
    nT, nP = plan.num_dates, plan.num_paths
    rows = int(lib().ref_amc_rows(plan.handle))
    x = np.zeros(nT * nP, np.float32)
    d = np.zeros(nT * nP, np.float32)
    ex = np.zeros(max(rows, 1) * nP, np.float32)
    e = _err()
    if lib().ref_amc_states(plan.handle, threads, x, d, ex, e, 512):
        raise ValueError(e.value.decode())
    return x.reshape(nT, nP), d.reshape(nT, nP), ex[: rows * nP].reshape(rows, nP)


SUMMARY_FIELDS = ("ev", "ee", "ene", "pfe", "dee", "dene", "cva_inc", "mean_survival", "mean_deflator")


def summarise(plan: RefPlan, sums: np.ndarray, values: np.ndarray) -> dict:
    """gpu::summarise on a read-back: the profile and the CVA inputs per reporting date."""
    nR = len(plan.reporting)
    out = np.zeros(9 * nR + 1)
    e = _err()
    if lib().ref_summarise(plan.handle, np.ascontiguousarray(sums, np.float32), np.ascontiguousarray(values, np.float32), out, e, 512):
        raise ValueError(e.value.decode())
    r = {k: out[i * nR:(i + 1) * nR] for i, k in enumerate(SUMMARY_FIELDS)}
    r["times"] = plan.times[plan.reporting.astype(np.int64)]
    r["pathwise_cva_04"] = out[9 * nR]
    return r


VIEW_FIELDS = ("value_change_quantile", "conditional_im_discounted", "conditional_im_mean", "conditional_im_band_05",
               "conditional_im_band_50", "conditional_im_band_95", "conditional_discounted_ee",
               "conditional_im_audit_ratio", "conditional_im_discounted_uncorrected")
TRADE_FIELDS = ("marginal_discounted", "marginal", "incremental_discounted", "standalone_discounted", "standalone")


def summarise_views(plan: RefPlan, sums: np.ndarray, values: np.ndarray) -> dict:
    """The rest of gpu::summarise's FusedResult per reporting date (NaN rows where the result has none), with
    the nested-IM audit the reference runs inside summarise; "trades" holds one dict per trade group."""
    nR, nTr = len(plan.reporting), int(plan.header[18])
    out = np.zeros((9 + 5 * nTr) * nR)
    e = _err()
    if lib().ref_summarise_views(plan.handle, np.ascontiguousarray(sums, np.float32), np.ascontiguousarray(values, np.float32),
                                 out, out.size, e, 512):
        raise ValueError(e.value.decode())
    r = {k: out[i * nR:(i + 1) * nR] for i, k in enumerate(VIEW_FIELDS)}
    r["trades"] = [{k: out[(9 + 5 * t + i) * nR:(10 + 5 * t + i) * nR] for i, k in enumerate(TRADE_FIELDS)} for t in range(nTr)]
    return r


PROFILE_FIELDS = ("times", "ev", "ee", "ene", "pfe", "dee", "dene")


def summarise_full(plan: RefPlan, sums: np.ndarray, values: np.ndarray) -> dict:
    """The whole FusedResult of gpu::summarise (with the reference's own nested-margin audit) as nested dicts
    and arrays, under the key names of zlatko_b200.summary.summarise."""
    s, v = np.ascontiguousarray(sums, np.float32), np.ascontiguousarray(values, np.float32)
    e = _err()
    n = lib().ref_summarise_full(plan.handle, s, v, None, 0, e, 512)
    if n < 0:
        raise ValueError(e.value.decode())
    flat = np.zeros(n)
    lib().ref_summarise_full(plan.handle, s, v, flat.ctypes.data, n, e, 512)
    pos = 0

    def scalar():
        nonlocal pos
        pos += 1
        return float(flat[pos - 1])

    def vec():
        k = int(scalar())
        nonlocal pos
        pos += k
        return flat[pos - k:pos].copy()

    def mat():
        return [vec() for _ in range(int(scalar()))]

    def profile():
        return {k: vec() for k in PROFILE_FIELDS}

    r = profile()
    for k in ("mean_survival", "market_survival", "cva_inc", "conditional_discounted_ee", "mean_deflator",
              "value_change_quantile", "conditional_im_discounted", "conditional_im_mean"):
        r[k] = vec()
    r["conditional_im_bands"] = mat()
    r["conditional_im_audit_ratio"] = vec()
    r["conditional_im_discounted_uncorrected"] = vec()
    r["trades"] = [{k: vec() for k in TRADE_FIELDS} for _ in range(int(scalar()))]
    for k in ("exposure_samples", "netted_samples", "collateral_samples", "collateral_bands"):
        r[k] = mat()
    r["gross_profile"] = profile() if scalar() else None
    r["histogram_time"] = scalar()
    r["histogram_edges"], r["histogram_counts"] = vec(), vec()
    r["trade_views"] = [{"profile": profile(), "samples": mat(), "bands": mat(), "mean_deflated": vec()}
                        for _ in range(int(scalar()))]
    r["exercise"] = [{"distribution": vec(), "sample_index": vec()} for _ in range(int(scalar()))]
    r["factors"] = None
    if scalar():
        f = {"rate_samples": mat(), "rate_bands": mat(), "rate_mean": vec(), "deflator_mean": vec(), "bond_mean": vec()}
        f["assets"] = [{"samples": mat(), "bands": mat(), "mean": vec(), "deflated_mean": vec()} for _ in range(int(scalar()))]
        f["credits"] = [{"intensity_samples": mat(), "intensity_bands": mat(), "survival_samples": mat(), "survival_mean": vec()}
                        for _ in range(int(scalar()))]
        k = int(scalar())
        f["increment_correlation"] = flat[pos:pos + k * k].reshape(k, k).copy()
        pos += k * k
        r["factors"] = f
    assert pos == n
    return r


@dataclass
class EngineResult:
    times: np.ndarray          # simulation grid
    reporting: np.ndarray      # indices of the reporting dates
    profile: dict              # ev, ee, ene, pfe, dee, dene over the reporting dates
    netted: np.ndarray         # [path][date]
    collateral: np.ndarray
    deflator: np.ndarray
    rate_state: np.ndarray
    survival: np.ndarray       # [credit][path][date]
    trades: np.ndarray         # [trade][path][date]
    pathwise_cva_04: float


def engine_run(model: np.ndarray, ns: np.ndarray, pfe: float, normals: Optional[np.ndarray] = None,
               streams: int = 0) -> EngineResult:
    """ExposureEngine::run (src/exposure/exposure_engine.cpp:50-81), FP64, on the reference's own normals or on
    injected ones laid out [step][normal][stream]."""
    e = _err()
    if normals is not None:
        normals = np.ascontiguousarray(normals, np.float64)
        ptr = normals.ctypes.data_as(C.c_void_p)
    else:
        ptr = None
    h = lib().ref_engine_run(model, model.size, ns, ns.size, pfe, ptr, streams, e, 512)
    if not h:
        raise ValueError(e.value.decode())
    try:
        s = np.zeros(5, np.uint64)
        lib().ref_engine_sizes(h, s)
        nP, nT, nR, nTr, nC = (int(v) for v in s)
        times = np.zeros(nT)
        rep = np.zeros(nR, np.uint64)
        prof = np.zeros(6 * nR)
        mats = [np.zeros((nP, nT)) for _ in range(4)]
        surv = np.zeros((nC, nP, nT))
        trades = np.zeros((nTr, nP, nT))
        ptrs = [a.ctypes.data_as(C.c_void_p) for a in [times, rep, prof] + mats + [surv, trades]]
        lib().ref_engine_get(h, *ptrs)
        pcva = lib().ref_engine_pathwise_cva(h, 0, 0.4) if nC > 0 else float("nan")
    finally:
        lib().ref_engine_free(h)
    names = ("ev", "ee", "ene", "pfe", "dee", "dene")
    profile = {k: prof[i * nR:(i + 1) * nR] for i, k in enumerate(names)}
    return EngineResult(times, rep.astype(np.int64), profile, mats[0], mats[1], mats[2], mats[3], surv, trades, pcva)


def unilateral_cva(times, dee, pillars, hazards, recovery: float) -> float:
    f = lambda a: np.ascontiguousarray(a, np.float64)
    t, d, p, h = f(times), f(dee), f(pillars), f(hazards)
    return lib().ref_unilateral_cva(t, d, t.size, p, h, p.size, recovery)


def bilateral_cva(times, dee, dene, cpty, own, rc: float, ro: float):
    f = lambda a: np.ascontiguousarray(a, np.float64)
    out = np.zeros(2)
    lib().ref_bilateral_cva(f(times), f(dee), f(dene), len(times), f(cpty[0]), f(cpty[1]), len(cpty[0]), f(own[0]),
                            f(own[1]), len(own[0]), rc, ro, out)
    return float(out[0]), float(out[1])


XVA_PARAM_ORDER = ("funding_spread_borrow", "funding_spread_lend", "margin_funding_spread", "hurdle_rate", "capital_ratio",
                   "risk_weight", "alpha")


def _f64(a):
    return np.ascontiguousarray(a, np.float64)


def xva(times, dee, dene, dim, cpty, rc: float, own, ro: float, params: dict) -> dict:
    """ccr::xva on a profile; cpty / own are (pillars, hazards); dim the discounted initial margin or None."""
    out = np.zeros(6)
    pr = _f64([params[k] for k in XVA_PARAM_ORDER])
    d = _f64(dim) if dim is not None else None
    lib().ref_xva(_f64(times), _f64(dee), _f64(dene), len(times), None if d is None else d.ctypes.data, _f64(cpty[0]),
                  _f64(cpty[1]), len(cpty[0]), rc, _f64(own[0]), _f64(own[1]), len(own[0]), ro, pr, out)
    return dict(zip(("cva", "dva", "fca", "fba", "mva", "kva"), out.tolist()))


def allocate_exposure_xva(times, contributions, cpty, rc: float, own, params: dict) -> np.ndarray:
    c = _f64(contributions)
    out = np.zeros((c.shape[0], 3))
    pr = _f64([params[k] for k in XVA_PARAM_ORDER])
    lib().ref_allocate_exposure_xva(_f64(times), len(times), c, c.shape[0], _f64(cpty[0]), _f64(cpty[1]), len(cpty[0]), rc,
                                    _f64(own[0]), _f64(own[1]), len(own[0]), pr, out)
    return out


def initial_margin_profile(values, deflator, times, q: float, mpr: float) -> np.ndarray:
    v, d = _f64(values), _f64(deflator)
    out = np.zeros(v.shape[1])
    lib().ref_initial_margin_profile(v, d, v.shape[0], _f64(times), v.shape[1], q, mpr, out)
    return out


def marginal_contributions(trade_values, netted, deflator=None) -> np.ndarray:
    tv, nv = _f64(trade_values), _f64(netted)
    d = _f64(deflator) if deflator is not None else None
    out = np.zeros((tv.shape[0], nv.shape[1]))
    lib().ref_marginal_contributions(tv, tv.shape[0], nv, None if d is None else d.ctypes.data, nv.shape[0], nv.shape[1], out)
    return out


def incremental_exposure(netted, new_trade, deflator=None) -> np.ndarray:
    nv, nt = _f64(netted), _f64(new_trade)
    d = _f64(deflator) if deflator is not None else None
    out = np.zeros(nv.shape[1])
    lib().ref_incremental_exposure(nv, nt, None if d is None else d.ctypes.data, nv.shape[0], nv.shape[1], out)
    return out


def _adaptive_opts(o) -> np.ndarray:
    return np.array([o.training_fraction, o.hermite_degree, o.inner_batch, o.min_inner_for_variance, o.max_inner_per_scenario,
                     o.inner_budget, o.max_scenarios_per_round, o.max_rounds, o.audit_per_bin, o.min_per_bin_for_misspecification,
                     float(o.refine_outside_training_range), 0.0] + list(o.bin_probabilities), np.float64)


def _inner_callback(simulate):
    def cb(scenario, seed, out, n, user):
        buf = np.ctypeslib.as_array(out, shape=(n,))
        simulate(int(scenario), int(seed), buf)
    return INNER_FN(cb)


def estimate_adaptive(features, payoff, weight, simulate, ee_rel: float, ee_abs: float, q: float, options) -> dict:
    """nested::estimateAdaptive with PositivePart(ee_rel, ee_abs) and Quantile(q, positive part); simulate(scenario,
    seed, out) fills out with inner payoffs."""
    F = np.ascontiguousarray(features, np.float64)
    y = np.ascontiguousarray(payoff, np.float64)
    w = None if weight is None else np.ascontiguousarray(weight, np.float64)
    opts = _adaptive_opts(options)
    cb = _inner_callback(simulate)
    e = _err()
    args = (F, F.shape[0], F.shape[1], y, None if w is None else w.ctypes.data, cb, None, ee_rel, ee_abs, q, opts, opts.size,
            int(options.seed))
    n = lib().ref_estimate_adaptive(*args, None, 0, e, 512)
    if n < 0:
        raise ValueError(e.value.decode())
    flat = np.zeros(n)
    lib().ref_estimate_adaptive(*args, flat.ctypes.data, n, e, 512)
    pos = 0

    def take(k):
        nonlocal pos
        pos += k
        return flat[pos - k:pos].copy()

    def vec():
        return take(int(take(1)[0]))

    r = {"estimate": take(2), "baseline": take(2), "regression": take(2), "training": vec(), "evaluation": vec(),
         "proxy": vec(), "value": vec(), "inner": vec()}
    for k in ("inner_paths", "audit_inner_paths", "refined_scenarios", "audited_scenarios", "rounds", "unresolved",
              "proxy_degree", "proxy_basis"):
        r[k] = int(take(1)[0])
    r["stop"] = ("converged", "scenario caps", "budget", "max rounds")[int(take(1)[0])]
    r["bins"] = [take(7) for _ in range(int(take(1)[0]))]
    return r


def estimate_uniform(weight, n: int, simulate, scenarios, per_scenario: int, ee_rel: float, ee_abs: float, q: float,
                     seed: int) -> np.ndarray:
    w = None if weight is None else np.ascontiguousarray(weight, np.float64)
    sc = np.ascontiguousarray(scenarios, np.uint64)
    out = np.zeros(2 + len(sc))
    e = _err()
    if lib().ref_estimate_uniform(None if w is None else w.ctypes.data, n, _inner_callback(simulate), None, sc.ctypes.data, len(sc),
                                  per_scenario, ee_rel, ee_abs, q, int(seed), out, e, 512):
        raise ValueError(e.value.decode())
    return out


def normal_stream(seed: int, n: int) -> np.ndarray:
    """The first n normals of the reference's NormalGenerator(seed) (mt19937_64, normal_distribution)."""
    out = np.zeros(n)
    lib().ref_normal_stream(seed, n, out)
    return out


NESTED_POINT_FIELDS = ("time", "ee_exact", "pfe_exact", "ee_regression", "pfe_regression", "ee_uniform", "pfe_uniform",
                       "ee_adaptive", "pfe_adaptive", "evaluated", "inner_paths", "audit_inner_paths", "refined", "rounds",
                       "uniform_inner_per_scenario", "live")


def nested_exposure(model: np.ndarray, ns: np.ndarray, reporting, pfe_quantile: float, adaptive, uniform: bool = True,
                    threads: int = 1):
    """nested::nestedExposure on the reference's own outer simulation (on `threads` threads): one dict per
    reporting point."""
    m, n, t = (np.ascontiguousarray(a, np.float64) for a in (model, ns, reporting))
    opts = _adaptive_opts(adaptive)
    e = _err()
    out = np.zeros(16 * (len(t) + 1))
    k = lib().ref_nested_exposure(m, m.size, n, n.size, t, t.size, pfe_quantile, opts, opts.size, int(adaptive.seed),
                                  int(uniform), threads, out.ctypes.data, out.size, e, 512)
    if k < 0:
        raise ValueError(e.value.decode())
    return [dict(zip(NESTED_POINT_FIELDS, out[16 * i:16 * (i + 1)].tolist())) for i in range(k)]


def counter_normal(seed: int, m: int) -> float:
    return lib().ref_counter_normal(seed, m)


def derive_seed(seed: int, a: int, b: int = 0, c: int = 0) -> int:
    return lib().ref_derive_seed(seed, a, b, c)


def quantile(values, p: float) -> float:
    v = np.ascontiguousarray(values, np.float64)
    return lib().ref_quantile(v, v.size, p)


def profile(values: np.ndarray, deflator: np.ndarray, times, q: float, horizon: float) -> dict:
    v = np.ascontiguousarray(values, np.float64)
    d = np.ascontiguousarray(deflator, np.float64)
    t = np.ascontiguousarray(times, np.float64)
    nP, nT = v.shape
    out = np.zeros(6 * nT + 3)
    lib().ref_profile(v, d, nP, t, nT, q, horizon, out)
    names = ("ev", "ee", "ene", "pfe", "dee", "dene")
    r = {k: out[i * nT:(i + 1) * nT] for i, k in enumerate(names)}
    r["epe"], r["eepe"], r["max_pfe"] = out[6 * nT], out[6 * nT + 1], out[6 * nT + 2]
    return r


def collateral(values: np.ndarray, times, hc, ho, mta, ia, mpr, kind=0, haircut=0.0, unit_price=None) -> np.ndarray:
    v = np.ascontiguousarray(values, np.float64)
    t = np.ascontiguousarray(times, np.float64)
    nP, nT = v.shape
    out = np.zeros((nP, nT))
    up = None if unit_price is None else np.ascontiguousarray(unit_price, np.float64)
    e = _err()
    if lib().ref_collateral(v, None if up is None else up.ctypes.data_as(C.c_void_p), nP, t, nT, hc, ho, mta, ia, mpr,
                            kind, haircut, out, e, 512):
        raise ValueError(e.value.decode())
    return out


def grid(model: np.ndarray, ns: np.ndarray, opts: np.ndarray, which: int) -> np.ndarray:
    """0: reporting grid, 1: engine simulation grid, 2: gpu::simulationGrid."""
    cap = 100000
    out = np.zeros(cap)
    n = lib().ref_grid(model, model.size, ns, ns.size, opts, opts.size, which, out, cap)
    return out[:n].copy()
