"""The fused exposure pipeline on a B200, behind the reference's ``ccr::gpu`` interface.

The reference splits the path into ``compile`` (netting set -> FusedPlan), a backend
``FusedOutput run(const FusedPlan&)`` and ``summarise`` (include/ccr/gpu/fused_exposure.hpp:338-392).
This module mirrors those three steps over the C ABI:

    plan = compile(model, netting_set, options)        # zk_compile (C++ host compiler)
    with Context() as ctx:
        sums, values = ctx.run(plan)                   # zk_run_plan: the CUDA kernels
    result = summarise(plan, sums, values)             # profiles, CVA increments, survival

``Plan.from_arrays`` wraps the buffers of any reference FusedPlan, so plans compiled by the reference
itself run unchanged.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import spec as S
from ._native import BatchInfo, Output, OutputF64, PlanView, PlanViewF64, ZkError, check, lib

STATS_PER_DATE = 8
H_QUANTILE, H_NUM_REPORTING, H_STATS = 14, 17, 16


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class Plan:
    """The tables of one gpu::FusedPlan, in the reference's binary layout."""

    header: np.ndarray            # uint32[32]
    indices: np.ndarray           # uint32
    params: np.ndarray            # float32[84]
    steps: np.ndarray             # float32[nT * 24]
    terms: np.ndarray             # float32[numTerms * 8]
    requests: np.ndarray          # float32[numRequests * 8]
    rows_total: int
    num_outputs: int
    times: np.ndarray             # simulation dates
    reporting: np.ndarray         # indices of the reporting dates
    market_survival: Optional[np.ndarray] = None
    tables64: Optional[Dict[str, np.ndarray]] = None  # double-precision params/steps/terms/requests (zk_compile)
    exercise_rows: int = 0
    amc_degrees: List[int] = field(default_factory=list)  # regression degree of each Bermudan (zk_fit_amc)
    im_audit_paths: int = 0          # the nested-IM audit (FusedPlan::imAuditPaths, imAuditInnerPaths); 0: off
    im_audit_inner_paths: int = 0
    options: Optional[S.Options] = None  # the options compiled (summarise decodes the views with them)

    def __post_init__(self):
        self.header = np.ascontiguousarray(self.header, np.uint32)
        self.indices = np.ascontiguousarray(self.indices, np.uint32)
        for k in ("params", "steps", "terms", "requests"):
            a = np.ascontiguousarray(getattr(self, k), np.float32)
            setattr(self, k, a if a.size else np.zeros(8, np.float32)[:0])
        self._keep: List = []

    @property
    def num_paths(self) -> int:
        return int(self.header[0])

    @property
    def num_dates(self) -> int:
        return int(self.header[1])

    @property
    def stats_per_date(self) -> int:
        return int(self.header[H_STATS])

    @property
    def num_reporting(self) -> int:
        return int(self.header[H_NUM_REPORTING])

    def sums_len(self) -> int:
        return self.num_dates * self.stats_per_date

    def values_len(self) -> int:
        return max(1, self.num_outputs)

    @staticmethod
    def from_arrays(header, indices, params, steps, terms, requests, rows_total, num_outputs, times, reporting,
                    market_survival=None) -> "Plan":
        return Plan(header, indices, params, steps, terms, requests, int(rows_total), int(num_outputs),
                    np.asarray(times, np.float64), np.asarray(reporting, np.int64), market_survival)

    def view(self) -> PlanView:
        # The view holds pointers into the plan's arrays: kept while they are the same objects (their contents
        # may change in place), rebuilt when a table is replaced.
        key = (self.header, self.indices, self.params, self.steps, self.terms, self.requests)
        cached = getattr(self, "_view", None)
        if cached is not None and all(a is b for a, b in zip(cached[0], key)) and \
                (cached[1].rows_total, cached[1].num_outputs) == (self.rows_total, self.num_outputs):
            return cached[1]
        terms = self.terms if self.terms.size else np.zeros(8, np.float32)
        reqs = self.requests if self.requests.size else np.zeros(8, np.float32)
        self._keep = [terms, reqs]
        v = PlanView(_ptr(self.header, C.c_uint32), self.header.size, _ptr(self.indices, C.c_uint32), self.indices.size,
                        _ptr(self.params, C.c_float), self.params.size, _ptr(self.steps, C.c_float), self.steps.size,
                        _ptr(terms, C.c_float), self.terms.size, _ptr(reqs, C.c_float), self.requests.size,
                        self.rows_total, self.num_outputs)
        self._view = (key, v)
        return v

    def view64(self) -> PlanViewF64:
        if self.tables64 is None:
            raise ValueError("this plan has no double-precision tables (compile it with zlatko_b200.gpu.compile)")
        t = self.tables64
        terms = t["terms"] if t["terms"].size else np.zeros(8)
        reqs = t["requests"] if t["requests"].size else np.zeros(8)
        self._keep = [terms, reqs]
        return PlanViewF64(_ptr(self.header, C.c_uint32), self.header.size, _ptr(self.indices, C.c_uint32), self.indices.size,
                           _ptr(t["params"], C.c_double), t["params"].size, _ptr(t["steps"], C.c_double), t["steps"].size,
                           _ptr(terms, C.c_double), t["terms"].size, _ptr(reqs, C.c_double), t["requests"].size,
                           self.rows_total, self.num_outputs)


def to_bf16_bits(a: np.ndarray) -> np.ndarray:
    """Round to the nearest bf16 (ties to even) and return the raw 16-bit patterns."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def compile(model: S.Model, netting_set: S.NettingSet, options: Optional[S.Options] = None,
            fit: Optional["Context"] = None) -> Plan:
    """zk_compile: the host plan compiler (a restatement of gpu::compile, src/gpu/fused_exposure.cpp:214).
    Raises ValueError where the reference throws std::invalid_argument.  The reference's compile also fits
    the Longstaff-Schwartz regressions of the Bermudans; here that is zk_fit_amc on the GPU: pass a Context
    as `fit` (or call Context.fit_amc on the plan)."""
    options = options or S.Options()
    plan = compile_arrays(S.encode_model(model), S.encode_netting_set(netting_set), S.encode_options(options))
    if model.credits:
        from .summary import hazard_survival
        c = model.credits[options.counterparty]
        plan.market_survival = np.array([hazard_survival(c.pillars, c.hazards, t) for t in plan.times])
    if fit is not None and plan.amc_degrees:
        plan = fit.fit_amc(plan)
    return plan


def compile_arrays(m: np.ndarray, n: np.ndarray, o: np.ndarray) -> Plan:
    """zk_compile on the flat model / netting-set / options arrays of zlatko_b200.spec.  The plan's
    market_survival is that of no default (compile() fills in the counterparty's curve)."""
    m, n, o = (np.ascontiguousarray(a, np.float64) for a in (m, n, o))
    L = lib()
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    st = L.zk_compile(m.ctypes.data, m.size, n.ctypes.data, n.size, o.ctypes.data, o.size, C.byref(h), err, 512)
    if st != 0:
        raise ValueError(err.value.decode())
    try:
        v, v64 = PlanView(), PlanViewF64()
        check(L.zk_plan_view_of(h, C.byref(v)))
        check(L.zk_plan_view_f64_of(h, C.byref(v64)))
        sizes = (C.c_uint64 * 6)()
        check(L.zk_plan_sizes(h, sizes))
        nT, nR = int(sizes[0]), int(sizes[1])

        def arr(p, n, dt):
            return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)

        times = np.zeros(nT)
        rep = np.zeros(nR, np.uint64)
        check(L.zk_plan_dates(h, times.ctypes.data, nT, rep.ctypes.data, nR))
        plan = Plan(arr(v.header, v.header_len, np.uint32), arr(v.indices, v.indices_len, np.uint32),
                    arr(v.params, v.params_len, np.float32), arr(v.steps, v.steps_len, np.float32),
                    arr(v.terms, v.terms_len, np.float32), arr(v.requests, v.requests_len, np.float32),
                    int(v.rows_total), int(v.num_outputs), times, rep.astype(np.int64))
        plan.tables64 = {"params": arr(v64.params, v64.params_len, np.float64), "steps": arr(v64.steps, v64.steps_len, np.float64),
                         "terms": arr(v64.terms, v64.terms_len, np.float64),
                         "requests": arr(v64.requests, v64.requests_len, np.float64)}
        plan.exercise_rows = int(sizes[5])
        plan.market_survival = np.ones(nT)
        plan.amc_degrees = S.bermudan_degrees(n)
        plan.options = S.decode_options(o)
        if plan.options.im_inner_paths > 0 and plan.options.im_audit_paths > 0:
            plan.im_audit_paths, plan.im_audit_inner_paths = plan.options.im_audit_paths, plan.options.im_audit_inner_paths
        return plan
    finally:
        L.zk_plan_destroy(h)


class Batch:
    """Plans uploaded once and executed on the device (zk_batch_*): the inputs stay resident in HBM."""

    def __init__(self, ctx: "Context", plans: Sequence[Plan]):
        self.ctx, self.plans = ctx, list(plans)
        views = (PlanView * len(self.plans))(*[p.view() for p in self.plans])
        h = C.c_void_p()
        check(lib().zk_batch_create(ctx.handle, views, len(self.plans), C.byref(h)), ctx.handle)
        self.handle = h

    def execute(self) -> None:
        check(lib().zk_batch_execute(self.handle), self.ctx.handle)

    def set_tile_paths(self, tile_paths: int) -> None:
        """Pins the tile shape (paths per revalue CTA: 128, 256 or 512) instead of the autotuned one."""
        check(lib().zk_batch_set_tile_paths(self.handle, tile_paths), self.ctx.handle)

    def timings(self) -> np.ndarray:
        """Milliseconds of the last execute: simulate, revalue, reduce, row statistics."""
        ms = (C.c_float * 4)()
        check(lib().zk_batch_timings(self.handle, ms), self.ctx.handle)
        return np.array(ms[:], np.float64)

    def info(self) -> BatchInfo:
        i = BatchInfo()
        check(lib().zk_batch_info_get(self.handle, C.byref(i)), self.ctx.handle)
        return i

    def read(self):
        outs, bufs = self.ctx._outputs(self.plans)
        check(lib().zk_batch_read(self.handle, outs), self.ctx.handle)
        return bufs

    def close(self) -> None:
        if self.handle:
            lib().zk_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


class Context:
    """A zk_context on one GPU.  Calls on one context run in order on its stream."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        h = C.c_void_p()
        st = lib().zk_context_create(device, C.byref(h))
        if st != 0:
            raise ZkError(st, "zk_context_create failed (no CUDA device?)")
        self.handle = h
        if stream:
            check(lib().zk_context_set_stream(h, C.c_void_p(stream)), h)

    def close(self) -> None:
        if self.handle:
            lib().zk_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def _outputs(plans: Sequence[Plan], f64: bool = False):
        """Output records of every plan over two shared buffers (one for the sums, one for the values): the
        records are written as one array in the C layout {pointer, length, pointer, length}."""
        T, dt = (OutputF64, np.float64) if f64 else (Output, np.float32)
        sl = np.array([p.sums_len() for p in plans], np.int64)
        vl = np.array([p.values_len() for p in plans], np.int64)
        so, vo = np.cumsum(sl) - sl, np.cumsum(vl) - vl
        sums, values = np.zeros(max(int(sl.sum()), 1), dt), np.zeros(max(int(vl.sum()), 1), dt)
        rec = np.zeros((len(plans), 4), np.uint64)
        rec[:, 0] = sums.ctypes.data + so * sums.itemsize
        rec[:, 1] = sl
        rec[:, 2] = values.ctypes.data + vo * values.itemsize
        rec[:, 3] = vl
        outs = (T * len(plans)).from_buffer(rec)
        outs._bufs = (rec, sums, values)  # the records and the buffers they point into live as long as outs
        bufs = [(sums[a:a + n], values[b:b + m]) for a, n, b, m in zip(so.tolist(), sl.tolist(), vo.tolist(), vl.tolist())]
        return outs, bufs

    def run(self, plan: Plan, rows: bool = False):
        """zk_run_plan: the drop-in for gpu::runFusedReference.  Returns (sums, values) as float32, and with
        rows=True also the per-path rows [row][path] the fused kernel wrote (zk_run_plan_rows)."""
        if not rows:
            return self.run_many([plan])[0]
        v = plan.view()
        outs, bufs = self._outputs([plan])
        r = np.zeros(max(plan.rows_total, 1) * plan.num_paths, np.float32)
        check(lib().zk_run_plan_rows(self.handle, C.byref(v), outs, r.ctypes.data), self.handle)
        sums, values = bufs[0]
        return sums, values, r[: plan.rows_total * plan.num_paths].reshape(plan.rows_total, plan.num_paths)

    def set_row_budget(self, nbytes: int) -> None:
        """zk_context_set_row_budget: device bytes for per-path rows and partials at once (0: automatic); books
        beyond it run in waves of netting sets with the same results."""
        check(lib().zk_context_set_row_budget(self.handle, int(nbytes)), self.handle)

    BASIS_AUTO, BASIS_OFF, BASIS_ALL = 0, 1, 2

    def set_basis(self, mode: int) -> None:
        """zk_context_set_basis: which netting sets run on the tensor-core basis kernel (BASIS_AUTO: groups of at
        least 24 eligible netting sets; BASIS_OFF: none; BASIS_ALL: every eligible one)."""
        check(lib().zk_context_set_basis(self.handle, int(mode)), self.handle)

    def set_exact_decisions(self, guard: float) -> None:
        """zk_context_set_exact_decisions: with guard > 0, run / run_plans / run(rows=True) take every margin call
        and exercise decision as the FP64 mode does on the same normals (paths with a decision inside the guard band
        re-run in FP64); 0 turns it off."""
        check(lib().zk_context_set_exact_decisions(self.handle, float(guard)), self.handle)

    def exact_stats(self) -> tuple:
        """zk_context_exact_stats: (paths re-run in FP64, paths checked) since the last call."""
        f, n = C.c_uint64(0), C.c_uint64(0)
        check(lib().zk_context_exact_stats(self.handle, C.byref(f), C.byref(n)), self.handle)
        return int(f.value), int(n.value)

    def call_timings(self) -> dict:
        """zk_context_call_timings: host wall milliseconds of the last run / run_many call by phase."""
        ms = (C.c_double * 5)()
        check(lib().zk_context_call_timings(self.handle, ms), self.handle)
        return dict(zip(("lower", "upload", "device", "exact_check", "read"), [float(v) for v in ms]))

    INJECT_FAIL_LAUNCH, INJECT_ROW_ROUNDS = 1, 2

    def inject(self, what: int, value: int) -> None:
        """zk_debug_inject (tests): INJECT_FAIL_LAUNCH makes the value-th kernel launch from now fail on the host
        instead of launching; INJECT_ROW_ROUNDS caps the row statistics' quantile search at value rounds."""
        check(lib().zk_debug_inject(self.handle, what, value), self.handle)

    def summarise(self, plan: Plan, sums: np.ndarray, values: np.ndarray):
        """summary.summarise with this context as the backend of the nested-IM audit (gpu::summarise runs the
        audit on the reference's CPU kernels; here it runs on the GPU)."""
        from .summary import summarise
        return summarise(plan, sums, values, run=self.run)

    def run_many(self, plans: Sequence[Plan]):
        views = (PlanView * len(plans))(*[p.view() for p in plans])
        outs, bufs = self._outputs(plans)
        check(lib().zk_run_plans(self.handle, views, len(plans), outs), self.handle)
        return bufs

    def amc_states(self, plan: Plan, exercise_rows: int):
        nT, nP = plan.num_dates, plan.num_paths
        x = np.zeros(nT * nP, np.float32)
        d = np.zeros(nT * nP, np.float32)
        ex = np.zeros(max(exercise_rows, 1) * nP, np.float32)
        v = plan.view()
        check(lib().zk_amc_states(self.handle, C.byref(v), x.ctypes.data, d.ctypes.data, ex.ctypes.data, exercise_rows), self.handle)
        return x.reshape(nT, nP), d.reshape(nT, nP), ex[: exercise_rows * nP].reshape(exercise_rows, nP)

    def gemm_bf16(self, a: np.ndarray, b: np.ndarray, bias: Optional[np.ndarray] = None, act: int = 0) -> np.ndarray:
        """zk_gemm_bf16: a @ b.T on the tensor cores, a [M][K] and b [N][K] rounded to bf16, FP32 result."""
        A, B = to_bf16_bits(a), to_bf16_bits(b)
        M, K = A.shape
        N = B.shape[0]
        out = np.zeros((M, N), np.float32)
        bs = None if bias is None else np.ascontiguousarray(bias, np.float32)
        check(lib().zk_gemm_bf16(self.handle, A.ctypes.data, B.ctypes.data, M, N, K, None if bs is None else bs.ctypes.data,
                                 act, out.ctypes.data), self.handle)
        return out

    def fit_amc(self, plan: Plan) -> Plan:
        """zk_fit_amc: the plan with its Bermudans' policy and continuation regressions fitted on the GPU
        (the fit gpu::compile runs; fused_exposure.cpp:103-156)."""
        out = plan.terms.copy()
        deg = np.ascontiguousarray(plan.amc_degrees, np.uint32)
        v = plan.view()
        check(lib().zk_fit_amc(self.handle, C.byref(v), deg.ctypes.data, deg.size, out.ctypes.data, out.size), self.handle)
        return dataclasses.replace(plan, terms=out)

    def fit_amc_f64(self, plan: Plan, normals: Optional[np.ndarray] = None, streams: int = 0) -> Plan:
        """zk_fit_amc_f64: the fit in the FP64 mode on the FP64 state pass (optionally on injected normals);
        returns the plan with fitted double-precision terms."""
        v = plan.view64()
        out = plan.tables64["terms"].copy()
        deg = np.ascontiguousarray(plan.amc_degrees, np.uint32)
        z = None if normals is None else np.ascontiguousarray(normals, np.float64)
        check(lib().zk_fit_amc_f64(self.handle, C.byref(v), None if z is None else z.ctypes.data, streams, deg.ctypes.data,
                                   deg.size, out.ctypes.data, out.size), self.handle)
        t64 = dict(plan.tables64)
        t64["terms"] = out
        return dataclasses.replace(plan, tables64=t64)

    def run_f64(self, plan: Plan, normals: Optional[np.ndarray] = None, streams: int = 0, rows: bool = False):
        """FP64 mode (zk_run_plan_f64), optionally on injected normals [step][normal][stream]."""
        v = plan.view64()
        outs, bufs = self._outputs([plan], f64=True)
        z = None if normals is None else np.ascontiguousarray(normals, np.float64)
        r = np.zeros(plan.rows_total * plan.num_paths) if rows else None
        check(lib().zk_run_plan_f64(self.handle, C.byref(v), None if z is None else z.ctypes.data, streams, outs,
                                    None if r is None else r.ctypes.data), self.handle)
        sums, values = bufs[0]
        return (sums, values, r.reshape(plan.rows_total, plan.num_paths)) if rows else (sums, values)

    def factor_paths_f64(self, plan: Plan, normals: Optional[np.ndarray] = None, streams: int = 0) -> np.ndarray:
        """zk_factor_paths_f64: [2 + nA][nT][nP] = x, D and every asset level on every date and path (FP64)."""
        v = plan.view64()
        nA = int(plan.header[2])
        out = np.zeros((2 + nA) * plan.num_dates * plan.num_paths)
        z = None if normals is None else np.ascontiguousarray(normals, np.float64)
        check(lib().zk_factor_paths_f64(self.handle, C.byref(v), None if z is None else z.ctypes.data, streams,
                                        out.ctypes.data, out.size), self.handle)
        return out.reshape(2 + nA, plan.num_dates, plan.num_paths)

    def run_injected(self, plan: Plan, normals: np.ndarray, streams: int, rows: bool = False):
        """FP32 kernels on injected normals (zk_run_plan_injected)."""
        v = plan.view()
        outs, bufs = self._outputs([plan])
        z = np.ascontiguousarray(normals, np.float64)
        r = np.zeros(plan.rows_total * plan.num_paths, np.float32) if rows else None
        check(lib().zk_run_plan_injected(self.handle, C.byref(v), z.ctypes.data, streams, outs,
                                         None if r is None else r.ctypes.data), self.handle)
        sums, values = bufs[0]
        return (sums, values, r.reshape(plan.rows_total, plan.num_paths)) if rows else (sums, values)

    def batch(self, plans: Sequence[Plan]) -> Batch:
        return Batch(self, plans)


NOALLOC_SCRATCH_BYTES = 32 << 20  # ZK_NOALLOC_SCRATCH_BYTES


def basis_check(plans: Sequence[Plan], x: np.ndarray, S: np.ndarray, xf: np.ndarray) -> dict:
    """zk_debug_basis (host only, no GPU): lowers the plans as one basis group and compares, along one path of
    factor values x[nT], S[nT][4], xf[nT][2], the group's FP16 hi/lo product with the plans' terms summed one by
    one (both in double).  Returns the largest difference relative to the gross basis sum, and the counts."""
    views = (PlanView * len(plans))(*[p.view() for p in plans])
    x = np.ascontiguousarray(x, np.float64)
    S = np.ascontiguousarray(S, np.float64)
    xf = np.ascontiguousarray(xf, np.float64)
    out = np.zeros(5, np.float64)
    err = C.create_string_buffer(512)
    st = lib().zk_debug_basis(views, len(plans), x.ctypes.data, S.ctypes.data, xf.ctypes.data, out.ctypes.data, err, 512)
    if st != 0:
        raise RuntimeError(f"zk_debug_basis: status {st}: {err.value.decode()}")
    return {"rel_err": float(out[0]), "columns": int(out[1]), "linear_terms": int(out[2]), "fixing_slots": int(out[3]),
            "chunks": int(out[4])}


def run_plan_noalloc(plan: Plan, device: int = 0, stream: Optional[int] = None):
    """zk_run_plan_noalloc: one plan without any device allocation (all scratch in the library's fixed
    per-device array of NOALLOC_SCRATCH_BYTES).  For callers that may not call cudaMalloc.  Returns
    (sums, values); raises ZkError for plans that need more scratch than the array holds."""
    v = plan.view()
    outs, bufs = Context._outputs([plan])
    err = C.create_string_buffer(512)
    st = lib().zk_run_plan_noalloc(device, C.c_void_p(stream) if stream else None, C.byref(v), outs, err, 512)
    if st != 0:
        raise ZkError(st, err.value.decode())
    return bufs[0]
