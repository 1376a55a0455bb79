"""ORACLE / TEST INFRASTRUCTURE ONLY: ctypes access to oracle/_ref/liboracle.so, the plain-C restatement of
the reference's exposure path (oracle/fused_oracle.c, oracle/engine_oracle.c; declared in oracle/oracle.h).

Unlike oracle/ref.py, which needs the reference's sources to build, this library builds from the files of
this directory alone (``make -C oracle restatement``), so it is the checker wherever the reference is not
present.  Only tests/, the smoke check and bench.py's CPU-baseline leg may import this module.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "liboracle.so")
_lib: Optional[C.CDLL] = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def build() -> None:
    """Builds the restatement with the system C compiler (no reference sources needed)."""
    subprocess.run(["make", "-s", "-C", _HERE, "restatement"], check=True)


def available() -> bool:
    return os.path.exists(_LIB_PATH)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not available():
            build()
        L = C.CDLL(_LIB_PATH)
        sz = C.c_size_t
        L.orc_run_fused.restype = C.c_int
        L.orc_run_fused.argtypes = [_up, _up, sz, _fp, _fp, _fp, sz, _fp, sz, C.c_uint32, C.c_uint32, _fp, _fp,
                                    C.c_void_p, C.c_char_p, sz]
        L.orc_amc_states.restype = C.c_int
        L.orc_amc_states.argtypes = [_up, _up, _fp, _fp, _fp, C.c_uint32, _up, _fp, _fp, _fp, C.c_char_p, sz]
        L.orc_reg_fit.restype = None
        L.orc_reg_fit.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_void_p, sz]
        L.orc_reg2_fit.restype = None
        L.orc_reg2_fit.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, C.c_void_p, sz]
        L.orc_fit_amc.restype = C.c_int
        L.orc_fit_amc.argtypes = [_up, _up, _fp, _fp, _fp, C.c_uint32, _up, sz, C.c_char_p, sz]
        L.orc_engine_run.restype = C.c_int
        L.orc_engine_run.argtypes = [_dp, sz, _dp, sz, C.c_double, _dp, sz, sz, _dp, _u64p, C.POINTER(C.c_size_t), _dp,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, sz]
        L.orc_quantile.restype = C.c_double
        L.orc_quantile.argtypes = [_dp, sz, C.c_double]
        L.orc_collateral.restype = C.c_int
        L.orc_collateral.argtypes = [_dp, C.c_void_p, sz, _dp, sz] + [C.c_double] * 5 + [C.c_int, C.c_double, _dp]
        L.orc_profile.restype = None
        L.orc_profile.argtypes = [_dp, _dp, sz, _dp, sz, C.c_double, C.c_double, _dp]
        L.orc_unilateral_cva.restype = C.c_double
        L.orc_unilateral_cva.argtypes = [_dp, _dp, sz, _dp, _dp, sz, C.c_double]
        L.orc_bilateral_cva.restype = None
        L.orc_bilateral_cva.argtypes = [_dp, _dp, _dp, sz, _dp, _dp, sz, _dp, _dp, sz, C.c_double, C.c_double, _dp]
        L.orc_pathwise_cva.restype = C.c_double
        L.orc_pathwise_cva.argtypes = [_dp, _dp, _dp, sz, sz, _u64p, sz, C.c_double]
        _lib = L
    return _lib


def _err() -> C.Array:
    return C.create_string_buffer(512)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, np.float32)


def run_fused(header, indices, params, steps, terms, requests, rows_total: int, num_outputs: int, rows: bool = False):
    """The fused pipeline in single precision on a plan in the reference's layout (the tables of a
    zlatko_b200.gpu.Plan, or of the reference's own compile).  Returns (sums, values[, rows])."""
    h = np.ascontiguousarray(header, np.uint32)
    idx = np.ascontiguousarray(indices, np.uint32)
    nT, nS, nP = int(h[1]), int(h[16]), int(h[0])
    t, q = _f32(terms), _f32(requests)
    sums = np.zeros(nT * nS, np.float32)
    values = np.zeros(max(1, num_outputs), np.float32)
    out_rows = np.zeros(max(1, rows_total) * nP, np.float32) if rows else None
    e = _err()
    rc = lib().orc_run_fused(h, idx, idx.size, _f32(params), _f32(steps), t, t.size // 8, q, q.size // 8, rows_total,
                             num_outputs, sums, values, None if out_rows is None else out_rows.ctypes.data_as(C.c_void_p),
                             e, 512)
    if rc:
        raise ValueError(e.value.decode())
    if rows:
        return sums, values, out_rows[: rows_total * nP].reshape(rows_total, nP)
    return sums, values


def run_plan(plan, rows: bool = False):
    """run_fused on a zlatko_b200.gpu.Plan."""
    return run_fused(plan.header, plan.indices, plan.params, plan.steps, plan.terms, plan.requests, plan.rows_total,
                     plan.num_outputs, rows)


def exercise_offsets(terms) -> np.ndarray:
    """First exercise row of each of the (up to 4) Bermudans: a Bermudan's rows are its decide terms'
    exercise indices (code >> 12), in Bermudan then exercise order."""
    t = np.asarray(terms, np.float32).reshape(-1, 8)
    code = t[:, 0].astype(np.int64)
    rows = np.zeros(4, np.int64)
    for c in code[(code & 15) == 6]:
        b = min((c >> 8) & 15, 3)
        rows[b] = max(rows[b], (c >> 12) + 1)
    return np.concatenate([[0], np.cumsum(rows)]).astype(np.uint32)


def amc_states(plan):
    """gpu::runAmcStates on a zlatko_b200.gpu.Plan: x and deflator [date][path], exercise values [row][path]."""
    off = exercise_offsets(plan.terms)
    rows, nT, nP = int(off[-1]), plan.num_dates, plan.num_paths
    x, d = np.zeros(nT * nP, np.float32), np.zeros(nT * nP, np.float32)
    ex = np.zeros(max(rows, 1) * nP, np.float32)
    e = _err()
    if lib().orc_amc_states(plan.header, plan.indices, _f32(plan.params), _f32(plan.steps), _f32(plan.terms),
                            plan.rows_total, off, x, d, ex, e, 512):
        raise ValueError(e.value.decode())
    return x.reshape(nT, nP), d.reshape(nT, nP), ex[: rows * nP].reshape(rows, nP)


class _Regression(C.Structure):
    _fields_ = [("center", C.c_double), ("scale", C.c_double), ("coef", C.c_double * 4), ("ncoef", C.c_int)]


def fit_regression(x, y, degree: int, mask=None) -> dict:
    """PolynomialRegression::fit (regression.cpp:33-80): center, scale and coefficients in the standardised
    regressor."""
    xs, ys = np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64)
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    r = _Regression()
    lib().orc_reg_fit(C.byref(r), degree, xs, ys, None if m is None else m.ctypes.data_as(C.c_void_p), xs.size)
    return {"center": r.center, "scale": r.scale, "ncoef": r.ncoef, "coef": list(r.coef)[: r.ncoef]}


class _Regression2(C.Structure):
    _fields_ = [("cx", C.c_double), ("sx", C.c_double), ("cs", C.c_double), ("ss", C.c_double),
                ("coef", C.c_double * 10), ("degree", C.c_int)]


def fit_regression2(x, s, y, degree: int, mask=None) -> dict:
    """The two-regressor basis (orc_reg2_fit, this library's extension): centers, scales, the 10 graded coefficients
    in the standardised regressors and the degree used (-1: no sample)."""
    xs, ss, ys = (np.ascontiguousarray(a, np.float64) for a in (x, s, y))
    m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
    r = _Regression2()
    lib().orc_reg2_fit(C.byref(r), degree, xs, ss, ys, None if m is None else m.ctypes.data_as(C.c_void_p), xs.size)
    return {"cx": r.cx, "sx": r.sx, "cs": r.cs, "ss": r.ss, "coef": np.array(list(r.coef)), "degree": r.degree}


def predict_regression2(r: dict, x, s) -> np.ndarray:
    """orc_reg2_predict over arrays: sum_i coef[i] basis_i in graded order (1, z, w, z^2, z w, w^2, z^3, z^2 w, z w^2,
    w^3), the terms beyond the degree zero."""
    if r["degree"] < 0:
        return np.zeros(np.shape(x))
    z, w = (np.asarray(x, np.float64) - r["cx"]) / r["sx"], (np.asarray(s, np.float64) - r["cs"]) / r["ss"]
    rows = [np.ones_like(z), z, w, z * z, z * w, w * w, z * z * z, z * z * w, z * w * w, w * w * w]
    count = {0: 1, 1: 3, 2: 6}.get(r["degree"], 10)
    v = np.zeros_like(z)
    for i in range(count):
        v = v + r["coef"][i] * rows[i]
    return v


def fit_amc2(plan, degrees) -> np.ndarray:
    """fitAmc (src/gpu/fused_exposure.cpp:103-156) extended to the two-regressor basis of this library, on the
    oracle's AMC pass (amc_states): the Bermudans whose policy / continuation records are followed by extension
    records (kind 15) regress on the short rate x and the co-terminal swap rate s = sum_14 c A e^{-B x} /
    sum_13 c A e^{-B x} over the annuity (13) and float-leg (14) records before each record; the others are fitted
    by fit_amc.  Records: cx, 1 / sx, cs, 1 / ss, c0, c1; c2..c8 in the first extension record's fields 1..7, c9 in
    the second's field 1.  At most 4 Bermudans (the code's Bermudan field)."""
    terms = fit_amc(plan, degrees).reshape(-1, 8)
    x, D, E = amc_states(plan)
    off = exercise_offsets(plan.terms)
    nT = plan.num_dates
    ind = np.asarray(plan.indices, np.int64)[: nT + 1]
    code = terms[:, 0].astype(np.int64)
    kind = code & 15
    date_of = np.repeat(np.arange(nT), np.diff(ind))
    decide, cont = {}, {}
    for t in np.flatnonzero((kind == 6) | (kind == 7)):
        b = min((int(code[t]) >> 8) & 15, 3)
        if t + 1 >= ind[date_of[t] + 1] or kind[t + 1] != 15:
            continue
        if kind[t] == 6:
            decide.setdefault(b, {})[int(code[t]) >> 12] = (int(t), int(date_of[t]))
        else:
            cont.setdefault(b, {})[int(date_of[t])] = int(t)

    def swap_rate(t, xs):
        u = t
        while u > ind[date_of[t]] and kind[u - 1] in (13, 14):
            u -= 1
        ann, flt = np.zeros_like(xs), np.zeros_like(xs)
        for q in range(u, t):
            c, A, B = (float(v) for v in terms[q, 2:5])
            if kind[q] == 13:
                ann = ann + c * (A * np.exp(-B * xs))
            else:
                flt = flt + c * (A * np.exp(-B * xs))
        return np.where(ann != 0.0, flt / np.where(ann != 0.0, ann, 1.0), 0.0)

    def write(t, r):
        rec = terms[t]
        rec[2], rec[3], rec[4], rec[5] = r["cx"], 1.0 / r["sx"], r["cs"], 1.0 / r["ss"]
        rec[6], rec[7] = r["coef"][0], r["coef"][1]
        terms[t + 1, 1:8] = r["coef"][2:9]
        terms[t + 2, 1] = r["coef"][9]

    for b, dec in decide.items():
        nE = len(dec)
        realised = np.zeros(plan.num_paths)
        for k in range(nE - 1, -1, -1):
            t, j = dec[k]
            xs, Dj = x[j].astype(np.float64), D[j].astype(np.float64)
            e = E[off[b] + k].astype(np.float64)
            s = swap_rate(t, xs)
            r = fit_regression2(xs, s, realised / Dj, int(degrees[b]), e > 0.0)
            write(t, r)
            go = (e > 0.0) & (e > predict_regression2(r, xs, s))
            realised[go] = Dj[go] * e[go]
            lo = dec[k - 1][1] if k > 0 else 0
            for jc, tc in sorted(cont.get(b, {}).items()):
                if lo <= jc < j:
                    xc, Dc = x[jc].astype(np.float64), D[jc].astype(np.float64)
                    write(tc, fit_regression2(xc, swap_rate(tc, xc), realised / Dc, int(degrees[b])))
    return terms.reshape(-1)


def fit_amc(plan, degrees) -> np.ndarray:
    """fitAmc on a plan's tables: a copy of the term table with the Bermudans' policy and continuation
    coefficients fitted (degrees[b]: regression degree of Bermudan b)."""
    terms = _f32(plan.terms).copy()
    deg = np.ascontiguousarray(degrees, np.uint32)
    e = _err()
    if lib().orc_fit_amc(np.ascontiguousarray(plan.header, np.uint32), np.ascontiguousarray(plan.indices, np.uint32),
                         _f32(plan.params), _f32(plan.steps), terms, plan.rows_total, deg, deg.size, e, 512):
        raise ValueError(e.value.decode())
    return terms


@dataclass
class EngineResult:
    times: np.ndarray       # simulation grid
    reporting: np.ndarray   # indices of the reporting dates in it
    profile: dict           # ev, ee, ene, pfe, dee, dene over the reporting dates
    netted: np.ndarray      # [path][date]
    collateral: np.ndarray
    deflator: np.ndarray
    survival: np.ndarray    # credit 0, [path][date]
    pathwise_cva_04: float
    exercise: np.ndarray    # [bermudan][path]: first exercise taken, -1 never


def engine_run(model: np.ndarray, ns: np.ndarray, pfe: float, normals: np.ndarray, streams: int,
               num_paths: int) -> EngineResult:
    """The FP64 exposure engine on injected normals laid out [step][normal][stream]."""
    cap = 4096
    times = np.zeros(cap)
    rep = np.zeros(cap, np.uint64)
    sizes = (C.c_size_t * 2)()
    prof = np.zeros(6 * cap)
    mats = [np.zeros(num_paths * cap) for _ in range(4)]
    from zlatko_b200.spec import bermudan_degrees

    nb = max(4, len(bermudan_degrees(ns)))
    exercise = np.full(nb * num_paths, -1.0)
    e = _err()
    z = np.ascontiguousarray(normals, np.float64)
    m, n = np.ascontiguousarray(model, np.float64), np.ascontiguousarray(ns, np.float64)
    rc = lib().orc_engine_run(m, m.size, n, n.size, pfe, z, streams, cap, times, rep, sizes, prof,
                              *[a.ctypes.data_as(C.c_void_p) for a in mats], exercise.ctypes.data_as(C.c_void_p), e, 512)
    if rc:
        raise ValueError(e.value.decode())
    nT, nR = sizes[0], sizes[1]
    netted, coll, defl, surv = (a[: num_paths * nT].reshape(num_paths, nT) for a in mats)
    names = ("ev", "ee", "ene", "pfe", "dee", "dene")
    p = {k: prof[i * nR:(i + 1) * nR].copy() for i, k in enumerate(names)}
    reporting = rep[:nR].copy()
    expo = np.ascontiguousarray(netted - coll)
    pcva = lib().orc_pathwise_cva(expo, np.ascontiguousarray(defl), np.ascontiguousarray(surv), num_paths, nT, reporting,
                                  nR, 0.4)
    return EngineResult(times[:nT].copy(), reporting.astype(np.int64), p, netted, coll, defl, surv, pcva,
                        exercise.reshape(nb, num_paths))


def quantile(values, p: float) -> float:
    v = np.ascontiguousarray(values, np.float64)
    return lib().orc_quantile(v, v.size, p)


def profile(values: np.ndarray, deflator: np.ndarray, times, q: float, horizon: float) -> dict:
    v = np.ascontiguousarray(values, np.float64)
    d = np.ascontiguousarray(deflator, np.float64)
    t = np.ascontiguousarray(times, np.float64)
    nP, nT = v.shape
    out = np.zeros(6 * nT + 3)
    lib().orc_profile(v, d, nP, t, nT, q, horizon, out)
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
    if lib().orc_collateral(v, None if up is None else up.ctypes.data_as(C.c_void_p), nP, t, nT, hc, ho, mta, ia, mpr,
                            kind, haircut, out):
        raise ValueError("simulateCollateral: invalid collateral agreement")
    return out


def unilateral_cva(times, dee, pillars, hazards, recovery: float) -> float:
    f = lambda a: np.ascontiguousarray(a, np.float64)
    t, d, p, h = f(times), f(dee), f(pillars), f(hazards)
    return lib().orc_unilateral_cva(t, d, t.size, p, h, p.size, recovery)


def bilateral_cva(times, dee, dene, cpty, own, rc: float, ro: float):
    f = lambda a: np.ascontiguousarray(a, np.float64)
    out = np.zeros(2)
    lib().orc_bilateral_cva(f(times), f(dee), f(dene), len(times), f(cpty[0]), f(cpty[1]), len(cpty[0]), f(own[0]),
                            f(own[1]), len(own[0]), rc, ro, out)
    return float(out[0]), float(out[1])


# ---- the reference's outer normals (src/models/scenario_generator.cpp:89 reads ccr::NormalGenerator) ----
class Mt19937_64:
    """std::mt19937_64 (the C++ standard's parameters)."""

    def __init__(self, seed: int):
        M = (1 << 64) - 1
        self.mt = [seed & M]
        for i in range(1, 312):
            prev = self.mt[-1]
            self.mt.append((6364136223846793005 * (prev ^ (prev >> 62)) + i) & M)
        self.i = 312

    def __call__(self) -> int:
        M = (1 << 64) - 1
        if self.i >= 312:
            mt = self.mt
            for k in range(312):
                y = (mt[k] & 0xFFFFFFFF80000000) | (mt[(k + 1) % 312] & 0x7FFFFFFF)
                mt[k] = mt[(k + 156) % 312] ^ (y >> 1) ^ (0xB5026F5AA96619E9 if y & 1 else 0)
            self.i = 0
        y = self.mt[self.i]
        self.i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & M


def normal_stream(seed: int, n: int) -> np.ndarray:
    """The first n draws of ccr::NormalGenerator(seed) (include/ccr/core/random.hpp): std::normal_distribution on
    std::mt19937_64 as GCC's libstdc++ implements it (the image's compiler): the Marsaglia polar method on
    generate_canonical<double, 53> (one 64-bit draw scaled by 2^-64), the y half returned first and the x half
    kept for the next call."""
    g = Mt19937_64(seed)
    out = np.zeros(n)
    k = 0
    while k < n:
        while True:
            x = 2.0 * (float(g()) * 2.0 ** -64) - 1.0
            y = 2.0 * (float(g()) * 2.0 ** -64) - 1.0
            r2 = x * x + y * y
            if not (r2 > 1.0 or r2 == 0.0):
                break
        mult = math.sqrt(-2.0 * math.log(r2) / r2)
        out[k] = y * mult
        if k + 1 < n:
            out[k + 1] = x * mult
        k += 2
    return out
