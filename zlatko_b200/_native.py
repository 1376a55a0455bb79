"""ctypes binding of the C ABI in include/zlatko_b200.h (the library zlatko_b200/_lib/libzlatko_b200.so).

The product path has no fallback: if the library is missing, importing the kernels fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libzlatko_b200.so")

ZK_OK = 0
STATUS_NAMES = {0: "ZK_OK", 1: "ZK_ERR_INVALID_ARGUMENT", 2: "ZK_ERR_INVALID_PLAN", 3: "ZK_ERR_UNSUPPORTED",
                4: "ZK_ERR_OUT_OF_MEMORY", 5: "ZK_ERR_CUDA", 6: "ZK_ERR_DEVICE_TIMEOUT", 7: "ZK_ERR_NO_DEVICE"}


class ZkError(RuntimeError):
    """A non-zero zk_status.  ``status`` is its name; the invalid-plan and unsupported cases are the ones
    where the reference throws std::invalid_argument."""

    def __init__(self, status: int, message: str):
        self.code = status
        self.status = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.status}: {message}")


class PlanView(C.Structure):
    _fields_ = [("header", C.POINTER(C.c_uint32)), ("header_len", C.c_size_t),
                ("indices", C.POINTER(C.c_uint32)), ("indices_len", C.c_size_t),
                ("params", C.POINTER(C.c_float)), ("params_len", C.c_size_t),
                ("steps", C.POINTER(C.c_float)), ("steps_len", C.c_size_t),
                ("terms", C.POINTER(C.c_float)), ("terms_len", C.c_size_t),
                ("requests", C.POINTER(C.c_float)), ("requests_len", C.c_size_t),
                ("rows_total", C.c_uint32), ("num_outputs", C.c_uint32)]


class PlanViewF64(C.Structure):
    _fields_ = [("header", C.POINTER(C.c_uint32)), ("header_len", C.c_size_t),
                ("indices", C.POINTER(C.c_uint32)), ("indices_len", C.c_size_t),
                ("params", C.POINTER(C.c_double)), ("params_len", C.c_size_t),
                ("steps", C.POINTER(C.c_double)), ("steps_len", C.c_size_t),
                ("terms", C.POINTER(C.c_double)), ("terms_len", C.c_size_t),
                ("requests", C.POINTER(C.c_double)), ("requests_len", C.c_size_t),
                ("rows_total", C.c_uint32), ("num_outputs", C.c_uint32)]


class Output(C.Structure):
    _fields_ = [("sums", C.POINTER(C.c_float)), ("sums_len", C.c_size_t),
                ("values", C.POINTER(C.c_float)), ("values_len", C.c_size_t)]


class OutputF64(C.Structure):
    _fields_ = [("sums", C.POINTER(C.c_double)), ("sums_len", C.c_size_t),
                ("values", C.POINTER(C.c_double)), ("values_len", C.c_size_t)]


class BatchInfo(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("num_plans", "num_launch_groups", "num_paths", "num_dates", "num_trades_hint",
                                          "num_terms", "term_evaluations", "exp_evaluations", "table_bytes", "row_bytes",
                                          "kernels_per_execute", "tile_paths", "graph_replay", "num_waves",
                                          "num_basis_netting_sets", "basis_columns", "basis_terms",
                                          "basis_bytes")]


# Every entry point declared in include/zlatko_b200.h.
EXPORTS = ["zk_abi_version", "zk_context_create", "zk_context_destroy", "zk_last_error", "zk_context_set_stream", "zk_context_set_row_budget", "zk_context_set_basis", "zk_debug_basis",
           "zk_context_set_exact_decisions", "zk_context_exact_stats", "zk_context_call_timings",
           "zk_run_plan", "zk_run_plan_rows", "zk_run_plans", "zk_amc_states", "zk_fit_amc", "zk_fit_amc_f64", "zk_run_plan_f64", "zk_run_plan_injected", "zk_run_plan_noalloc", "zk_debug_inject",
           "zk_batch_create", "zk_batch_execute", "zk_batch_set_tile_paths", "zk_batch_timings", "zk_batch_read", "zk_batch_info_get",
           "zk_batch_destroy", "zk_peak_ex2", "zk_gemm_bf16", "zk_surrogate_create", "zk_surrogate_destroy",
           "zk_surrogate_train", "zk_surrogate_predict", "zk_surrogate_gradients", "zk_surrogate_params",
           "zk_surrogate_features", "zk_surrogate_book", "zk_compile", "zk_plan_view_of", "zk_plan_view_f64_of", "zk_plan_dates", "zk_plan_sizes",
           "zk_plan_destroy", "zk_factor_paths_f64", "zk_nest_create", "zk_nest_run", "zk_nest_events", "zk_nest_destroy",
           "zk_zero_bond_coefficients", "zk_hermite_fit", "zk_hermite_predict", "zk_hermite_info", "zk_hermite_destroy", "zk_erfc_array"]

_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """The loaded library; raises if it has not been built (there is no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"zlatko_b200: the CUDA library {LIB_PATH} is missing; build it with "
                           "`python -m zlatko_b200.build` (there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, sz, st = C.c_void_p, C.c_size_t, C.c_int
    P = C.POINTER
    sig = {
        "zk_abi_version": (C.c_int, []),
        "zk_context_create": (st, [C.c_int, P(vp)]),
        "zk_context_destroy": (None, [vp]),
        "zk_last_error": (C.c_char_p, [vp]),
        "zk_context_set_stream": (st, [vp, vp]),
        "zk_context_set_row_budget": (st, [vp, C.c_uint64]),
        "zk_context_set_basis": (st, [vp, C.c_uint32]),
        "zk_context_set_exact_decisions": (st, [vp, C.c_double]),
        "zk_context_exact_stats": (st, [vp, P(C.c_uint64), P(C.c_uint64)]),
        "zk_context_call_timings": (st, [vp, P(C.c_double)]),
        "zk_run_plan": (st, [vp, P(PlanView), P(Output)]),
        "zk_run_plans": (st, [vp, P(PlanView), sz, P(Output)]),
        "zk_amc_states": (st, [vp, P(PlanView), vp, vp, vp, sz]),
        "zk_fit_amc": (st, [vp, P(PlanView), vp, sz, vp, sz]),
        "zk_run_plan_rows": (st, [vp, P(PlanView), P(Output), vp]),
        "zk_gemm_bf16": (st, [vp, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, C.c_uint32, vp]),
        "zk_surrogate_create": (st, [vp, C.c_uint32, vp]),
        "zk_surrogate_destroy": (None, [vp]),
        "zk_surrogate_train": (st, [vp, vp, vp, sz, C.c_uint32, C.c_uint32, C.c_float, C.c_float, vp]),
        "zk_surrogate_predict": (st, [vp, vp, sz, vp]),
        "zk_surrogate_gradients": (st, [vp, vp, vp, sz, vp, vp]),
        "zk_surrogate_params": (st, [vp, vp, vp, vp, vp]),
        "zk_surrogate_features": (st, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp, C.c_uint32, vp, vp, vp, vp]),
        "zk_surrogate_book": (st, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp, C.c_uint32, vp, vp, vp, C.c_uint32, vp, vp,
                                   vp, vp, C.c_uint32, vp]),
        "zk_fit_amc_f64": (st, [vp, P(PlanViewF64), vp, sz, vp, sz, vp, sz]),
        "zk_run_plan_f64": (st, [vp, P(PlanViewF64), vp, sz, P(OutputF64), vp]),
        "zk_run_plan_injected": (st, [vp, P(PlanView), vp, sz, P(Output), vp]),
        "zk_run_plan_noalloc": (st, [C.c_int, vp, P(PlanView), P(Output), C.c_char_p, sz]),
        "zk_debug_inject": (st, [vp, C.c_uint32, C.c_uint64]),
        "zk_debug_basis": (st, [P(PlanView), sz, vp, vp, vp, vp, C.c_char_p, sz]),
        "zk_batch_create": (st, [vp, P(PlanView), sz, P(vp)]),
        "zk_batch_execute": (st, [vp]),
        "zk_batch_set_tile_paths": (st, [vp, C.c_uint64]),
        "zk_factor_paths_f64": (st, [vp, P(PlanViewF64), vp, sz, vp, sz]),
        "zk_nest_create": (st, [vp, vp, sz, vp, sz, vp, sz, C.c_double, vp, vp, vp, sz, sz, P(vp)]),
        "zk_nest_run": (st, [vp, vp, vp, vp, sz, vp]),
        "zk_nest_events": (st, [vp, P(C.c_uint64)]),
        "zk_nest_destroy": (None, [vp]),
        "zk_zero_bond_coefficients": (st, [vp, sz, vp, sz, vp]),
        "zk_hermite_fit": (st, [vp, sz, sz, vp, vp, sz, C.c_uint32, C.c_double, P(vp), C.c_char_p, sz]),
        "zk_hermite_predict": (st, [vp, vp, sz, sz, vp, sz, vp, vp]),
        "zk_hermite_info": (st, [vp, P(C.c_uint64)]),
        "zk_hermite_destroy": (None, [vp]),
        "zk_erfc_array": (st, [vp, sz, vp]),
        "zk_batch_timings": (st, [vp, P(C.c_float)]),
        "zk_batch_read": (st, [vp, P(Output)]),
        "zk_batch_info_get": (st, [vp, P(BatchInfo)]),
        "zk_batch_destroy": (None, [vp]),
        "zk_peak_ex2": (st, [C.c_int, P(C.c_double)]),
        "zk_compile": (st, [vp, sz, vp, sz, vp, sz, P(vp), C.c_char_p, sz]),
        "zk_plan_view_of": (st, [vp, P(PlanView)]),
        "zk_plan_view_f64_of": (st, [vp, P(PlanViewF64)]),
        "zk_plan_dates": (st, [vp, vp, sz, vp, sz]),
        "zk_plan_sizes": (st, [vp, P(C.c_uint64)]),
        "zk_plan_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status: int, ctx=None, message: str = "") -> None:
    if status != ZK_OK:
        if not message and ctx:
            message = (lib().zk_last_error(ctx) or b"").decode()
        raise ZkError(status, message)
