"""ctypes bindings of ``include/moao_b200.h`` (the C ABI of libmoao_b200.so).

The library is loaded from the package directory only; a missing or unloadable
library raises immediately, so no code path can silently run without the CUDA
implementation.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmoao_b200.so")

MOAO_OK = 0
STATUS = {0: "MOAO_OK", 1: "MOAO_ERR_BAD_ARG", 2: "MOAO_ERR_NOT_SPD", 3: "MOAO_ERR_OOM",
          4: "MOAO_ERR_CUDA", 5: "MOAO_ERR_IO", 6: "MOAO_ERR_TIMEOUT", 7: "MOAO_ERR_UNSUPPORTED",
          8: "MOAO_ERR_BUSY", 9: "MOAO_ERR_CANCELLED"}
PREC = {"fp64": 0, "mixed": 1}

vp = C.c_void_p
dp = C.c_void_p  # double* (device or host address as an integer)
i32 = C.c_int
i64 = C.c_long


class TomoInfo(C.Structure):
    _fields_ = [("nW", i32), ("nLgs", i32), ("nNgs", i32), ("nTarget", i32), ("nLayer", i32),
                ("Nx", i32), ("nmeas", i64), ("nmeasts", i64), ("diam", C.c_double),
                ("obs", C.c_double), ("lgsCst", C.c_double), ("nssp_ts", i32)]


class SolveReport(C.Structure):
    _fields_ = [("info", i32), ("refine_steps", i32), ("refine_resid", C.c_double),
                ("ms_factor", C.c_double), ("ms_solve", C.c_double), ("ms_refine", C.c_double),
                ("fallback", i32), ("est_error", C.c_double)]


class IsampleInfo(C.Structure):
    _fields_ = [("N", i64), ("np", i64), ("nidx", i64), ("lambda_", C.c_double),
                ("dactupix", C.c_double)]


class ServerOpts(C.Structure):
    _fields_ = [("device", i32), ("slots", i32), ("hbm_budget_gb", C.c_double),
                ("queue_capacity", i32), ("nb", i32), ("dry_run", i32)]


class Request(C.Structure):
    _fields_ = [("system", i32), ("nlayer", i32), ("cn2", vp), ("h", vp), ("L0", vp),
                ("target", i32), ("prec", i32), ("R", vp), ("Cvv", vp), ("psf", vp),
                ("dry_run_ms", C.c_double)]


class RequestResult(C.Structure):
    _fields_ = [("status", i32), ("info", i32), ("slot", i32), ("refine_steps", i32),
                ("refine_resid", C.c_double), ("queue_ms", C.c_double), ("run_ms", C.c_double),
                ("latency_ms", C.c_double), ("start_ms", C.c_double), ("end_ms", C.c_double),
                ("footprint_gb", C.c_double),
                ("message", C.c_char * 256)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("failed", C.c_longlong),
                ("cancelled", C.c_longlong), ("rejected", C.c_longlong), ("max_in_flight", i32),
                ("peak_admitted_gb", C.c_double), ("budget_gb", C.c_double)]


class BatchItem(C.Structure):
    _fields_ = [("tomo", vp), ("d_R", vp), ("nb", i32), ("status", i32), ("info", i32),
                ("nb_used", i32), ("stream", i32), ("packed", i32)]


class BatchOpts(C.Structure):
    _fields_ = [("prec", i32), ("streams", i32), ("hbm_budget_gb", C.c_double),
                ("packed_max", C.c_long), ("gemm_tile", i32),
                ("ms_device", C.c_double),
                ("ms_build", C.c_double), ("graph_nodes", C.c_longlong),
                ("streams_used", i32), ("failed", i32), ("device_gb", C.c_double),
                ("packed_count", i32), ("packed_tasks", C.c_longlong)]


# name -> (restype, argtypes)
SIGNATURES = {
    "moao_status_string": (C.c_char_p, [i32]),
    "moao_last_error": (C.c_char_p, []),
    "moao_tomo_create": (i32, [C.c_char_p, C.c_char_p, C.POINTER(vp)]),
    "moao_tomo_update_atm": (i32, [vp, C.c_char_p]),
    "moao_tomo_set_profile": (i32, [vp, i32, dp, dp, dp]),
    "moao_tomo_set_target": (i32, [vp, i32]),
    "moao_tomo_get_info": (i32, [vp, C.POINTER(TomoInfo)]),
    "moao_tomo_table": (i64, [vp, C.c_char_p, dp, i64]),
    "moao_tomo_destroy": (None, [vp]),
    "moao_ctx_create": (i32, [i32, C.POINTER(vp)]),
    "moao_ctx_destroy": (None, [vp]),
    "moao_ctx_set_stream": (i32, [vp, vp]),
    "moao_ctx_use_own_stream": (i32, [vp]),
    "moao_ctx_stream": (vp, [vp]),
    "moao_ctx_synchronize": (i32, [vp]),
    "moao_ctx_launch_count": (C.c_longlong, [vp]),
    "moao_ctx_set_block": (i32, [vp, i32]),
    "moao_ctx_set_kernel_timing": (i32, [vp, i32]),
    "moao_ctx_set_mixed": (i32, [vp, i32, i32, i32, i32, C.c_double, i32]),
    "moao_ctx_set_offsets": (i32, [vp, i32, vp, vp, vp]),
    "moao_ctx_set_host_precision": (i32, [vp, i32]),
    "moao_ctx_set_wait_limit": (i32, [vp, C.c_longlong]),
    "moao_ctx_set_accuracy": (i32, [vp, C.c_double]),
    "moao_ctx_set_lookahead_max": (i32, [vp, i32]),
    "moao_ctx_set_gemm_tile": (i32, [vp, i32]),
    "moao_ctx_set_tc_pair": (i32, [vp, i32]),
    "moao_ctx_set_residual": (i32, [vp, i32]),
    "moao_ctx_set_host_cache": (i32, [vp, i32]),
    "moao_dense_potrf_inv": (i32, [vp, i64, vp, i64, vp, i64, C.POINTER(i32)]),
    "moao_dense_gemm": (i32, [vp, i32, i32, i64, i64, i64, C.c_double, vp, i64, vp, i64,
                              C.c_double, vp, i64]),
    "moao_tuning_get_packed": (i32, [vp, i32, C.POINTER(C.c_long)]),
    "moao_tuning_get_gemm": (i32, [vp, i32, vp]),
    "moao_packed_task_list": (i32, [i32, vp, vp, vp, C.c_long, C.POINTER(C.c_long),
                                    C.POINTER(i32)]),
    "moao_intersample_inputs": (i32, [vp, i64, C.c_double, C.c_double, C.c_double, vp, vp, vp, vp,
                                      vp]),
    "moao_intersample_create_synth": (i32, [vp, i64, C.c_double, C.c_double, C.c_double, vp]),
    "moao_ctx_set_factor_format": (i32, [vp, i32]),
    "moao_ctx_set_lookahead": (i32, [vp, i32]),
    "moao_server_create": (i32, [C.POINTER(ServerOpts), C.POINTER(vp)]),
    "moao_server_add_system_synth": (i32, [vp, C.c_char_p, C.c_char_p, C.c_long, vp, C.c_double,
                                           C.POINTER(i32)]),
    "moao_server_add_system": (i32, [vp, C.c_char_p, C.c_char_p, C.c_long, vp, vp, vp, vp,
                                     C.POINTER(i32)]),
    "moao_server_system_info": (i32, [vp, i32, C.POINTER(C.c_long), C.POINTER(C.c_long),
                                      C.POINTER(C.c_long), C.POINTER(C.c_long)]),
    "moao_serve_submit": (i32, [vp, C.POINTER(Request), C.POINTER(C.c_longlong)]),
    "moao_serve_poll": (i32, [vp, C.c_longlong, C.POINTER(RequestResult)]),
    "moao_serve_wait": (i32, [vp, C.c_longlong, C.c_double, C.POINTER(RequestResult)]),
    "moao_serve_cancel": (i32, [vp, C.c_longlong]),
    "moao_server_get_stats": (i32, [vp, C.POINTER(ServerStats)]),
    "moao_server_destroy": (None, [vp]),
    "moao_batch_reconstructors": (i32, [vp, i32, vp, C.POINTER(BatchOpts)]),
    "moao_autotune": (i32, [vp, i32, vp, i32, vp, i32]),
    "moao_tuning_get": (i32, [vp, i32, vp, C.POINTER(i32)]),
    "moao_tuning_save": (i32, [vp, C.c_char_p]),
    "moao_tuning_load": (i32, [vp, C.c_char_p]),
    "moao_fits_read_f64": (i32, [C.c_char_p, C.POINTER(C.c_long), C.POINTER(C.c_long), vp, C.c_long]),
    "moao_fits_read_i64": (i32, [C.c_char_p, C.POINTER(C.c_long), C.POINTER(C.c_long), vp, C.c_long]),
    "moao_fits_write_f64": (i32, [C.c_char_p, C.c_long, C.c_long, vp]),
    "moao_fits_write_i64": (i32, [C.c_char_p, C.c_long, C.c_long, vp]),
    "moao_ctx_set_offsets_from_tomo": (i32, [vp, vp]),
    "moao_ctx_kernel_stats": (i32, [vp, C.c_char_p, C.POINTER(C.c_longlong), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)]),
    "moao_ctx_reset_kernel_stats": (i32, [vp]),
    "moao_matcov_tile": (i32, [vp, vp, dp, i32, i32, i32, i32, i32, i32]),
    "moao_matcov_tile_host": (i32, [vp, vp, dp, i32, i32, i32, i32, i32, i32]),
    "moao_reconstructor": (i32, [vp, i64, i64, dp, i64, dp, i64, i64, i32, C.POINTER(SolveReport)]),
    "moao_reconstructor_host": (i32, [vp, i64, i64, dp, i64, dp, i64, i64, C.POINTER(SolveReport)]),
    "moao_reconstructor_noalloc": (i32, [i64, i64, dp, i64, dp, i64, i64, vp, C.POINTER(i32)]),
    "moao_cee_cvv": (i32, [vp, i64, i64, i64] + [dp, i64] * 8),
    "moao_cee_cvv_host": (i32, [vp, i64, i64, i64] + [dp, i64] * 8),
    "moao_cee_cvv_prec": (i32, [vp, i64, i64, i64] + [dp, i64] * 8 + [i32]),
    "moao_intersample_create": (i32, [vp, i64, i64, C.c_double, dp, dp, dp, C.POINTER(vp)]),
    "moao_intersample_get_info": (i32, [vp, C.POINTER(IsampleInfo)]),
    "moao_intersample_process": (i32, [vp, dp, dp]),
    "moao_intersample_process_host": (i32, [vp, dp, dp]),
    "moao_intersample_destroy": (None, [vp]),
    "moao_debug_tc_gemm": (i32, [vp, i32, i64, i64, i64, dp, i64, i32, dp, i64, i32, i32, dp, dp, dp,
                                 i64, C.c_float, C.c_float, dp, dp, i32, i32]),
    "moao_debug_residual": (i32, [vp, i32, i64, i64, dp, i64, dp, i64, dp, i64, dp, i64]),
    "moao_debug_crt_moduli": (i32, [i32, i64]),
}


class MoaoError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        self.name = STATUS.get(status, str(status))
        super().__init__(f"{where}: {self.name}" + (f" ({detail})" if detail else ""))


class NotSPDError(MoaoError):
    """Cholesky met a non-positive pivot; ``column`` is the 1-based column."""

    def __init__(self, status, where, detail="", column=0):
        super().__init__(status, where, detail)
        self.column = column


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"moao_b200: {LIB_PATH} is missing; build it with `python -m moao_b200.build` "
                "(the CUDA implementation is the only implementation)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str, **kw):
    if status != MOAO_OK:
        detail = lib().moao_last_error().decode(errors="replace")
        if status == 2:
            raise NotSPDError(status, where, detail, **kw)
        raise MoaoError(status, where, detail)
