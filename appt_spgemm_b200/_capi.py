"""ctypes binding of the engine's C ABI (include/spgemm_b200.h).

The shared library is built in-tree into ``appt_spgemm_b200/_lib``; importing
this module loads it and fails loudly when it is missing — there is no
Python or CPU fallback for any engine call.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int32, c_int64,
                    c_uint64, c_void_p)

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libspgemm_b200.so")
CUSPARSE_LIB_PATH = os.path.join(LIB_DIR, "libspg_cusparse_baseline.so")
CLI_PATH = os.path.join(LIB_DIR, "spgemm_b200_cli")

# spg_status
SPG_OK = 0
STATUS_NAMES = {
    0: "SPG_OK", 1: "SPG_ERR_INVALID_ARG", 2: "SPG_ERR_INVALID_CSR", 3: "SPG_ERR_OOM",
    4: "SPG_ERR_CUDA", 5: "SPG_ERR_HASH_FULL", 6: "SPG_ERR_TIMEOUT",
    7: "SPG_ERR_UNSUPPORTED", 8: "SPG_ERR_BUDGET", 9: "SPG_ERR_NOT_READY", 10: "SPG_ERR_IO",
}
SPG_ERR_INVALID_ARG = 1
SPG_ERR_INVALID_CSR = 2
SPG_ERR_OOM = 3
SPG_ERR_CUDA = 4
SPG_ERR_HASH_FULL = 5
SPG_ERR_TIMEOUT = 6
SPG_ERR_UNSUPPORTED = 7
SPG_ERR_BUDGET = 8
SPG_ERR_NOT_READY = 9
SPG_ERR_IO = 10

# spg_task
TASKS = {"AA": 0, "AAt": 1, "AAtS": 2}


class SpgCsrDev(Structure):
    _fields_ = [("n", c_int32), ("nnz", c_int64), ("rowptr", c_void_p), ("col", c_void_p),
                ("val", c_void_p)]


class SpgCsrOut(Structure):
    _fields_ = [("n", c_int32), ("nnz", c_int64), ("rowptr", c_void_p), ("col", c_void_p),
                ("val", c_void_p)]


class SpgConfig(Structure):
    _fields_ = [("struct_size", c_int32), ("device", c_int32), ("lanes_per_row", c_int32),
                ("max_smem_slots", c_int32), ("heavy_threads", c_int32),
                ("window_bits", c_int32), ("force_heavy", c_int32), ("sym_load_pct", c_int32),
                ("num_load_pct", c_int32), ("heavy_split", c_int32),
                ("pool_release_bytes", c_int64), ("heavy_block_budget", c_int64),
                ("grid_sms", c_int64), ("small_max_nnz", c_int64), ("heavy_vcap", c_int64),
                ("dense_max_words", c_int64), ("bin_streams", c_int32), ("pad0", c_int32)]


class SpgEngResult(Structure):
    _fields_ = [("ms", c_float), ("nnz", c_int64), ("s", c_double), ("as_", c_double),
                ("sq", c_double)]


class SpgPlanInfo(Structure):
    _fields_ = [("n", c_int32), ("task", c_int32), ("nnz_a", c_int64), ("nnz_c", c_int64),
                ("products", c_int64), ("products_computed", c_int64),
                ("max_row_products", c_int64), ("max_row_nnz", c_int64),
                ("heavy_rows", c_int64), ("workspace_bytes", c_int64),
                ("output_bytes", c_int64), ("bins_used", c_int32), ("symmetric_pattern", c_int32),
                ("exec_workspace_bytes", c_int64)]


class SpgDescriptors(Structure):
    _fields_ = [("n", c_int32), ("nnz", c_int64), ("mean_deg", c_double), ("deg_cv", c_double),
                ("fill_aa", c_double), ("fill_aat", c_double), ("products_aa", c_int64),
                ("products_aat", c_int64), ("max_deg", c_int32), ("max_col_deg", c_int32),
                ("bandwidth", c_int32), ("reserved", c_int32), ("pattern_symmetry", c_double)]


class SpgHostCsr(Structure):
    _fields_ = [("n", c_int32), ("nnz", c_int64), ("rowptr", POINTER(c_int32)),
                ("col", POINTER(c_int32)), ("val", POINTER(c_double))]


class SpgServerConfig(Structure):
    _fields_ = [("struct_size", c_int32), ("workers", c_int32), ("memory_budget_bytes", c_int64),
                ("batch_rows", c_int32), ("batch_max", c_int32), ("reserved", c_int64 * 4)]


class SpgRequestInfo(Structure):
    _fields_ = [("id", c_uint64), ("status", c_int32), ("task", c_int32), ("n", c_int32),
                ("batched", c_int32), ("nnz_c", c_int64), ("products", c_int64),
                ("reserved_bytes", c_int64), ("submit_ms", c_double), ("start_ms", c_double),
                ("done_ms", c_double), ("planned_ms", c_double), ("run_ms", c_double)]


class SpgServerStats(Structure):
    _fields_ = [("submitted", c_int64), ("completed", c_int64), ("rejected", c_int64),
                ("failed", c_int64), ("batches", c_int64), ("products_completed", c_int64),
                ("budget_bytes", c_int64), ("reserved_bytes", c_int64),
                ("peak_reserved_bytes", c_int64), ("p50_ms", c_double), ("p99_ms", c_double),
                ("max_ms", c_double), ("first_submit_ms", c_double), ("last_done_ms", c_double),
                ("held_bytes", c_int64), ("peak_held_bytes", c_int64)]


_ctx_p = c_void_p
_plan_p = c_void_p
_srv_p = c_void_p

# name → (restype, argtypes); every function declared in include/spgemm_b200.h
SIGNATURES = {
    "spg_abi_version": (c_int32, []),
    "spg_last_error_string": (c_char_p, []),
    "spg_status_string": (c_char_p, [c_int32]),
    "spg_create": (c_int32, [POINTER(_ctx_p), POINTER(SpgConfig)]),
    "spg_destroy": (c_int32, [_ctx_p]),
    "spg_check_device_status": (c_int32, [_ctx_p, c_void_p]),
    "spg_plan_create": (c_int32, [_ctx_p, c_int32, POINTER(SpgCsrDev), c_void_p,
                                  POINTER(_plan_p)]),
    "spg_plan_get_info": (c_int32, [_plan_p, POINTER(SpgPlanInfo)]),
    "spg_plan_workspace_bound": (c_int32, [_ctx_p, c_int32, c_int32, POINTER(SpgCsrDev), c_int32,
                                           POINTER(c_int64)]),
    "spg_execute": (c_int32, [_plan_p, POINTER(SpgCsrOut), c_void_p]),
    "spg_plan_destroy": (c_int32, [_plan_p]),
    "spg_multiply": (c_int32, [_ctx_p, c_int32, POINTER(SpgCsrDev), POINTER(SpgCsrOut),
                               c_void_p]),
    "spg_free": (c_int32, [_ctx_p, c_void_p, c_void_p]),
    "spg_plan_create_batched": (c_int32, [_ctx_p, c_int32, c_int32, POINTER(SpgCsrDev), c_void_p,
                                          POINTER(_plan_p)]),
    "spg_plan_batch_offsets": (c_int32, [_plan_p, POINTER(c_int64), POINTER(c_int64)]),
    "spg_graph_capture": (c_int32, [_plan_p, POINTER(SpgCsrOut), c_void_p, POINTER(c_void_p)]),
    "spg_graph_launch": (c_int32, [c_void_p, c_void_p]),
    "spg_graph_destroy": (c_int32, [c_void_p]),
    "spg_server_create": (c_int32, [POINTER(SpgServerConfig), POINTER(_srv_p)]),
    "spg_server_submit": (c_int32, [_srv_p, c_int32, POINTER(SpgCsrDev), POINTER(c_uint64)]),
    "spg_server_poll": (c_int32, [_srv_p, c_uint64, POINTER(SpgRequestInfo)]),
    "spg_server_wait": (c_int32, [_srv_p, c_uint64, c_int32, POINTER(SpgRequestInfo)]),
    "spg_server_copy_result": (c_int32, [_srv_p, c_uint64, c_void_p, c_void_p, c_void_p]),
    "spg_server_release": (c_int32, [_srv_p, c_uint64]),
    "spg_server_stats_get": (c_int32, [_srv_p, POINTER(SpgServerStats)]),
    "spg_server_destroy": (c_int32, [_srv_p]),
    "spg_set_config": (c_int32, [_ctx_p, POINTER(SpgConfig)]),
    "spg_get_config": (c_int32, [_ctx_p, POINTER(SpgConfig)]),
    "spg_autotune": (c_int32, [_ctx_p, c_int32, c_int32, POINTER(SpgCsrDev), c_int32,
                               POINTER(SpgConfig), c_void_p]),
    "spg_autotune_trials": (c_int32, [_ctx_p, POINTER(c_int32), POINTER(c_int32)]),
    "spg_profile_enable": (c_int32, [_ctx_p, c_int32]),
    "spg_profile_reset": (c_int32, [_ctx_p]),
    "spg_profile_read": (c_int32, [_ctx_p, c_char_p, c_uint64]),
    "spg_drop_zeros": (c_int32, [_ctx_p, POINTER(SpgCsrOut), c_void_p]),
    "spg_transpose": (c_int32, [_ctx_p, POINTER(SpgCsrDev), c_void_p, c_void_p, c_void_p,
                                c_void_p]),
    "spg_transpose_noalloc": (c_int32, [POINTER(SpgCsrDev), c_void_p, c_void_p, c_void_p,
                                        c_void_p]),
    "spg_describe": (c_int32, [_ctx_p, POINTER(SpgCsrDev), POINTER(SpgDescriptors), c_void_p]),
    "spg_run_ours": (c_int32, [c_char_p, c_void_p, c_void_p, c_void_p, c_int32, c_int64,
                               c_int32, POINTER(SpgEngResult)]),
    "spg_checksum": (c_int32, [c_void_p, c_int64, POINTER(c_double), POINTER(c_double),
                               POINTER(c_double)]),
    "spg_csr1_read": (c_int32, [c_char_p, POINTER(SpgHostCsr)]),
    "spg_csr1_write": (c_int32, [c_char_p, POINTER(SpgHostCsr)]),
    "spg_host_csr_free": (None, [POINTER(SpgHostCsr)]),
    "spg_host_csr_validate": (c_int32, [POINTER(SpgHostCsr)]),
    "spg_gen_laplace2d": (c_int32, [c_int32, POINTER(SpgHostCsr)]),
    "spg_gen_stencil27": (c_int32, [c_int32, c_uint64, POINTER(SpgHostCsr)]),
    "spg_gen_rmat": (c_int32, [c_int32, c_int32, c_double, c_double, c_double, c_uint64,
                               POINTER(SpgHostCsr)]),
    "spg_gen_banded": (c_int32, [c_int32, c_int32, c_double, c_uint64, POINTER(SpgHostCsr)]),
    "spg_gen_er": (c_int32, [c_int32, c_double, c_uint64, POINTER(SpgHostCsr)]),
    "spg_gen_uniform": (c_int32, [c_int32, c_int32, c_uint64, POINTER(SpgHostCsr)]),
}


class SpgemmError(RuntimeError):
    """An engine call returned a status other than SPG_OK."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.status_name}: {message}")


_lib = None


def lib():
    """The loaded engine library (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"engine library not built: {LIB_PATH} is missing "
                "(run `make -C appt_spgemm_b200/csrc` or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, what: str = "") -> None:
    if status != SPG_OK:
        msg = lib().spg_last_error_string()
        msg = msg.decode() if msg else ""
        raise SpgemmError(status, f"{what}: {msg}" if what else msg)
