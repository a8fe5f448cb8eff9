"""ctypes binding of libts_b200.so (include/ts_b200.h).

The library is built in-tree (``make`` in the package directory).  Loading it
needs no GPU; every compute entry point fails with ``TsError`` when no CUDA
device is visible -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libts_b200.so")

OK, ERR_INVALID_ARG, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_UNSUPPORTED, ERR_DEVICE, ERR_STATE, ERR_NO_DEVICE = range(8)

STRUCT_CSR, STRUCT_HASH, STRUCT_WSWAP, STRUCT_CSR_BITSET, STRUCT_CSR_BB, STRUCT_CSR_BITSET_BB = range(6)
STRUCT_NAMES = ["csr", "hash", "wswap", "csr-bitset", "csr-bb", "csr-bitset-bb"]
PROBLEM_MDP, PROBLEM_MAXBS = 0, 1
TENURE_REF, TENURE_FIXED = 0, 1
PASS_AUTO, PASS_TILE, PASS_ROWS = 0, 1, 2

# Every symbol include/ts_b200.h declares.
EXPORTS = [
    "ts_abi_version", "ts_status_string", "ts_last_error", "ts_struct_from_name", "ts_struct_name",
    "ts_graph_create", "ts_graph_create_device", "ts_graph_info_get", "ts_graph_destroy",
    "ts_lookup", "ts_lookup_host", "ts_params_default", "ts_solver_create", "ts_solver_init",
    "ts_solver_step", "ts_solver_result", "ts_solver_state", "ts_solver_trace",
    "ts_solver_destroy", "ts_solver_info_get", "ts_random_start", "ts_perturb_draws", "ts_solver_prepare",
    "ts_solver_enqueue", "ts_solver_sync", "ts_best_swap_noalloc",
    "ts_batch_create", "ts_batch_launch", "ts_batch_sync", "ts_batch_results", "ts_batch_info_get",
    "ts_batch_destroy", "ts_batch_run", "ts_solver_set_perturbations",
    "ts_server_create", "ts_server_submit", "ts_server_poll", "ts_server_stats_get", "ts_server_now",
    "ts_server_destroy",
]


class TsError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__(f"{where}: status {status}: {message}")


class GraphInfo(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32), ("kind", ctypes.c_int32), ("num_edges", ctypes.c_int64),
        ("num_entries", ctypes.c_int64), ("max_weighted_degree", ctypes.c_int64),
        ("device_bytes", ctypes.c_int64), ("hash_slots", ctypes.c_int64),
        ("bitset_words_per_row", ctypes.c_int64),
    ]


class SolverInfo(ctypes.Structure):
    _fields_ = [
        ("grid", ctypes.c_int32), ("tile_rows", ctypes.c_int32), ("chunk_cols", ctypes.c_int32),
        ("n_chunks", ctypes.c_int32), ("threads", ctypes.c_int32), ("dyn_smem_bytes", ctypes.c_int32),
        ("key_bytes", ctypes.c_int32), ("w_bytes", ctypes.c_int32), ("slices", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 7),
    ]


class Params(ctypes.Structure):
    _fields_ = [
        ("problem", ctypes.c_int32), ("m", ctypes.c_int32), ("max_iter", ctypes.c_int64),
        ("tenure_policy", ctypes.c_int32), ("tenure", ctypes.c_int32), ("maxt", ctypes.c_int32),
        ("piter", ctypes.c_int32), ("gamma", ctypes.c_int32), ("seed", ctypes.c_uint32),
        ("trace", ctypes.c_int32), ("pass_", ctypes.c_int32), ("reserved", ctypes.c_int32 * 6),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int64), ("evaluations", ctypes.c_int64), ("cur", ctypes.c_int64),
        ("best", ctypes.c_int64), ("best_true", ctypes.c_int64), ("perturbations", ctypes.c_int64),
        ("stopped", ctypes.c_int32), ("m", ctypes.c_int32), ("n", ctypes.c_int32),
        ("device_error", ctypes.c_int32),
    ]


class BatchJob(ctypes.Structure):
    _fields_ = [
        ("graph", ctypes.c_void_p), ("params", Params), ("initial", ctypes.c_void_p),
        ("cluster", ctypes.c_int32), ("reserved", ctypes.c_int32 * 3),
    ]


class BatchOpts(ctypes.Structure):
    _fields_ = [("max_bytes", ctypes.c_int64), ("max_slots", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 5)]


class BatchInfo(ctypes.Structure):
    _fields_ = [
        ("jobs", ctypes.c_int32), ("groups", ctypes.c_int32), ("slots", ctypes.c_int64),
        ("slot_bytes", ctypes.c_int64), ("input_bytes", ctypes.c_int64),
        ("best_sol_words", ctypes.c_int64),
    ]


class Request(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32), ("num_edges", ctypes.c_int64), ("u", ctypes.c_void_p),
        ("v", ctypes.c_void_p), ("w", ctypes.c_void_p), ("kind", ctypes.c_int32),
        ("drop_self_loops", ctypes.c_int32), ("params", Params), ("initial", ctypes.c_void_p),
        ("best_sol", ctypes.c_void_p),
    ]


class ServerOpts(ctypes.Structure):
    _fields_ = [("max_bytes", ctypes.c_int64), ("round_ms", ctypes.c_double),
                ("plain_min_pairs", ctypes.c_int64), ("reserved", ctypes.c_int32 * 8)]


class Served(ctypes.Structure):
    _fields_ = [
        ("ticket", ctypes.c_int64), ("status", ctypes.c_int32), ("executor", ctypes.c_int32),
        ("kind", ctypes.c_int32), ("pad", ctypes.c_int32), ("result", Result),
        ("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double),
        ("footprint_bytes", ctypes.c_int64),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_int64), ("admitted", ctypes.c_int64), ("completed", ctypes.c_int64),
        ("queued", ctypes.c_int64), ("active", ctypes.c_int64), ("rounds", ctypes.c_int64),
        ("bytes_in_use", ctypes.c_int64), ("bytes_budget", ctypes.c_int64), ("busy_s", ctypes.c_double),
    ]


TRACE_DTYPE = np.dtype([
    ("iter", "<i8"), ("idx", "<i8"), ("key", "<i8"), ("cur", "<i8"), ("best", "<i8"),
    ("kind", "<i4"), ("tenure", "<i4"), ("tenure2", "<i4"), ("pad", "<i4"),
])

_lib = None


def lib():
    """Loads the library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise TsError(ERR_STATE, "load", f"{LIB_PATH} not built; run build() or make")
    L = ctypes.CDLL(LIB_PATH)
    P, I32, I64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    st = ctypes.c_int
    L.ts_abi_version.restype = I32
    L.ts_status_string.restype = ctypes.c_char_p
    L.ts_status_string.argtypes = [st]
    L.ts_last_error.restype = ctypes.c_char_p
    L.ts_struct_from_name.restype = I32
    L.ts_struct_from_name.argtypes = [ctypes.c_char_p]
    L.ts_struct_name.restype = ctypes.c_char_p
    L.ts_struct_name.argtypes = [I32]
    L.ts_graph_create.restype = st
    L.ts_graph_create.argtypes = [I32, I64, P, P, P, I32, I32, P, ctypes.POINTER(P)]
    L.ts_graph_create_device.restype = st
    L.ts_graph_create_device.argtypes = [I32, I64, P, P, P, I32, I32, P, ctypes.POINTER(P)]
    L.ts_graph_info_get.restype = st
    L.ts_graph_info_get.argtypes = [P, ctypes.POINTER(GraphInfo)]
    L.ts_graph_destroy.restype = st
    L.ts_graph_destroy.argtypes = [P]
    L.ts_lookup.restype = st
    L.ts_lookup.argtypes = [P, I64, P, P, P]
    L.ts_lookup_host.restype = st
    L.ts_lookup_host.argtypes = [P, I64, P, P, P]
    L.ts_params_default.restype = st
    L.ts_params_default.argtypes = [I32, ctypes.POINTER(Params)]
    L.ts_solver_create.restype = st
    L.ts_solver_create.argtypes = [P, ctypes.POINTER(Params), ctypes.POINTER(P)]
    L.ts_solver_init.restype = st
    L.ts_solver_init.argtypes = [P, P]
    L.ts_solver_set_perturbations.restype = st
    L.ts_solver_set_perturbations.argtypes = [P, P, I64]
    L.ts_solver_step.restype = st
    L.ts_solver_step.argtypes = [P, I64, ctypes.POINTER(I64)]
    L.ts_solver_result.restype = st
    L.ts_solver_result.argtypes = [P, ctypes.POINTER(Result), P]
    L.ts_solver_state.restype = st
    L.ts_solver_state.argtypes = [P, P, P, P, P]
    L.ts_solver_trace.restype = st
    L.ts_solver_trace.argtypes = [P, P, I64, ctypes.POINTER(I64)]
    L.ts_solver_destroy.restype = st
    L.ts_solver_destroy.argtypes = [P]
    L.ts_solver_info_get.restype = st
    L.ts_solver_info_get.argtypes = [P, ctypes.POINTER(SolverInfo)]
    L.ts_solver_prepare.restype = st
    L.ts_solver_prepare.argtypes = [P, I64, ctypes.POINTER(I64)]
    L.ts_solver_enqueue.restype = st
    L.ts_solver_enqueue.argtypes = [P, I64]
    L.ts_solver_sync.restype = st
    L.ts_solver_sync.argtypes = [P, ctypes.POINTER(I64)]
    L.ts_random_start.restype = st
    L.ts_random_start.argtypes = [I32, I32, I32, ctypes.c_uint32, P]
    L.ts_perturb_draws.restype = st
    L.ts_perturb_draws.argtypes = [I32, ctypes.c_uint32, I32, I32, I32, P]
    L.ts_batch_create.restype = st
    L.ts_batch_create.argtypes = [P, I32, ctypes.POINTER(BatchOpts), P, ctypes.POINTER(P)]
    L.ts_batch_launch.restype = st
    L.ts_batch_launch.argtypes = [P]
    L.ts_batch_sync.restype = st
    L.ts_batch_sync.argtypes = [P]
    L.ts_batch_results.restype = st
    L.ts_batch_results.argtypes = [P, P, P]
    L.ts_batch_info_get.restype = st
    L.ts_batch_info_get.argtypes = [P, ctypes.POINTER(BatchInfo)]
    L.ts_batch_destroy.restype = st
    L.ts_batch_destroy.argtypes = [P]
    L.ts_batch_run.restype = st
    L.ts_batch_run.argtypes = [P, I32, ctypes.POINTER(BatchOpts), P, P]
    L.ts_server_create.restype = st
    L.ts_server_create.argtypes = [ctypes.POINTER(ServerOpts), ctypes.POINTER(P)]
    L.ts_server_submit.restype = st
    L.ts_server_submit.argtypes = [P, ctypes.POINTER(Request), ctypes.POINTER(I64)]
    L.ts_server_poll.restype = st
    L.ts_server_poll.argtypes = [P, P, I32, ctypes.POINTER(I32), I32]
    L.ts_server_stats_get.restype = st
    L.ts_server_stats_get.argtypes = [P, ctypes.POINTER(ServerStats)]
    L.ts_server_now.restype = ctypes.c_double
    L.ts_server_now.argtypes = [P]
    L.ts_server_destroy.restype = st
    L.ts_server_destroy.argtypes = [P]
    _lib = L
    return L


def check(status: int, where: str) -> None:
    if status != OK:
        msg = lib().ts_last_error().decode(errors="replace")
        raise TsError(status, where, msg)


def ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)
