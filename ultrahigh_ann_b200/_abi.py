"""ctypes declarations of the C ABI in include/uha_b200.h.

The shared library is built in-tree (ultrahigh_ann_b200/libuha_b200.so). There
is no fallback: when the library is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes
from ctypes import (POINTER, c_char, c_char_p, c_double, c_int, c_uint32, c_uint64,
                    c_void_p)
from pathlib import Path

LIBRARY_PATH = Path(__file__).resolve().parent / "libuha_b200.so"

# uha_status
OK = 0
INVALID_ARGUMENT = 1
LENGTH_ERROR = 2
RUNTIME_ERROR = 3
OVERFLOW_ERROR = 4
OUT_OF_RANGE = 5
DOMAIN_ERROR = 6
LOGIC_ERROR = 7

# uha_metric
L2 = 0
L1 = 1

# uha_pair_backend
PAIRS_DIRECT = 0
PAIRS_GRAM = 1
PAIRS_DIRECT_MAX32 = 2
PAIRS_GRAM_MAX32 = 3

# uha_strategy
DIRECT = 0
GEMM = 1
GEMM_BF16_RERANK = 2
GEMM_FP8_RERANK = 3
GEMM_BF16_RERANK_FP32 = 4
GEMM_FP8_RERANK_FP32 = 5
REPLAY_BINARY64 = 0
REPLAY_EMULATED = 1


class TuneReport(ctypes.Structure):
    _fields_ = [("candidates", ctypes.c_uint32), ("kernel", ctypes.c_uint32),
                ("queries_per_pass", ctypes.c_uint32), ("tile_queries", ctypes.c_uint32),
                ("splits", ctypes.c_uint32), ("best_ms", c_double),
                ("default_ms", c_double)]


class BatchStats(ctypes.Structure):
    _fields_ = [("pairs", c_uint64), ("queries", c_uint64), ("graph_nodes", c_uint64),
                ("kernel_launches", c_uint64), ("replayed_queries", c_uint64),
                ("device_ms", c_double)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", c_uint64), ("max_batch", ctypes.c_uint32),
                ("slots", ctypes.c_uint32), ("queries_on_device", c_int)]


class ServerResult(ctypes.Structure):
    _fields_ = [("tag", c_uint64), ("index_id", ctypes.c_uint32),
                ("status", ctypes.c_uint32), ("row", c_uint64), ("distance", c_double),
                ("latency_us", c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", c_uint64), ("completed", c_uint64), ("failed", c_uint64),
                ("batches", c_uint64), ("mean_batch", c_double), ("p50_us", c_double),
                ("p99_us", c_double), ("max_us", c_double), ("throughput_qps", c_double),
                ("workspace_bytes", c_uint64), ("peak_workspace_bytes", c_uint64),
                ("admission_waits", c_uint64), ("evictions", c_uint64),
                ("peak_in_flight", ctypes.c_uint32)]


VALUES_F32 = 0
VALUES_BF16 = 1


class DeviceMatrix(ctypes.Structure):
    _fields_ = [("data", c_void_p), ("type", c_int), ("rows", c_uint64),
                ("columns", c_uint64), ("row_stride", c_uint64)]


class SpaceUsage(ctypes.Structure):
    _fields_ = [("index_payload_bytes", c_uint64),
                ("query_workspace_payload_bytes", c_uint64),
                ("unique_query_coordinates", c_uint64),
                ("sampled_multiplicity", c_uint64)]


class DeviceInfo(ctypes.Structure):
    _fields_ = [("device", c_int),
                ("device_name", c_char * 256),
                ("compute_capability_major", c_int),
                ("compute_capability_minor", c_int),
                ("total_global_memory_bytes", c_uint64),
                ("compiled_runtime_version", c_int),
                ("runtime_version", c_int),
                ("driver_version", c_int)]


class QueryStats(ctypes.Structure):
    _fields_ = [("query_count", c_uint64),
                ("certified_queries", c_uint64),
                ("replayed_queries", c_uint64),
                ("kernel_launches", c_uint64),
                ("scan_ms", c_double),
                ("device_ms", c_double),
                ("timed_scans", c_uint64)]


class ProbabilityReport(ctypes.Structure):
    _fields_ = [("pair_count", c_uint64),
                ("pair_chunks", c_uint64),
                ("device_working_set_bytes", c_uint64),
                ("host_to_device_ms", c_double),
                ("inverse_distance_ms", c_double),
                ("coordinate_maximum_ms", c_double),
                ("device_to_host_ms", c_double),
                ("total_ms", c_double)]


_F = POINTER(ctypes.c_float)
_D = POINTER(c_double)
_U = POINTER(c_uint64)
_H = POINTER(c_void_p)

# name -> (restype, argtypes)
SIGNATURES = {
    "uha_last_error": (c_char_p, []),
    "uha_cuda_available": (c_int, []),
    "uha_device_info_get": (c_int, [c_int, POINTER(DeviceInfo)]),
    "uha_exact_index_create": (c_int, [c_int, c_int, c_void_p, c_uint64, c_uint64, _H]),
    "uha_weighted_l1_index_create": (c_int, [c_int, c_void_p, c_uint64, c_uint64, c_void_p, _H]),
    "uha_sampled_index_create": (c_int, [c_int, c_int, c_void_p, c_uint64, c_uint64,
                                          c_void_p, c_void_p, c_void_p, c_uint64, _H]),
    "uha_hierarchical_index_create": (c_int, [c_int, c_int, c_void_p, c_uint64, c_uint64,
                                               c_void_p, c_void_p, c_void_p, c_uint64,
                                               c_void_p, c_uint64, _H]),
    "uha_exact_index_create_device": (c_int, [c_int, c_int, POINTER(DeviceMatrix), _H]),
    "uha_sampled_index_create_device": (c_int, [c_int, c_int, POINTER(DeviceMatrix),
                                                 c_void_p, c_void_p, c_void_p, c_uint64,
                                                 _H]),
    "uha_hierarchical_index_create_device": (c_int, [c_int, c_int, POINTER(DeviceMatrix),
                                                      c_void_p, c_void_p, c_void_p,
                                                      c_uint64, c_void_p, c_uint64, _H]),
    "uha_index_destroy": (None, [c_void_p]),
    "uha_index_space_usage": (c_int, [c_void_p, POINTER(SpaceUsage)]),
    "uha_index_device": (c_int, [c_void_p, POINTER(c_int), c_char_p, c_uint64]),
    "uha_workspace_create": (c_int, [c_void_p, c_uint64, _H]),
    "uha_workspace_destroy": (None, [c_void_p]),
    "uha_workspace_info": (c_int, [c_void_p, _U, _U]),
    "uha_query": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_int, c_int,
                          c_void_p, c_void_p]),
    "uha_query_many": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_uint64, c_int,
                               c_int, c_void_p, c_void_p]),
    "uha_query_noalloc": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_void_p,
                                  c_void_p]),
    "uha_workspace_last_stats": (c_int, [c_void_p, POINTER(QueryStats)]),
    "uha_workspace_set_timing": (c_int, [c_void_p, c_int]),
    "uha_workspace_stream": (c_void_p, [c_void_p]),
    "uha_workspace_set_candidates": (c_int, [c_void_p, c_uint32]),
    "uha_workspace_set_replay": (c_int, [c_void_p, c_int]),
    "uha_workspace_autotune": (c_int, [c_void_p, c_uint64, c_int, POINTER(TuneReport)]),
    "uha_batch_create": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_int, _H]),
    "uha_batch_create_persistent": (c_int, [c_void_p, c_void_p, c_uint64, c_int, _H]),
    "uha_batch_query_buffer": (c_void_p, [c_void_p, c_uint64]),
    "uha_batch_run": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "uha_batch_stats_get": (c_int, [c_void_p, POINTER(BatchStats)]),
    "uha_batch_stage_times": (c_int, [c_void_p, c_void_p, c_uint64, POINTER(c_uint64)]),
    "uha_batch_tuning": (c_int, [c_void_p, c_uint64, POINTER(TuneReport)]),
    "uha_batch_destroy": (None, [c_void_p]),
    "uha_server_create": (c_int, [c_int, POINTER(ServerConfig), _H]),
    "uha_server_add_index": (c_int, [c_void_p, c_void_p, c_int, POINTER(ctypes.c_uint32)]),
    "uha_server_reserve": (c_int, [c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                    POINTER(ctypes.c_uint32)]),
    "uha_server_submit": (c_int, [c_void_p, ctypes.c_uint32, c_void_p, c_uint64]),
    "uha_server_replay": (c_int, [c_void_p, c_uint64, c_void_p, c_void_p, c_void_p,
                                   c_void_p]),
    "uha_server_drain": (c_int, [c_void_p]),
    "uha_server_poll": (c_int, [c_void_p, c_void_p, c_uint64, _U]),
    "uha_server_stats_get": (c_int, [c_void_p, POINTER(ServerStats)]),
    "uha_server_reset_stats": (c_int, [c_void_p]),
    "uha_server_destroy": (None, [c_void_p]),
    "uha_precision_scores": (c_int, [c_void_p, c_void_p, c_void_p, c_uint64, c_int,
                                      c_void_p, c_void_p]),
    "uha_importance_probabilities": (c_int, [c_int, c_int, c_void_p, c_uint64, c_uint64,
                                              c_int, c_uint64, c_void_p,
                                              POINTER(ProbabilityReport)]),
    "uha_importance_probabilities_host": (c_int, [c_int, c_void_p, c_uint64, c_uint64,
                                                   c_int, c_void_p]),
    "uha_importance_probabilities_device": (c_int, [c_int, c_int, c_void_p, c_uint64,
                                                     c_uint64, c_int, c_uint64, c_void_p,
                                                     POINTER(ProbabilityReport)]),
    "uha_sha256": (c_int, [c_void_p, c_uint64, c_void_p]),
    "uha_sha256_file": (c_int, [c_char_p, c_void_p]),
    "uha_probabilities_save": (c_int, [c_char_p, c_int, c_uint64, c_void_p, c_void_p,
                                        c_uint64]),
    "uha_probabilities_load": (c_int, [c_char_p, POINTER(c_int), _U, c_void_p, c_void_p,
                                        c_uint64, _U]),
    "uha_npy_load_f32": (c_int, [c_char_p, c_void_p, c_uint64, _U, _U]),
    "uha_npy_load_u16": (c_int, [c_char_p, c_void_p, c_uint64, _U]),
    "uha_rng_create": (c_int, [c_uint64, _H]),
    "uha_rng_destroy": (None, [c_void_p]),
    "uha_rng_state": (c_int, [c_void_p, c_char_p, c_uint64, _U]),
    "uha_rng_set_state": (c_int, [c_void_p, c_char_p]),
    "uha_sample_coordinates": (c_int, [c_void_p, c_uint64, c_uint64, c_void_p,
                                        c_void_p, c_void_p, c_void_p, _U]),
    "uha_jl_matrix": (c_int, [c_void_p, c_void_p, c_uint64, c_uint64, c_void_p, c_void_p]),
    "uha_cauchy_matrix": (c_int, [c_void_p, c_void_p, c_uint64, c_uint64, c_void_p, c_void_p]),
    "uha_gaussian_jl_matrix": (c_int, [c_void_p, c_void_p, c_uint64, c_uint64, c_void_p,
                                       c_void_p]),
}

_lib: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    """Loads the engine library once; raises if it is absent."""
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            raise RuntimeError(
                f"CUDA engine library {LIBRARY_PATH} is missing; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'`")
        lib = ctypes.CDLL(str(LIBRARY_PATH))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib
