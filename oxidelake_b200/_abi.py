"""ctypes binding of liboxb200.so (include/oxb200.h).

Loads the in-tree, ahead-of-time built library.  There is no fallback: if
the library is missing, importing the GPU path raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from .errors import error_for

LIB_PATH = Path(os.environ.get("OXB200_LIB", Path(__file__).resolve().parent / "lib" / "liboxb200.so"))

OXB_MAX_AGGREGATES = 16
OXB_MAX_PREDICATE_LEAVES = 64
OXB_NOALLOC_MAX_ROWS = 1 << 24

TYPE_INT64, TYPE_FLOAT64, TYPE_INT32, TYPE_FLOAT32, TYPE_VECTOR_F32 = 1, 2, 3, 4, 5


class Column(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("dim", C.c_int32),
        ("length", C.c_int64),
        ("values", C.c_void_p),
        ("validity", C.c_void_p),
    ]


class _Lit(C.Union):
    _fields_ = [("i", C.c_int64), ("f", C.c_double)]


class Leaf(C.Structure):
    _fields_ = [
        ("column", C.c_int32),
        ("op", C.c_int32),
        ("lit_type", C.c_int32),
        ("reserved", C.c_int32),
        ("lit", _Lit),
    ]


class MemoryInfo(C.Structure):
    _fields_ = [
        ("total_bytes", C.c_uint64),
        ("free_bytes", C.c_uint64),
        ("pinned_supported", C.c_int32),
        ("reserved", C.c_int32),
    ]


class FilterProjectArgs(C.Structure):
    _fields_ = [
        ("input", C.c_void_p),
        ("leaves", C.POINTER(Leaf)),
        ("nleaves", C.c_int32),
        ("projection", C.POINTER(C.c_int32)),
        ("nprojection", C.c_int32),
    ]


class JoinIndex(C.Structure):
    _fields_ = [
        ("keys", C.POINTER(C.c_int64)),
        ("starts", C.POINTER(C.c_uint32)),
        ("counts", C.POINTER(C.c_uint32)),
        ("ndistinct", C.c_int64),
        ("rows", C.POINTER(C.c_uint32)),
        ("nrows", C.c_int64),
    ]


class JoinBuildArgs(C.Structure):
    _fields_ = [
        ("build", C.c_void_p),
        ("key", C.c_int32),
        ("reserved", C.c_int32),
        ("index", C.POINTER(JoinIndex)),
    ]


class JoinProbeArgs(C.Structure):
    _fields_ = [
        ("probe", C.c_void_p),
        ("key", C.c_int32),
        ("reserved", C.c_int32),
        ("table", C.c_void_p),
    ]


class HashJoinArgs(C.Structure):
    _fields_ = [
        ("left", C.c_void_p),
        ("right", C.c_void_p),
        ("table", C.c_void_p),
        ("matches", C.c_void_p),
        ("first", C.c_uint64),
        ("rows", C.c_uint64),
        ("projection", C.POINTER(C.c_int32)),
        ("nprojection", C.c_int32),
        ("reserved", C.c_int32),
    ]


class AggregateSpecC(C.Structure):
    _fields_ = [
        ("group_by", C.c_int32),
        ("naggregates", C.c_int32),
        ("funcs", C.c_int32 * OXB_MAX_AGGREGATES),
        ("columns", C.c_int32 * OXB_MAX_AGGREGATES),
    ]


class AggregateArgs(C.Structure):
    _fields_ = [
        ("input", C.c_void_p),
        ("spec", C.POINTER(AggregateSpecC)),
        ("leaves", C.POINTER(Leaf)),
        ("nleaves", C.c_int32),
        ("reserved", C.c_int32),
    ]


class AggregateBatchesArgs(C.Structure):
    _fields_ = [
        ("inputs", C.c_void_p),
        ("ninputs", C.c_int32),
        ("reserved", C.c_int32),
        ("spec", C.c_void_p),
        ("leaves", C.c_void_p),
        ("nleaves", C.c_int32),
        ("reserved2", C.c_int32),
    ]


class ServerConfig(C.Structure):
    _fields_ = [("memory_budget", C.c_uint64), ("workers", C.c_int32), ("max_batch", C.c_int32)]


class TopkRequest(C.Structure):
    _fields_ = [
        ("index", C.c_void_p),
        ("input", C.c_void_p),
        ("leaves", C.c_void_p),
        ("nleaves", C.c_int32),
        ("qleaf", C.c_int32),
        ("query", C.c_void_p),
        ("dim", C.c_int32),
        ("k", C.c_int32),
        ("metric", C.c_int32),
        ("reserved", C.c_int32),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("completed", C.c_int64),
        ("rejected", C.c_int64),
        ("dispatches", C.c_int64),
        ("batched_queries", C.c_int64),
        ("peak_bytes", C.c_int64),
        ("p50_us", C.c_double),
        ("p99_us", C.c_double),
        ("qps", C.c_double),
    ]


class VectorTopkArgs(C.Structure):
    _fields_ = [
        ("index", C.c_void_p),
        ("input", C.c_void_p),
        ("leaves", C.c_void_p),
        ("nleaves", C.c_int32),
        ("nqueries", C.c_int32),
        ("queries", C.c_void_p),
        ("dim", C.c_int32),
        ("k", C.c_int32),
        ("metric", C.c_int32),
        ("overfetch", C.c_int32),
        ("exact", C.c_int32),
        ("qleaf_column", C.c_int32),
        ("qleaf_op", C.c_int32),
        ("qleaf_type", C.c_int32),
        ("reserved", C.c_int32),
        ("qleaf_lits", C.c_void_p),
    ]


class VectorTopkStats(C.Structure):
    _fields_ = [
        ("reranked", C.c_int64),
        ("exact_queries", C.c_int64),
        ("max_score_error", C.c_double),
        ("mean_score_error", C.c_double),
    ]


class VectorDistanceArgs(C.Structure):
    _fields_ = [
        ("input", C.c_void_p),
        ("column", C.c_int32),
        ("metric", C.c_int32),
        ("query", C.POINTER(C.c_float)),
        ("dim", C.c_int32),
        ("reserved", C.c_int32),
    ]


class JoinAggregateArgs(C.Structure):
    _fields_ = [
        ("probe", C.c_void_p),
        ("probe_key", C.c_int32),
        ("reserved", C.c_int32),
        ("table", C.c_void_p),
        ("build", C.c_void_p),
        ("leaves", C.POINTER(Leaf)),
        ("nleaves", C.c_int32),
        ("group_side", C.c_int32),
        ("group_column", C.c_int32),
        ("naggregates", C.c_int32),
        ("funcs", C.c_int32 * OXB_MAX_AGGREGATES),
        ("sides", C.c_int32 * OXB_MAX_AGGREGATES),
        ("columns", C.c_int32 * OXB_MAX_AGGREGATES),
    ]


OP_TRANSFER, OP_FILTER, OP_JOIN, OP_AGGREGATE, OP_VECTOR = 0, 1, 2, 3, 4


class ArrowSchema(C.Structure):
    """struct ArrowSchema of the Arrow C data interface."""


ArrowSchema._fields_ = [
    ("format", C.c_char_p), ("name", C.c_char_p), ("metadata", C.c_char_p), ("flags", C.c_int64),
    ("n_children", C.c_int64), ("children", C.POINTER(C.POINTER(ArrowSchema))),
    ("dictionary", C.POINTER(ArrowSchema)), ("release", C.CFUNCTYPE(None, C.POINTER(ArrowSchema))),
    ("private_data", C.c_void_p),
]


class ArrowArray(C.Structure):
    """struct ArrowArray of the Arrow C data interface."""


ArrowArray._fields_ = [
    ("length", C.c_int64), ("null_count", C.c_int64), ("offset", C.c_int64), ("n_buffers", C.c_int64),
    ("n_children", C.c_int64), ("buffers", C.POINTER(C.c_void_p)), ("children", C.POINTER(C.POINTER(ArrowArray))),
    ("dictionary", C.POINTER(ArrowArray)), ("release", C.CFUNCTYPE(None, C.POINTER(ArrowArray))),
    ("private_data", C.c_void_p),
]


class CallStats(C.Structure):
    _fields_ = [
        ("op", C.c_int32),
        ("status", C.c_int32),
        ("batches", C.c_uint64),
        ("rows_in", C.c_uint64),
        ("rows_out", C.c_uint64),
        ("elapsed_ns", C.c_uint64),
        ("device_ns", C.c_uint64),
        ("bytes_h2d", C.c_uint64),
        ("bytes_d2h", C.c_uint64),
    ]


class OperatorStats(C.Structure):
    _fields_ = [
        ("calls", C.c_uint64),
        ("batches", C.c_uint64),
        ("rows_in", C.c_uint64),
        ("rows_out", C.c_uint64),
        ("elapsed_ns", C.c_uint64),
        ("device_ns", C.c_uint64),
        ("bytes_h2d", C.c_uint64),
        ("bytes_d2h", C.c_uint64),
        ("unsupported", C.c_uint64),
        ("failed", C.c_uint64),
        ("fallback_batches", C.c_uint64),
    ]


_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_S = C.c_int  # oxb_status

# name -> (restype, argtypes)
PROTOTYPES = {
    "oxb_last_error": (C.c_char_p, []),
    "oxb_abi_version": (C.c_int32, []),
    "oxb_backend_create": (_S, [C.c_int32, _PP]),
    "oxb_backend_destroy": (None, [_P]),
    "oxb_backend_kind": (C.c_char_p, [_P]),
    "oxb_backend_device_id": (C.c_int32, [_P]),
    "oxb_memory_info_get": (_S, [_P, C.POINTER(MemoryInfo)]),
    "oxb_alloc_device": (_S, [_P, C.c_size_t, _PP]),
    "oxb_buffer_device_ptr": (C.c_void_p, [_P]),
    "oxb_buffer_len": (C.c_size_t, [_P]),
    "oxb_buffer_free": (None, [_P]),
    "oxb_alloc_pinned_host": (_S, [_P, C.c_size_t, _PP]),
    "oxb_host_buffer_ptr": (C.c_void_p, [_P]),
    "oxb_host_buffer_len": (C.c_size_t, [_P]),
    "oxb_host_buffer_is_pinned": (C.c_int32, [_P]),
    "oxb_host_buffer_free": (None, [_P]),
    "oxb_stream_create": (_S, [_P, _PP]),
    "oxb_stream_wrap": (_S, [_P, C.c_void_p, _PP]),
    "oxb_stream_cuda_handle": (C.c_void_p, [_P]),
    "oxb_stream_synchronize": (_S, [_P, _P]),
    "oxb_stream_destroy": (None, [_P]),
    "oxb_copy_h2d": (_S, [_P, _P, _P, _P]),
    "oxb_copy_d2h": (_S, [_P, _P, _P, _P]),
    "oxb_upload": (_S, [_P, _P, C.POINTER(Column), C.c_int32, C.c_int64, _PP]),
    "oxb_batch_from_device": (_S, [_P, C.POINTER(Column), C.c_int32, C.c_int64, _PP]),
    "oxb_batch_num_rows": (C.c_int64, [_P]),
    "oxb_batch_num_columns": (C.c_int32, [_P]),
    "oxb_batch_column": (_S, [_P, C.c_int32, C.POINTER(Column)]),
    "oxb_download_column": (_S, [_P, _P, _P, C.c_int32, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)]),
    "oxb_download": (_S, [_P, _P, _P, C.c_int32, _PP, _PP, C.POINTER(C.c_int32)]),
    "oxb_import_arrow": (_S, [_P, _P, C.POINTER(ArrowArray), C.POINTER(ArrowSchema), _PP]),
    "oxb_export_arrow": (_S, [_P, _P, _P, C.POINTER(C.c_char_p), C.POINTER(ArrowArray), C.POINTER(ArrowSchema)]),
    "oxb_batch_free": (None, [_P]),
    "oxb_filter_project": (_S, [_P, _P, C.POINTER(FilterProjectArgs), _PP]),
    "oxb_filter_project_noalloc": (
        _S,
        [_P, _P, C.POINTER(FilterProjectArgs), _PP, _PP, C.c_int64, C.POINTER(C.c_int64)],
    ),
    "oxb_prepare_join_build": (_S, [_P, _P, C.POINTER(JoinBuildArgs), _PP]),
    "oxb_join_table_distinct_keys": (C.c_int64, [_P]),
    "oxb_join_table_rows": (C.c_int64, [_P]),
    "oxb_join_table_free": (None, [_P]),
    "oxb_probe_join": (_S, [_P, _P, C.POINTER(JoinProbeArgs), _PP]),
    "oxb_join_matches_len": (C.c_uint64, [_P]),
    "oxb_join_matches_probe_rows": (C.c_int64, [_P]),
    "oxb_join_matches_free": (None, [_P]),
    "oxb_hash_join": (_S, [_P, _P, C.POINTER(HashJoinArgs), _PP]),
    "oxb_aggregate": (_S, [_P, _P, C.POINTER(AggregateArgs), _PP]),
    "oxb_join_aggregate": (_S, [_P, _P, C.POINTER(JoinAggregateArgs), _PP]),
    "oxb_join_aggregate_many": (_S, [_P, _P, C.POINTER(JoinAggregateArgs), C.c_int32, _PP]),
    "oxb_vector_distance": (_S, [_P, _P, C.POINTER(VectorDistanceArgs), _PP]),
    "oxb_aggregate_batches": (_S, [_P, _P, C.POINTER(AggregateBatchesArgs), _PP]),
    "oxb_server_create": (_S, [_P, C.POINTER(ServerConfig), _PP]),
    "oxb_server_destroy": (None, [_P]),
    "oxb_server_submit_topk": (_S, [_P, C.POINTER(TopkRequest), C.POINTER(C.c_uint64)]),
    "oxb_server_submit_join_aggregate": (_S, [_P, C.POINTER(JoinAggregateArgs), C.POINTER(C.c_uint64)]),
    "oxb_server_wait_topk": (_S, [_P, C.c_uint64, _P, _P, C.POINTER(C.c_double)]),
    "oxb_server_wait_batch": (_S, [_P, C.c_uint64, _PP, C.POINTER(C.c_double)]),
    "oxb_server_stats_get": (_S, [_P, C.POINTER(ServerStats), C.c_int32]),
    "oxb_vector_index_build": (_S, [_P, _P, _P, C.c_int32, _PP]),
    "oxb_vector_index_free": (None, [_P]),
    "oxb_vector_topk": (_S, [_P, _P, C.POINTER(VectorTopkArgs), _P, _P, C.POINTER(VectorTopkStats)]),
    "oxb_set_kernel_timing": (_S, [_P, C.c_int32]),
    "oxb_last_kernel_time": (_S, [_P, C.c_char_p, C.c_int32, C.POINTER(C.c_float)]),
    "oxb_kernel_launches": (C.c_uint64, []),
    "oxb_set_autotune": (_S, [_P, C.c_int32]),
    "oxb_set_upload_staging": (_S, [_P, C.c_int32]),
    "oxb_set_agg_variant": (_S, [_P, C.c_int32, C.c_int32]),
    "oxb_last_call_stats": (_S, [C.POINTER(CallStats)]),
    "oxb_operator_stats_get": (_S, [_P, C.c_int32, C.POINTER(OperatorStats), C.c_int32]),
    "oxb_supports_predicate": (C.c_int32, [_P, C.POINTER(Leaf), C.c_int32]),
    "oxb_supports_hash_join": (C.c_int32, [_P]),
    "oxb_supports_aggregate": (C.c_int32, [_P]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded library with every prototype bound.  Raises if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"liboxb200.so not built at {LIB_PATH}: run `python -m oxidelake_b200.build` "
                "(the GPU operator path has no CPU fallback)"
            )
        l = C.CDLL(str(LIB_PATH))
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(status: int) -> None:
    if status != 0:
        msg = lib().oxb_last_error().decode("utf-8", "replace")
        raise error_for(status, msg)
