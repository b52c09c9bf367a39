"""ctypes binding of the C ABI declared in include/qdb_gb.h (the library the reference's FFI would bind).

Loading fails loudly when the CUDA library has not been built: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqdbgb.so")
GEN_PATH = os.path.join(HERE, "libqdbgen.so")

# status codes (include/qdb_gb.h, mirroring QueryEngineErrorType of qikkDB/QueryEngine/GPUError.h:17-28)
QDB_OK = 0
QDB_ERROR = 1
QDB_DIVISION_BY_ZERO = 2
QDB_INTEGER_OVERFLOW = 3
QDB_HASH_TABLE_FULL = 4
QDB_UNKNOWN_AGG_FUN = 5
QDB_NOT_FOUND = 6
QDB_ERR_INVALID = 100
QDB_ERR_NOMEM = 101
QDB_ERR_CUDA = 102
QDB_ERR_TIMEOUT = 103
QDB_ERR_TOO_LARGE = 104

# element types (qikkDB/DataType.h COLUMN_* codes)
QDB_INT32, QDB_INT64, QDB_FLOAT, QDB_DOUBLE, QDB_INT8 = 8, 9, 10, 11, 15

# aggregates
QDB_AGG_MIN, QDB_AGG_MAX, QDB_AGG_SUM, QDB_AGG_AVG, QDB_AGG_COUNT = 1, 2, 4, 8, 16

# filter operators (FilterConditions::*)
(QDB_GREATER, QDB_GREATER_EQUAL, QDB_LESS, QDB_LESS_EQUAL, QDB_EQUAL, QDB_NOT_EQUAL, QDB_LOGICAL_AND,
 QDB_LOGICAL_OR) = range(8)

QDB_PLACE_AUTO, QDB_PLACE_SHARED, QDB_PLACE_GLOBAL = 0, 1, 2


class qdb_pred(C.Structure):
    _fields_ = [
        ("col", C.c_void_p),
        ("type", C.c_int32),
        ("op", C.c_int32),
        ("const_type", C.c_int32),
        ("reserved", C.c_int32),
        ("const_i", C.c_int64),
        ("const_f", C.c_double),
        ("nulls", C.c_void_p),
    ]


class qdb_aafl_col(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("type", C.c_int32),
        ("reserved", C.c_int32),
        ("rows", C.c_int64),
        ("elements", C.c_int64),
        ("blocks", C.c_int64),
        ("min_bits", C.c_int64),
        ("max_bits", C.c_int64),
    ]


class qdb_gb_query(C.Structure):
    _fields_ = [
        ("agg_mask", C.c_int32),
        ("key_type", C.c_int32),
        ("val_type", C.c_int32),
        ("reserved", C.c_int32),
        ("keys", C.c_void_p),
        ("vals", C.c_void_p),
        ("n_rows", C.c_int64),
        ("max_groups", C.c_int64),
        ("key_mod", C.c_int64),
        ("pred", qdb_pred),
    ]


class qdb_gb_batch_cfg(C.Structure):
    _fields_ = [
        ("placement", C.c_int32),
        ("smem_slots", C.c_int32),
        ("replicas", C.c_int32),
        ("warps", C.c_int32),
        ("rows_per_thread", C.c_int32),
        ("reserved", C.c_int32),
        ("chunk_rows", C.c_int64),
    ]


class qdb_server_result(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("n_cols", C.c_int32),
        ("n_groups", C.c_int64),
        ("keys", C.c_void_p),
        ("cols", C.c_void_p),
        ("submit_ns", C.c_int64),
        ("start_ns", C.c_int64),
        ("done_ns", C.c_int64),
        ("retries", C.c_int32),
        ("batch_size", C.c_int32),
        ("max_groups", C.c_int64),
    ]


class qdb_server_stats(C.Structure):
    _fields_ = [(f, C.c_int64) for f in ("submitted", "completed", "batches", "retries", "rejected",
                                         "queries_in_batches", "table_budget_bytes", "hbm_free_at_create",
                                         "plain_queries")]


P = C.c_void_p
PP = C.POINTER(C.c_void_p)
I32 = C.c_int32
I64 = C.c_int64
PI64 = C.POINTER(C.c_int64)

# (name, restype, argtypes) of every entry point declared in include/qdb_gb.h
SIGNATURES = [
    ("qdb_last_error", C.c_char_p, []),
    ("qdb_version", C.c_char_p, []),
    ("qdb_launch_count", I64, []),
    ("qdb_device_count", I32, [C.POINTER(I32)]),
    ("qdb_malloc", I32, [PP, I64, P]),
    ("qdb_free", I32, [P, P]),
    ("qdb_memcpy_h2d", I32, [P, P, I64, P]),
    ("qdb_memcpy_d2h", I32, [P, P, I64, P]),
    ("qdb_memcpy_d2d", I32, [P, P, I64, P]),
    ("qdb_memset", I32, [P, I32, I64, P]),
    ("qdb_stream_sync", I32, [P]),
    ("qdb_set_device", I32, [I32]),
    ("qdb_get_device", I32, [C.POINTER(I32)]),
    ("qdb_memcpy_peer", I32, [P, I32, P, I32, I64]),
    ("qdb_gb_create", I32, [PP, I32, I32, I32, I32, I64, I32, P]),
    ("qdb_gb_destroy", I32, [P]),
    ("qdb_gb_max_hash_count", I32, [P, PI64]),
    ("qdb_gb_group_count", I32, [P, PI64, P]),
    ("qdb_gb_process", I32, [P, PP, PP, P, P, I64, C.POINTER(qdb_pred), P, P]),
    ("qdb_gb_process_host", I32, [P, PP, PP, P, P, I64, C.POINTER(qdb_pred), P, I64, P]),
    ("qdb_gb_check", I32, [P, P]),
    ("qdb_gb_process_sync", I32, [P, PP, PP, P, P, I64, C.POINTER(qdb_pred), P, P]),
    ("qdb_gb_results", I32, [P, I32, PP, PP, PP, PP, PI64, P]),
    ("qdb_gb_results_multi", I32, [P, I32, C.POINTER(I32), PP, PP, PP, PP, PI64, P]),
    ("qdb_gb_reset", I32, [P, P]),
    ("qdb_gb_state_words", I32, [P, C.POINTER(I32)]),
    ("qdb_gb_export_partitioned", I32, [P, I32, PP, PP, PP, PI64, P]),
    ("qdb_gb_merge_partial", I32, [P, P, P, P, I64, P]),
    ("qdb_filter", I32, [I32, I32, I32, P, I32, I32, P, P, P, I64, P]),
    ("qdb_arith_mod", I32, [I32, P, I64, P, I64, P]),
    ("qdb_reconstruct_keep", I32, [I32, P, P, I64, PP, PI64, P, PP, P]),
    ("qdb_reconstruct_keep_noalloc", I32, [I32, P, P, I64, P, I64, PI64, P, P, P]),
    ("qdb_generate_indexes", I32, [P, I64, PP, PI64, P]),
    ("qdb_prefix_sum", I32, [P, I64, P, P]),
    ("qdb_compress_null_mask", I32, [P, I64, PP, P]),
    ("qdb_gb_batch_create", I32, [PP, I32, I64, I64, P]),
    ("qdb_gb_batch_destroy", I32, [P]),
    ("qdb_gb_batch_set", I32, [P, C.POINTER(qdb_gb_query), I32, P]),
    ("qdb_gb_batch_run", I32, [P, I32, P]),
    ("qdb_gb_batch_fetch", I32, [P, PI64, C.POINTER(I32), P]),
    ("qdb_gb_batch_result", I32, [P, I32, PP, PP, C.POINTER(I32), PI64]),
    ("qdb_gb_batch_copy_results", I32, [P, I32, I32, P, I64, PI64, P]),
    ("qdb_gb_batch_get_cfg", I32, [P, I32, C.POINTER(qdb_gb_batch_cfg)]),
    ("qdb_gb_batch_set_cfg", I32, [P, I32, C.POINTER(qdb_gb_batch_cfg)]),
    ("qdb_gb_batch_autotune", I32, [P, P]),
    ("qdb_gb_batch_item_times", I32, [P, PI64, P]),
    ("qdb_gb_batch_required", I32, [C.POINTER(qdb_gb_query), I32, PI64, PI64]),
    ("qdb_gb_batch_set_sharing", I32, [P, I32]),
    ("qdb_gb_batch_tuning_reset", I32, []),
    ("qdb_gb_plain_run", I32, [C.POINTER(qdb_gb_query), I32, I32, PI64, P]),
    ("qdb_order_by_column", I32, [I32, P, P, I32, I64, I32, P, P]),
    ("qdb_order_by", I32, [I32, P, P, P, P, I64, P, P]),
    ("qdb_reorder", I32, [I32, P, P, I64, I64, P, P]),
    ("qdb_reorder_nulls", I32, [P, P, I64, I64, P, P]),
    ("qdb_scalar_create", I32, [PP, I32, P]),
    ("qdb_scalar_destroy", I32, [P]),
    ("qdb_scalar_reset", I32, [P, P]),
    ("qdb_scalar_process", I32, [P, P, P, I64, C.POINTER(qdb_pred), P, P]),
    ("qdb_scalar_result", I32, [P, I32, P, C.POINTER(I32), P]),
    ("qdb_gbs_create", I32, [PP, I32, I32, I64, I64, P]),
    ("qdb_gbs_destroy", I32, [P]),
    ("qdb_gbs_reset", I32, [P, P]),
    ("qdb_gbs_process", I32, [P, P, P, P, P, P, P, I64, P]),
    ("qdb_gbs_check", I32, [P, P]),
    ("qdb_gbs_results", I32, [P, I32, P, PP, PP, PP, PP, PP, C.POINTER(I64), P]),
    ("qdb_gbs_export", I32, [P, PP, PP, PP, PP, C.POINTER(I64), P]),
    ("qdb_gbs_merge_exported", I32, [P, P, P, P, P, I64, P]),
    ("qdb_gbs_state_words", I32, [P, C.POINTER(I32)]),
    ("qdb_aafl_decompress", I32, [C.POINTER(qdb_aafl_col), P, P]),
    ("qdb_aafl_compress", I32, [I32, P, I64, I64, I64, PP, C.POINTER(I64), P]),
    ("qdb_gb_process_aafl", I32, [P, C.POINTER(qdb_aafl_col), P, C.POINTER(qdb_pred), P]),
    ("qdb_gb_process_mod", I32, [P, P, I64, P, C.POINTER(qdb_pred), I64, P]),
    ("qdb_pred_block_may_pass", I32, [C.POINTER(qdb_pred), P, P, C.POINTER(I32)]),
    ("qdb_server_create", I32, [PP, I32, I32, I64, I64]),
    ("qdb_server_destroy", I32, [P]),
    ("qdb_server_submit", I32, [P, C.POINTER(qdb_gb_query), C.POINTER(C.c_uint64)]),
    ("qdb_server_wait", I32, [P, C.c_uint64, I64, C.POINTER(qdb_server_result)]),
    ("qdb_server_release", I32, [P, C.c_uint64]),
    ("qdb_server_stats_get", I32, [P, C.POINTER(qdb_server_stats)]),
    ("qdb_server_set_plain_route", I32, [P, I64, I64]),
    ("qdb_server_run_open_loop", I32, [P, C.POINTER(qdb_gb_query), I32, PI64, PI64, C.POINTER(I32), PI64]),
]

_lib = None
_gen = None


class QdbError(RuntimeError):
    """A non-zero status of the C ABI; `code` is the status (QueryEngineErrorType values 0..8)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"qdb status {code}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    """The CUDA library.  Raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m qikkdb_b200.build` "
                              "(the GROUP BY path has no CPU fallback)")
        handle = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(handle, name)
            f.restype = res
            f.argtypes = args
        _lib = handle
    return _lib


def gen() -> C.CDLL:
    global _gen
    if _gen is None:
        if not os.path.exists(GEN_PATH):
            raise ImportError(f"{GEN_PATH} is missing: build it with `python -m qikkdb_b200.build`")
        g = C.CDLL(GEN_PATH)
        U64 = C.c_uint64
        g.qdbgen_uniform_i32.argtypes = [U64, U64, I64, I32, I32, P, I32]
        g.qdbgen_uniform_i64.argtypes = [U64, U64, I64, I64, I64, P, I32]
        g.qdbgen_uniform_f32.argtypes = [U64, U64, I64, C.c_float, C.c_float, P, I32]
        g.qdbgen_lognormal_f32.argtypes = [U64, U64, I64, C.c_double, C.c_double, P, I32]
        g.qdbgen_zipf_i64.argtypes = [U64, U64, I64, I64, C.c_double, I32, P, I32]
        g.qdbgen_loguniform_i64.argtypes = [U64, U64, I64, I64, I64, P, I32]
        g.qdbgen_rank_key.argtypes = [I64]
        g.qdbgen_rank_key.restype = I64
        for name in ("qdbgen_uniform_i32", "qdbgen_uniform_i64", "qdbgen_uniform_f32", "qdbgen_lognormal_f32",
                     "qdbgen_zipf_i64", "qdbgen_loguniform_i64", "qdbgen_version"):
            getattr(g, name).restype = I32
        _gen = g
    return _gen


def check(rc: int) -> None:
    if rc != QDB_OK:
        raise QdbError(rc, lib().qdb_last_error().decode(errors="replace"))


def exported_symbols() -> list[str]:
    return [name for name, _, _ in SIGNATURES]
