"""Batched GROUP BY over the C ABI (``qdb_gb_batch_*``): many independent queries in one persistent launch.

The reference issues one ``GPUGroupBy`` per query (qikkDB/GpuSqlParser/Dispatcher/
GpuSqlDispatcherAggregationFunctions.h:377-507).  ``GroupByBatch`` holds up to ``max_instances`` such queries
over device-resident columns and executes all of them with one work-queue-driven persistent kernel, optionally
replayed as a CUDA graph.  Each query's results are the same as ``GroupByTable`` / ``GPUGroupBy`` produce for it
alone (keys and integer aggregates bit-exact; float SUM/AVG accumulated in FP64).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from . import _capi as capi
from .groupby import AGG_CODES, CODE_TO_NP, _ptr, _stream, type_code

AGG_ORDER = ("min", "max", "sum", "avg", "count")  # column order of a query's results (agg bit order)


@dataclass
class Query:
    """One GROUP BY of a batch: GROUP BY keys [% key_mod] with `aggs` of vals, WHERE pred."""
    keys: torch.Tensor
    vals: Optional[torch.Tensor]
    aggs: Sequence[str]
    max_groups: int
    key_mod: int = 0
    pred: Optional[tuple] = None  # (column tensor, op, constant[, constant dtype])
    n_rows: Optional[int] = None
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> capi.qdb_gb_query:
        q = capi.qdb_gb_query()
        mask = 0
        for a in self.aggs:
            mask |= AGG_CODES[a]
        q.agg_mask = mask
        q.key_type = type_code(self.keys.dtype)
        q.val_type = type_code(self.vals.dtype) if self.vals is not None else 0
        q.keys = _ptr(self.keys)
        q.vals = _ptr(self.vals)
        q.n_rows = int(self.keys.numel() if self.n_rows is None else self.n_rows)
        q.max_groups = int(self.max_groups)
        q.key_mod = int(self.key_mod)
        if self.pred is not None:
            col, op, const = self.pred[:3]
            cdt = self.pred[3] if len(self.pred) > 3 else (np.float64 if isinstance(const, float) else np.int64)
            q.pred.col = _ptr(col)
            q.pred.type = type_code(col.dtype)
            q.pred.op = op
            ct = type_code(cdt)
            q.pred.const_type = ct
            if ct in (capi.QDB_FLOAT, capi.QDB_DOUBLE):
                q.pred.const_f = float(np.float32(const)) if ct == capi.QDB_FLOAT else float(const)
            else:
                q.pred.const_i = int(const)
        return q


def _out_dtype(agg: str, val_dtype) -> np.dtype:
    if agg == "count":
        return np.dtype(np.int64)
    return np.dtype(CODE_TO_NP[type_code(val_dtype)])


class GroupByBatch:
    """A batch of GROUP BY queries executed together (C ABI qdb_gb_batch_*)."""

    def __init__(self, max_instances: int, table_bytes: int, result_bytes: int, stream=None):
        h = C.c_void_p()
        capi.check(capi.lib().qdb_gb_batch_create(C.byref(h), int(max_instances), int(table_bytes),
                                                  int(result_bytes), _stream(stream)))
        self.handle = h
        self.queries: list[Query] = []
        self.counts = np.zeros(0, np.int64)
        self.status = np.zeros(0, np.int32)

    def __del__(self):
        try:
            if getattr(self, "handle", None) and self.handle.value:
                capi.lib().qdb_gb_batch_destroy(self.handle)
                self.handle = C.c_void_p()
        except Exception:
            pass

    def set(self, queries: Sequence[Query], stream=None) -> None:
        arr = (capi.qdb_gb_query * max(len(queries), 1))(*[q.to_c() for q in queries])
        capi.check(capi.lib().qdb_gb_batch_set(self.handle, arr, len(queries), _stream(stream)))
        self.queries = list(queries)

    def run(self, graph: bool = False, stream=None) -> None:
        capi.check(capi.lib().qdb_gb_batch_run(self.handle, 1 if graph else 0, _stream(stream)))

    def fetch(self, stream=None):
        n = len(self.queries)
        self.counts = np.zeros(max(n, 1), np.int64)
        self.status = np.zeros(max(n, 1), np.int32)
        capi.check(capi.lib().qdb_gb_batch_fetch(self.handle, self.counts.ctypes.data_as(capi.PI64),
                                                 self.status.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 _stream(stream)))
        self.counts = self.counts[:n]
        self.status = self.status[:n]
        return self.counts, self.status

    def _decode(self, i: int, keys_w: np.ndarray, cols_w: list) -> dict:
        q = self.queries[i]
        out = {"n_groups": int(keys_w.size), "keys": [keys_w.astype(CODE_TO_NP[type_code(q.keys.dtype)])]}
        names = [a for a in AGG_ORDER if a in q.aggs]
        for a, w in zip(names, cols_w):
            dt = _out_dtype(a, q.vals.dtype if q.vals is not None else torch.int64)
            out[a] = w.view(np.float64).astype(dt) if dt.kind == "f" else w.astype(dt)
        return out

    def result(self, i: int, stream=None) -> dict:
        """Query i's results of the last run (call fetch() first): {'n_groups', 'keys': [arr], agg: arr}."""
        kp = C.c_void_p()
        cp = C.c_void_p()
        nc = C.c_int32()
        stride = C.c_int64()
        capi.check(capi.lib().qdb_gb_batch_result(self.handle, i, C.byref(kp), C.byref(cp), C.byref(nc),
                                                  C.byref(stride)))
        n = int(self.counts[i])
        keys_w = np.empty(n, np.int64)
        capi.check(capi.lib().qdb_memcpy_d2h(keys_w.ctypes.data, kp.value, n * 8, _stream(stream)))
        cols = []
        for j in range(nc.value):
            w = np.empty(n, np.int64)
            capi.check(capi.lib().qdb_memcpy_d2h(w.ctypes.data, cp.value + j * stride.value * 8, n * 8,
                                                 _stream(stream)))
            cols.append(w)
        return self._decode(i, keys_w, cols)

    def results_all(self, stream=None) -> list:
        """Every query's results with one device-to-host copy of the result region."""
        n = len(self.queries)
        if n == 0:
            return []
        need = C.c_int64()
        capi.check(capi.lib().qdb_gb_batch_copy_results(self.handle, 0, n, None, 0, C.byref(need), _stream(stream)))
        buf = np.empty(need.value // 8, np.int64)
        capi.check(capi.lib().qdb_gb_batch_copy_results(self.handle, 0, n, buf.ctypes.data, need.value,
                                                        C.byref(need), _stream(stream)))
        out, off = [], 0
        for i, q in enumerate(self.queries):
            rows = int(q.max_groups) + 2
            ncol = sum(1 for a in AGG_ORDER if a in q.aggs)
            c = int(self.counts[i])
            keys_w = buf[off:off + c]
            cols = [buf[off + (j + 1) * rows: off + (j + 1) * rows + c] for j in range(ncol)]
            out.append(self._decode(i, keys_w, cols))
            off += rows * (1 + ncol)
        return out

    def get_cfg(self, i: int) -> dict:
        c = capi.qdb_gb_batch_cfg()
        capi.check(capi.lib().qdb_gb_batch_get_cfg(self.handle, i, C.byref(c)))
        return {f: getattr(c, f) for f, _ in capi.qdb_gb_batch_cfg._fields_ if f != "reserved"}

    def set_cfg(self, i: int, **kw) -> None:
        cur = self.get_cfg(i)
        cur.update(kw)
        c = capi.qdb_gb_batch_cfg()
        for k, v in cur.items():
            setattr(c, k, int(v))
        capi.check(capi.lib().qdb_gb_batch_set_cfg(self.handle, i, C.byref(c)))

    def set_sharing(self, share: bool) -> None:
        capi.check(capi.lib().qdb_gb_batch_set_sharing(self.handle, 1 if share else 0))

    def autotune(self, stream=None) -> None:
        capi.check(capi.lib().qdb_gb_batch_autotune(self.handle, _stream(stream)))

    def item_times(self, stream=None) -> np.ndarray:
        ns = np.zeros(max(len(self.queries), 1), np.int64)
        capi.check(capi.lib().qdb_gb_batch_item_times(self.handle, ns.ctypes.data_as(capi.PI64), _stream(stream)))
        return ns[:len(self.queries)]


def required_bytes(queries: Sequence[Query]) -> tuple:
    """(table bytes, result bytes) that a batch of these queries needs (qdb_gb_batch_required)."""
    arr = (capi.qdb_gb_query * max(len(queries), 1))(*[q.to_c() for q in queries])
    t, r = C.c_int64(), C.c_int64()
    capi.check(capi.lib().qdb_gb_batch_required(arr, len(queries), C.byref(t), C.byref(r)))
    return t.value, r.value


def plain_run(queries: Sequence[Query], results_to_host: bool = True, stream=None) -> np.ndarray:
    """The same queries one at a time through the plain path, looped in C (qdb_gb_plain_run): per query the
    `key % key_mod` column, a table, ProcessBlock with the fused WHERE, GetResults, optionally the results copied to
    host memory, then everything freed.  Returns every query's group count."""
    arr = (capi.qdb_gb_query * max(len(queries), 1))(*[q.to_c() for q in queries])
    groups = np.zeros(max(len(queries), 1), np.int64)
    capi.check(capi.lib().qdb_gb_plain_run(arr, len(queries), 1 if results_to_host else 0,
                                           groups.ctypes.data_as(C.POINTER(C.c_int64)), _stream(stream)))
    return groups[:len(queries)]


def tuning_reset() -> None:
    capi.check(capi.lib().qdb_gb_batch_tuning_reset())
