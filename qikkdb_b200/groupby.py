"""Python mirror of the reference's GROUP BY operator surface over the C ABI.

Names, argument meaning and error behaviour follow qikkDB's C++ operators so that tests read like the
reference's own (qikkDB_test/GPUGroupByTests.cu, GPUFilterTests.cu, GPUReconstructTests.cu):

* ``GPUGroupBy(agg, O, K, V, maxHashCount, keySizeMultiplier)`` with ``ProcessBlock`` / ``GetResults`` /
  ``GetMaxHashCount`` (qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:285-587), including the multi-key form
  ``GPUGroupBy(agg, O, [COLUMN_INT, COLUMN_INT], V, ...)`` (GPUGroupByMultiKey.cuh:330-912);
* ``GPUBinary.Binary(op, outMask, A, B, n, nullBitMask)`` for filters (GPUBinary.cuh:555-579);
* ``GPUReconstruct.reconstructColKeep / GenerateIndexesKeep / PrefixSum / CompressNullMask``
  (GPUReconstruct.cuh:272-640).

Device columns are torch CUDA tensors; results come back as ``DeviceBuffer`` objects owned by the caller
(freed with qdb_free when garbage-collected, like GPUMemory::free).  A non-zero status raises
``QueryEngineError`` carrying the QueryEngineErrorType code (GPU_HASH_TABLE_FULL = 4 ...).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np
import torch

from . import _capi as capi
from ._capi import QdbError as QueryEngineError  # noqa: F401  (reference name: query_engine_error)

GPU_EXTENSION_SUCCESS = 0
GPU_EXTENSION_ERROR = 1
GPU_DIVISION_BY_ZERO_ERROR = 2
GPU_INTEGER_OVERFLOW_ERROR = 3
GPU_HASH_TABLE_FULL = 4
GPU_UNKNOWN_AGG_FUN = 5

# DataType codes of key / value columns (qikkDB/DataType.h:7-27)
COLUMN_INT, COLUMN_LONG, COLUMN_FLOAT, COLUMN_DOUBLE, COLUMN_INT8_T = 8, 9, 10, 11, 15

TORCH_TO_CODE = {torch.int32: capi.QDB_INT32, torch.int64: capi.QDB_INT64, torch.float32: capi.QDB_FLOAT,
                 torch.float64: capi.QDB_DOUBLE, torch.int8: capi.QDB_INT8}
NP_TO_CODE = {np.dtype(np.int32): capi.QDB_INT32, np.dtype(np.int64): capi.QDB_INT64,
              np.dtype(np.float32): capi.QDB_FLOAT, np.dtype(np.float64): capi.QDB_DOUBLE,
              np.dtype(np.int8): capi.QDB_INT8}
CODE_TO_NP = {capi.QDB_INT32: np.int32, capi.QDB_INT64: np.int64, capi.QDB_FLOAT: np.float32,
              capi.QDB_DOUBLE: np.float64, capi.QDB_INT8: np.int8}
CODE_TO_TORCH = {v: k for k, v in TORCH_TO_CODE.items()}


class AggregationFunctions:
    """Aggregate tags (AggregationFunctions::{min,max,sum,avg,count,none})."""
    min = "min"
    max = "max"
    sum = "sum"
    avg = "avg"
    count = "count"
    none = "none"


AGG_CODES = {"min": capi.QDB_AGG_MIN, "max": capi.QDB_AGG_MAX, "sum": capi.QDB_AGG_SUM, "avg": capi.QDB_AGG_AVG,
             "count": capi.QDB_AGG_COUNT, "none": 0}


class FilterConditions:
    """Filter operators (FilterConditions::*, GPUFilterConditions.cuh:9-180)."""
    greater = capi.QDB_GREATER
    greaterEqual = capi.QDB_GREATER_EQUAL
    less = capi.QDB_LESS
    lessEqual = capi.QDB_LESS_EQUAL
    equal = capi.QDB_EQUAL
    notEqual = capi.QDB_NOT_EQUAL
    logicalAnd = capi.QDB_LOGICAL_AND
    logicalOr = capi.QDB_LOGICAL_OR


def type_code(dtype) -> int:
    if isinstance(dtype, torch.dtype):
        return TORCH_TO_CODE[dtype]
    if isinstance(dtype, int):
        return dtype
    return NP_TO_CODE[np.dtype(dtype)]


def _stream(stream=None) -> int:
    if stream is not None:
        return int(stream)
    return torch.cuda.current_stream().cuda_stream


def _ptr(t) -> Optional[int]:
    if t is None:
        return None
    if isinstance(t, DeviceBuffer):
        return t.ptr
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise ValueError("device columns must be CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("device columns must be contiguous")
    return t.data_ptr()


class DeviceBuffer:
    """A device allocation returned by the library (freed with qdb_free unless `owned` is False)."""

    def __init__(self, ptr: Optional[int], count: int, dtype, owned: bool = True):
        self.ptr = int(ptr) if ptr else 0
        self.count = int(count)
        self.dtype = np.dtype(dtype)
        self.owned = owned and bool(self.ptr)

    @property
    def nbytes(self) -> int:
        return self.count * self.dtype.itemsize

    def numpy(self, stream=None) -> np.ndarray:
        out = np.empty(self.count, dtype=self.dtype)
        if self.count and self.ptr:
            capi.check(capi.lib().qdb_memcpy_d2h(out.ctypes.data, self.ptr, self.nbytes, _stream(stream)))
        return out

    def torch(self, stream=None) -> torch.Tensor:
        tdt = {np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64, np.dtype(np.float32): torch.float32,
               np.dtype(np.float64): torch.float64, np.dtype(np.int8): torch.int8,
               np.dtype(np.uint64): torch.int64, np.dtype(np.uint8): torch.uint8}[self.dtype]
        t = torch.empty(self.count, dtype=tdt, device="cuda")
        if self.count and self.ptr:
            capi.check(capi.lib().qdb_memcpy_d2d(t.data_ptr(), self.ptr, self.nbytes, _stream(stream)))
        return t

    def free(self, stream=None) -> None:
        if self.owned and self.ptr:
            capi.lib().qdb_free(self.ptr, _stream(stream) if torch.cuda.is_available() else None)
        self.ptr = 0
        self.owned = False

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def nullmask_words(n: int) -> int:
    """NullValues::GetNullBitMaskSize (qikkDB/QueryEngine/GPUCore/NullValues.cu:13-16)."""
    return (n + 63) // 64


def pack_nullmask(flags) -> np.ndarray:
    """bool[n] -> bit-packed uint64 words (bit i%64 of word i/64)."""
    flags = np.asarray(flags, dtype=bool)
    words = np.zeros(nullmask_words(len(flags)), dtype=np.uint64)
    if len(flags):
        padded = np.zeros(len(words) * 64, dtype=bool)
        padded[:len(flags)] = flags
        words = np.packbits(padded, bitorder="little").view(np.uint64).copy()
    return words


def unpack_nullmask(words: np.ndarray, n: int) -> np.ndarray:
    if n == 0:
        return np.zeros(0, dtype=bool)
    w = np.ascontiguousarray(np.asarray(words).view(np.uint64))
    return np.unpackbits(w.view(np.uint8), bitorder="little")[:n].astype(bool)


def device_nullmask(flags) -> Optional[torch.Tensor]:
    if flags is None:
        return None
    return torch.from_numpy(pack_nullmask(flags).view(np.int64)).cuda()


def make_pred(col: torch.Tensor, op: int, constant, const_dtype=None, nulls: Optional[torch.Tensor] = None):
    """A fused predicate `col OP constant` for ProcessBlock / GroupByTable.process."""
    p = capi.qdb_pred()
    p.col = _ptr(col)
    p.type = type_code(col.dtype)
    p.op = op
    if const_dtype is None:
        const_dtype = np.float64 if isinstance(constant, float) else np.int64
    ct = type_code(const_dtype)
    p.const_type = ct
    if ct in (capi.QDB_FLOAT, capi.QDB_DOUBLE):
        p.const_f = float(np.float32(constant)) if ct == capi.QDB_FLOAT else float(constant)
    else:
        p.const_i = int(constant)
    p.nulls = _ptr(nulls)
    p._keep = (col, nulls)  # the struct holds raw pointers: keep the tensors alive with it
    return p


class GroupByTable:
    """A multi-aggregate GROUP BY table (one fused pass computes every aggregate in `aggs`)."""

    def __init__(self, aggs: Sequence[str], key_dtype, val_dtype, max_groups: int, n_key_cols: int = 1,
                 placement: int = capi.QDB_PLACE_AUTO, stream=None):
        self.aggs = [a for a in aggs if a != "none"]
        self.key_code = type_code(key_dtype)
        self.val_code = type_code(val_dtype) if val_dtype is not None else 0
        self.n_key_cols = n_key_cols
        mask = 0
        for a in self.aggs:
            mask |= AGG_CODES[a]
        h = C.c_void_p()
        capi.check(capi.lib().qdb_gb_create(C.byref(h), mask, self.key_code, n_key_cols, self.val_code,
                                            int(max_groups), placement, _stream(stream)))
        self.handle = h

    def __del__(self):
        try:
            if getattr(self, "handle", None) and self.handle.value:
                capi.lib().qdb_gb_destroy(self.handle)
                self.handle = C.c_void_p()
        except Exception:
            pass

    def process(self, keys, values=None, n: Optional[int] = None, key_nulls=None, value_nulls=None, pred=None,
                mask=None, stream=None, sync: bool = True) -> None:
        keys = list(keys) if isinstance(keys, (list, tuple)) else [keys]
        if n is None:
            n = keys[0].numel()
        kc = (C.c_void_p * len(keys))(*[_ptr(k) for k in keys])
        kn = None
        if key_nulls is not None:
            key_nulls = list(key_nulls) if isinstance(key_nulls, (list, tuple)) else [key_nulls]
            kn = (C.c_void_p * len(key_nulls))(*[_ptr(k) for k in key_nulls])
        fn = capi.lib().qdb_gb_process_sync if sync else capi.lib().qdb_gb_process
        capi.check(fn(self.handle, kc, kn, _ptr(values), _ptr(value_nulls), int(n),
                      C.byref(pred) if pred is not None else None, _ptr(mask), _stream(stream)))

    def process_host(self, keys, values=None, key_nulls=None, value_nulls=None, pred=None, mask=None,
                     chunk_rows: int = 1 << 24, stream=None) -> None:
        """qdb_gb_process_host: host (numpy / pinned CPU tensor) columns, streamed to the GPU in chunks.
        pred: (host column, op, constant, constant dtype[, host null words]).  Asynchronous: the host arrays must
        stay alive until `stream` has passed this call."""
        def hp(x):
            if x is None:
                return None
            if isinstance(x, torch.Tensor):
                assert not x.is_cuda and x.is_contiguous()
                return x.data_ptr()
            return np.ascontiguousarray(x).ctypes.data
        keys = list(keys) if isinstance(keys, (list, tuple)) else [keys]
        n = len(keys[0])
        kc = (C.c_void_p * len(keys))(*[hp(k) for k in keys])
        kn = None
        if key_nulls is not None:
            key_nulls = list(key_nulls) if isinstance(key_nulls, (list, tuple)) else [key_nulls]
            kn = (C.c_void_p * len(key_nulls))(*[hp(k) for k in key_nulls])
        p = None
        if pred is not None:
            col, op, const, cdt = pred[:4]
            pn = pred[4] if len(pred) > 4 else None
            p = capi.qdb_pred()
            p.col = hp(col)
            p.type = type_code(col.dtype)
            p.op = op
            ct = type_code(cdt)
            p.const_type = ct
            if ct in (capi.QDB_FLOAT, capi.QDB_DOUBLE):
                p.const_f = float(np.float32(const)) if ct == capi.QDB_FLOAT else float(const)
            else:
                p.const_i = int(const)
            p.nulls = hp(pn)
        capi.check(capi.lib().qdb_gb_process_host(self.handle, kc, kn, hp(values), hp(value_nulls), int(n),
                                                  C.byref(p) if p is not None else None, hp(mask), int(chunk_rows),
                                                  _stream(stream)))

    def check(self, stream=None) -> None:
        capi.check(capi.lib().qdb_gb_check(self.handle, _stream(stream)))

    def results(self, aggs: Optional[Sequence[str]] = None, stream=None):
        """(keys: list[DeviceBuffer], key_nulls: list[DeviceBuffer], {agg: (values, nulls)}, count)."""
        aggs = list(self.aggs if aggs is None else aggs)
        nk = self.n_key_cols
        ok = (C.c_void_p * nk)()
        okn = (C.c_void_p * nk)()
        na = len(aggs)
        codes = (C.c_int32 * max(na, 1))(*[AGG_CODES[a] for a in aggs])
        ov = (C.c_void_p * max(na, 1))()
        ovn = (C.c_void_p * max(na, 1))()
        cnt = C.c_int64()
        capi.check(capi.lib().qdb_gb_results_multi(self.handle, na, codes, ok, okn, ov if na else None,
                                                   ovn if na else None, C.byref(cnt), _stream(stream)))
        n = cnt.value
        kdt = CODE_TO_NP[capi.QDB_INT32 if nk == 2 else self.key_code]
        keys = [DeviceBuffer(ok[c], n, kdt) for c in range(nk)]
        knulls = [DeviceBuffer(okn[c], nullmask_words(n), np.uint64) for c in range(nk)]
        vals = {}
        vdt = CODE_TO_NP.get(self.val_code, np.int64)
        for i, a in enumerate(aggs):
            dt = np.int64 if a == "count" else vdt
            vals[a] = (DeviceBuffer(ov[i], n, dt), DeviceBuffer(ovn[i], nullmask_words(n), np.uint64))
        return keys, knulls, vals, n

    def results_numpy(self, aggs: Optional[Sequence[str]] = None, stream=None) -> dict:
        """Results copied to host: {'n_groups': g, 'keys': [arr...], 'key_nulls': [bool arr...], agg: arr,
        agg + '_null': bool arr}."""
        keys, knulls, vals, n = self.results(aggs, stream)
        out = {"n_groups": n, "keys": [k.numpy() for k in keys],
               "key_nulls": [unpack_nullmask(kn.numpy(), n) for kn in knulls]}
        for a, (v, vn) in vals.items():
            out[a] = v.numpy()
            out[a + "_null"] = unpack_nullmask(vn.numpy(), n)
        return out

    def group_count(self, stream=None) -> int:
        v = C.c_int64()
        capi.check(capi.lib().qdb_gb_group_count(self.handle, C.byref(v), _stream(stream)))
        return v.value

    def reset(self, stream=None) -> None:
        capi.check(capi.lib().qdb_gb_reset(self.handle, _stream(stream)))


class GPUGroupBy:
    """GPUGroupBy<AGG, O, K, V> (qikkDB/QueryEngine/GPUCore/GPUGroupBy.cuh:285-587).

    K is a key dtype, or a list of DataType codes for the multi-key form (GPUGroupByMultiKey.cuh:330)."""

    def __init__(self, agg: str, O, K, V, maxHashCount: int, keySizeMultiplier: int = 1,
                 placement: int = capi.QDB_PLACE_AUTO):
        if agg not in AGG_CODES:
            raise QueryEngineError(GPU_UNKNOWN_AGG_FUN, f"unknown aggregation {agg!r}")
        if agg == "count" and np.dtype(O) != np.dtype(np.int64):
            raise QueryEngineError(GPU_EXTENSION_ERROR, "Output value data type in GROUP BY with COUNT must be int64_t")
        if agg in ("min", "max", "sum") and np.dtype(O) != np.dtype(V):
            raise QueryEngineError(GPU_EXTENSION_ERROR, "Input and output value data type must be the same in GROUP BY")
        self.agg = agg
        self.string_keys = K is str
        if self.string_keys:
            # GPUGroupBy<AGG, O, std::string, V> (qikkDB/QueryEngine/GPUCore/GPUGroupByString.cuh:171-785)
            self.n_key_cols = 1
            self.max_groups = min(int(maxHashCount) * int(keySizeMultiplier), 1 << 30)
            self.table = StringGroupByTable([agg] if agg != "none" else [], V if agg != "none" else None,
                                            self.max_groups)
            return
        multi = isinstance(K, (list, tuple))
        if multi and (len(K) != 2 or any(k != COLUMN_INT for k in K)):
            raise QueryEngineError(GPU_EXTENSION_ERROR, "multi-key GROUP BY supports (COLUMN_INT, COLUMN_INT) keys")
        self.n_key_cols = 2 if multi else 1
        key_dtype = np.int32 if multi else K
        self.max_groups = min(int(maxHashCount) * int(keySizeMultiplier), 1 << 30)
        self.table = GroupByTable([agg] if agg != "none" else [], key_dtype, V if agg != "none" else None,
                                  self.max_groups, self.n_key_cols, placement)

    def ProcessBlock(self, inKeys, inValues, dataElementCount: int, inKeysNullMask=None, inValuesNullMask=None):
        if dataElementCount <= 0:
            return
        self.table.process(inKeys, inValues if self.agg != "none" else None, dataElementCount, inKeysNullMask,
                           inValuesNullMask if self.agg != "none" else None)

    def GetMaxHashCount(self) -> int:
        if self.string_keys:
            return self.max_groups + 1
        v = C.c_int64()
        capi.check(capi.lib().qdb_gb_max_hash_count(self.table.handle, C.byref(v)))
        return v.value

    def GetResults(self):
        """(outKeys, outValues, outDataElementCount, outKeysNullMask, outValuesNullMask); outKeys is a list of
        DeviceBuffers for the multi-key form.  outValues is None for AGG none."""
        aggs = [] if self.agg == "none" else [self.agg]
        if self.string_keys:
            keys, knull, vals, n = self.table.results(aggs)
            v, vn = vals.get(self.agg, (None, None))
            return keys, v, n, knull, vn
        keys, knulls, vals, n = self.table.results(aggs)
        if self.agg == "count" and n:
            # COUNT is never NULL: the reference allocates an all-zero mask (GPUGroupBy.cuh:571-583).
            pass
        v, vn = vals.get(self.agg, (None, None))
        if self.n_key_cols == 2:
            return keys, v, n, knulls, vn
        return keys[0], v, n, knulls[0], vn


class GPUBinary:
    """GPUBinary<FilterConditions::OP, int8_t, L, R>::Binary (qikkDB/QueryEngine/GPUCore/GPUBinary.cuh:555-579)."""

    @staticmethod
    def Binary(op: int, outMask: torch.Tensor, A, B, dataElementCount: int, nullBitMask=None, stream=None) -> None:
        def side(x):
            if isinstance(x, torch.Tensor):
                return type_code(x.dtype), 1, _ptr(x), None
            arr = np.array([x]) if not isinstance(x, np.ndarray) else x.reshape(1)
            if not isinstance(x, np.generic) and not isinstance(x, np.ndarray):
                arr = np.array([x], dtype=np.float32 if isinstance(x, float) else np.int32)
            return type_code(arr.dtype), 0, arr.ctypes.data, arr

        at, ac, ap, akeep = side(A)
        bt, bc, bp, bkeep = side(B)
        capi.check(capi.lib().qdb_filter(op, at, ac, ap, bt, bc, bp, _ptr(nullBitMask), _ptr(outMask),
                                         int(dataElementCount), _stream(stream)))
        del akeep, bkeep


class GPUReconstruct:
    """GPUReconstruct (qikkDB/QueryEngine/GPUCore/GPUReconstruct.cuh:204-640)."""

    @staticmethod
    def reconstructColKeep(inCol: torch.Tensor, inMask: Optional[torch.Tensor], dataElementCount: int,
                           nullMask=None, stream=None):
        """(outCol DeviceBuffer, outDataElementCount, outNullMask DeviceBuffer or None)."""
        out = C.c_void_p()
        cnt = C.c_int64()
        onm = C.c_void_p()
        esz = inCol.element_size()
        capi.check(capi.lib().qdb_reconstruct_keep(esz, _ptr(inCol), _ptr(inMask), int(dataElementCount),
                                                   C.byref(out), C.byref(cnt), _ptr(nullMask),
                                                   C.byref(onm) if nullMask is not None else None, _stream(stream)))
        owned = inMask is not None
        dt = {1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[esz]
        if inCol.dtype in (torch.float32, torch.float64):
            dt = np.float32 if esz == 4 else np.float64
        col = DeviceBuffer(out.value, cnt.value, dt, owned=owned)
        nm = DeviceBuffer(onm.value, nullmask_words(cnt.value), np.uint64, owned=owned) if nullMask is not None else None
        return col, cnt.value, nm

    @staticmethod
    def reconstructCol(inCol, inMask, dataElementCount: int, nullMask=None, stream=None):
        """Host-output form: (numpy array, count, null bits or None)."""
        col, n, nm = GPUReconstruct.reconstructColKeep(inCol, inMask, dataElementCount, nullMask, stream)
        return col.numpy(), n, (unpack_nullmask(nm.numpy(), n) if nm is not None else None)

    @staticmethod
    def GenerateIndexesKeep(inMask: torch.Tensor, dataElementCount: int, stream=None):
        out = C.c_void_p()
        cnt = C.c_int64()
        capi.check(capi.lib().qdb_generate_indexes(_ptr(inMask), int(dataElementCount), C.byref(out), C.byref(cnt),
                                                   _stream(stream)))
        return DeviceBuffer(out.value, cnt.value, np.int32), cnt.value

    @staticmethod
    def GenerateIndexes(inMask: torch.Tensor, dataElementCount: int, stream=None):
        buf, n = GPUReconstruct.GenerateIndexesKeep(inMask, dataElementCount, stream)
        return buf.numpy(), n

    @staticmethod
    def PrefixSum(inMask: torch.Tensor, dataElementCount: int, stream=None) -> torch.Tensor:
        out = torch.empty(dataElementCount, dtype=torch.int32, device="cuda")
        capi.check(capi.lib().qdb_prefix_sum(_ptr(inMask), int(dataElementCount), _ptr(out), _stream(stream)))
        return out

    @staticmethod
    def CompressNullMask(inArray: torch.Tensor, dataElementCount: int, stream=None) -> DeviceBuffer:
        out = C.c_void_p()
        capi.check(capi.lib().qdb_compress_null_mask(_ptr(inArray), int(dataElementCount), C.byref(out),
                                                     _stream(stream)))
        return DeviceBuffer(out.value, nullmask_words(dataElementCount), np.uint64)


class GPUOrderBy:
    """GPUOrderBy (qikkDB/QueryEngine/GPUCore/GPUOrderBy.cuh:88-195): the dispatcher calls OrderByColumn for the
    ORDER BY columns from the last to the first, then reorders every result column by the indices
    (ReOrderByIdx / ReOrderNullValuesByIdx).  NULL rows order as lowest(T); ties keep their input order."""

    ASC = 0   # OrderBy::Order::ASC
    DESC = 1  # OrderBy::Order::DESC

    def __init__(self, dataElementCount: int, stream=None):
        self.n = int(dataElementCount)
        self.indices = torch.empty(max(self.n, 1), dtype=torch.int32, device="cuda")
        self.first = True
        self.stream = stream

    def OrderByColumn(self, outIndices: Optional[torch.Tensor], inCol: torch.Tensor, nullBitMask,
                      dataElementCount: int, order: int) -> None:
        capi.check(capi.lib().qdb_order_by_column(type_code(inCol.dtype), _ptr(inCol), _ptr(nullBitMask), int(order),
                                                  int(dataElementCount), 1 if self.first else 0, _ptr(self.indices),
                                                  _stream(self.stream)))
        self.first = False
        if outIndices is not None and dataElementCount:
            outIndices[:dataElementCount].copy_(self.indices[:dataElementCount])

    @staticmethod
    def ReOrderByIdx(outCol: torch.Tensor, inIndices: torch.Tensor, inCol: torch.Tensor, dataElementCount: int,
                     offset: int = 0, stream=None) -> None:
        """outCol[i] = inCol[inIndices[offset + i]] for i < dataElementCount (OFFSET / LIMIT)."""
        capi.check(capi.lib().qdb_reorder(inCol.element_size(), _ptr(inCol), _ptr(inIndices), int(offset),
                                          int(dataElementCount), _ptr(outCol), _stream(stream)))

    @staticmethod
    def ReOrderNullValuesByIdx(outNullBitMask: torch.Tensor, indices: torch.Tensor, inNullBitMask: torch.Tensor,
                               rowCount: int, offset: int = 0, stream=None) -> None:
        capi.check(capi.lib().qdb_reorder_nulls(_ptr(inNullBitMask), _ptr(indices), int(offset), int(rowCount),
                                                _ptr(outNullBitMask), _stream(stream)))


def order_by(cols: Sequence[torch.Tensor], descending: Optional[Sequence[bool]] = None, nulls=None,
             stream=None) -> torch.Tensor:
    """Row permutation of ORDER BY cols[0], cols[1], ... (qdb_order_by): int32 device tensor."""
    n = cols[0].numel()
    out = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    k = len(cols)
    types = (C.c_int32 * k)(*[type_code(c.dtype) for c in cols])
    ptrs = (C.c_void_p * k)(*[_ptr(c) for c in cols])
    nl = (C.c_void_p * k)(*[_ptr(x) for x in nulls]) if nulls is not None else None
    desc = (C.c_int32 * k)(*[int(bool(d)) for d in (descending or [False] * k)])
    capi.check(capi.lib().qdb_order_by(k, types, ptrs, nl, desc, n, _ptr(out), _stream(stream)))
    return out[:n]


class GPUString:
    """GPUMemory::GPUString (qikkDB/QueryEngine/GPUCore/GPUMemory.cuh): `allChars` every string's characters
    concatenated (uint8), `stringIndices` the int64 end offset of each string (string i is
    allChars[stringIndices[i-1] if i else 0 : stringIndices[i]]).  Either member is a torch CUDA tensor or a
    DeviceBuffer."""

    def __init__(self, allChars, stringIndices):
        self.allChars = allChars
        self.stringIndices = stringIndices

    @staticmethod
    def from_strings(strings, device="cuda") -> "GPUString":
        """StringFactory::PrepareGPUString: uploads a list of str/bytes (None stands for an empty string)."""
        bs = [b"" if x is None else (x.encode() if isinstance(x, str) else bytes(x)) for x in strings]
        ends = np.cumsum(np.fromiter((len(b) for b in bs), dtype=np.int64, count=len(bs)), dtype=np.int64)
        chars = np.frombuffer(b"".join(bs), dtype=np.uint8).copy()
        return GPUString(torch.from_numpy(chars).to(device), torch.from_numpy(ends).to(device))

    def __len__(self) -> int:
        x = self.stringIndices
        return x.numel() if isinstance(x, torch.Tensor) else x.count

    def to_strings(self) -> list:
        """GPUReconstruct::ReconstructStringCol to host: the strings as bytes."""
        def host(x):
            return x.cpu().numpy() if isinstance(x, torch.Tensor) else x.numpy()
        ends = host(self.stringIndices) if len(self) else np.zeros(0, dtype=np.int64)
        chars = host(self.allChars) if len(self) and int(ends[-1]) else np.zeros(0, dtype=np.uint8)
        out, b = [], 0
        for e in ends:
            out.append(chars[b:int(e)].tobytes())
            b = int(e)
        return out


class StringGroupByTable:
    """A multi-aggregate GROUP BY table over string keys (qdb_gbs_*)."""

    def __init__(self, aggs: Sequence[str], val_dtype, max_groups: int, max_key_bytes: int = 0, stream=None):
        self.aggs = [a for a in aggs if a != "none"]
        self.val_code = type_code(val_dtype) if val_dtype is not None else 0
        mask = 0
        for a in self.aggs:
            mask |= AGG_CODES[a]
        h = C.c_void_p()
        capi.check(capi.lib().qdb_gbs_create(C.byref(h), mask, self.val_code, int(max_groups), int(max_key_bytes),
                                             _stream(stream)))
        self.handle = h

    def __del__(self):
        try:
            if getattr(self, "handle", None) and self.handle.value:
                capi.lib().qdb_gbs_destroy(self.handle)
                self.handle = C.c_void_p()
        except Exception:
            pass

    def process(self, keys: GPUString, values=None, n: Optional[int] = None, key_nulls=None, value_nulls=None,
                mask=None, stream=None, sync: bool = True) -> None:
        n = len(keys) if n is None else n
        capi.check(capi.lib().qdb_gbs_process(self.handle, _ptr(keys.allChars), _ptr(keys.stringIndices),
                                              _ptr(key_nulls), _ptr(values), _ptr(value_nulls), _ptr(mask), int(n),
                                              _stream(stream)))
        if sync:
            self.check(stream)

    def check(self, stream=None) -> None:
        capi.check(capi.lib().qdb_gbs_check(self.handle, _stream(stream)))

    def reset(self, stream=None) -> None:
        capi.check(capi.lib().qdb_gbs_reset(self.handle, _stream(stream)))

    def results(self, aggs: Optional[Sequence[str]] = None, stream=None):
        """(keys: GPUString of DeviceBuffers, key_nulls: DeviceBuffer, {agg: (values, nulls)}, count)."""
        aggs = list(self.aggs if aggs is None else aggs)
        na = len(aggs)
        codes = (C.c_int32 * max(na, 1))(*[AGG_CODES[a] for a in aggs])
        ov = (C.c_void_p * max(na, 1))()
        ovn = (C.c_void_p * max(na, 1))()
        oc, oe, okn = C.c_void_p(), C.c_void_p(), C.c_void_p()
        cnt = C.c_int64()
        capi.check(capi.lib().qdb_gbs_results(self.handle, na, codes, C.byref(oc), C.byref(oe), C.byref(okn),
                                              ov if na else None, ovn if na else None, C.byref(cnt), _stream(stream)))
        n = cnt.value
        ends = DeviceBuffer(oe.value, n, np.int64)
        nchars = int(ends.numpy()[-1]) if n else 0
        keys = GPUString(DeviceBuffer(oc.value, nchars, np.uint8), ends)
        vals = {}
        vdt = CODE_TO_NP.get(self.val_code, np.int64)
        for i, a in enumerate(aggs):
            vals[a] = (DeviceBuffer(ov[i], n, np.int64 if a == "count" else vdt),
                       DeviceBuffer(ovn[i], nullmask_words(n), np.uint64))
        return keys, DeviceBuffer(okn.value, nullmask_words(n), np.uint64), vals, n

    def merge_from(self, other: "StringGroupByTable", stream=None) -> None:
        """Adds every group of `other` (same aggregates and value type, same device) to this table: the string form
        of GetResults over several tables (qdb_gbs_export + qdb_gbs_merge_exported)."""
        oc, oe, ost, ofl = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        n = C.c_int64()
        capi.check(capi.lib().qdb_gbs_export(other.handle, C.byref(oc), C.byref(oe), C.byref(ost), C.byref(ofl),
                                             C.byref(n), _stream(stream)))
        bufs = [DeviceBuffer(x.value, 1, np.uint8) for x in (oc, oe, ost, ofl)]
        capi.check(capi.lib().qdb_gbs_merge_exported(self.handle, oc.value, oe.value, ost.value, ofl.value, n.value,
                                                     _stream(stream)))
        self.check(stream)
        for b in bufs:
            b.free(stream)

    def results_host(self, aggs: Optional[Sequence[str]] = None, stream=None) -> dict:
        """{key bytes, or None for the NULL key: {agg: value, or None for a NULL aggregate}}."""
        keys, knull, vals, n = self.results(aggs, stream)
        ks = keys.to_strings()
        kn = unpack_nullmask(knull.numpy(), n) if n else np.zeros(0, dtype=bool)
        host = {a: (v.numpy(), unpack_nullmask(vn.numpy(), n)) for a, (v, vn) in vals.items()} if n else {}
        out = {}
        for i in range(n):
            key = None if kn[i] else ks[i]
            assert key not in out, f"duplicate group {key!r}"
            out[key] = {a: (None if (a != "count" and hv[1][i]) else hv[0][i].item()) for a, hv in host.items()}
        return out


class AaflBlock:
    """An AAFL-compressed column block on the device (the block format of qikkDB's CompressionGPU::compressDataAAFL:
    header, per-group position ids and bit lengths, packed words) with the block's min and max, which the
    decompression needs (the dispatcher passes the block statistics).  `data` is a CUDA tensor holding the block."""

    def __init__(self, data: torch.Tensor, dtype, vmin, vmax):
        self.data = data
        self.dtype = np.dtype(dtype)
        hdr = data.view(torch.uint8)[:24].cpu().numpy().view(np.int64)
        self.rows, self.elements, self.blocks = int(hdr[0]), int(hdr[1]), int(hdr[2])
        self.vmin, self.vmax = vmin, vmax

    @staticmethod
    def from_host(block: np.ndarray, vmin, vmax, device="cuda") -> "AaflBlock":
        return AaflBlock(torch.from_numpy(np.ascontiguousarray(block)).to(device), block.dtype, vmin, vmax)

    def c(self):
        d = capi.qdb_aafl_col()
        d.data = _ptr(self.data)
        d.type = NP_TO_CODE[self.dtype]
        d.rows, d.elements, d.blocks = self.rows, self.elements, self.blocks
        raw = lambda x: int(np.array([x], dtype=self.dtype).view(np.int32 if self.dtype.itemsize == 4 else np.int64)[0])  # noqa: E731
        d.min_bits, d.max_bits = raw(self.vmin), raw(self.vmax)
        return d

    @staticmethod
    def compress(col: torch.Tensor, vmin=None, vmax=None, stream=None) -> Optional["AaflBlock"]:
        """qdb_aafl_compress of a CUDA column (int32, int64 or float32) with its min and max (default: the column's
        own); None when the block stays plain."""
        dt = np.dtype({torch.int32: np.int32, torch.int64: np.int64, torch.float32: np.float32}[col.dtype])
        vmin = col.min().item() if vmin is None else vmin
        vmax = col.max().item() if vmax is None else vmax
        bits = lambda x: int(np.array([x], dtype=dt).view(np.int32 if dt.itemsize == 4 else np.int64)[0])  # noqa: E731
        out = C.c_void_p()
        elems = C.c_int64()
        capi.check(capi.lib().qdb_aafl_compress(NP_TO_CODE[dt], _ptr(col), col.numel(), bits(vmin), bits(vmax),
                                                C.byref(out), C.byref(elems), _stream(stream)))
        if not out.value:
            return None
        buf = DeviceBuffer(out.value, elems.value, dt)
        blk = AaflBlock(buf.torch(stream), dt, vmin, vmax)
        buf.free(stream)
        return blk

    def decompress(self, stream=None) -> torch.Tensor:
        """qdb_aafl_decompress: the block's rows as a CUDA tensor."""
        out = torch.empty(max(self.rows, 1), dtype=CODE_TO_TORCH[NP_TO_CODE[self.dtype]], device=self.data.device)
        d = self.c()
        capi.check(capi.lib().qdb_aafl_decompress(C.byref(d), _ptr(out), _stream(stream)))
        return out[:self.rows]


def process_aafl(table: "GroupByTable", keys: AaflBlock, values=None, pred=None, stream=None, sync: bool = True):
    """qdb_gb_process_aafl: ProcessBlock of a single-key table whose key column is an AAFL block."""
    d = keys.c()
    capi.check(capi.lib().qdb_gb_process_aafl(table.handle, C.byref(d), _ptr(values),
                                              C.byref(pred) if pred is not None else None, _stream(stream)))
    if sync:
        table.check(stream)


def process_mod(table: "GroupByTable", keys, key_mod: int, values=None, pred=None, n: int | None = None,
                stream=None, sync: bool = True):
    """qdb_gb_process_mod: ProcessBlock of key % key_mod (the GPUBinary modulo column and the GROUP BY fused)."""
    rows = int(keys.numel()) if n is None else int(n)
    capi.check(capi.lib().qdb_gb_process_mod(table.handle, _ptr(keys), int(key_mod), _ptr(values),
                                             C.byref(pred) if pred is not None else None, rows, _stream(stream)))
    if sync:
        table.check(stream)


class ScalarAggregate:
    """Scalar aggregation over a query's blocks (qdb_scalar_*): COUNT, SUM, MIN, MAX (and AVG) of one value column,
    filtered by an optional `col OP constant` predicate and mask, NULL values skipped."""

    def __init__(self, val_dtype, stream=None):
        h = C.c_void_p()
        self.val_code = type_code(val_dtype)
        capi.check(capi.lib().qdb_scalar_create(C.byref(h), self.val_code, _stream(stream)))
        self.handle = h

    def __del__(self):
        try:
            if self.handle:
                capi.lib().qdb_scalar_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def reset(self, stream=None) -> None:
        capi.check(capi.lib().qdb_scalar_reset(self.handle, _stream(stream)))

    def process(self, values: torch.Tensor, n: Optional[int] = None, value_nulls=None, pred=None, mask=None,
                stream=None) -> None:
        n = values.numel() if n is None else n
        capi.check(capi.lib().qdb_scalar_process(self.handle, _ptr(values), _ptr(value_nulls), int(n),
                                                 C.byref(pred) if pred is not None else None, _ptr(mask),
                                                 _stream(stream)))

    def result(self, agg: str, stream=None):
        """The aggregate as a Python number, or None for MIN/MAX/SUM/AVG over no row."""
        code = CODE_TO_NP[self.val_code] if agg != "count" else np.int64
        out = np.zeros(1, dtype=code)
        isnull = C.c_int32()
        capi.check(capi.lib().qdb_scalar_result(self.handle, AGG_CODES[agg], out.ctypes.data, C.byref(isnull),
                                                _stream(stream)))
        return None if isnull.value else out[0].item()


class GPUAggregation:
    """GPUAggregation::col<AGG, OUT, IN> (qikkDB/QueryEngine/GPUCore/GPUAggregation.cuh:15-37): one aggregate of a
    whole column (here optionally filtered and with NULL values skipped)."""

    @staticmethod
    def col(agg: str, ACol: torch.Tensor, dataElementCount: int, nullMask=None, pred=None, mask=None, stream=None):
        a = ScalarAggregate(ACol.dtype, stream)
        a.process(ACol, dataElementCount, nullMask, pred, mask, stream)
        return a.result(agg, stream)


def block_may_pass(pred_dtype, op: int, constant, const_dtype, block_min, block_max) -> bool:
    """qdb_pred_block_may_pass: whether a block whose predicate column spans [block_min, block_max] can hold a row
    passing `col OP constant` (GpuSqlDispatcher::WhereEvaluation's block skipping)."""
    p = capi.qdb_pred()
    p.col = 1  # not read: only the type, op and constant matter here
    p.type = type_code(pred_dtype)
    p.op = op
    ct = type_code(const_dtype)
    p.const_type = ct
    if ct in (capi.QDB_FLOAT, capi.QDB_DOUBLE):
        p.const_f = float(np.float32(constant)) if ct == capi.QDB_FLOAT else float(constant)
    else:
        p.const_i = int(constant)
    npdt = CODE_TO_NP[p.type]
    lo = np.array([block_min], dtype=npdt)
    hi = np.array([block_max], dtype=npdt)
    m = C.c_int32()
    capi.check(capi.lib().qdb_pred_block_may_pass(C.byref(p), lo.ctypes.data, hi.ctypes.data, C.byref(m)))
    return bool(m.value)
