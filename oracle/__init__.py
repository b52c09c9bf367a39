"""ORACLE - test infrastructure only (see oracle.cpp).  Imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py; never by the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None

T_INT32, T_INT64, T_FLOAT, T_DOUBLE, T_INT8 = 8, 9, 10, 11, 15
NP_CODE = {np.dtype(np.int32): T_INT32, np.dtype(np.int64): T_INT64, np.dtype(np.float32): T_FLOAT,
           np.dtype(np.float64): T_DOUBLE, np.dtype(np.int8): T_INT8}


def build() -> str:
    src = os.path.join(HERE, "oracle.cpp")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P, I32, I64 = C.c_void_p, C.c_int32, C.c_int64
        L.oracle_groupby.restype = P
        L.oracle_groupby.argtypes = [I32, I32, P, P, P, P, I32, P, P, I64, I32, P, P, I32, I32, I64, C.c_double, P,
                                     I32, I32]
        L.oracle_result_count.restype = I64
        L.oracle_result_count.argtypes = [P]
        L.oracle_result_seconds.restype = C.c_double
        L.oracle_result_seconds.argtypes = [P]
        L.oracle_result_threads.restype = I32
        L.oracle_result_threads.argtypes = [P]
        L.oracle_result_fetch.argtypes = [P] * 11
        L.oracle_result_free.argtypes = [P]
        L.oracle_filter.argtypes = [I32, I32, I32, P, I32, I32, P, P, P, I64]
        L.oracle_compact.restype = I64
        L.oracle_compact.argtypes = [I32, P, P, I64, P, P, P]
        L.oracle_indexes.restype = I64
        L.oracle_indexes.argtypes = [P, I64, P]
        L.oracle_prefix_sum.argtypes = [P, I64, P]
        L.oracle_reference_filter_inputs.argtypes = [I32, I32, I64, P, P]
        L.oracle_order_by.argtypes = [I32, P, P, P, P, I64, P]
        L.oracle_aafl_compress.restype = I64
        L.oracle_aafl_compress.argtypes = [I32, P, I64, P, P, P, I64]
        L.oracle_aafl_decompress.argtypes = [I32, P, P, P, P]
        L.oracle_string_ids.restype = I64
        L.oracle_string_ids.argtypes = [P, P, P, I64, P]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else np.ascontiguousarray(a).ctypes.data


def groupby(keys, vals=None, key_nulls=None, val_nulls=None, pred=None, mask=None, threads: int = 0,
            sort: bool = True, timing_only: bool = False) -> dict:
    """CPU GROUP BY.  keys: array or [a, b] (composite int32).  key_nulls/val_nulls: packed uint64 masks.
    pred: (col, op, const, const_dtype, packed_nulls or None).  Returns a dict of host arrays sorted by key:
    keys (list), key_nulls (list of bool), cnt, sum, min, max, avg, val_null, plus 'seconds' and 'threads'."""
    keys = list(keys) if isinstance(keys, (list, tuple)) else [keys]
    keys = [np.ascontiguousarray(k) for k in keys]
    n = len(keys[0])
    kt = NP_CODE[keys[0].dtype]
    kn = list(key_nulls) if isinstance(key_nulls, (list, tuple)) else [key_nulls, None]
    kn = [None if x is None else np.ascontiguousarray(x, dtype=np.uint64) for x in kn] + [None]
    vt = 0
    if vals is not None:
        vals = np.ascontiguousarray(vals)
        vt = NP_CODE[vals.dtype]
    vn = None if val_nulls is None else np.ascontiguousarray(val_nulls, dtype=np.uint64)
    pt, pc, pn, pop, ct, ci, cf = 0, None, None, 0, 0, 0, 0.0
    if pred is not None:
        pcol, pop, const, cdt, pnul = pred
        pc = np.ascontiguousarray(pcol)
        pt = NP_CODE[pc.dtype]
        ct = NP_CODE[np.dtype(cdt)]
        if ct in (T_FLOAT, T_DOUBLE):
            cf = float(np.float32(const)) if ct == T_FLOAT else float(const)
        else:
            ci = int(const)
        pn = None if pnul is None else np.ascontiguousarray(pnul, dtype=np.uint64)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int8)
    L = lib()
    r = L.oracle_groupby(kt, len(keys), _p(keys[0]), _p(keys[1]) if len(keys) > 1 else None, _p(kn[0]), _p(kn[1]),
                         vt, _p(vals), _p(vn), n, pt, _p(pc), _p(pn), pop, ct, ci, cf, _p(m), threads,
                         1 if sort else 0)
    try:
        g = L.oracle_result_count(r)
        out = {"count": g, "seconds": L.oracle_result_seconds(r), "threads": L.oracle_result_threads(r)}
        if timing_only:
            return out
        kf = kt in (T_FLOAT, T_DOUBLE)
        k0 = np.empty(g, dtype=np.float64 if kf else np.int64)
        k1 = np.empty(g, dtype=np.int64) if len(keys) > 1 else None
        n0 = np.empty(g, dtype=np.uint8)
        n1 = np.empty(g, dtype=np.uint8) if len(keys) > 1 else None
        vf = vt in (T_FLOAT, T_DOUBLE)
        vd = np.float64 if vf else np.int64
        cnt = np.empty(g, dtype=np.int64)
        s, mn, mx, av = (np.empty(g, dtype=vd) for _ in range(4))
        vnull = np.empty(g, dtype=np.uint8)
        L.oracle_result_fetch(r, _p(k0), _p(k1), _p(n0), _p(n1), _p(cnt), _p(s), _p(mn), _p(mx), _p(av), _p(vnull))
        out.update({"keys": [k0] + ([k1] if k1 is not None else []),
                    "key_nulls": [n0.astype(bool)] + ([n1.astype(bool)] if n1 is not None else []),
                    "cnt": cnt, "sum": s, "min": mn, "max": mx, "avg": av, "val_null": vnull.astype(bool)})
        return out
    finally:
        L.oracle_result_free(r)


def pack_strings(strings) -> tuple[np.ndarray, np.ndarray]:
    """GPUString layout of a list of str/bytes (None counts as an empty string): (uint8 chars, int64 end offsets)."""
    bs = [b"" if s is None else (s.encode() if isinstance(s, str) else bytes(s)) for s in strings]
    lens = np.fromiter((len(b) for b in bs), dtype=np.int64, count=len(bs))
    ends = np.cumsum(lens, dtype=np.int64)
    chars = np.frombuffer(b"".join(bs), dtype=np.uint8).copy() if bs else np.zeros(0, dtype=np.uint8)
    return chars, ends


def string_at(chars: np.ndarray, ends: np.ndarray, i: int) -> bytes:
    b = int(ends[i - 1]) if i else 0
    return chars[b:int(ends[i])].tobytes()


def groupby_string(chars, ends, vals=None, key_nulls=None, val_nulls=None, mask=None, threads: int = 0) -> dict:
    """CPU GROUP BY over string keys: every string maps to the row of its first occurrence, then the integer GROUP BY
    runs over those ids.  Returns {key (bytes, or None for the NULL key): {cnt, sum, min, max, avg, val_null}}."""
    chars = np.ascontiguousarray(chars, dtype=np.uint8)
    ends = np.ascontiguousarray(ends, dtype=np.int64)
    n = len(ends)
    ids = np.empty(n, dtype=np.int64)
    kn = None if key_nulls is None else np.ascontiguousarray(key_nulls, dtype=np.uint64)
    lib().oracle_string_ids(_p(chars) if len(chars) else None, _p(ends), _p(kn), n, _p(ids))
    r = groupby(ids, vals, key_nulls=kn, val_nulls=val_nulls, mask=mask, threads=threads)
    out = {}
    for j in range(r["count"]):
        key = None if r["key_nulls"][0][j] else string_at(chars, ends, int(r["keys"][0][j]))
        out[key] = {f: r[f][j] for f in ("cnt", "sum", "min", "max", "avg", "val_null")}
    return out


def aafl_compress(values: np.ndarray, vmin=None, vmax=None):
    """AAFL block of a column (int32, int64 or float32) with its min and max (default: the column's own), or None
    when the block stays plain.  Returns the block as an array of the column's dtype."""
    v = np.ascontiguousarray(values)
    dt = v.dtype
    mn = np.array([v.min() if vmin is None else vmin], dtype=dt)
    mx = np.array([v.max() if vmax is None else vmax], dtype=dt)
    out = np.zeros(len(v) + 64, dtype=dt)
    r = lib().oracle_aafl_compress(NP_CODE[dt], _p(v), len(v), _p(mn), _p(mx), _p(out), len(out))
    if r <= 0:
        return None
    return out[:r].copy()


def aafl_header(block: np.ndarray) -> tuple:
    """(rows, elements, blocks) of an AAFL block."""
    h = np.frombuffer(np.ascontiguousarray(block).tobytes()[:24], dtype=np.int64)
    return int(h[0]), int(h[1]), int(h[2])


def aafl_decompress(block: np.ndarray, vmin, vmax) -> np.ndarray:
    b = np.ascontiguousarray(block)
    dt = b.dtype
    rows = aafl_header(b)[0]
    out = np.empty(rows, dtype=dt)
    mn = np.array([vmin], dtype=dt)
    mx = np.array([vmax], dtype=dt)
    lib().oracle_aafl_decompress(NP_CODE[dt], _p(b), _p(mn), _p(mx), _p(out))
    return out


def filter_mask(op: int, a, b, nulls=None, n: int | None = None) -> np.ndarray:
    """a / b: numpy column or numpy scalar (constant)."""
    def side(x):
        if isinstance(x, np.ndarray) and x.ndim == 1:
            return NP_CODE[x.dtype], 1, np.ascontiguousarray(x)
        arr = np.array([x]) if not isinstance(x, np.generic) else np.array([x], dtype=x.dtype)
        return NP_CODE[arr.dtype], 0, arr
    at, ac, aa = side(a)
    bt, bc, bb = side(b)
    if n is None:
        n = len(aa) if ac else len(bb)
    out = np.empty(n, dtype=np.int8)
    lib().oracle_filter(op, at, ac, _p(aa), bt, bc, _p(bb), _p(nulls), _p(out), n)
    return out


def compact(col: np.ndarray, mask: np.ndarray, nulls=None):
    col = np.ascontiguousarray(col)
    out = np.empty_like(col)
    nout = np.zeros((len(col) + 63) // 64 + 1, dtype=np.uint64) if nulls is not None else None
    c = lib().oracle_compact(col.dtype.itemsize, _p(col), _p(np.ascontiguousarray(mask, dtype=np.int8)), len(col),
                             _p(out), _p(nulls), _p(nout))
    return out[:c], (nout if nout is not None else None), c


def order_by(cols, descending=None, nulls=None) -> np.ndarray:
    """Row permutation of ORDER BY cols[0], cols[1], ... (descending[c] per column; nulls[c] packed words or None)."""
    cols = [np.ascontiguousarray(c) for c in cols]
    n = len(cols[0])
    k = len(cols)
    types = (C.c_int32 * k)(*[NP_CODE[c.dtype] for c in cols])
    ptrs = (C.c_void_p * k)(*[c.ctypes.data for c in cols])
    nl = None
    keep = []
    if nulls is not None:
        nw = [None if x is None else np.ascontiguousarray(x, dtype=np.uint64) for x in nulls]
        keep = nw
        nl = (C.c_void_p * k)(*[None if x is None else x.ctypes.data for x in nw])
    desc = (C.c_int32 * k)(*[int(bool(d)) for d in (descending or [0] * k)])
    out = np.empty(n, dtype=np.int32)
    lib().oracle_order_by(k, types, ptrs, nl, desc, n, _p(out))
    del keep
    return out


def indexes(mask: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(mask, dtype=np.int8)
    out = np.empty(len(m), dtype=np.int32)
    c = lib().oracle_indexes(_p(m), len(m), _p(out))
    return out[:c]


def prefix_sum(mask: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(mask, dtype=np.int8)
    out = np.empty(len(m), dtype=np.int32)
    lib().oracle_prefix_sum(_p(m), len(m), _p(out))
    return out


def reference_filter_inputs(dtype, mode: int, n: int = 1 << 18):
    """Inputs of qikkDB_test/GPUFilterTests.cu (mode 0: col-col arrays; mode 1: column and one constant)."""
    dt = np.dtype(dtype)
    a = np.empty(n, dtype=dt)
    b = np.empty(n if mode == 0 else 1, dtype=dt)
    lib().oracle_reference_filter_inputs(NP_CODE[dt], mode, n, _p(a), _p(b))
    return a, (b if mode == 0 else b[0])
