"""Seeded synthetic columns for the GROUP BY workloads (wraps libqdbgen.so, csrc/datagen.cpp).

Every generator is a pure function of (seed, stream, row): the bytes do not depend on the thread count,
so the oracle and the GPU path see identical inputs.
"""
from __future__ import annotations

import numpy as np

from . import _capi as capi


def _out(n: int, dtype, out=None) -> np.ndarray:
    if out is None:
        return np.empty(n, dtype=dtype)
    assert out.dtype == np.dtype(dtype) and out.size >= n and out.flags.c_contiguous
    return out


def uniform_i32(seed: int, stream: int, n: int, lo: int, hi: int, threads: int = 0, out=None) -> np.ndarray:
    a = _out(n, np.int32, out)
    assert capi.gen().qdbgen_uniform_i32(seed, stream, n, lo, hi, a.ctypes.data, threads) == 0
    return a


def uniform_i64(seed: int, stream: int, n: int, lo: int, hi: int, threads: int = 0, out=None) -> np.ndarray:
    a = _out(n, np.int64, out)
    assert capi.gen().qdbgen_uniform_i64(seed, stream, n, lo, hi, a.ctypes.data, threads) == 0
    return a


def uniform_f32(seed: int, stream: int, n: int, lo: float = 0.0, hi: float = 1.0, threads: int = 0,
                out=None) -> np.ndarray:
    a = _out(n, np.float32, out)
    assert capi.gen().qdbgen_uniform_f32(seed, stream, n, lo, hi, a.ctypes.data, threads) == 0
    return a


def lognormal_f32(seed: int, stream: int, n: int, mu: float, sigma: float, threads: int = 0,
                  out=None) -> np.ndarray:
    a = _out(n, np.float32, out)
    assert capi.gen().qdbgen_lognormal_f32(seed, stream, n, mu, sigma, a.ctypes.data, threads) == 0
    return a


def zipf_i64(seed: int, stream: int, n: int, n_distinct: int, s: float, map_keys: bool = True, threads: int = 0,
             out=None) -> np.ndarray:
    a = _out(n, np.int64, out)
    assert capi.gen().qdbgen_zipf_i64(seed, stream, n, n_distinct, s, 1 if map_keys else 0, a.ctypes.data,
                                      threads) == 0
    return a


def loguniform_i64(seed: int, stream: int, n: int, lo: int, hi: int, threads: int = 0) -> np.ndarray:
    a = np.empty(n, dtype=np.int64)
    assert capi.gen().qdbgen_loguniform_i64(seed, stream, n, lo, hi, a.ctypes.data, threads) == 0
    return a


def rank_key(rank: int) -> int:
    return int(capi.gen().qdbgen_rank_key(rank))
