"""The serving loop of the C ABI (``qdb_server_*``): continuous batching of GROUP BY queries over device-resident
columns.

Queries (``batch.Query``; ``max_groups=0`` lets the server size the table from a cardinality estimate) are
submitted from any thread and return a ticket at once; a native scheduler thread admits them into batches as
batch slots and the table budget free up, keeps up to ``in_flight`` batches on the GPU, and hands every query's
results back on the host.  ``run_open_loop`` replays an arrival schedule (open loop: queries arrive whether or not
earlier ones are done) and reports each query's latency from its arrival to its results on the host.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _capi as capi
from .batch import AGG_ORDER, Query, _out_dtype
from .groupby import CODE_TO_NP, type_code


class Server:
    def __init__(self, max_batch: int = 32, in_flight: int = 2, table_budget: int = 1 << 32,
                 result_budget: int = 1 << 30, plain_rows: int | None = None, plain_groups: int | None = None):
        """plain_rows / plain_groups: queries of at least plain_rows rows, or whose table capacity is at least
        plain_groups, run alone through the single-query fast pass (qdb_server_set_plain_route; <= 0 is off; None
        keeps the library's default: 2^22 rows, groups off)."""
        h = C.c_void_p()
        capi.check(capi.lib().qdb_server_create(C.byref(h), int(max_batch), int(in_flight), int(table_budget),
                                                int(result_budget)))
        self.handle = h
        self._alive: dict[int, Query] = {}
        if plain_rows is not None or plain_groups is not None:
            capi.check(capi.lib().qdb_server_set_plain_route(
                h, int(1 << 22 if plain_rows is None else plain_rows), int(plain_groups or 0)))

    def close(self) -> None:
        if getattr(self, "handle", None) and self.handle.value:
            capi.lib().qdb_server_destroy(self.handle)
            self.handle = C.c_void_p()
            self._alive.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, q: Query) -> int:
        t = C.c_uint64()
        cq = q.to_c()
        capi.check(capi.lib().qdb_server_submit(self.handle, C.byref(cq), C.byref(t)))
        self._alive[t.value] = q  # the query's device columns must outlive it
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1, release: bool = True) -> dict:
        """{'status', 'n_groups', 'keys': [arr], agg: arr, 'retries', 'batch_size', 'max_groups',
        'latency_ns' (submit to results on host), 'queue_ns' (submit to batch launch)}"""
        r = capi.qdb_server_result()
        capi.check(capi.lib().qdb_server_wait(self.handle, C.c_uint64(ticket), int(timeout_ms), C.byref(r)))
        q = self._alive[ticket]
        n = r.n_groups
        words = np.ctypeslib.as_array(C.cast(r.keys, C.POINTER(C.c_int64)), shape=(n * (1 + r.n_cols),)).copy() \
            if n > 0 else np.zeros(0, np.int64)
        out = {"status": r.status, "n_groups": n, "retries": r.retries, "batch_size": r.batch_size,
               "max_groups": r.max_groups, "latency_ns": r.done_ns - r.submit_ns, "queue_ns": r.start_ns - r.submit_ns,
               "keys": [words[:n].astype(CODE_TO_NP[type_code(q.keys.dtype)])]}
        names = [a for a in AGG_ORDER if a in q.aggs]
        for j, a in enumerate(names):
            w = words[(j + 1) * n:(j + 2) * n]
            dt = _out_dtype(a, q.vals.dtype if q.vals is not None else np.int64)
            out[a] = w.view(np.float64).astype(dt) if dt.kind == "f" else w.astype(dt)
        if release:
            self.release(ticket)
        return out

    def release(self, ticket: int) -> None:
        capi.check(capi.lib().qdb_server_release(self.handle, C.c_uint64(ticket)))
        self._alive.pop(ticket, None)

    def stats(self) -> dict:
        s = capi.qdb_server_stats()
        capi.check(capi.lib().qdb_server_stats_get(self.handle, C.byref(s)))
        return {f: getattr(s, f) for f, _ in capi.qdb_server_stats._fields_}

    def run_open_loop(self, queries: Sequence[Query], arrival_ns: Sequence[int]):
        """Submits queries[i] at arrival_ns[i] after the call; returns (latency_ns, status, wall_ns)."""
        n = len(queries)
        arr = (capi.qdb_gb_query * max(n, 1))(*[q.to_c() for q in queries])
        at = np.ascontiguousarray(arrival_ns, dtype=np.int64)
        lat = np.zeros(max(n, 1), np.int64)
        st = np.zeros(max(n, 1), np.int32)
        wall = C.c_int64()
        capi.check(capi.lib().qdb_server_run_open_loop(self.handle, arr, n, at.ctypes.data_as(capi.PI64),
                                                       lat.ctypes.data_as(capi.PI64),
                                                       st.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(wall)))
        return lat[:n], st[:n], wall.value


def poisson_arrivals(rate_qps: float, n: int, seed: int) -> np.ndarray:
    """Arrival times (ns) of an open-loop Poisson stream: exponential inter-arrival gaps of mean 1 / rate."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1e9 / rate_qps, size=n)
    return np.cumsum(gaps).astype(np.int64) - int(gaps[0])


def percentile_ms(lat_ns: np.ndarray, p: float) -> float:
    return float(np.percentile(lat_ns, p)) / 1e6 if lat_ns.size else float("nan")


__all__ = ["Server", "poisson_arrivals", "percentile_ms"]
