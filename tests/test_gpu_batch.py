"""Batched GROUP BY (qdb_gb_batch_*) against the oracle: every query of a mixed batch must give the same result
as the oracle on that query alone (keys and integer aggregates bit-exact, float SUM/AVG within FLOAT_RTOL), under
every execution plan (shared-memory replicas, global table, warp-group widths, rows per thread), across CUDA-graph
replays, and the same result as the plain single-query path."""
import numpy as np
import pytest
import torch

import oracle
from gpu_compare import compare
from qikkdb_b200 import _capi as capi
from qikkdb_b200 import datagen as dg
from qikkdb_b200.batch import AGG_ORDER, GroupByBatch, Query, tuning_reset
from qikkdb_b200.groupby import FilterConditions, GroupByTable, QueryEngineError

pytestmark = pytest.mark.gpu

AGG_SETS = [["sum", "min", "max", "count"], ["sum", "avg"], ["sum", "count", "max"], list(AGG_ORDER)]


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


class Spec:
    """Host columns of one query plus its device tensors and its oracle result."""

    def __init__(self, seed, kdt, vdt, n, card, aggs, key_mod=0, pred=None, neg_keys=False, max_groups=None):
        self.n = n
        lo = -card if neg_keys else 0
        if kdt == np.int32:
            self.k = dg.uniform_i32(seed, 0, n, lo, card - 1)
        else:
            self.k = dg.uniform_i64(seed, 0, n, lo, card - 1) * 1_000_003 if neg_keys else dg.uniform_i64(
                seed, 0, n, lo, card - 1)
        if vdt is None:
            self.v = None
        elif vdt == np.int32:
            self.v = dg.uniform_i32(seed, 1, n, -1000, 1000)
        elif vdt == np.int64:
            self.v = dg.uniform_i64(seed, 1, n, -(1 << 40), 1 << 40)
        elif vdt == np.float32:
            self.v = dg.lognormal_f32(seed, 1, n, 2.0, 1.0)
        else:
            self.v = dg.uniform_f32(seed, 1, n, -100.0, 100.0).astype(np.float64)
        self.aggs = list(aggs) if vdt is not None else ["count"]
        self.key_mod = key_mod
        self.pred = None
        if pred is not None:
            pdt, op, const, cdt = pred
            if pdt in (np.float32, np.float64):
                pc = dg.uniform_f32(seed, 2, n).astype(pdt)
            else:
                pc = dg.uniform_i32(seed, 2, n, -50, 50).astype(pdt)
            self.pred = (pc, op, const, cdt)
        ek = np.fmod(self.k, key_mod).astype(self.k.dtype) if key_mod else self.k
        distinct = len(np.unique(ek)) if n else 0
        self.max_groups = max_groups if max_groups is not None else max(1, distinct)
        self.ref = oracle.groupby(ek, self.v, pred=(self.pred + (None,)) if self.pred else None)
        self.dk = _dev(self.k)
        self.dv = _dev(self.v) if self.v is not None else None
        self.dp = _dev(self.pred[0]) if self.pred else None

    def query(self):
        pred = (self.dp, self.pred[1], self.pred[2], self.pred[3]) if self.pred else None
        return Query(self.dk, self.dv, self.aggs, self.max_groups, self.key_mod, pred)

    def check(self, res):
        g = dict(res)
        g["key_nulls"] = [np.zeros(g["n_groups"], bool)]
        for a in self.aggs:
            g[a + "_null"] = np.zeros(g["n_groups"], bool)
        vf = self.v is not None and self.v.dtype.kind == "f"
        return compare(g, self.ref, self.aggs, vf)


def mixed_specs(seed=0):
    rng = np.random.default_rng(seed)
    specs = []
    shapes = [  # (key dtype, value dtype, rows, cardinality)
        (np.int32, np.int32, 1 << 20, 1000), (np.int64, np.float32, 300_000, 50_000), (np.int32, np.int64, 70_000, 4),
        (np.int32, np.float32, 200_000, 1), (np.int64, np.int64, 65, 7), (np.int32, np.float64, 1, 1),
        (np.int32, None, 123_457, 300), (np.int64, np.float64, 500_000, 200_000), (np.int32, np.int32, 0, 5),
        (np.int32, np.float32, 3, 3), (np.int64, np.int32, 64, 64), (np.int32, np.int64, 2_000_000, 17),
        (np.int32, np.float32, 1_000_000, 8000), (np.int64, np.float32, 100_000, 100_000),
    ]
    for i, (kdt, vdt, n, card) in enumerate(shapes):
        aggs = AGG_SETS[int(rng.integers(len(AGG_SETS)))]
        specs.append(Spec(100 + i, kdt, vdt, n, card, aggs))
    # key modulus and predicates of every column type
    specs.append(Spec(200, np.int32, np.float32, 400_000, 100_000, ["sum", "avg"], key_mod=97, neg_keys=True))
    specs.append(Spec(201, np.int64, np.int64, 300_001, 1 << 20, ["sum", "min", "max", "count"], key_mod=5000,
                      neg_keys=True))
    specs.append(Spec(202, np.int64, np.float32, 500_000, 1000, ["sum", "avg"],
                      pred=(np.float32, FilterConditions.less, 0.5, np.float32)))
    specs.append(Spec(203, np.int32, np.int32, 250_000, 77, ["min", "max", "count"],
                      pred=(np.int32, FilterConditions.greaterEqual, 10, np.int64)))
    specs.append(Spec(204, np.int32, np.float64, 100_000, 3000, ["sum", "count"],
                      pred=(np.float64, FilterConditions.notEqual, 0.25, np.float64)))
    specs.append(Spec(205, np.int64, np.int32, 150_000, 40, ["sum", "max"],
                      pred=(np.int64, FilterConditions.lessEqual, -20, np.int32)))
    specs.append(Spec(206, np.int32, np.float32, 90_000, 12, ["avg", "min"],
                      pred=(np.float32, FilterConditions.greater, 2.0, np.float32)))  # no row passes
    return specs


def run_batch(specs, graph=False, stream=None, cfgs=None, runs=1):
    b = GroupByBatch(len(specs), 1 << 30, 1 << 28)
    b.set([s.query() for s in specs], stream=stream)
    if cfgs:
        for i, c in cfgs.items():
            b.set_cfg(i, **c)
    out = None
    for _ in range(runs):
        b.run(graph=graph, stream=stream)
        counts, status = b.fetch(stream=stream)
        assert (status == 0).all(), f"statuses {status}"
        out = b.results_all(stream=stream)
    return b, out


def test_batch_mixed_parity(cuda):
    specs = mixed_specs()
    _, res = run_batch(specs)
    for s, r in zip(specs, res):
        s.check(r)


def test_batch_graph_replays(cuda):
    """The captured graph replays: the result kernel leaves every table clean for the next run."""
    specs = mixed_specs(1)
    st = torch.cuda.Stream()
    b, res = run_batch(specs, graph=True, stream=st.cuda_stream, runs=3)
    for s, r in zip(specs, res):
        s.check(r)
    # a new set of queries through the same graph
    specs2 = mixed_specs(2)[::-1]
    b.set([s.query() for s in specs2], stream=st.cuda_stream)
    b.run(graph=True, stream=st.cuda_stream)
    _, status = b.fetch(stream=st.cuda_stream)
    assert (status == 0).all()
    for s, r in zip(specs2, b.results_all(stream=st.cuda_stream)):
        s.check(r)


PLANS = [
    {"placement": capi.QDB_PLACE_GLOBAL, "warps": 12, "rows_per_thread": 4},
    {"placement": capi.QDB_PLACE_GLOBAL, "warps": 3, "rows_per_thread": 1},
    {"placement": capi.QDB_PLACE_SHARED, "replicas": 1, "warps": 12, "rows_per_thread": 2},
    {"placement": capi.QDB_PLACE_SHARED, "replicas": 4, "warps": 6, "rows_per_thread": 4},
    {"placement": capi.QDB_PLACE_SHARED, "replicas": 4, "warps": 3, "rows_per_thread": 1},
]


@pytest.mark.parametrize("plan", range(len(PLANS)))
def test_batch_every_plan(cuda, plan):
    """The same queries under a forced plan: placement, replicas, warp-group width, rows per thread, and work
    items cut small (many items per query, several merges into one global table)."""
    specs = [Spec(300, np.int32, np.int32, 400_000, 60, AGG_SETS[3]),
             Spec(301, np.int64, np.float32, 300_000, 900, ["sum", "avg", "max"]),
             Spec(302, np.int32, np.int64, 100_003, 5, ["sum", "min", "count"],
                  pred=(np.float32, FilterConditions.less, 0.3, np.float32)),
             Spec(303, np.int32, np.float64, 77_777, 20_000, ["sum", "count"], key_mod=1500, neg_keys=True)]
    b = GroupByBatch(len(specs), 1 << 28, 1 << 26)
    b.set([s.query() for s in specs])
    p = dict(PLANS[plan])
    for i, s in enumerate(specs):
        c = dict(p)
        c["chunk_rows"] = 8192
        if c["placement"] == capi.QDB_PLACE_SHARED:
            slots = 64
            while slots < 2 * (s.max_groups + 1):
                slots *= 2
            c["smem_slots"] = min(slots, 2048)
            c["replicas"] = min(c["replicas"], c["warps"])
            while True:  # shrink until the tables fit the group's shared memory (undersized tables spill)
                try:
                    b.set_cfg(i, **c)
                    break
                except QueryEngineError as e:
                    assert e.code == capi.QDB_ERR_TOO_LARGE
                    if c["replicas"] > 1:
                        c["replicas"] //= 2
                    else:
                        assert c["smem_slots"] > 64
                        c["smem_slots"] //= 2
        else:
            b.set_cfg(i, **c)
    b.run()
    _, status = b.fetch()
    assert (status == 0).all()
    for s, r in zip(specs, b.results_all()):
        s.check(r)


def test_batch_undersized_shared_table_spills_to_global(cuda):
    """A shared table far smaller than the key count: rows whose probe fails go to the global table."""
    s = Spec(310, np.int32, np.int64, 500_000, 30_000, ["sum", "min", "max", "count"])
    b = GroupByBatch(1, 1 << 28, 1 << 26)
    b.set([s.query()])
    b.set_cfg(0, placement=capi.QDB_PLACE_SHARED, smem_slots=256, replicas=2, warps=12, chunk_rows=65536)
    b.run()
    _, status = b.fetch()
    assert status[0] == 0
    s.check(b.results_all()[0])


def test_batch_table_full_is_per_query(cuda):
    ok = Spec(320, np.int32, np.int32, 100_000, 100, ["sum"])
    full = Spec(321, np.int32, np.int32, 100_000, 5000, ["sum"], max_groups=1000)
    b = GroupByBatch(2, 1 << 26, 1 << 24)
    b.set([ok.query(), full.query()])
    b.run()
    _, status = b.fetch()
    assert status[0] == 0 and status[1] == capi.QDB_HASH_TABLE_FULL
    ok.check(b.result(0))
    # the next run of a corrected batch starts from clean tables
    full2 = Spec(321, np.int32, np.int32, 100_000, 5000, ["sum"])
    b.set([ok.query(), full2.query()])
    b.run()
    _, status = b.fetch()
    assert (status == 0).all()
    ok.check(b.result(0))
    full2.check(b.result(1))


def test_batch_escape_key_and_extremes(cuda):
    """INT64_MIN (the empty-slot pattern) is an ordinary key; int32 extremes and key % m of negative keys."""
    n = 50_000
    k = dg.uniform_i64(330, 0, n, -3, 3)
    k[::7] = np.iinfo(np.int64).min
    k[::11] = np.iinfo(np.int64).max
    v = dg.uniform_i64(330, 1, n, -(1 << 62), 1 << 62)  # sums wrap in int64
    s = Spec.__new__(Spec)
    s.n, s.k, s.v, s.aggs, s.key_mod, s.pred = n, k, v, list(AGG_ORDER), 0, None
    s.max_groups = 9
    s.ref = oracle.groupby(k, v)
    s.dk, s.dv, s.dp = _dev(k), _dev(v), None
    k32 = dg.uniform_i32(331, 0, n, -2**31, 2**31 - 1)
    s2 = Spec.__new__(Spec)
    s2.n, s2.k, s2.v, s2.aggs, s2.key_mod, s2.pred = n, k32, dg.uniform_i32(331, 1, n, -2**31, 2**31 - 1), \
        ["sum", "avg", "min", "max"], 1 << 31, None
    ek = np.fmod(k32.astype(np.int64), 1 << 31).astype(np.int32)
    s2.max_groups = len(np.unique(ek))
    s2.ref = oracle.groupby(ek, s2.v)
    s2.dk, s2.dv, s2.dp = _dev(k32), _dev(s2.v), None
    _, res = run_batch([s, s2])
    s.check(res[0])
    s2.check(res[1])


def test_batch_same_as_plain_path(cuda):
    """Each query's result in the mix equals the plain single-query path's result for it alone."""
    specs = [Spec(340 + i, np.int32, np.int64, 200_000 + 1000 * i, 10 ** (1 + i % 4), ["sum", "min", "max", "count"])
             for i in range(6)]
    _, res = run_batch(specs)
    for s, r in zip(specs, res):
        t = GroupByTable(s.aggs, np.int32, np.int64, s.max_groups)
        t.process(s.dk, s.dv)
        g = t.results_numpy()
        order_b = np.argsort(r["keys"][0])
        order_p = np.argsort(g["keys"][0])
        assert (r["keys"][0][order_b] == g["keys"][0][order_p]).all()
        for a in s.aggs:
            assert (r[a][order_b] == g[a][order_p]).all(), a


def test_batch_autotune(cuda):
    tuning_reset()
    specs = mixed_specs(3)[:10]
    b = GroupByBatch(len(specs), 1 << 30, 1 << 28)
    b.set([s.query() for s in specs])
    b.autotune()
    cfgs = [b.get_cfg(i) for i in range(len(specs))]
    assert all(c["warps"] in (12, 6, 3) and c["rows_per_thread"] in (1, 2, 4) for c in cfgs)
    b.run()
    _, status = b.fetch()
    assert (status == 0).all()
    ns = b.item_times()
    assert (ns[[i for i, s in enumerate(specs) if s.n > 0]] > 0).all()
    for s, r in zip(specs, b.results_all()):
        s.check(r)
    # the tuning table now plans a fresh batch of the same classes
    b2 = GroupByBatch(len(specs), 1 << 30, 1 << 28)
    b2.set([s.query() for s in specs])
    assert [b2.get_cfg(i) for i in range(len(specs))] == cfgs
    tuning_reset()


def test_batch_rejects_bad_queries(cuda):
    b = GroupByBatch(2, 1 << 20, 1 << 20)
    k = torch.zeros(1025, dtype=torch.int32, device="cuda")
    v = torch.zeros(1025, dtype=torch.int32, device="cuda")
    with pytest.raises(QueryEngineError) as e:
        b.set([Query(k[1:], v[1:], ["sum"], 10)])  # not 16-byte aligned
    assert e.value.code == capi.QDB_ERR_INVALID
    with pytest.raises(QueryEngineError) as e:
        b.set([Query(k, v, ["sum"], 1 << 22)])  # table larger than the batch's table budget
    assert e.value.code == capi.QDB_ERR_TOO_LARGE
    with pytest.raises(QueryEngineError) as e:
        b.set([Query(k, None, ["sum"], 10)])
    assert e.value.code == capi.QDB_ERR_INVALID
    with pytest.raises(QueryEngineError) as e:
        b.set([Query(k.float(), v, ["sum"], 10)])
    assert e.value.code == capi.QDB_ERR_INVALID


@pytest.mark.parametrize("share", [True, False])
def test_batch_shared_scan(cuda, share):
    """Queries over the same columns (different WHERE constants, key moduli, aggregates, placements) aggregated in
    shared scans: each result equals the oracle on that query alone."""
    n = 600_000
    k = dg.uniform_i64(400, 0, n, -(1 << 40), 1 << 40)
    v = dg.lognormal_f32(400, 1, n, 2.0, 1.0)
    p = dg.uniform_f32(400, 2, n)
    dk, dv, dp = _dev(k), _dev(v), _dev(p)
    specs = []
    for i, (mod, sel, aggs) in enumerate([(10, 0.9, ["sum", "avg"]), (1000, 0.05, ["sum", "count", "max"]),
                                          (7, 0.5, list(AGG_ORDER)), (100_000, 0.3, ["sum", "avg"]),
                                          (64, 1.0, ["min", "count"]), (2, 0.01, ["sum"]),
                                          (300, 0.7, ["max", "sum"]), (5000, 0.2, ["count"]),
                                          (33, 0.6, ["sum", "avg", "count"]), (1 << 20, 0.4, ["sum", "count"])]):
        s = Spec.__new__(Spec)
        s.n, s.k, s.v, s.aggs, s.key_mod = n, k, v, aggs, mod
        s.pred = (p, FilterConditions.less, sel, np.float32)
        ek = np.fmod(k, mod)
        keep = p < np.float32(sel)
        s.max_groups = max(1, len(np.unique(ek[keep])))
        s.ref = oracle.groupby(ek, v, pred=(p, FilterConditions.less, sel, np.float32, None))
        s.dk, s.dv, s.dp = dk, dv, dp
        specs.append(s)
    b = GroupByBatch(len(specs), 1 << 30, 1 << 28)
    b.set_sharing(share)
    b.set([s.query() for s in specs])
    b.run()
    _, status = b.fetch()
    assert (status == 0).all()
    for s, r in zip(specs, b.results_all()):
        s.check(r)


def test_batch_float_sums_outside_fixed_point_window(cuda):
    """Shared-table float sums are fixed point per work item, scaled from the item's first tile: values far from
    those magnitudes (lognormal with sigma 10, some negative, zeros) take the FP64 global path, and every sum stays
    within tolerance of the FP64 oracle; a chunk above 2^24 rows is rejected."""
    specs = []
    for i, (n, card) in enumerate([(400_000, 50), (300_000, 900)]):
        s = Spec(400 + i, np.int32, np.float32, n, card, ["sum", "avg", "min", "max", "count"])
        v = dg.lognormal_f32(400 + i, 5, n, 0.0, 10.0)
        v[::11] *= -1.0
        v[::7] = 0.0
        s.v = v
        s.dv = _dev(v)
        s.ref = oracle.groupby(s.k, v)
        specs.append(s)
    b = GroupByBatch(len(specs), 1 << 28, 1 << 26)
    b.set([s.query() for s in specs])
    for i, s in enumerate(specs):
        slots = 64
        while slots < 2 * (s.max_groups + 1):
            slots *= 2
        b.set_cfg(i, placement=capi.QDB_PLACE_SHARED, replicas=1, warps=12, rows_per_thread=2, chunk_rows=65536,
                  smem_slots=min(slots, 2048))
    with pytest.raises(QueryEngineError):
        b.set_cfg(0, chunk_rows=(1 << 24) + 64)
    b.run()
    _, status = b.fetch()
    assert (status == 0).all()
    for s, r in zip(specs, b.results_all()):
        s.check(r)
