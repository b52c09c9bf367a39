"""The serving loop (qdb_server_*): queries submitted concurrently over shared device-resident columns are batched
together, and every query's result is the same as the oracle's (and the same as the query run alone): keys and
integer aggregates bit-exact, float SUM/AVG within FLOAT_RTOL.  Also: tables sized from the server's cardinality
estimate, resubmission after HASH_TABLE_FULL, admission against the table budget, and the open-loop driver."""
import threading

import numpy as np
import pytest
import torch

import oracle
from gpu_compare import compare
from qikkdb_b200 import _capi as capi
from qikkdb_b200 import datagen as dg
from qikkdb_b200.batch import AGG_ORDER, GroupByBatch, Query
from qikkdb_b200.groupby import FilterConditions
from qikkdb_b200.serve import Server, poisson_arrivals

pytestmark = pytest.mark.gpu

N = 1 << 20


@pytest.fixture(scope="module")
def columns(cuda):
    h = {"k32": dg.uniform_i32(500, 0, N, 0, (1 << 31) - 1), "k64": dg.uniform_i64(500, 1, N, 0, 1 << 62),
         "p": dg.uniform_f32(500, 2, N), "v": dg.lognormal_f32(500, 3, N, 2.0, 1.0),
         "vi": dg.uniform_i64(500, 4, N, -(1 << 40), 1 << 40), "v32": dg.uniform_i32(500, 5, N, -(1 << 20), 1 << 20)}
    d = {k: torch.from_numpy(a).cuda() for k, a in h.items()}
    return h, d


SHAPES = [("k32", "v", ["sum", "min", "max", "count"]), ("k64", "v", ["sum", "avg"]),
          ("k64", "vi", ["sum", "count", "max"]), ("k32", "vi", list(AGG_ORDER))]


def make_queries(cols, n_q, seed, max_groups_known=False, shapes=SHAPES):
    h, d = cols
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_q):
        kc, vc, aggs = shapes[i % len(shapes)]
        card = int(np.exp(rng.uniform(np.log(10), np.log(200_000))))
        sel = float(np.float32(rng.uniform(0.01, 1.0)))
        ek = np.fmod(h[kc], card)
        mg = 0
        if max_groups_known:
            mg = max(1, len(np.unique(ek[h["p"] < np.float32(sel)])))
        q = Query(d[kc], d[vc], aggs, mg, key_mod=card, pred=(d["p"], FilterConditions.less, sel, np.float32))
        ref = oracle.groupby(ek, h[vc], pred=(h["p"], FilterConditions.less, sel, np.float32, None))
        out.append((q, ref, h[vc].dtype.kind == "f"))
    return out


def check(res, ref, aggs, vf):
    g = dict(res)
    g["key_nulls"] = [np.zeros(g["n_groups"], bool)]
    for a in aggs:
        g[a + "_null"] = np.zeros(g["n_groups"], bool)
    return compare(g, ref, aggs, vf)


def test_server_concurrent_mix_matches_oracle(columns):
    qs = make_queries(columns, 40, 1)
    srv = Server(max_batch=8, in_flight=2, table_budget=1 << 30, result_budget=1 << 28)
    tickets = [None] * len(qs)

    def submitter(idx):
        for i in idx:
            tickets[i] = srv.submit(qs[i][0])

    ths = [threading.Thread(target=submitter, args=(range(j, len(qs), 4),)) for j in range(4)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    sizes = []
    for (q, ref, vf), t in zip(qs, tickets):
        r = srv.wait(t)
        assert r["status"] == 0
        sizes.append(r["batch_size"])
        check(r, ref, q.aggs, vf)
    st = srv.stats()
    assert st["completed"] == len(qs) and st["batches"] < len(qs)  # queries were batched together
    assert max(sizes) > 1
    srv.close()


def test_server_result_same_alone_and_in_mix(columns):
    """The same query alone (a batch of one, no shared scan) and in the server's mix gives the same keys and
    integer aggregates bit for bit and float aggregates within the tolerance."""
    qs = make_queries(columns, 12, 2, max_groups_known=True)
    srv = Server(max_batch=12, in_flight=1, table_budget=1 << 30, result_budget=1 << 28)
    tickets = [srv.submit(q) for q, _, _ in qs]
    mixed = [srv.wait(t) for t in tickets]
    srv.close()
    for (q, ref, vf), m in zip(qs, mixed):
        b = GroupByBatch(1, 1 << 28, 1 << 26)
        b.set_sharing(False)
        b.set([q])
        b.run()
        b.fetch()
        alone = b.results_all()[0]
        oa = np.argsort(alone["keys"][0])
        om = np.argsort(m["keys"][0])
        assert (alone["keys"][0][oa] == m["keys"][0][om]).all()
        for a in q.aggs:
            x, y = alone[a][oa], m[a][om]
            if vf and a in ("sum", "avg"):
                assert np.allclose(x, y, rtol=1e-5, atol=0), a
            else:
                assert (x == y).all(), a
        check(m, ref, q.aggs, vf)


def test_server_retries_when_table_overflows(columns):
    h, d = columns
    card = 5000
    ek = np.fmod(h["k32"], card)
    q = Query(d["k32"], d["vi"], ["sum", "count"], 100, key_mod=card)  # far too small: HASH_TABLE_FULL
    ref = oracle.groupby(ek, h["vi"])
    srv = Server(max_batch=4, in_flight=2, table_budget=1 << 28, result_budget=1 << 26)
    r = srv.wait(srv.submit(q))
    assert r["status"] == 0 and r["retries"] >= 1 and r["max_groups"] >= card
    check(r, ref, q.aggs, False)
    srv.close()


def test_server_rejects_query_over_budget(columns):
    h, d = columns
    srv = Server(max_batch=4, in_flight=2, table_budget=1 << 20, result_budget=1 << 26)
    r = srv.wait(srv.submit(Query(d["k64"], d["v"], ["sum"], 1 << 20)))
    assert r["status"] == capi.QDB_ERR_TOO_LARGE
    ok = Query(d["k32"], d["v"], ["sum"], 0, key_mod=10)
    r = srv.wait(srv.submit(ok))
    assert r["status"] == 0 and r["n_groups"] == 10
    srv.close()


def test_server_open_loop(columns):
    qs = make_queries(columns, 24, 3)
    srv = Server(max_batch=8, in_flight=2, table_budget=1 << 30, result_budget=1 << 28)
    lat, st, wall = srv.run_open_loop([q for q, _, _ in qs], poisson_arrivals(2000.0, len(qs), 7))
    assert (st == 0).all() and (lat > 0).all() and wall > 0
    assert srv.stats()["completed"] == len(qs)
    srv.close()


PLAIN_SHAPES = SHAPES + [("k64", "v32", list(AGG_ORDER)), ("k32", "v", list(AGG_ORDER))]


@pytest.mark.parametrize("route", [{"plain_rows": 1}, {"plain_rows": 0, "plain_groups": 50_000}])
def test_server_plain_route_matches_oracle(columns, route):
    """Queries routed through the single-query fast pass (every query by its row count, or those whose estimated
    tables reach 50K groups) give the oracle's results in the server's result words: int32 and int64 keys, int32 /
    int64 / float aggregates of every kind."""
    qs = make_queries(columns, 18, 11, shapes=PLAIN_SHAPES)
    srv = Server(max_batch=6, in_flight=2, table_budget=1 << 30, result_budget=1 << 28, **route)
    tickets = [srv.submit(q) for q, _, _ in qs]
    for (q, ref, vf), t in zip(qs, tickets):
        r = srv.wait(t)
        assert r["status"] == 0
        check(r, ref, q.aggs, vf)
    st = srv.stats()
    assert st["completed"] == len(qs)
    if route.get("plain_rows") == 1:
        assert st["plain_queries"] == len(qs) and st["batches"] == 0
    else:
        assert 0 < st["plain_queries"] < len(qs) and st["batches"] > 0
    srv.close()


def test_server_plain_route_off_batches_everything(columns):
    qs = make_queries(columns, 8, 12)
    srv = Server(max_batch=8, in_flight=2, table_budget=1 << 30, result_budget=1 << 28, plain_rows=0, plain_groups=0)
    for (q, ref, vf), t in zip(qs, [srv.submit(q) for q, _, _ in qs]):
        r = srv.wait(t)
        assert r["status"] == 0
        check(r, ref, q.aggs, vf)
    assert srv.stats()["plain_queries"] == 0
    srv.close()


def test_server_plain_route_retries_when_table_overflows(columns):
    """A plain-routed query whose table is far too small reports HASH_TABLE_FULL from the fast pass and is resubmitted
    with twice the table until it fits."""
    h, d = columns
    card = 70_000
    ek = np.fmod(h["k64"], card)
    q = Query(d["k64"], d["v32"], ["min", "sum", "count"], 1000, key_mod=card)
    ref = oracle.groupby(ek, h["v32"])
    srv = Server(max_batch=4, in_flight=2, table_budget=1 << 30, result_budget=1 << 28, plain_groups=1)
    r = srv.wait(srv.submit(q))
    assert r["status"] == 0 and r["retries"] >= 1 and r["max_groups"] >= card
    check(r, ref, q.aggs, False)
    assert srv.stats()["plain_queries"] == 1 + r["retries"]
    srv.close()


def test_server_plain_route_without_modulus(columns):
    """A query grouping by the key column itself (key_mod 0) on the single-query route: ProcessBlock over the column
    as it is, its table sized by the server's estimate of the key's distinct count."""
    h, d = columns
    n = 1 << 16
    keys = (h["k32"][:n] % 3000).astype(np.int64)
    kd = torch.from_numpy(keys).cuda()
    q = Query(kd, d["v32"][:n], ["min", "max", "sum", "count"], 0,
              pred=(d["p"][:n], FilterConditions.less, 0.5, np.float32))
    ref = oracle.groupby(keys, h["v32"][:n], pred=(h["p"][:n], FilterConditions.less, 0.5, np.float32, None))
    srv = Server(max_batch=4, in_flight=2, table_budget=1 << 28, result_budget=1 << 26, plain_rows=1)
    r = srv.wait(srv.submit(q))
    assert r["status"] == 0 and r["batch_size"] == 1
    check(r, ref, q.aggs, False)
    assert srv.stats()["plain_queries"] >= 1
    srv.close()
