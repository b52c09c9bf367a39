"""ORDER BY of GROUP BY results on the GPU (qdb_order_by_column / qdb_order_by / qdb_reorder, the replacement of
GPUOrderBy, qikkDB/QueryEngine/GPUCore/GPUOrderBy.cuh:88-195) against the oracle: the reference's GROUP BY +
ORDER BY known answers, then random multi-column orders with NULLs, ties, descending columns, IEEE edge values and
row counts around the 2048-row tile, OFFSET / LIMIT through the gather, and an ORDER BY of the 16.8M-group result
of the composite-key GROUP BY.  Permutations must equal the oracle's exactly (the sort is stable)."""
import json
import os

import numpy as np
import pytest
import torch

import oracle
from qikkdb_b200 import datagen as dg
from qikkdb_b200.groupby import GPUOrderBy, GroupByTable, order_by, pack_nullmask, unpack_nullmask

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_group_by_order_by_reference_kats(cuda):
    """DispatcherGroupByTests.cpp:1551-1588 through the operator mirror: GROUP BY on the GPU, then GPUOrderBy
    OrderByColumn + ReOrderByIdx over the result columns, as the dispatcher runs them."""
    with open(os.path.join(HERE, "golden", "reference_kats.json")) as f:
        cases = json.load(f)["order_by_cases"]
    for c in cases:
        k = np.asarray(c["keys"], dtype=np.int32)
        v = np.asarray(c["values"], dtype=np.int32)
        t = GroupByTable(["sum"], np.int32, np.int32, 1024)
        t.process([_dev(k)], _dev(v), len(k))
        keys, _, vals, n = t.results(["sum"])
        kd, sd = keys[0].torch(), vals["sum"][0].torch()
        ob = GPUOrderBy(n)
        idx = torch.empty(n, dtype=torch.int32, device="cuda")
        ob.OrderByColumn(idx, kd if c["order_by"] == "key" else sd, None, n,
                         GPUOrderBy.DESC if c["descending"] else GPUOrderBy.ASC)
        ok, os_ = torch.empty_like(kd), torch.empty_like(sd)
        GPUOrderBy.ReOrderByIdx(ok, idx, kd, n)
        GPUOrderBy.ReOrderByIdx(os_, idx, sd, n)
        got = [[int(a), int(b)] for a, b in zip(ok.cpu().numpy(), os_.cpu().numpy())]
        assert got == c["expected"], (c["name"], got)


def _random_cols(rng, n, spec):
    cols, nulls = [], []
    for dt, card, null_frac in spec:
        if dt in (np.float32, np.float64):
            x = rng.integers(-card, card, n).astype(dt) * dt(0.5)
            edge = np.array([0.0, -0.0, np.inf, -np.inf, np.finfo(dt).max, -np.finfo(dt).max], dtype=dt)
            pick = rng.random(n) < 0.05
            x[pick] = edge[rng.integers(0, len(edge), int(pick.sum()))]
        else:
            x = rng.integers(-card, card, n).astype(dt)
            pick = rng.random(n) < 0.01
            x[pick] = np.iinfo(dt).min
        cols.append(x)
        nulls.append(pack_nullmask(rng.random(n) < null_frac) if null_frac > 0 else None)
    return cols, nulls


@pytest.mark.parametrize("n", [0, 1, 2047, 2048, 2049, 100_003])
def test_order_by_random_against_oracle(cuda, n):
    rng = np.random.default_rng(n + 7)
    spec = [(np.int32, 50, 0.05), (np.float64, 1000, 0.0), (np.int64, 1 << 40, 0.1), (np.float32, 30, 0.02)]
    cols, nulls = _random_cols(rng, n, spec)
    desc = [False, True, False, True]
    exp = oracle.order_by(cols, desc, nulls)
    got = order_by([_dev(c) for c in cols], desc,
                   [None if x is None else _dev(x.view(np.int64)) for x in nulls]).cpu().numpy()
    assert (got == exp).all()


def test_order_by_offset_limit_and_nulls(cuda):
    rng = np.random.default_rng(11)
    n = 50_000
    v = rng.integers(-1000, 1000, n).astype(np.int32)
    nflags = rng.random(n) < 0.1
    nw = pack_nullmask(nflags)
    exp = oracle.order_by([v], [True], [nw])
    idx = order_by([_dev(v)], [True], [_dev(nw.view(np.int64))])
    offset, limit = 123, 4567
    out = torch.empty(limit, dtype=torch.int32, device="cuda")
    GPUOrderBy.ReOrderByIdx(out, idx, _dev(v), limit, offset=offset)
    assert (out.cpu().numpy() == v[exp[offset:offset + limit]]).all()
    onull = torch.zeros((limit + 63) // 64, dtype=torch.int64, device="cuda")
    GPUOrderBy.ReOrderNullValuesByIdx(onull, idx, _dev(nw.view(np.int64)), limit, offset=offset)
    assert (unpack_nullmask(onull.cpu().numpy(), limit) == nflags[exp[offset:offset + limit]]).all()


def test_order_by_composite_groupby_results(cuda):
    """ORDER BY SUM DESC, key0, key1 over the 16.8M groups of a 2^26-row composite-key GROUP BY."""
    n = 1 << 26
    a = dg.uniform_i32(43, 0, n, 0, 4095)
    b = dg.uniform_i32(43, 1, n, 0, 4095)
    v = dg.uniform_i64(43, 2, n, 0, (1 << 31) - 1)
    t = GroupByTable(["sum"], np.int32, np.int64, 1 << 24, n_key_cols=2)
    t.process([_dev(a), _dev(b)], _dev(v), n)
    keys, _, vals, g = t.results(["sum"])
    k0, k1, s = keys[0].torch(), keys[1].torch(), vals["sum"][0].torch()
    idx = order_by([s, k0, k1], [True, False, False]).cpu().numpy()
    exp = oracle.order_by([s.cpu().numpy(), k0.cpu().numpy(), k1.cpu().numpy()], [True, False, False])
    assert g > 10_000_000 and (idx == exp).all()
