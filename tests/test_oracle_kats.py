"""The oracle against every known-answer case transcribed from the reference's tests (CPU only)."""
import numpy as np
import pytest

import oracle
from kat_util import OPS, expected_map, kat_inputs, load_kats, result_map
from qikkdb_b200.groupby import pack_nullmask

CASES = load_kats()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_kat(case):
    keys, kn, vals, vn = kat_inputs(case)
    pred = None
    if case.get("pred"):
        p = case["pred"]
        pred = (np.asarray(p["col"], dtype=np.int32), OPS[p["op"]], p["const"], np.int32, None)
    r = oracle.groupby(keys if len(keys) > 1 else keys[0], vals,
                       key_nulls=[pack_nullmask(x) for x in kn] if kn is not None else None,
                       val_nulls=pack_nullmask(vn) if vn is not None else None, pred=pred, threads=4)
    agg = case["agg"]
    if "expected_groups" in case:
        assert r["count"] == case["expected_groups"]
        assert (r[agg] == case["expected_value_all"]).all()
        return
    col = {"sum": "sum", "min": "min", "max": "max", "avg": "avg", "count": "cnt"}.get(agg)
    values = r[col] if col else None
    vnull = None if agg in ("count", "none") else r["val_null"]
    got = result_map(r["keys"], r["key_nulls"], values, vnull)
    assert got == expected_map(case)


def test_oracle_threads_agree():
    rng = np.random.default_rng(5)
    k = rng.integers(0, 5000, 300_000).astype(np.int64)
    v = rng.standard_normal(300_000).astype(np.float32)
    a = oracle.groupby(k, v, threads=1)
    b = oracle.groupby(k, v, threads=8)
    assert a["count"] == b["count"] == len(np.unique(k))
    assert (a["keys"][0] == b["keys"][0]).all() and (a["cnt"] == b["cnt"]).all()
    np.testing.assert_allclose(a["sum"], b["sum"], rtol=1e-12, atol=1e-9)
    assert (a["min"] == b["min"]).all() and (a["max"] == b["max"]).all()


def test_oracle_int_sum_wraps_like_int32_atomics():
    k = np.zeros(3, dtype=np.int32)
    v = np.array([2**31 - 1, 5, 7], dtype=np.int32)
    r = oracle.groupby(k, v, threads=1)
    wrapped = (2**31 - 1 + 12) - 2**32  # int32 two's-complement wrap
    assert r["sum"][0] == wrapped
    # AVG divides the wrapped sum with C++ truncation toward zero (GPUBinary<div> on the int32 sum)
    assert r["avg"][0] == int(wrapped / 3)


def test_oracle_filter_and_compaction():
    rng = np.random.default_rng(1)
    a = rng.integers(-100, 100, 1000).astype(np.int32)
    b = rng.standard_normal(1000).astype(np.float32) * 50
    for op, f in [(0, np.greater), (1, np.greater_equal), (2, np.less), (3, np.less_equal), (4, np.equal),
                  (5, np.not_equal)]:
        m = oracle.filter_mask(op, a, b)
        assert (m.astype(bool) == f(a.astype(np.float32), b)).all()
        mc = oracle.filter_mask(op, a, np.int32(7))
        assert (mc.astype(bool) == f(a, 7)).all()
    m = (a > 0).astype(np.int8)
    out, _, c = oracle.compact(b, m)
    assert (out == b[a > 0]).all() and c == (a > 0).sum()
    assert (oracle.indexes(m) == np.nonzero(a > 0)[0]).all()
    assert (oracle.prefix_sum(m) == np.cumsum(m)).all()


def test_oracle_order_by_reference_kats():
    """GROUP BY + ORDER BY known answers (qikkDB_test/DispatcherGroupByTests.cpp:1551-1588): the oracle's GROUP BY
    result ordered by the oracle's ORDER BY equals the rows the reference's tests assert, in order."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")) as f:
        cases = json.load(f)["order_by_cases"]
    assert len(cases) == 2
    for c in cases:
        k = np.asarray(c["keys"], dtype=np.int32)
        v = np.asarray(c["values"], dtype=np.int32)
        r = oracle.groupby(k, v)
        keys = r["keys"][0].astype(np.int32)
        sums = r["sum"].astype(np.int32)
        by = keys if c["order_by"] == "key" else sums
        perm = oracle.order_by([by], [c["descending"]])
        got = [[int(keys[i]), int(sums[i])] for i in perm]
        assert got == c["expected"], (c["name"], got)


def test_oracle_order_by_semantics():
    """Ties keep input order; NULL rows order as lowest(T) (ascending first, descending last, tied with a real
    lowest(T)); IEEE values order by their bits (-0.0 before +0.0); the first column is most significant."""
    a = np.array([3, 1, 2, 1, 3, np.iinfo(np.int32).min], dtype=np.int32)
    nulls = np.zeros(1, dtype=np.uint64)
    nulls[0] = 1 << 2  # row 2 is NULL
    assert list(oracle.order_by([a], [False], [nulls])) == [2, 5, 1, 3, 0, 4]
    assert list(oracle.order_by([a], [True], [nulls])) == [0, 4, 1, 3, 2, 5]
    f = np.array([0.0, -0.0, -1.5, np.inf, -np.inf, 2.0], dtype=np.float32)
    assert list(oracle.order_by([f])) == [4, 2, 1, 0, 5, 3]
    b = np.array([5, 4, 3, 2, 1, 0], dtype=np.int64)
    assert list(oracle.order_by([np.array([1, 0, 1, 0, 1, 0], dtype=np.int32), b], [False, True])) == [1, 3, 5, 0, 2, 4]


def _string_kat_oracle(case):
    from kat_util import string_blocks
    keys, vals, vn, mask = [], [], [], []
    have_vals = case["blocks_values"] is not None
    for k, v, n, m in string_blocks(case):
        keys += k
        if have_vals:
            vals.append(v)
            vn.append(n if n is not None else np.zeros(len(k), dtype=bool))
        mask.append(m if m is not None else np.ones(len(k), dtype=np.int8))
    chars, ends = oracle.pack_strings(keys)
    kn = np.array([k is None for k in keys], dtype=bool)
    v = np.concatenate(vals) if have_vals else None
    vnul = np.concatenate(vn) if have_vals else None
    return oracle.groupby_string(chars, ends, v, key_nulls=pack_nullmask(kn) if kn.any() else None,
                                 val_nulls=pack_nullmask(vnul) if vnul is not None and vnul.any() else None,
                                 mask=np.concatenate(mask), threads=1)


def test_oracle_string_groupby_reference_kats():
    """GROUP BY over string keys (qikkDB_test/GPUGroupByTests.cu:474-516, DispatcherGroupByTests.cpp:1422-1467,
    DispatcherNullTests.cpp:1372-1750): the oracle's groups and aggregates equal what the reference's tests assert."""
    from kat_util import load_string_kats, string_expected
    cases = load_string_kats()
    assert len(cases) == 17
    for c in cases:
        r = _string_kat_oracle(c)
        col = {"sum": "sum", "min": "min", "max": "max", "avg": "avg", "count": "cnt"}[c["agg"]]
        got = {k: (None if (c["agg"] != "count" and s["val_null"]) else int(s[col])) for k, s in r.items()}
        assert got == string_expected(c), (c["name"], got)


def test_oracle_aafl_reference_kats():
    """AAFL blocks (qikkDB_test/GPUCompressionTests.cpp:79-233): the compressed header words the reference's tests
    assert, the blocks it leaves plain, and the round trip."""
    from kat_util import compression_column, load_compression_kats
    cases = load_compression_kats()
    assert len(cases) == 6
    for c in cases:
        v = compression_column(c["name"])
        b = oracle.aafl_compress(v)
        want = c.get("head32", c.get("head64"))
        if want == "plain":
            assert b is None, c["name"]
            continue
        head = b.view(np.int32)[:8] if "head32" in c else b.view(np.int64)[:8]
        assert head.tolist() == want, (c["name"], head.tolist())
        d = oracle.aafl_decompress(b, v.min(), v.max())
        assert d.tobytes() == v.tobytes(), c["name"]


def test_oracle_aafl_round_trips():
    """Ragged lengths, constant groups (bit length 0), full-width groups, negative ranges, offset 0 (a range wider
    than the type), and 64-bit values."""
    rng = np.random.default_rng(4)
    for n in (1, 31, 33, 1023, 1025, 2047, 2049, 5000, 70_001):
        for dt, lo, hi in ((np.int32, -50, 900), (np.int64, -(1 << 40), -(1 << 39)), (np.int32, 7, 8),
                           (np.int64, 0, 1 << 20)):
            v = rng.integers(lo, hi, n).astype(dt)
            b = oracle.aafl_compress(v)
            if b is None:
                continue
            assert oracle.aafl_header(b) == (n, len(b), (n + 31) // 32)
            assert np.array_equal(oracle.aafl_decompress(b, v.min(), v.max()), v)
    # a stated range wider than the type's positive half: offset 0, negative values take full width
    v = np.array([-5, 3, 2_000_000_000, -2_000_000_000] * 400, dtype=np.int32)
    assert oracle.aafl_compress(v) is None  # full width never shrinks the block
    v = np.zeros(4096, dtype=np.int64)
    b = oracle.aafl_compress(v)
    assert b is not None and np.array_equal(oracle.aafl_decompress(b, 0, 0), v)
