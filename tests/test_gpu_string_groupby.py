"""GROUP BY over string keys on the GPU (qdb_gbs_*) against the reference's known answers and the oracle.

The known answers are the reference's own string GROUP BY tests (qikkDB_test/GPUGroupByTests.cu:474-516,
DispatcherGroupByTests.cpp:1422-1467, DispatcherNullTests.cpp:1372-1750), run block by block through
GPUGroupBy<AGG, O, std::string, V> as those tests do.  Random cases compare every aggregate with the oracle:
integers bit-exact, float SUM/AVG within 1e-5 relative of the FP64 oracle.
"""
import numpy as np
import pytest
import torch

import oracle
from kat_util import load_string_kats, string_blocks, string_expected
from qikkdb_b200.groupby import (GPU_HASH_TABLE_FULL, GPUGroupBy, GPUString, QueryEngineError, StringGroupByTable,
                                 pack_nullmask)

pytestmark = pytest.mark.gpu

STRING_CASES = load_string_kats()
AGGS = ["min", "max", "sum", "avg", "count"]


def _dev(x):
    return None if x is None else torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("case", STRING_CASES, ids=[c["name"] for c in STRING_CASES])
def test_string_groupby_reference_kat(case):
    agg = case["agg"]
    have_vals = case["blocks_values"] is not None
    O = np.int64 if agg == "count" else np.int32
    gb = GPUGroupBy(agg, O, str, np.int32 if have_vals else None, 8)
    for keys, vals, vn, mask in string_blocks(case):
        kn = np.array([k is None for k in keys], dtype=bool)
        gs = GPUString.from_strings(keys)
        if mask is not None:
            # WHERE: the block's mask feeds the operator like the reconstructed block does
            gb.table.process(gs, _dev(vals), len(keys), _dev(pack_nullmask(kn)) if kn.any() else None,
                             _dev(pack_nullmask(vn)) if vn is not None else None, mask=_dev(mask))
        else:
            gb.ProcessBlock(gs, _dev(vals), len(keys), _dev(pack_nullmask(kn)) if kn.any() else None,
                            _dev(pack_nullmask(vn)) if vn is not None else None)
    got = gb.table.results_host()
    got = {k: v[agg] for k, v in got.items()}
    assert got == string_expected(case)
    outKeys, outValues, n, _, _ = gb.GetResults()
    assert n == len(string_expected(case))
    assert sorted(outKeys.to_strings()) == sorted(k if k is not None else b"" for k in string_expected(case))


def _vocab(rng, n_distinct, max_len):
    """n_distinct distinct byte strings: lengths 0..max_len, bytes 0..255 (NUL included)."""
    out, seen = [], set()
    while len(out) < n_distinct:
        ln = int(rng.integers(0, max_len + 1))
        s = rng.integers(0, 256, ln, dtype=np.uint8).tobytes()
        if s not in seen:
            seen.add(s)
            out.append(s)
    return out


def _check_against_oracle(tab, chars, ends, vals, kn, vn, mask, vdt):
    r = oracle.groupby_string(chars, ends, vals, key_nulls=kn, val_nulls=vn, mask=mask)
    got = tab.results_host()
    assert set(got) == set(r)
    fl = np.dtype(vdt).kind == "f"
    for k, st in r.items():
        g = got[k]
        assert g["count"] == st["cnt"], k
        if st["val_null"]:
            assert g["min"] is None and g["max"] is None and g["sum"] is None and g["avg"] is None
            continue
        if fl:
            assert g["min"] == st["min"] and g["max"] == st["max"], k
            for a in ("sum", "avg"):
                assert abs(g[a] - st[a]) <= 1e-5 * max(1.0, abs(st[a])), (k, a, g[a], st[a])
        else:
            for a in ("min", "max", "sum", "avg"):
                assert g[a] == st[a], (k, a, g[a], st[a])


@pytest.mark.parametrize("vdt", [np.int32, np.int64, np.float32, np.float64])
def test_string_groupby_random_matches_oracle(vdt):
    rng = np.random.default_rng(11)
    vocab = _vocab(rng, 20_000, 40)
    n = 1 << 20
    pick = np.minimum(rng.zipf(1.2, n) - 1, len(vocab) - 1)
    keys = [vocab[i] for i in pick]
    chars, ends = oracle.pack_strings(keys)
    if np.dtype(vdt).kind == "f":
        vals = rng.lognormal(2.0, 1.0, n).astype(vdt)
    else:
        vals = rng.integers(-(1 << 30), 1 << 30, n).astype(vdt)
    kn_f = rng.random(n) < 0.01
    vn_f = rng.random(n) < 0.05
    mask = (rng.random(n) < 0.7).astype(np.int8)
    kn, vn = pack_nullmask(kn_f), pack_nullmask(vn_f)
    tab = StringGroupByTable(AGGS, vdt, 40_000)
    # four blocks, each through its own ProcessBlock
    step = n // 4
    for b in range(0, n, step):
        e = b + step
        cb = chars[(ends[b - 1] if b else 0):ends[e - 1]]
        eb = ends[b:e] - (ends[b - 1] if b else 0)
        tab.process(GPUString(_dev(cb), _dev(eb)), _dev(vals[b:e]), step, _dev(pack_nullmask(kn_f[b:e])),
                    _dev(pack_nullmask(vn_f[b:e])), mask=_dev(mask[b:e]))
    _check_against_oracle(tab, chars, ends, vals, kn, vn, mask, vdt)


def test_string_groupby_high_cardinality():
    """1M distinct keys over 4M rows, keys of every length 0..24 (word and partial-word tails)."""
    rng = np.random.default_rng(3)
    n, d = 1 << 22, 1 << 20
    ids = rng.integers(0, d, n)
    keys = [b"k%07x" % i + b"#" * (i % 17) for i in ids]
    chars, ends = oracle.pack_strings(keys)
    vals = rng.integers(-1000, 1000, n).astype(np.int64)
    tab = StringGroupByTable(AGGS, np.int64, d)
    tab.process(GPUString(_dev(chars), _dev(ends)), _dev(vals))
    _check_against_oracle(tab, chars, ends, vals, None, None, None, np.int64)


def test_string_groupby_near_keys_are_distinct():
    """Prefixes of each other, keys that differ only past a word boundary, embedded NULs, and the empty string."""
    base = [b"", b"a", b"aa", b"aaaaaaa", b"aaaaaaaa", b"aaaaaaaaa", b"aaaaaaab", b"aaaaaaaab", b"\x00", b"\x00\x00",
            b"a\x00", b"\x00a", b"abcdefghijklmnop", b"abcdefghijklmnoq", b"bbcdefghijklmnop"]
    keys = base * 50
    vals = np.arange(len(keys), dtype=np.int32)
    chars, ends = oracle.pack_strings(keys)
    tab = StringGroupByTable(AGGS, np.int32, 64)
    tab.process(GPUString(_dev(chars), _dev(ends)), _dev(vals))
    got = tab.results_host()
    assert set(got) == set(base)
    for i, k in enumerate(base):
        idx = np.arange(i, len(keys), len(base))
        assert got[k]["count"] == 50 and got[k]["sum"] == int(idx.sum()) and got[k]["min"] == i


def test_string_groupby_long_keys_use_the_arena():
    """Keys of 5..195 bytes (inline words and arena words), many sharing long prefixes, against the oracle."""
    rng = np.random.default_rng(8)
    base = [b"p" * int(L) + b"%05d" % i for i, L in enumerate(rng.integers(0, 190, 3000))]
    n = 200_000
    keys = [base[i] for i in rng.integers(0, len(base), n)]
    chars, ends = oracle.pack_strings(keys)
    vals = rng.integers(-100, 100, n).astype(np.int32)
    tab = StringGroupByTable(AGGS, np.int32, 4096, max_key_bytes=4096 * 200)
    tab.process(GPUString(_dev(chars), _dev(ends)), _dev(vals))
    _check_against_oracle(tab, chars, ends, vals, None, None, None, np.int32)


def test_string_groupby_unaligned_character_buffer():
    """A character buffer that starts at an odd address (a slice of a larger buffer)."""
    keys = [b"alpha", b"beta", b"", b"gamma-delta-epsilon-zeta-eta", b"beta", b"alpha"] * 1000
    chars, ends = oracle.pack_strings(keys)
    dpad = _dev(np.concatenate([np.zeros(3, dtype=np.uint8), chars]))
    vals = np.arange(len(keys), dtype=np.int32)
    tab = StringGroupByTable(AGGS, np.int32, 16)
    tab.process(GPUString(dpad[3:], _dev(ends)), _dev(vals))
    _check_against_oracle(tab, chars, ends, vals, None, None, None, np.int32)


def test_string_groupby_count_rows_without_values():
    keys = ["x", "y", None, "x", None, "z", "x"]
    chars, ends = oracle.pack_strings(keys)
    kn = pack_nullmask(np.array([k is None for k in keys]))
    tab = StringGroupByTable(["count"], None, 8)
    tab.process(GPUString(_dev(chars), _dev(ends)), None, key_nulls=_dev(kn))
    assert {k: v["count"] for k, v in tab.results_host().items()} == {b"x": 3, b"y": 1, b"z": 1, None: 2}


def test_string_groupby_table_full_and_arena_full():
    keys = [b"key%d" % i for i in range(1000)]
    chars, ends = oracle.pack_strings(keys)
    vals = np.ones(len(keys), dtype=np.int32)
    tab = StringGroupByTable(["sum"], np.int32, 100)
    with pytest.raises(QueryEngineError) as e:
        tab.process(GPUString(_dev(chars), _dev(ends)), _dev(vals))
    assert e.value.code == GPU_HASH_TABLE_FULL
    # keys longer than the 24 bytes a slot keeps inline need the arena: 64 bytes of it hold four 16-byte tails
    long_keys = [b"%040d" % i for i in range(10)]
    lc, le = oracle.pack_strings(long_keys)
    tab2 = StringGroupByTable(["sum"], np.int32, 2000, max_key_bytes=64)
    with pytest.raises(QueryEngineError) as e:
        tab2.process(GPUString(_dev(lc), _dev(le)), _dev(np.ones(10, dtype=np.int32)))
    assert e.value.code == GPU_HASH_TABLE_FULL
    # the same keys fit a table sized for them
    tab3 = StringGroupByTable(["sum"], np.int32, 1000)
    tab3.process(GPUString(_dev(chars), _dev(ends)), _dev(vals))
    assert len(tab3.results_host()) == 1000


def test_string_groupby_empty_and_reset():
    tab = StringGroupByTable(AGGS, np.float32, 16)
    empty = GPUString(torch.zeros(0, dtype=torch.uint8, device="cuda"), torch.zeros(0, dtype=torch.int64, device="cuda"))
    tab.process(empty, torch.zeros(0, dtype=torch.float32, device="cuda"), 0)
    assert tab.results_host() == {}
    chars, ends = oracle.pack_strings(["a", "b", "a"])
    tab.process(GPUString(_dev(chars), _dev(ends)), _dev(np.array([1.5, 2.0, 0.5], dtype=np.float32)))
    assert tab.results_host()[b"a"]["sum"] == 2.0
    tab.reset()
    assert tab.results_host() == {}


def test_string_tables_merge_like_getresults_over_gpus():
    """Two tables over the two halves of the rows (NULL keys and NULL values included), merged with
    qdb_gbs_export + qdb_gbs_merge_exported, equal the oracle over all rows: the per-GPU partial tables that
    GetResults(..., tables) combines (GPUGroupByString.cuh:565-785)."""
    rng = np.random.default_rng(17)
    vocab = _vocab(rng, 3000, 30)
    n = 200_000
    keys = [vocab[i] for i in np.minimum(rng.zipf(1.3, n) - 1, len(vocab) - 1)]
    chars, ends = oracle.pack_strings(keys)
    vals = rng.integers(-10_000, 10_000, n).astype(np.int64)
    kn_f = rng.random(n) < 0.02
    vn_f = rng.random(n) < 0.05
    half = n // 2
    ta = StringGroupByTable(AGGS, np.int64, 4096)
    tb = StringGroupByTable(AGGS, np.int64, 4096)
    for t, b0, b1 in ((ta, 0, half), (tb, half, n)):
        c0 = int(ends[b0 - 1]) if b0 else 0
        t.process(GPUString(_dev(chars[c0:int(ends[b1 - 1])]), _dev(ends[b0:b1] - c0)), _dev(vals[b0:b1]), b1 - b0,
                  _dev(pack_nullmask(kn_f[b0:b1])), _dev(pack_nullmask(vn_f[b0:b1])))
    ta.merge_from(tb)
    _check_against_oracle(ta, chars, ends, vals, pack_nullmask(kn_f), pack_nullmask(vn_f), None, np.int64)
