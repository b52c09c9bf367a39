"""AAFL compressed column blocks on the GPU (qdb_aafl_compress / qdb_aafl_decompress / qdb_gb_process_aafl) against
the oracle's restatement of the reference's format (qikkDB/Compression/GPUCompression.cu, feathergpu AAFL), which
tests/test_oracle_kats.py pins to qikkDB_test/GPUCompressionTests.cpp.  Blocks are bit-exact; GROUP BY results over a
compressed key column equal the oracle's over the plain column (integers exact, float SUM/AVG within 1e-5)."""
import numpy as np
import pytest
import torch

import oracle
from gpu_compare import FLOAT_RTOL
from kat_util import compression_column, load_compression_kats
from qikkdb_b200 import _capi as capi
from qikkdb_b200.groupby import AaflBlock, FilterConditions, GroupByTable, make_pred, process_aafl

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _col(rng, dt, n, lo, hi):
    if np.dtype(dt).kind == "f":
        return rng.uniform(lo, hi, n).astype(dt)
    return rng.integers(lo, hi, n).astype(dt)


def test_aafl_reference_blocks(cuda):
    """The columns of GPUCompressionTests.cpp: the GPU compresses them byte for byte as the oracle does (so the
    asserted header words hold), leaves the same ones plain, and decompresses them to the column."""
    for c in load_compression_kats():
        v = compression_column(c["name"])
        want = oracle.aafl_compress(v)
        got = AaflBlock.compress(_dev(v))
        if want is None:
            assert got is None, c["name"]
            continue
        assert got is not None, c["name"]
        assert got.data.cpu().numpy().tobytes() == want.tobytes(), c["name"]
        blk = AaflBlock.from_host(want, v.min(), v.max())
        assert blk.decompress().cpu().numpy().tobytes() == v.tobytes(), c["name"]


@pytest.mark.parametrize("dt,lo,hi", [(np.int32, -3000, 70000), (np.int64, -(1 << 44), 1 << 20),
                                       (np.float32, 1.0, 3.0), (np.float32, -9.0, -2.0), (np.int32, 5, 6)])
def test_aafl_round_trip_ragged(cuda, dt, lo, hi):
    """Ragged row counts (partial last groups, word regions that start unaligned: rows/32 blocks of 9 metadata bytes),
    constant groups (0 bits), and the oracle's blocks decoded on the GPU."""
    rng = np.random.default_rng(21)
    for n in (33, 1025, 2047, 4097, 100_003, 1 << 20):
        v = _col(rng, dt, n, lo, hi)
        want = oracle.aafl_compress(v)
        got = AaflBlock.compress(_dev(v))
        assert (want is None) == (got is None), n
        if want is None:
            continue
        assert got.data.cpu().numpy().tobytes() == want.tobytes(), n
        out = AaflBlock.from_host(want, v.min(), v.max()).decompress()
        assert out.cpu().numpy().tobytes() == v.tobytes(), n


def test_aafl_malformed_block_is_rejected(cuda):
    """A position id pointing past the packed words is caught by the decoder's bounds check, not read."""
    v = np.arange(5000, dtype=np.int32)
    b = oracle.aafl_compress(v)
    bad = b.copy()
    bad.view(np.uint8)[24:32] = np.frombuffer(np.int64(1 << 40).tobytes(), dtype=np.uint8)  # group 0's position
    with pytest.raises(capi.QdbError) as e:
        AaflBlock.from_host(bad, v.min(), v.max()).decompress()
    assert e.value.code == capi.QDB_ERR_INVALID


def _groupby_compare(keys, vals, table, pred_np=None, aggs=("sum", "count", "min", "max", "avg")):
    r = oracle.groupby(keys, vals, pred=pred_np)
    g = table.results_numpy(list(aggs))
    assert g["n_groups"] == r["count"]
    order = np.argsort(g["keys"][0], kind="stable")
    kf = np.dtype(keys.dtype).kind == "f"
    if kf:
        assert np.array_equal(g["keys"][0][order].astype(np.float64), r["keys"][0])
    else:
        assert np.array_equal(g["keys"][0][order].astype(np.int64), r["keys"][0])
    vf = np.dtype(vals.dtype).kind == "f"
    for a in aggs:
        got = g[a][order]
        exp = r["cnt" if a == "count" else a]
        if vf and a in ("sum", "avg"):
            assert np.all(np.abs(got - exp) <= FLOAT_RTOL * np.maximum(np.abs(exp), 1.0)), a
        else:
            assert np.array_equal(got.astype(exp.dtype), exp), a


@pytest.mark.parametrize("kdt,n", [(np.int64, 1 << 22), (np.int32, (1 << 22) + 777), (np.int64, 1500),
                                   (np.float32, 1 << 21)])
def test_groupby_over_compressed_keys(cuda, kdt, n):
    """GROUP BY whose key column is an AAFL block: the fused fast pass (2^21-2^22 rows) and the decompress-first path
    (1500 rows), Zipf keys over 1M values with a filtered float value column."""
    from qikkdb_b200 import datagen as dg
    ranks = dg.zipf_i64(31, 0, n, 1_000_000, 1.1, map_keys=False)
    keys = (ranks * 3 - 7).astype(kdt) if np.dtype(kdt).kind != "f" else (1.0 + ranks / 4096.0).astype(kdt)
    vals = dg.lognormal_f32(31, 1, n, 2.0, 1.0)
    p = dg.uniform_f32(31, 2, n)
    blk = AaflBlock.compress(_dev(keys))
    assert blk is not None
    t = GroupByTable(["sum", "count", "min", "max", "avg"], kdt, np.float32, 1 << 20)
    pred = make_pred(_dev(p), FilterConditions.less, 0.5, np.float32)
    process_aafl(t, blk, _dev(vals), pred)
    _groupby_compare(keys, vals, t, pred_np=(p, FilterConditions.less, 0.5, np.float32, None))
    # the same block a second time accumulates into the same table
    process_aafl(t, blk, _dev(vals), pred)
    g = t.results_numpy(["count"])
    r = oracle.groupby(keys, vals, pred=(p, FilterConditions.less, 0.5, np.float32, None))
    assert int(g["count"].sum()) == 2 * int(r["cnt"].sum())


def test_groupby_over_compressed_keys_count_only_and_null_predicate(cuda):
    """A COUNT-only table (the fast pass without a value column) and a predicate with a NULL mask (the
    decompress-first path) over an AAFL key block."""
    from qikkdb_b200 import datagen as dg
    from qikkdb_b200.groupby import pack_nullmask
    n = (1 << 20) + 333
    keys = (dg.zipf_i64(41, 0, n, 50_000, 1.2, map_keys=False) - 25_000).astype(np.int32)
    blk = AaflBlock.compress(_dev(keys))
    t = GroupByTable(["count"], np.int32, None, 1 << 16)
    process_aafl(t, blk, None, None)
    g = t.results_numpy(["count"])
    r = oracle.groupby(keys)
    order = np.argsort(g["keys"][0], kind="stable")
    assert np.array_equal(g["keys"][0][order].astype(np.int64), r["keys"][0])
    assert np.array_equal(g["count"][order], r["cnt"])

    vals = dg.uniform_i64(41, 1, n, -(1 << 40), 1 << 40)
    p = dg.uniform_f32(41, 2, n)
    pn = np.random.default_rng(41).random(n) < 0.1
    t2 = GroupByTable(["sum", "count", "max"], np.int32, np.int64, 1 << 16)
    pred = make_pred(_dev(p), FilterConditions.greater, 0.3, np.float32, _dev(pack_nullmask(pn).view(np.int64)))
    process_aafl(t2, blk, _dev(vals), pred)
    _groupby_compare(keys, vals, t2, pred_np=(p, FilterConditions.greater, 0.3, np.float32, pack_nullmask(pn)),
                     aggs=("sum", "count", "max"))
