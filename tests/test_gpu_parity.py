"""GPU GROUP BY against the oracle on seeded inputs: the workload shapes at oracle-friendly sizes, every key and
value type, NULLs, predicates and masks, both table placements, and the edge cases of the reference's tests."""
import numpy as np
import pytest
import torch

import oracle
from gpu_compare import FLOAT_RTOL, compare
from qikkdb_b200 import datagen as dg
from qikkdb_b200.groupby import (GPU_HASH_TABLE_FULL, FilterConditions, GroupByTable, QueryEngineError,
                                 device_nullmask, make_pred, pack_nullmask)

pytestmark = pytest.mark.gpu
ALL = ["min", "max", "sum", "avg", "count"]


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_both(keys, vals, aggs, max_groups, placement=0, key_nulls=None, val_nulls=None, pred=None, mask=None,
             val_is_float=False, key_is_float=False, blocks=1):
    """Runs the GPU table (optionally over several ProcessBlock calls) and the oracle; compares."""
    keys = keys if isinstance(keys, list) else [keys]
    n = len(keys[0])
    t = GroupByTable(aggs, keys[0].dtype, vals.dtype if vals is not None else None, max_groups, len(keys), placement)
    bounds = np.linspace(0, n, blocks + 1).astype(np.int64)
    for b0, b1 in zip(bounds[:-1], bounds[1:]):
        if b1 == b0:
            continue
        kn = [device_nullmask(x[b0:b1]) for x in key_nulls] if key_nulls is not None else None
        p = None
        if pred is not None:
            pcol, op, const, cdt, pnull = pred
            p = make_pred(_dev(pcol[b0:b1]), op, const, cdt, device_nullmask(pnull[b0:b1]) if pnull is not None else None)
        t.process([_dev(k[b0:b1]) for k in keys], _dev(vals[b0:b1]) if vals is not None else None, int(b1 - b0), kn,
                  device_nullmask(val_nulls[b0:b1]) if val_nulls is not None else None, pred=p,
                  mask=_dev(mask[b0:b1]) if mask is not None else None)
    g = t.results_numpy()
    opred = None
    if pred is not None:
        pcol, op, const, cdt, pnull = pred
        opred = (pcol, op, const, cdt, pack_nullmask(pnull) if pnull is not None else None)
    r = oracle.groupby(keys if len(keys) > 1 else keys[0], vals,
                       key_nulls=[pack_nullmask(x) for x in key_nulls] if key_nulls is not None else None,
                       val_nulls=pack_nullmask(val_nulls) if val_nulls is not None else None, pred=opred, mask=mask)
    return compare(g, r, aggs, val_is_float, key_is_float), g, r


@pytest.mark.parametrize("placement", [0, 1, 2])
def test_plain_groupby_1m_int32(cuda, placement):
    """Plain GROUP BY, one block: 1M rows, int32 key in [0,1000), int32 value in [-1000,1000]; SUM, MIN, MAX,
    COUNT (and AVG) in one fused table; bit-exact."""
    n = 1 << 20
    k = dg.uniform_i32(11, 0, n, 0, 999)
    v = dg.uniform_i32(11, 1, n, -1000, 1000)
    run_both(k, v, ALL, 1000, placement)


@pytest.mark.parametrize("placement", [0, 2])
def test_filtered_zipf_int64_float(cuda, placement):
    """Filtered GROUP BY shape at 4M rows: f32 predicate p < 0.5, int64 Zipf(1.1) keys over 1M ranks, f32
    lognormal(2, 1) values; SUM and AVG within 1e-5 relative of FP64."""
    n = 1 << 22
    p = dg.uniform_f32(21, 0, n)
    k = dg.zipf_i64(21, 1, n, 1_000_000, 1.1)
    v = dg.lognormal_f32(21, 2, n, 2.0, 1.0)
    rel, g, _ = run_both(k, v, ["sum", "avg", "count"], 1 << 20, placement,
                         pred=(p, FilterConditions.less, 0.5, np.float32, None), val_is_float=True)
    assert rel <= FLOAT_RTOL
    print(f"max relative error SUM/AVG: {rel:.3e} over {g['n_groups']} groups")


def test_composite_high_cardinality(cuda):
    """Composite (int32, int32) keys uniform over 4096 x 4096, int64 values in [0, 2^31); SUM/COUNT/MAX exact."""
    n = 1 << 23
    a = dg.uniform_i32(31, 0, n, 0, 4095)
    b = dg.uniform_i32(31, 1, n, 0, 4095)
    v = dg.uniform_i64(31, 2, n, 0, (1 << 31) - 1)
    run_both([a, b], v, ["sum", "count", "max"], 1 << 23)


KT = [np.int32, np.int64, np.float32, np.float64]


@pytest.mark.parametrize("kt", KT, ids=lambda t: np.dtype(t).name)
@pytest.mark.parametrize("vt", KT, ids=lambda t: np.dtype(t).name)
def test_type_matrix_with_nulls(cuda, kt, vt):
    rng = np.random.default_rng(hash((np.dtype(kt).name, np.dtype(vt).name)) & 0xffff)
    n = 50_000 + 3  # not a multiple of 4: exercises the tail
    k = rng.integers(-300, 300, n).astype(kt)
    if np.dtype(vt).kind == "f":
        v = (rng.random(n) * 1000).astype(vt)
    else:
        v = rng.integers(-(1 << 20), 1 << 20, n).astype(vt)
    kn = rng.random(n) < 0.05
    vn = rng.random(n) < 0.1
    for placement in (1, 2):
        run_both(k, v, ALL, 1024, placement, key_nulls=[kn], val_nulls=vn, val_is_float=np.dtype(vt).kind == "f",
                 key_is_float=np.dtype(kt).kind == "f")


@pytest.mark.parametrize("ptype", [np.int32, np.int64, np.float32, np.float64], ids=lambda t: np.dtype(t).name)
@pytest.mark.parametrize("op", range(6))
def test_predicate_types_and_ops(cuda, ptype, op):
    rng = np.random.default_rng(op * 7 + np.dtype(ptype).itemsize)
    n = 30_001
    k = rng.integers(0, 50, n).astype(np.int32)
    v = rng.integers(-100, 100, n).astype(np.int64)
    pc = (rng.integers(-5, 5, n)).astype(ptype)
    pn = rng.random(n) < 0.1
    const, cdt = (1.5, np.float64) if op % 2 else (1, np.int32)
    run_both(k, v, ALL, 64, 0, pred=(pc, op, const, cdt, pn))


def test_mask_and_predicate_combined_multiblock(cuda):
    rng = np.random.default_rng(3)
    n = 200_000
    k = rng.integers(0, 5000, n).astype(np.int64)
    v = rng.integers(-1000, 1000, n).astype(np.int32)
    m = (rng.random(n) < 0.7).astype(np.int8)
    pc = rng.random(n).astype(np.float32)
    run_both(k, v, ALL, 8192, 0, pred=(pc, FilterConditions.greaterEqual, 0.25, np.float32, None), mask=m, blocks=7)


def test_escape_and_extreme_keys(cuda):
    """INT64_MIN (the empty-slot marker) and INT32_MIN keys are ordinary groups here."""
    k = np.array([np.iinfo(np.int64).min, 5, np.iinfo(np.int64).min, -1, np.iinfo(np.int64).max, 0, 5],
                 dtype=np.int64)
    v = np.arange(7, dtype=np.int32)
    run_both(k, v, ALL, 16, 1)
    run_both(k, v, ALL, 16, 2)
    a = np.array([np.iinfo(np.int32).min, np.iinfo(np.int32).min, 3, 3], dtype=np.int32)
    b = np.array([0, 0, 0, np.iinfo(np.int32).min], dtype=np.int32)
    run_both([a, b], np.arange(4, dtype=np.int64), ALL, 16)


def test_float_keys_negative_zero(cuda):
    k = np.array([0.0, -0.0, 1.5, -1.5, 1.5, -0.0], dtype=np.float32)
    v = np.arange(6, dtype=np.float64)
    run_both(k, v, ALL, 16, 0, val_is_float=True, key_is_float=True)


def test_empty_and_all_filtered(cuda):
    t = GroupByTable(["sum"], np.int32, np.int32, 16)
    r = t.results_numpy()
    assert r["n_groups"] == 0
    k = np.arange(100, dtype=np.int32)
    run_both(k, k.copy(), ALL, 128, 0, mask=np.zeros(100, dtype=np.int8))


def test_hash_table_full_at_capacity_plus_one(cuda):
    for placement in (1, 2):
        cap = 1000
        t = GroupByTable(["count"], np.int32, np.int32, cap, 1, placement)
        k = np.arange(cap, dtype=np.int32)
        t.process([_dev(k)], _dev(k), cap)  # exactly full: fine
        assert t.group_count() == cap
        with pytest.raises(QueryEngineError) as e:
            t.process([_dev(np.array([cap], dtype=np.int32))], _dev(np.zeros(1, dtype=np.int32)), 1)
        assert e.value.code == GPU_HASH_TABLE_FULL


def test_unaligned_columns(cuda):
    rng = np.random.default_rng(9)
    n = 10_001
    kbig = _dev(rng.integers(0, 100, n + 1).astype(np.int32))
    vbig = _dev(rng.integers(0, 100, n + 1).astype(np.int32))
    t = GroupByTable(ALL, np.int32, np.int32, 128)
    t.process([kbig[1:]], vbig[1:], n)  # 4-byte offset: scalar load path
    r = oracle.groupby(kbig[1:].cpu().numpy(), vbig[1:].cpu().numpy())
    compare(t.results_numpy(), r, ALL, False)


def test_partial_export_merge_roundtrip(cuda):
    """Three row shards -> three tables -> export bucketed by owner -> merge per owner: the union of the owners'
    results equals one GROUP BY over all rows (the merge step of a multi-GPU GROUP BY, run on one GPU)."""
    from qikkdb_b200.dist import export_partitioned, merge_partial
    rng = np.random.default_rng(4)
    n = 300_000
    k = rng.integers(0, 20_000, n).astype(np.int64)
    v = (rng.random(n) * 10).astype(np.float32)
    kn = rng.random(n) < 0.01
    shards = np.array_split(np.arange(n), 3)
    owners = [GroupByTable(ALL, np.int64, np.float32, 1 << 15) for _ in range(2)]
    for idx in shards:
        t = GroupByTable(ALL, np.int64, np.float32, 1 << 15)
        t.process([_dev(k[idx])], _dev(v[idx]), len(idx), [device_nullmask(kn[idx])])
        parts = export_partitioned(t, 2)
        for o, part in zip(owners, parts):
            merge_partial(o, part)
    res = [o.results_numpy() for o in owners]
    g = {"n_groups": sum(r["n_groups"] for r in res), "keys": [np.concatenate([r["keys"][0] for r in res])],
         "key_nulls": [np.concatenate([r["key_nulls"][0] for r in res])]}
    for a in ALL:
        g[a] = np.concatenate([r[a] for r in res])
        g[a + "_null"] = np.concatenate([r[a + "_null"] for r in res])
    ref = oracle.groupby(k, v, key_nulls=[pack_nullmask(kn)])
    compare(g, ref, ALL, True)
