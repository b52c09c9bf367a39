"""Scalar aggregation (qdb_scalar_*, the replacement of GPUAggregation::col, qikkDB/QueryEngine/GPUCore/
GPUAggregation.cuh:15-37) against the oracle (a GROUP BY whose keys are all equal has one group: the scalar result),
over value types, a predicate with NULLs, NULL values, several blocks accumulated and an empty selection; and the
block skipping of GpuSqlDispatcher::WhereEvaluation (qdb_pred_block_may_pass) against the rows themselves."""
import numpy as np
import pytest
import torch

import oracle
from gpu_compare import FLOAT_RTOL
from qikkdb_b200 import datagen as dg
from qikkdb_b200.groupby import (FilterConditions, GPUAggregation, ScalarAggregate, block_may_pass, make_pred,
                                 pack_nullmask)

pytestmark = pytest.mark.gpu
AGGS = ["sum", "min", "max", "count", "avg"]


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("vt", [np.int32, np.int64, np.float32, np.float64], ids=lambda t: np.dtype(t).name)
def test_scalar_against_oracle(cuda, vt):
    rng = np.random.default_rng(5 + np.dtype(vt).itemsize)
    n = 3_000_001
    if np.dtype(vt).kind == "f":
        v = (rng.standard_normal(n) * 1000).astype(vt)
    else:
        v = rng.integers(np.iinfo(vt).min // 2, np.iinfo(vt).max // 2, n, dtype=np.int64).astype(vt)
    p = dg.uniform_f32(9, 0, n)
    pn = rng.random(n) < 0.03
    vn = rng.random(n) < 0.05
    pw, vw = pack_nullmask(pn), pack_nullmask(vn)
    acc = ScalarAggregate(vt)
    bounds = [0, 1_000_000, 2_500_000, n]  # three blocks, as the dispatcher feeds them
    for b0, b1 in zip(bounds[:-1], bounds[1:]):
        pred = make_pred(_dev(p[b0:b1]), FilterConditions.less, 0.4, np.float32,
                         _dev(pack_nullmask(pn[b0:b1]).view(np.int64)))
        acc.process(_dev(v[b0:b1]), b1 - b0, _dev(pack_nullmask(vn[b0:b1]).view(np.int64)), pred)
    r = oracle.groupby(np.zeros(n, np.int32), v, val_nulls=vw, pred=(p, FilterConditions.less, 0.4, np.float32, pw))
    assert r["count"] == 1
    for a in AGGS:
        got = acc.result(a)
        exp = r["cnt" if a == "count" else a][0]
        if np.dtype(vt).kind == "f" and a in ("sum", "avg"):
            assert abs(got - exp) <= FLOAT_RTOL * abs(exp), a
        else:
            assert got == exp, (a, got, exp)


def test_scalar_empty_selection_and_column(cuda):
    v = _dev(np.arange(1000, dtype=np.int32))
    p = _dev(np.zeros(1000, dtype=np.float32))
    acc = ScalarAggregate(np.int32)
    acc.process(v, 1000, pred=make_pred(p, FilterConditions.greater, 1.0, np.float32))
    assert [acc.result(a) for a in AGGS] == [None, None, None, 0, None]
    assert GPUAggregation.col("count", v, 0) == 0 and GPUAggregation.col("max", v, 0) is None
    assert GPUAggregation.col("max", v, 1000) == 999 and GPUAggregation.col("sum", v, 1000) == 499500


@pytest.mark.parametrize("op", [FilterConditions.less, FilterConditions.greaterEqual, FilterConditions.equal,
                                FilterConditions.notEqual])
def test_block_skipping_agrees_with_rows(cuda, op):
    """A block is skippable exactly when no row of it passes (the predicate's interval misses [min, max])."""
    rng = np.random.default_rng(op)
    for _ in range(200):
        lo = int(rng.integers(-50, 50))
        block = rng.integers(lo, lo + int(rng.integers(0, 20)) + 1, 64).astype(np.int32)
        c = int(rng.integers(-60, 60))
        passing = {FilterConditions.less: block < c, FilterConditions.greaterEqual: block >= c,
                   FilterConditions.equal: block == c, FilterConditions.notEqual: block != c}[op]
        may = block_may_pass(np.int32, op, c, np.int32, block.min(), block.max())
        if not may:
            assert not passing.any()
        if op != FilterConditions.equal:  # == with a value strictly inside [min, max] may still miss every row
            assert may == bool(passing.any())
