"""qdb_gb_process_host (host columns streamed to the GPU in chunks, the copies overlapped with the aggregation)
against the oracle: pageable numpy and pinned torch columns, a predicate, NULL masks, a ragged last chunk, and a
table large enough to use the spill."""
import numpy as np
import pytest
import torch

import oracle
from gpu_compare import FLOAT_RTOL, compare
from qikkdb_b200 import datagen as dg
from qikkdb_b200.groupby import FilterConditions, GroupByTable, pack_nullmask

pytestmark = pytest.mark.gpu
ALL = ["sum", "avg", "count", "min", "max"]


def test_host_columns_pageable_with_predicate_and_spill(cuda):
    n = (1 << 20) + 777  # a ragged last chunk
    k = dg.zipf_i64(101, 0, n, 300_000, 1.1)
    v = dg.lognormal_f32(101, 1, n, 2.0, 1.0)
    p = dg.uniform_f32(101, 2, n)
    t = GroupByTable(ALL, np.int64, np.float32, 1 << 19)
    t.process_host([k], v, pred=(p, FilterConditions.less, 0.4, np.float32), chunk_rows=1 << 16)
    torch.cuda.synchronize()
    t.check()
    r = oracle.groupby(k, v, pred=(p, FilterConditions.less, 0.4, np.float32, None))
    assert compare(t.results_numpy(), r, ALL, True) <= FLOAT_RTOL


def test_host_columns_pinned_with_nulls(cuda):
    rng = np.random.default_rng(102)
    n = 300_001
    k = torch.from_numpy(rng.integers(0, 5_000, n).astype(np.int32)).pin_memory()
    v = torch.from_numpy(rng.integers(-(1 << 30), 1 << 30, n).astype(np.int64)).pin_memory()
    kn = rng.random(n) < 0.02
    vn = rng.random(n) < 0.05
    kw, vw = pack_nullmask(kn), pack_nullmask(vn)
    t = GroupByTable(ALL, np.int32, np.int64, 8192)
    t.process_host([k], v, key_nulls=[kw], value_nulls=vw, chunk_rows=1 << 15)
    torch.cuda.synchronize()
    t.check()
    r = oracle.groupby(k.numpy(), v.numpy(), key_nulls=[kw], val_nulls=vw)
    compare(t.results_numpy(), r, ALL, False)


def test_host_columns_back_to_back_on_two_streams(cuda):
    # The staging buffers are shared by every call of a thread: a call on a second stream must not overwrite a
    # buffer that the first stream's aggregation still reads.
    n = (1 << 21) + 4099
    k1 = dg.zipf_i64(103, 0, n, 400_000, 1.1)
    v1 = dg.lognormal_f32(103, 1, n, 2.0, 1.0)
    k2 = dg.zipf_i64(104, 0, n, 50_000, 1.3)
    v2 = dg.lognormal_f32(104, 1, n, 1.0, 2.0)
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    ta = GroupByTable(ALL, np.int64, np.float32, 1 << 19)
    tb = GroupByTable(ALL, np.int64, np.float32, 1 << 16)
    torch.cuda.synchronize()
    ta.process_host([k1], v1, chunk_rows=1 << 18, stream=sa.cuda_stream)
    tb.process_host([k2], v2, chunk_rows=1 << 18, stream=sb.cuda_stream)
    torch.cuda.synchronize()
    ta.check()
    tb.check()
    assert compare(ta.results_numpy(), oracle.groupby(k1, v1), ALL, True) <= FLOAT_RTOL
    assert compare(tb.results_numpy(), oracle.groupby(k2, v2), ALL, True) <= FLOAT_RTOL
