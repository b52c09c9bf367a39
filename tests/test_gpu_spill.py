"""GPU GROUP BY edge cases of the shared-table accumulators and the hash-partitioned spill, against the oracle:
a spill whose cells overflow (every key in one partition), float values outside a CTA's fixed-point window,
signed integer sums that wrap, and negative float sums."""
import numpy as np
import pytest

from gpu_compare import FLOAT_RTOL
from qikkdb_b200 import datagen as dg
from qikkdb_b200.groupby import FilterConditions
from test_gpu_parity import run_both

pytestmark = pytest.mark.gpu

# The aggregation pass picks a row's spill partition from the top bits of key * C (mod 2^64); the global table hashes
# keys with the independent mix64.
SPILL_HASH = 0x9E3779B97F4A7C15


def keys_in_partition_zero(count: int, seed: int) -> np.ndarray:
    """Distinct int64 keys whose spill partition is 0 for every partition count up to 2^14 (first and second level
    together): k = t * C^-1 mod 2^64 with t < 2^50, so the top 14 bits of k * C are zero."""
    inv = pow(SPILL_HASH, -1, 1 << 64)
    rng = np.random.default_rng(seed)
    t = np.unique(rng.integers(1, 1 << 50, count + count // 8, dtype=np.uint64))[:count]
    k = (t * np.uint64(inv)).astype(np.int64)  # wraps modulo 2^64
    assert len(np.unique(k)) == count
    return k


def test_spill_cells_overflow_to_global_default_tables(cuda):
    """200000 keys in spill partition 0 with the default table sizes: the CTAs' cells of that partition overflow and
    the spill pass's table cannot hold the partition, so rows take the global-table path on both sides."""
    n = 1 << 21
    uniq = keys_in_partition_zero(200_000, 5)
    pick = dg.uniform_i32(51, 0, n, 0, len(uniq) - 1)
    k = uniq[pick]
    v = dg.lognormal_f32(51, 1, n, 2.0, 1.0)
    p = dg.uniform_f32(51, 2, n)
    rel, g, _ = run_both(k, v, ["sum", "avg", "count", "min", "max"], 1 << 20, 0,
                         pred=(p, FilterConditions.less, 0.7, np.float32, None), val_is_float=True)
    assert rel <= FLOAT_RTOL and g["n_groups"] > 100_000


@pytest.mark.parametrize("levels", [1, 2])
def test_spill_cells_overflow_to_global(cuda, monkeypatch, levels):
    """Every key lands in spill partition 0.  With both shared tables cut down (64 buckets in the aggregation pass,
    8 KB in the spill pass, hence 8192 partitions, written in one level or, with at most 1024 partitions per pass, in
    two), the CTAs' cells of that partition overflow and the spill pass's table cannot hold the partition, so rows
    take the global-table path on every side."""
    monkeypatch.setenv("QDB_FAST_BUCKETS", "64")
    monkeypatch.setenv("QDB_SPILL_SMEM_KB", "8")
    if levels == 2:
        monkeypatch.setenv("QDB_SPILL_BITS_MAX", "10")
    n = 1 << 19
    uniq = keys_in_partition_zero(3000, 5)
    pick = dg.uniform_i32(51, 0, n, 0, len(uniq) - 1)
    k = uniq[pick]
    v = dg.lognormal_f32(51, 1, n, 2.0, 1.0)
    p = dg.uniform_f32(51, 2, n)
    rel, g, _ = run_both(k, v, ["sum", "avg", "count", "min", "max"], 1 << 20, 0,
                         pred=(p, FilterConditions.less, 0.7, np.float32, None), val_is_float=True)
    assert rel <= FLOAT_RTOL and g["n_groups"] == 3000


def test_float_values_outside_fixed_point_window(cuda):
    """Values spread over e^-50 .. e^50 (and exact zeros): those far from a CTA's first-tile magnitudes take the
    FP64 global path, the rest the fixed-point shared path; sums stay within tolerance of FP64."""
    n = 1 << 20
    k = dg.zipf_i64(61, 0, n, 50_000, 1.1)
    v32 = dg.lognormal_f32(61, 1, n, 0.0, 12.0)
    v32[::97] = 0.0
    rel, _, _ = run_both(k, v32, ["sum", "avg", "count", "min", "max"], 1 << 16, 0, val_is_float=True)
    assert rel <= FLOAT_RTOL
    v64 = v32.astype(np.float64) * np.exp(dg.uniform_f32(61, 2, n).astype(np.float64) * 40.0)
    rel, _, _ = run_both(k, v64, ["sum", "avg", "count"], 1 << 16, 0, val_is_float=True)
    assert rel <= FLOAT_RTOL


def test_integer_sums_wrap_through_limbs(cuda):
    """int64 values near +-2^62 make the per-CTA two-limb accumulators carry and the sums wrap: SUM and AVG are
    the reference's wrapping int64 results, bit for bit."""
    rng = np.random.default_rng(71)
    n = 1 << 20
    k = rng.integers(0, 100_000, n).astype(np.int64)
    v = rng.integers(-(1 << 62), 1 << 62, n, dtype=np.int64)
    run_both(k, v, ["sum", "avg", "count", "min", "max"], 1 << 17, 0)
    k32 = rng.integers(0, 500, n).astype(np.int32)
    v32 = rng.integers(np.iinfo(np.int32).min, np.iinfo(np.int32).max, n, dtype=np.int64).astype(np.int32)
    run_both(k32, v32, ["sum", "avg", "count", "min", "max"], 512, 0)


def test_negative_float_sums(cuda):
    """Values of both signs in the 96-bit fixed-point accumulators (two's-complement limbs)."""
    rng = np.random.default_rng(81)
    n = 1 << 20
    k = rng.integers(0, 100, n).astype(np.int32)
    v = (rng.random(n) * 2000.0 - 1000.0).astype(np.float32)
    rel, _, _ = run_both(k, v, ["sum", "avg", "count", "min", "max"], 128, 0, val_is_float=True)
    assert rel <= FLOAT_RTOL


def test_tables_on_two_streams_share_the_spill_area(cuda):
    """Two spilling tables fed alternately on two streams: the per-device spill area is ordered between the calls
    by its event, so both results equal the oracle's."""
    import torch

    import oracle
    from gpu_compare import compare
    from qikkdb_b200.groupby import GroupByTable

    n = 1 << 21
    cols = []
    for seed in (91, 92):
        k = dg.zipf_i64(seed, 0, n, 200_000, 1.05)
        v = dg.lognormal_f32(seed, 1, n, 1.0, 1.0)
        cols.append((k, v))
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    tables = [GroupByTable(["sum", "count", "max"], np.int64, np.float32, 1 << 18, stream=s.cuda_stream)
              for s in streams]
    blocks = 8
    bounds = np.linspace(0, n, blocks + 1).astype(np.int64)
    dev = []
    for (k, v), s in zip(cols, streams):
        with torch.cuda.stream(s):
            dev.append((torch.from_numpy(k).cuda(), torch.from_numpy(v).cuda()))
    torch.cuda.synchronize()
    for b0, b1 in zip(bounds[:-1], bounds[1:]):
        for t, (dk, dv), s in zip(tables, dev, streams):
            t.process([dk[b0:b1]], dv[b0:b1], int(b1 - b0), stream=s.cuda_stream, sync=False)
    for t, s in zip(tables, streams):
        s.synchronize()
        t.check(stream=s.cuda_stream)
    for t, (k, v) in zip(tables, cols):
        rel = compare(t.results_numpy(), oracle.groupby(k, v), ["sum", "count", "max"], True)
        assert rel <= FLOAT_RTOL


def test_two_level_spill_composite(cuda, monkeypatch):
    """A composite-key table whose groups need 4096 spill partitions, written as 1024 first-level partitions of 4
    sub-partitions each (the two-level spill): SUM/COUNT/MAX bit for bit."""
    monkeypatch.setenv("QDB_SPILL_BITS_MAX", "10")
    n = 1 << 23
    a = dg.uniform_i32(32, 0, n, 0, 4095)
    b = dg.uniform_i32(32, 1, n, 0, 4095)
    v = dg.uniform_i64(32, 2, n, 0, (1 << 31) - 1)
    run_both([a, b], v, ["sum", "count", "max"], 1 << 23)
