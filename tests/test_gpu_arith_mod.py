"""qdb_arith_mod (GPUBinary<ArithmeticOperations::mod, T, T*, T>, GPUBinary.cuh:145-166): out = in % m with the C++
remainder (sign of the dividend), computed with a multiply-high instead of a division; checked bit-exact against
numpy's fmod on extreme dividends and divisors (1, powers of two, odd, near 2^31 and 2^62, negative)."""
import numpy as np
import pytest
import torch

from qikkdb_b200 import _capi as capi
from qikkdb_b200 import datagen as dg

pytestmark = pytest.mark.gpu


def _mod(a: np.ndarray, m: int) -> np.ndarray:
    d = torch.from_numpy(a).cuda()
    out = torch.empty_like(d)
    code = capi.QDB_INT32 if a.dtype == np.int32 else capi.QDB_INT64
    capi.check(capi.lib().qdb_arith_mod(code, d.data_ptr(), int(m), out.data_ptr(), a.size,
                                        torch.cuda.current_stream().cuda_stream))
    return out.cpu().numpy()


@pytest.mark.parametrize("m", [1, 2, 3, 7, 10, 64, 1000, 65537, 2**31 - 1, -5, -(2**31)])
def test_mod_int32(cuda, m):
    a = dg.uniform_i32(600, 0, 1 << 18, -(2**31), 2**31 - 1)
    a[:6] = [0, 1, -1, 2**31 - 1, -(2**31), -(2**31) + 1]
    assert (_mod(a, m) == np.fmod(a.astype(np.int64), m).astype(np.int32)).all()


@pytest.mark.parametrize("m", [1, 2, 3, 10, 2**20, 1_000_003, 2**32 + 15, 2**62 + 1, 2**63 - 1, -9, -(2**40)])
def test_mod_int64(cuda, m):
    a = dg.uniform_i64(601, 0, 1 << 18, -(2**63), 2**63 - 1)
    a[:6] = [0, 1, -1, 2**63 - 1, -(2**63), -(2**63) + 1]
    ref = np.array([int(np.sign(x)) * (abs(int(x)) % abs(m)) for x in a[:4096]], dtype=np.int64)
    assert (_mod(a, m)[:4096] == ref).all()
    assert (_mod(a, m) == np.fmod(a, np.int64(m))).all()


def test_mod_by_zero(cuda):
    a = np.arange(10, dtype=np.int32)
    with pytest.raises(capi.QdbError) as e:
        _mod(a, 0)
    assert e.value.code == capi.QDB_DIVISION_BY_ZERO


@pytest.mark.parametrize("dt", [np.int32, np.int64])
@pytest.mark.parametrize("n,off", [(1, 0), (3, 0), (5, 0), (4097, 0), ((1 << 20) + 3, 0), (4099, 1), (4099, 3)])
def test_mod_ragged_and_unaligned(cuda, dt, n, off):
    """Row counts that leave 1-3 rows after the 4-row vector steps, and columns starting off a 16-byte boundary
    (the scalar form), against numpy's fmod."""
    a = (dg.uniform_i32(602, 0, n + off, -(2**31), 2**31 - 1) if dt == np.int32
         else dg.uniform_i64(602, 0, n + off, -(2**63), 2**63 - 1))
    d = torch.from_numpy(a).cuda()[off:]
    out = torch.full((n + off,), 7, dtype=d.dtype, device="cuda")[off:]
    code = capi.QDB_INT32 if dt == np.int32 else capi.QDB_INT64
    for m in (3, 1000, -77):
        capi.check(capi.lib().qdb_arith_mod(code, d.data_ptr(), m, out.data_ptr(), n,
                                            torch.cuda.current_stream().cuda_stream))
        assert (out.cpu().numpy() == np.fmod(a[off:], dt(m))).all(), (n, off, m)


def _check_table(table, keys_mod, vals, pred_np, aggs):
    import oracle
    from gpu_compare import FLOAT_RTOL
    r = oracle.groupby(keys_mod, vals, pred=pred_np)
    g = table.results_numpy(list(aggs))
    assert g["n_groups"] == r["count"]
    order = np.argsort(g["keys"][0], kind="stable")
    assert np.array_equal(g["keys"][0][order].astype(np.int64), r["keys"][0])
    vf = vals is not None and vals.dtype.kind == "f"
    for a in aggs:
        got, exp = g[a][order], r["cnt" if a == "count" else a]
        if vf and a in ("sum", "avg"):
            assert np.all(np.abs(got - exp) <= FLOAT_RTOL * np.maximum(np.abs(exp), 1.0)), a
        else:
            assert np.array_equal(got.astype(exp.dtype), exp), a


@pytest.mark.parametrize("kdt,m,n,off", [
    (np.int32, 1000, 1 << 21, 0),            # fused, every group in the shared table
    (np.int32, -77, (1 << 20) + 5, 0),       # fused, negative modulus, ragged tail
    (np.int64, 300_000, 1 << 21, 0),         # fused, spilling table
    (np.int64, 2**40 + 3, 1 << 20, 0),       # fused, remainders beyond int32
    (np.int32, 5000, 1500, 0),               # too few rows for the fast pass: remainder column first
    (np.int64, 999, (1 << 20) + 1, 1),       # key column off a 16-byte boundary: remainder column first
])
def test_process_mod_matches_oracle(cuda, kdt, m, n, off):
    """qdb_gb_process_mod (GROUP BY key % m, the modulo fused into the aggregation pass or materialised first) against
    the oracle's GROUP BY over numpy's fmod column, with a fused WHERE and float or integer values."""
    from qikkdb_b200.groupby import FilterConditions, GroupByTable, make_pred, process_mod
    rng = np.random.default_rng(abs(m) % 1000 + n % 7)
    info = np.iinfo(kdt)
    keys = rng.integers(info.min, info.max, n + off, dtype=kdt)
    keys[off:off + 4] = [0, -1, info.max, info.min]
    p = rng.random(n).astype(np.float32)
    for vals, aggs in ((dg.lognormal_f32(603, 1, n, 2.0, 1.0), ("sum", "count", "min", "max", "avg")),
                       (dg.uniform_i32(603, 2, n, -1000, 1000), ("sum", "min", "avg", "count"))):
        kd = torch.from_numpy(keys).cuda()[off:]
        bound = int(min(abs(m) * 2, n))
        t = GroupByTable(list(aggs), kdt, vals.dtype, max(bound, 16))
        pred = make_pred(torch.from_numpy(p).cuda(), FilterConditions.less, 0.6, np.float32)
        process_mod(t, kd, m, torch.from_numpy(vals).cuda(), pred, n=n)
        _check_table(t, np.fmod(keys[off:], kdt(m)), vals, (p, FilterConditions.less, 0.6, np.float32, None), aggs)


def test_process_mod_count_only_and_errors(cuda):
    from qikkdb_b200.groupby import GroupByTable, process_mod
    n = 1 << 20
    keys = dg.uniform_i64(604, 0, n, -(1 << 62), 1 << 62)
    t = GroupByTable(["count"], np.int64, None, 8192)  # remainders of signed keys: (-4001, 4001)
    process_mod(t, torch.from_numpy(keys).cuda(), 4001)
    _check_table(t, np.fmod(keys, np.int64(4001)), None, None, ("count",))
    with pytest.raises(capi.QdbError) as e:
        process_mod(t, torch.from_numpy(keys).cuda(), 0)
    assert e.value.code == capi.QDB_DIVISION_BY_ZERO
    t32 = GroupByTable(["count"], np.int32, None, 64)
    with pytest.raises(capi.QdbError) as e:
        process_mod(t32, torch.zeros(4096, dtype=torch.int32, device="cuda"), 1 << 40)
    assert e.value.code == capi.QDB_ERR_INVALID
