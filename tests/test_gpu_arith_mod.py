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
