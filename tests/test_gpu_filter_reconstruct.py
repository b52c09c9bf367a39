"""Filter and compaction kernels against the oracle on the reference tests' own inputs
(qikkDB_test/GPUFilterTests.cu:175-700, GPUReconstructTests.cu:140-174) and on seeded edge cases."""
import numpy as np
import pytest
import torch

import oracle
from qikkdb_b200.groupby import GPUBinary, GPUReconstruct, QueryEngineError, device_nullmask, unpack_nullmask

pytestmark = pytest.mark.gpu
N = 1 << 18  # DATA_ELEMENT_COUNT of GPUFilterTests.cu:14


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("dtype", [np.int32, np.int64, np.float32], ids=lambda t: np.dtype(t).name)
@pytest.mark.parametrize("mode", ["colcol", "colconst", "constcol", "constconst"])
def test_filters_reference_inputs(cuda, dtype, mode):
    a, b = oracle.reference_filter_inputs(dtype, 0 if mode == "colcol" else 1, N)
    if mode == "constconst":
        a = a[0]
    for op in range(6):
        out = torch.empty(N, dtype=torch.int8, device="cuda")
        if mode == "colcol":
            GPUBinary.Binary(op, out, _dev(a), _dev(b), N)
            ref = oracle.filter_mask(op, a, b)
        elif mode == "colconst":
            GPUBinary.Binary(op, out, _dev(a), b, N)
            ref = oracle.filter_mask(op, a, b)
        elif mode == "constcol":
            GPUBinary.Binary(op, out, b, _dev(a), N)
            ref = oracle.filter_mask(op, b, a)
        else:
            GPUBinary.Binary(op, out, a, b, N)
            ref = oracle.filter_mask(op, a, b, n=N)
        assert (out.cpu().numpy() == ref).all(), f"op {op}"


def test_filter_mixed_types_nulls_and_logic(cuda):
    rng = np.random.default_rng(2)
    n = 100_003
    a = rng.integers(-50, 50, n).astype(np.int32)
    b = (rng.standard_normal(n) * 30).astype(np.float64)
    nulls = rng.random(n) < 0.2
    from qikkdb_b200.groupby import pack_nullmask
    for op in range(8):
        out = torch.empty(n, dtype=torch.int8, device="cuda")
        GPUBinary.Binary(op, out, _dev(a), _dev(b), n, device_nullmask(nulls))
        ref = oracle.filter_mask(op, a, b, nulls=pack_nullmask(nulls))
        assert (out.cpu().numpy() == ref).all(), f"op {op}"


@pytest.mark.parametrize("dtype", [np.int8, np.int32, np.int64, np.float32, np.float64], ids=lambda t: np.dtype(t).name)
@pytest.mark.parametrize("density", [0.0, 0.01, 0.5, 1.0])
def test_reconstruct_col_keep(cuda, dtype, density):
    rng = np.random.default_rng(int(density * 100))
    n = 123_457
    col = (rng.integers(-1000, 1000, n)).astype(dtype)
    mask = (rng.random(n) < density).astype(np.int8)
    nulls = rng.random(n) < 0.3
    from qikkdb_b200.groupby import pack_nullmask
    out, cnt, nm = GPUReconstruct.reconstructColKeep(_dev(col), _dev(mask), n, device_nullmask(nulls))
    ref, rnull, rc = oracle.compact(col, mask, pack_nullmask(nulls))
    assert cnt == rc
    if cnt == 0:
        assert out.ptr == 0 and (nm is None or nm.ptr == 0)
        return
    assert (out.numpy() == ref).all()
    assert (unpack_nullmask(nm.numpy(), cnt) == unpack_nullmask(rnull, cnt)).all()


def test_reconstruct_without_mask_returns_input(cuda):
    col = _dev(np.arange(10, dtype=np.int32))
    out, cnt, _ = GPUReconstruct.reconstructColKeep(col, None, 10)
    assert cnt == 10 and out.ptr == col.data_ptr() and not out.owned


@pytest.mark.parametrize("mask,expected", [([1, 1, 1, 1], [0, 1, 2, 3]), ([0, 0, 0, 0, 0, 0], []),
                                           ([0, 1, 0, 0, 1, 1, 1, 1], [1, 4, 5, 6, 7])])
def test_generate_indexes_kats(cuda, mask, expected):
    """GPUReconstructTests.cu:140-153, :171-174."""
    got, n = GPUReconstruct.GenerateIndexes(_dev(np.array(mask, dtype=np.int8)), len(mask))
    assert n == len(expected) and list(got) == expected


def test_generate_indexes_big_mask(cuda):
    """GPUReconstructTests.cu:155-169: 2^18 alternating mask."""
    m = (np.arange(1 << 18) % 2).astype(np.int8)
    got, n = GPUReconstruct.GenerateIndexes(_dev(m), len(m))
    assert n == (1 << 17) and (got == np.arange(1, 1 << 18, 2)).all()


def test_generate_indexes_requires_mask(cuda):
    with pytest.raises(QueryEngineError):
        GPUReconstruct.GenerateIndexesKeep(None, 4)


def test_prefix_sum_and_compress(cuda):
    rng = np.random.default_rng(7)
    n = 1_000_003
    m = (rng.random(n) < 0.37).astype(np.int8)
    ps = GPUReconstruct.PrefixSum(_dev(m), n).cpu().numpy()
    assert (ps == oracle.prefix_sum(m)).all()
    arr = (rng.random(n) < 0.5).astype(np.uint8)
    words = GPUReconstruct.CompressNullMask(_dev(arr), n).numpy()
    assert (unpack_nullmask(words, n) == arr.astype(bool)).all()
