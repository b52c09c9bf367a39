"""The allocation-free compaction entry point, checked against the allocating one through the C ABI.

qdb_reconstruct_keep_noalloc serves callers that own all device memory themselves (a buffer pool that accounts
every byte, a serving loop with a fixed HBM budget) and therefore cannot let the library allocate during a query.
It must select exactly what qdb_reconstruct_keep selects and what the CPU oracle's compaction selects.  Two calls
run back to back, because every call shares one scratch array that keeps the previous call's contents.  This file
is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from qikkdb_b200 import _capi
from qikkdb_b200.groupby import nullmask_words, pack_nullmask, unpack_nullmask

pytestmark = pytest.mark.gpu


def _reference(lib, col, mask, nulls, stream):
    out, cnt, onm = C.c_void_p(), C.c_int64(), C.c_void_p()
    _capi.check(lib.qdb_reconstruct_keep(col.element_size(), col.data_ptr(), mask.data_ptr(), col.numel(),
                                         C.byref(out), C.byref(cnt), nulls.data_ptr(), C.byref(onm), stream))
    n = cnt.value
    vals = torch.empty(n, dtype=col.dtype, device="cuda")
    words = torch.empty(nullmask_words(n), dtype=torch.int64, device="cuda")
    if n:
        _capi.check(lib.qdb_memcpy_d2d(vals.data_ptr(), out.value, n * col.element_size(), stream))
        _capi.check(lib.qdb_memcpy_d2d(words.data_ptr(), onm.value, words.numel() * 8, stream))
        lib.qdb_free(out.value, stream)
        lib.qdb_free(onm.value, stream)
    return n, vals.cpu().numpy(), unpack_nullmask(words.cpu().numpy(), n)


def test_noalloc_compaction_matches_allocating_form(cuda):
    lib = _capi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(77)
    for call, (n, dtype, density) in enumerate([(1_000_003, np.int64, 0.3), (257_000, np.float32, 0.9)]):
        col = torch.from_numpy((rng.standard_normal(n) * 1000).astype(dtype)).cuda()
        mask = torch.from_numpy((rng.random(n) < density).astype(np.int8)).cuda()
        nulls_h = rng.random(n) < 0.2
        nulls = torch.from_numpy(pack_nullmask(nulls_h).view(np.int64)).cuda()
        ref_n, ref_vals, ref_nulls = _reference(lib, col, mask, nulls, stream)
        # caller-owned outputs; filled with garbage first so stale contents would show
        out = torch.full((n,), 7, dtype=col.dtype, device="cuda")
        out_nulls = torch.full((nullmask_words(n),), -1, dtype=torch.int64, device="cuda")
        cnt = C.c_int64(-1)
        _capi.check(lib.qdb_reconstruct_keep_noalloc(col.element_size(), col.data_ptr(), mask.data_ptr(), n,
                                                     out.data_ptr(), n, C.byref(cnt), nulls.data_ptr(),
                                                     out_nulls.data_ptr(), stream))
        torch.cuda.synchronize()
        assert cnt.value == ref_n, f"call {call}: count {cnt.value} != {ref_n}"
        got = out[:ref_n].cpu().numpy()
        assert (got == ref_vals).all(), f"call {call}: compacted values differ"
        assert (unpack_nullmask(out_nulls.cpu().numpy(), ref_n) == ref_nulls).all(), f"call {call}: null bits differ"


def test_noalloc_rejects_oversize_and_short_output(cuda):
    lib = _capi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    cnt = C.c_int64()
    rc = lib.qdb_reconstruct_keep_noalloc(4, 16, 16, (1 << 28) + 1, 16, 1 << 29, C.byref(cnt), None, None, stream)
    assert rc == _capi.QDB_ERR_TOO_LARGE and b"268435456" in lib.qdb_last_error()
    col = torch.arange(1000, dtype=torch.int32, device="cuda")
    mask = torch.ones(1000, dtype=torch.int8, device="cuda")
    out = torch.empty(10, dtype=torch.int32, device="cuda")
    rc = lib.qdb_reconstruct_keep_noalloc(4, col.data_ptr(), mask.data_ptr(), 1000, out.data_ptr(), 10,
                                          C.byref(cnt), None, None, stream)
    assert rc == _capi.QDB_ERR_TOO_LARGE


def test_noalloc_compaction_matches_oracle_unaligned_mask(cuda):
    # A mask that starts one byte past a 16-byte boundary takes the kernels' scalar path, and row counts that are not
    # a multiple of the 4096-row tile leave a ragged last tile.
    lib = _capi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(78)
    for call, (n, dtype, density) in enumerate([(700_001, np.int32, 0.5), (12_345, np.float64, 0.07)]):
        col_h = (rng.standard_normal(n) * 1e4).astype(dtype)
        mask_h = (rng.random(n) < density).astype(np.int8)
        nulls_flags = rng.random(n) < 0.1
        words_h = pack_nullmask(nulls_flags)
        exp_vals, exp_words, exp_n = oracle.compact(col_h, mask_h, words_h)
        col = torch.from_numpy(col_h).cuda()
        mask_buf = torch.zeros(n + 16, dtype=torch.int8, device="cuda")
        mask_buf[1:n + 1] = torch.from_numpy(mask_h).cuda()
        mask = mask_buf[1:n + 1]
        assert mask.data_ptr() % 16 == 1
        nulls = torch.from_numpy(words_h.view(np.int64)).cuda()
        out = torch.full((n,), 3, dtype=col.dtype, device="cuda")
        out_nulls = torch.full((nullmask_words(n),), -1, dtype=torch.int64, device="cuda")
        cnt = C.c_int64(-1)
        _capi.check(lib.qdb_reconstruct_keep_noalloc(col.element_size(), col.data_ptr(), mask.data_ptr(), n,
                                                     out.data_ptr(), n, C.byref(cnt), nulls.data_ptr(),
                                                     out_nulls.data_ptr(), stream))
        torch.cuda.synchronize()
        assert cnt.value == exp_n, f"call {call}: count {cnt.value} != {exp_n}"
        assert (out[:exp_n].cpu().numpy() == exp_vals).all(), f"call {call}: compacted values differ from the oracle"
        got_nulls = unpack_nullmask(out_nulls.cpu().numpy(), exp_n)
        assert (got_nulls == unpack_nullmask(exp_words, exp_n)).all(), f"call {call}: null bits differ from the oracle"
