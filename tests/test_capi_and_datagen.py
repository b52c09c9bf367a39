"""CPU checks: the C-ABI library loads and exports every entry point include/qdb_gb.h declares (no GPU call),
the ctypes binding covers the header, and the synthetic generators are deterministic and well distributed."""
import os
import re
import subprocess

import numpy as np

from qikkdb_b200 import _capi
from qikkdb_b200 import datagen as dg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h") and name.startswith("qdb"):
            txt = open(os.path.join(ROOT, "include", name)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            syms |= set(re.findall(r"\b(qdb_[a-z0-9_]+)\s*\(", txt))
    return syms


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    declared = header_symbols()
    assert declared, "no declarations found"
    for s in declared:
        assert hasattr(lib, s), f"{s} declared in include/ but not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(qdb_[a-z0-9_]+)\b", out))
    assert declared <= exported


def test_ctypes_binding_covers_header():
    assert header_symbols() == set(_capi.exported_symbols())


def test_version_and_device_count_without_gpu():
    lib = _capi.lib()
    assert b"sm_100a" in lib.qdb_version()
    import ctypes
    n = ctypes.c_int32(-1)
    assert lib.qdb_device_count(ctypes.byref(n)) == 0 and n.value >= 0


def test_generators_are_deterministic_across_threads():
    a = dg.zipf_i64(5, 1, 300_000, 10_000, 1.1, threads=1)
    b = dg.zipf_i64(5, 1, 300_000, 10_000, 1.1, threads=7)
    assert (a == b).all()
    x = dg.lognormal_f32(5, 2, 200_000, 2.0, 1.0, threads=1)
    y = dg.lognormal_f32(5, 2, 200_000, 2.0, 1.0, threads=5)
    assert (x == y).all()
    # a piece regenerated alone equals the same rows of the full column (pure function of the row)
    u = dg.uniform_i32(9, 3, 1000, 0, 99)
    assert (dg.uniform_i32(9, 3, 1000, 0, 99, threads=3) == u).all()


def test_generator_distributions():
    n = 1 << 20
    p = dg.uniform_f32(1, 0, n)
    assert 0.0 <= p.min() and p.max() < 1.0 and abs((p < 0.5).mean() - 0.5) < 0.005
    z = dg.zipf_i64(1, 1, n, 1_000_000, 1.1, map_keys=False)
    top = (z == 1).mean()
    assert abs(top - 0.1239) < 0.005  # 1 / H(1e6, 1.1)
    v = dg.lognormal_f32(1, 2, n, 2.0, 1.0)
    assert abs(np.log(v).mean() - 2.0) < 0.01 and abs(np.log(v).std() - 1.0) < 0.01
    k = dg.uniform_i32(1, 3, n, 0, 999)
    assert k.min() == 0 and k.max() == 999
    lu = dg.loguniform_i64(1, 4, 10_000, 1_000, 4_000_000)
    assert lu.min() >= 1000 and lu.max() <= 4_000_000
    keys = dg.zipf_i64(1, 5, 1000, 100, 1.1)
    assert (keys != np.iinfo(np.int64).min).all()


def test_server_entry_points_reject_null_handles_without_gpu():
    """The serving loop's entry points check their arguments before any CUDA call: a null server is
    QDB_ERR_INVALID with a message, on a machine without a GPU too."""
    import ctypes
    lib = _capi.lib()
    st = _capi.qdb_server_stats()
    assert lib.qdb_server_set_plain_route(None, 1 << 22, 0) == _capi.QDB_ERR_INVALID
    assert b"qdb_server_set_plain_route" in lib.qdb_last_error()
    assert lib.qdb_server_stats_get(None, ctypes.byref(st)) == _capi.QDB_ERR_INVALID
    t = ctypes.c_uint64()
    assert lib.qdb_server_submit(None, None, ctypes.byref(t)) == _capi.QDB_ERR_INVALID
    assert lib.qdb_server_release(None, 1) == _capi.QDB_ERR_INVALID
    assert lib.qdb_server_destroy(None) == 0
