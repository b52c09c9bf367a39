"""The C++ drop-in header (include/qdb_groupby.hpp) compiled by g++ and linked against libqdbgb.so.

tests/cpp/dropin_kats.cpp is written the way a reference caller is: GPUGroupBy<AGG, O, K, V> and its multi-key
form, GPUBinary<FilterConditions::OP, int8_t, L, R>::Binary, GPUReconstruct::reconstructColKeep, GPUMemory and
query_engine_error, with the dispatcher's grow-and-restart on GPU_HASH_TABLE_FULL.  On the CPU the program must
compile, link and load the library; on the GPU it runs every known-answer case of the reference's tests
(tests/golden/reference_kats.json), including qikkDB_test/GPUGroupByTests.cu:520-540 (multi-key) and :620-628 (no
aggregate), and its groups must equal the expected ones.
"""
import os
import subprocess

import numpy as np
import pytest

from kat_util import OPS, expected_map, kat_inputs, load_kats

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "qikkdb_b200")
EXE = os.path.join(ROOT, "_build", "dropin_kats")


def build_program() -> str:
    src = os.path.join(ROOT, "tests", "cpp", "dropin_kats.cpp")
    hdrs = [os.path.join(ROOT, "include", h) for h in ("qdb_groupby.hpp", "qdb_gb.h")]
    lib = os.path.join(LIBDIR, "libqdbgb.so")
    newest = max(os.path.getmtime(p) for p in [src, lib, *hdrs])
    if not os.path.exists(EXE) or os.path.getmtime(EXE) < newest:
        os.makedirs(os.path.dirname(EXE), exist_ok=True)
        cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), src,
               "-L", LIBDIR, "-lqdbgb", f"-Wl,-rpath,{LIBDIR}", "-o", EXE + ".tmp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        os.replace(EXE + ".tmp", EXE)
    return EXE


def test_dropin_header_compiles_links_and_loads():
    exe = build_program()
    r = subprocess.run([exe, "version"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip(), "qdb_version() printed nothing"


def _serialise(case) -> str:
    keys, kn, vals, vn = kat_inputs(case)
    n = len(keys[0])
    pred = case.get("pred")
    agg = case["agg"]
    hdr = ["case", case["name"], agg, case["n_key_cols"], n, case.get("block") or n, case.get("table_size") or 0,
           int(bool(case.get("grow_on_full"))), int(vals is not None and agg != "none"), int(kn is not None),
           int(vn is not None and agg != "none"), OPS[pred["op"]] if pred else -1, int(pred["const"]) if pred else 0]
    parts = [" ".join(str(x) for x in hdr)]
    arr = lambda a: " ".join(str(int(x)) for x in np.asarray(a).astype(np.int64))  # noqa: E731
    parts += [arr(k) for k in keys]
    if kn is not None:
        parts += [arr(x) for x in kn]
    if vals is not None and agg != "none":
        parts.append(arr(vals))
        if vn is not None:
            parts.append(arr(vn))
    if pred:
        parts.append(arr(pred["col"]))
    return "\n".join(parts) + "\n"


def _parse(out: str, cases):
    res = {}
    lines = out.splitlines()
    i = 0
    by_name = {c["name"]: c for c in cases}
    while i < len(lines):
        tag, name, count, mult = lines[i].split()
        assert tag == "result"
        nk = by_name[name]["n_key_cols"]
        groups = {}
        for line in lines[i + 1:i + 1 + int(count)]:
            f = [int(x) for x in line.split()]
            key = tuple(None if f[nk + c] else f[c] for c in range(nk))
            assert key not in groups, f"{name}: duplicate group {key}"
            groups[key] = None if f[2 * nk] else f[2 * nk + 1]
        res[name] = (groups, int(count), int(mult))
        i += 1 + int(count)
    return res


@pytest.mark.gpu
def test_dropin_runs_reference_kats(cuda):
    exe = build_program()
    cases = load_kats()
    text = "".join(_serialise(c) for c in cases)
    r = subprocess.run([exe], input=text, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = _parse(r.stdout, cases)
    assert set(res) == {c["name"] for c in cases}
    for c in cases:
        groups, count, mult = res[c["name"]]
        if c.get("grow_on_full"):
            assert mult > 1, f"{c['name']}: the first table must overflow"
            assert count == c["expected_groups"]
            assert set(groups.values()) == {c["expected_value_all"]}
            continue
        exp = expected_map(c)
        if c["agg"] == "none":
            exp = {k: None for k in exp}
        assert groups == exp, f"{c['name']}: {groups} != {exp}"


@pytest.mark.gpu
def test_dropin_order_by_and_scalar_aggregation(cuda):
    """GPUOrderBy over GROUP BY results (DispatcherGroupByTests.cpp:1551-1588) and GPUAggregation::col on the inputs
    of GPUAggregationTests.cu:13-126 (2^18 default-seeded int32 draws as int32 and int64 columns, 0.25 as float),
    through the C++ drop-in."""
    import json

    import oracle
    exe = build_program()
    with open(os.path.join(ROOT, "tests", "golden", "reference_kats.json")) as f:
        cases = json.load(f)["order_by_cases"]
    text = ""
    for c in cases:
        text += f"ocase {c['name']} {int(c['order_by'] == 'value')} {int(c['descending'])} {len(c['keys'])}\n"
        text += " ".join(map(str, c["keys"])) + "\n" + " ".join(map(str, c["values"])) + "\n"
    r = subprocess.run([exe, "order"], input=text, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    i = 0
    for c in cases:
        tag, name, g = lines[i].split()
        assert tag == "oresult" and name == c["name"]
        got = [[int(x) for x in line.split()] for line in lines[i + 1:i + 1 + int(g)]]
        assert got == c["expected"], (name, got)
        i += 1 + int(g)

    n = 1 << 18
    a32, _ = oracle.reference_filter_inputs(np.int32, 1, n)
    a64, _ = oracle.reference_filter_inputs(np.int64, 1, n)
    f32 = np.full(n, 0.25, dtype=np.float32)
    text = "\n".join(f"{code} {n}\n" + " ".join(map(str, arr.tolist()))
                     for code, arr in ((8, a32), (9, a64), (10, f32))) + "\n"
    r = subprocess.run([exe, "scalar"], input=text, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = [line.split() for line in r.stdout.splitlines()]
    # the test's own expectations: T sum (int32 wraps), avg = sum / N truncated, cnt = N
    s32 = (int(a32.astype(np.int64).sum()) + (1 << 31)) % (1 << 32) - (1 << 31)
    assert [int(x) for x in out[0]] == [int(a32.min()), int(a32.max()), s32, int(s32 / n), n]
    s64 = int(a64.sum())
    assert [int(x) for x in out[1]] == [int(a64.min()), int(a64.max()), s64, int(s64 / n), n]
    assert [float(x) for x in out[2]] == [0.25, 0.25, 0.25 * n, 0.25, n]


@pytest.mark.gpu
def test_dropin_string_groupby(cuda):
    """GPUGroupBy<AGG, O, std::string, int32_t> through the C++ drop-in on the reference's string GROUP BY tests
    (GPUGroupByTests.cu:474-516, DispatcherGroupByTests.cpp:1422-1467, DispatcherNullTests.cpp:1372-1750)."""
    from kat_util import load_string_kats, string_blocks, string_expected
    exe = build_program()
    cases = load_string_kats()
    text = ""
    for c in cases:
        blocks = string_blocks(c)
        text += f"scase {c['name']} {c['agg']} {len(blocks)}\n"
        for keys, vals, vn, mask in blocks:
            text += f"{len(keys)}\n"
            for i, k in enumerate(keys):
                kt = "N" if k is None else ("-" if k == "" else k.encode().hex())
                vt = "X" if vals is None else ("N" if vn is not None and vn[i] else str(int(vals[i])))
                text += f"{kt} {vt} {1 if mask is None else int(mask[i])}\n"
    # "string": block by block through one table; "smerge": blocks dealt to two tables merged by GetResults(tables)
    for mode in ("string", "smerge"):
        r = subprocess.run([exe, mode], input=text, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        lines = r.stdout.splitlines()
        i = 0
        for c in cases:
            tag, name, g = lines[i].split()
            assert tag == "sresult" and name == c["name"]
            got = {}
            for line in lines[i + 1:i + 1 + int(g)]:
                k, v = line.split()
                key = None if k == "N" else (b"" if k == "-" else bytes.fromhex(k))
                got[key] = None if v == "N" else int(v)
            assert got == string_expected(c), (mode, name, got)
            i += 1 + int(g)


@pytest.mark.gpu
def test_dropin_compression_reference_columns(cuda):
    """CompressionGPU::compressDataAAFL / decompressDataAAFL / decompressDataAAFLOnDevice through the C++ drop-in on the
    columns of qikkDB_test/GPUCompressionTests.cpp: the header words the tests assert, the blocks left plain, and
    the round trip."""
    from kat_util import compression_column, load_compression_kats
    exe = build_program()
    cases = load_compression_kats()
    codes = {np.dtype(np.int32): 8, np.dtype(np.int64): 9, np.dtype(np.float32): 10}
    text = ""
    for c in cases:
        v = compression_column(c["name"])
        vals = " ".join(repr(float(x)) if v.dtype.kind == "f" else str(int(x)) for x in v)
        text += f"{codes[v.dtype]} {len(v)}\n{vals}\n"
    r = subprocess.run([exe, "compress"], input=text, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    i = 0
    for c in cases:
        want = c.get("head32", c.get("head64"))
        if want == "plain":
            assert lines[i] == "plain", c["name"]
            i += 1
            continue
        parts = lines[i].split()
        assert parts[0] == "block" and [int(x) for x in parts[1:]] == want, (c["name"], lines[i])
        assert lines[i + 1] == "roundtrip 1", c["name"]
        i += 2
