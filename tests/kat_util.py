"""Helpers that run the reference's known-answer GROUP BY cases (tests/golden/reference_kats.json)."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OPS = {"greater": 0, "greaterEqual": 1, "less": 2, "lessEqual": 3, "equal": 4, "notEqual": 5}


def load_kats():
    with open(os.path.join(HERE, "golden", "reference_kats.json")) as f:
        return json.load(f)["cases"]


def kat_inputs(case):
    """(keys list[np.int32], key_null_flags list or None, values np.int32 or None, value_null_flags or None)."""
    if "generator" in case:
        g = case["generator"]
        keys = [np.arange(g["n"], dtype=np.int64) % g["modulus"]]
        keys = [keys[0].astype(np.int32)]
        vals = np.full(g["n"], g["value"], dtype=np.int32)
        return keys, None, vals, None
    keys = [np.asarray(k, dtype=np.int32) for k in case["keys"]]
    kn = [np.asarray(x, dtype=bool) for x in case["key_nulls"]] if case.get("key_nulls") else None
    vals = np.asarray(case["values"], dtype=np.int32) if case.get("values") is not None else None
    vn = np.asarray(case["value_nulls"], dtype=bool) if case.get("value_nulls") else None
    return keys, kn, vals, vn


def expected_map(case):
    out = {}
    for e in case["expected"]:
        key = tuple(None if n else k for k, n in zip(e["key"], e["key_null"]))
        out[key] = e["value"]
    return out


def result_map(keys, key_nulls, values, value_nulls):
    """Builds {key tuple (None = NULL component): value or None} from host arrays."""
    out = {}
    n = len(keys[0])
    for i in range(n):
        key = tuple(None if (key_nulls is not None and key_nulls[c] is not None and key_nulls[c][i]) else int(keys[c][i])
                    for c in range(len(keys)))
        if values is None:
            v = None
        elif value_nulls is not None and value_nulls[i]:
            v = None
        else:
            v = int(values[i])
        assert key not in out, f"duplicate group {key}"
        out[key] = v
    return out


def load_string_kats():
    with open(os.path.join(HERE, "golden", "reference_kats.json")) as f:
        return json.load(f)["string_cases"]


def string_blocks(case):
    """Per block: (key strings with None for NULL, values np.int32 or None, value NULL flags or None, mask or None)."""
    out = []
    pv = case.get("pred_values_greater")
    for b, keys in enumerate(case["blocks_keys"]):
        vals = vn = None
        if case["blocks_values"] is not None:
            raw = case["blocks_values"][b]
            vn = np.array([v is None for v in raw], dtype=bool)
            vals = np.array([0 if v is None else v for v in raw], dtype=np.int32)
            if not vn.any():
                vn = None
        mask = None
        if pv is not None:
            mask = (np.asarray(pv["values"][b], dtype=np.int32) > pv["const"]).astype(np.int8)
        out.append((keys, vals, vn, mask))
    return out


def string_expected(case):
    return {(None if e["key"] is None else e["key"].encode()): e["value"] for e in case["expected"]}


def load_compression_kats():
    with open(os.path.join(HERE, "golden", "reference_kats.json")) as f:
        return json.load(f)["compression_cases"]


def compression_column(name: str) -> np.ndarray:
    """The 1024-row columns of qikkDB_test/GPUCompressionTests.cpp:44-52 (block size 1024)."""
    i = np.arange(1024)
    if name == "CompressionInt":
        return (i - 512).astype(np.int32)
    if name == "CompressionIntLarge":
        return ((i - 512) * 100000000).astype(np.int64).astype(np.int32)
    if name == "CompressionLong":
        return ((i - 512) * 100000).astype(np.int64)
    if name == "CompressionFloatPositive":
        return (i / 100.0 + 10).astype(np.float32)
    if name == "CompressionFloatNegative":
        return -((i / 1000.0 + 10).astype(np.float32))
    return ((i - 512) / 100.0).astype(np.float32)
