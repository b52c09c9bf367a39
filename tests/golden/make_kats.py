"""Transcribes the reference's GROUP BY known-answer tests into tests/golden/reference_kats.json.

Each case restates one test of qikkDB's own suite (file:line in `source`): its input columns, the
predicate when the test has a WHERE clause, the block size the test processes in, and the expected
(key -> aggregate) result exactly as the test asserts it.  Expected values of loop-generated tests are
computed here by the same loops the tests run.  Run: python tests/golden/make_kats.py
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
DGB = "qikkDB_test/DispatcherGroupByTests.cpp"
DNT = "qikkDB_test/DispatcherNullTests.cpp"
GGB = "qikkDB_test/GPUGroupByTests.cu"

cases = []


def single(name, src, agg, keys, values, expected, block=4, pred=None, key_nulls=None, value_nulls=None,
           table_size=None):
    """expected: list of (key or None for NULL, value or None for NULL)."""
    cases.append({
        "name": name, "source": src, "agg": agg, "n_key_cols": 1, "key_type": "int32", "value_type": "int32",
        "keys": [keys], "key_nulls": [key_nulls] if key_nulls else None, "values": values,
        "value_nulls": value_nulls, "pred": pred, "block": block, "table_size": table_size,
        "expected": [{"key": [k], "key_null": [k is None], "value": v} for k, v in expected],
    })


def multi(name, src, agg, ka, kb, values, expected, block=4, ka_nulls=None, kb_nulls=None, value_nulls=None,
          table_size=None):
    """expected: list of ((a or None, b or None), value or None)."""
    kn = None
    if ka_nulls or kb_nulls:
        kn = [ka_nulls or [False] * len(ka), kb_nulls or [False] * len(kb)]
    cases.append({
        "name": name, "source": src, "agg": agg, "n_key_cols": 2, "key_type": "int32", "value_type": "int32",
        "keys": [ka, kb], "key_nulls": kn, "values": values, "value_nulls": value_nulls, "pred": None,
        "block": block, "table_size": table_size,
        "expected": [{"key": [a, b], "key_null": [a is None, b is None], "value": v} for (a, b), v in expected],
    })


K9 = [0, 1, -1, -1, 0, 1, 2, 1, 1]
V9 = [1, 2, 2, 2, 1, 3, 15, 5, -4]
single("IntSimpleSum", DGB + ":1330", "sum", K9, V9, [(0, 2), (1, 6), (2, 15), (-1, 4)])
single("IntCollisionsSum", DGB + ":1336", "sum",
       [0, 1, -1, 2, 262143, 262144, 262145, 1048576, 1048577, 1, 1, 262144, 0],
       [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096],
       [(0, 4097), (1, 1538), (-1, 4), (2, 8), (262143, 16), (262144, 2080), (262145, 64), (1048576, 128),
        (1048577, 256)])
KS = [2, 30, 7, 2, 30, 7, 2, 2]
single("IntSparseKeysSum", DGB + ":1344", "sum", KS, [1, 15, 14, 1, 15, 14, 1, 1], [(2, 4), (7, 28), (30, 30)])
single("IntSparseKeysAvg", DGB + ":1349", "avg", KS, [1, 15, 14, 1, 15, 14, 1, 1], [(2, 1), (7, 14), (30, 15)])
single("IntSparseKeysCount", DGB + ":1355", "count", KS, [1, 15, 0, 1, 15, 0, 1, 1], [(2, 4), (7, 2), (30, 2)])
single("IntKeyWhereSimpleSum", DGB + ":1372", "sum", K9, V9, [(1, 6)],
       pred={"col": K9, "type": "int32", "op": "equal", "const": 1})
single("IntSimpleMin", DGB + ":1390", "min", K9, V9, [(0, 1), (1, -4), (2, 15), (-1, 2)])
single("IntSimpleMax", DGB + ":1396", "max", K9, V9, [(0, 1), (1, 5), (2, 15), (-1, 2)])
single("IntSimpleAvg", DGB + ":1402", "avg", K9, V9, [(0, 1), (1, 1), (2, 15), (-1, 2)])
single("IntSimpleCount", DGB + ":1408", "count", K9, V9, [(0, 2), (1, 4), (2, 1), (-1, 2)])
single("IntSimpleCountAsterisk", DGB + ":1414", "count", K9, V9, [(0, 2), (1, 4), (2, 1), (-1, 2)])
single("NullIntKeysWhere", DGB + ":1600", "sum", [1, -1, 1, -1, 2, -1, 2, 5], [1, 19, 2, 21, 4, -1, 8, -1],
       [(None, 19), (1, 2), (2, 12), (5, None)],
       pred={"col": [0, 8, 7, 1, 8, 2, 9, 7], "type": "int32", "op": "greater", "const": 4},
       key_nulls=[False, True, False, True, False, True, False, False],
       value_nulls=[False, False, False, False, False, True, False, True])

MA = [1, 1, 1, 2, 5, 7, -1, 5]
MB = [2, 2, 5, 1, 1, 7, -5, 1]
MV = [5, 5, 24, 1, 7, 1, 1, 2]
multi("MultiKeySingleBlockSum", DGB + ":1485", "sum", [1, 1, 1, 2], [2, 2, 5, 1], [5, 7, 24, 1],
      [((1, 2), 12), ((1, 5), 24), ((2, 1), 1)])
multi("MultiKeySimpleSum", DGB + ":1491", "sum", MA, MB, MV,
      [((1, 2), 10), ((1, 5), 24), ((2, 1), 1), ((5, 1), 9), ((7, 7), 1), ((-1, -5), 1)])
multi("MultiKeySimpleMin", DGB + ":1498", "min", MA, MB, MV,
      [((1, 2), 5), ((1, 5), 24), ((2, 1), 1), ((5, 1), 2), ((7, 7), 1), ((-1, -5), 1)])
multi("MultiKeySimpleMax", DGB + ":1505", "max", MA, MB, MV,
      [((1, 2), 5), ((1, 5), 24), ((2, 1), 1), ((5, 1), 7), ((7, 7), 1), ((-1, -5), 1)])
multi("MultiKeySimpleAvg", DGB + ":1512", "avg", MA, MB, MV,
      [((1, 2), 5), ((1, 5), 24), ((2, 1), 1), ((5, 1), 4), ((7, 7), 1), ((-1, -5), 1)])
multi("MultiKeySimpleCount", DGB + ":1519", "count", MA, MB, MV,
      [((1, 2), 2), ((1, 5), 1), ((2, 1), 1), ((5, 1), 2), ((7, 7), 1), ((-1, -5), 1)])

# GROUP BY without aggregation: the result is the key set (DispatcherGroupByTests.cpp:1623-1641).
for nm, line, keys in [("IntKeyNoAggSingleBlock", 1623, [7, 4, 7, 3]),
                       ("IntKeyNoAggMoreBlocks", 1628,
                        [0, 1, 2, 3, 4, 8, -1, 5, -3, -4, -5, -255, 2, 8, -5, 7, 9, 9, 5, 4])]:
    single(nm, DGB + f":{line}", "none", keys, None, [(k, None) for k in sorted(set(keys))])
for nm, line, blocks in [("GPUIntKeyNoAggOneBlock", 620, [[0, 1, 2, 3, 10, 7, 1, 2, 5, -1, 3, 2, 1, 0, 0, 7]]),
                         ("GPUIntKeyNoAggMoreBlocks", 625, [[0, 1, 2, 3], [0, 1, 2, 3], [3, 1, 0, 2], [1, 1, 3, -5]])]:
    keys = [k for b in blocks for k in b]
    single(nm, GGB + f":{line}", "none", keys, None, [(k, None) for k in sorted(set(keys))],
           block=len(blocks[0]), table_size=256)

# GPUGroupByTests multi-key cases run with a hash table of 8 entries (GPUGroupByTests.cu:110-112).
multi("GPUMultiKeyUnique", GGB + ":520", "sum", [1, 1, 1, 1, 2, 3, 4, 0], [1, 2, 3, 4, 1, 1, 1, 0], [1] * 8,
      [((1, 1), 1), ((1, 2), 1), ((1, 3), 1), ((1, 4), 1), ((2, 1), 1), ((3, 1), 1), ((4, 1), 1), ((0, 0), 1)],
      block=8, table_size=8)
multi("GPUMultiKeySimple", GGB + ":531", "sum", [1, 1, 1, 2, 1, 1, 2, 2], [1, 2, 3, 4, 1, 1, -1, -1], [1] * 8,
      [((1, 1), 3), ((1, 2), 1), ((1, 3), 1), ((2, 4), 1), ((2, -1), 2)], block=8, table_size=8)

# DispatcherNullTests single-key cases: 32 inserted rows, block size 8, value 2.
rows = range(32)
exp = {}
null_sum = 0
for i in rows:
    if i % 4 == 2:
        null_sum += 2
    else:
        exp[i % 4] = exp.get(i % 4, 0) + 2
single("GroupByNullKeySum", DNT + ":921", "sum", [i % 4 for i in rows], [2] * 32,
       [(None, null_sum)] + sorted(exp.items()), block=8, key_nulls=[i % 4 == 2 for i in rows])
single("GroupByNullKeyAvg", DNT + ":1005", "avg", [i % 4 for i in rows], [2] * 32,
       [(None, 2), (0, 2), (1, 2), (3, 2)], block=8, key_nulls=[i % 4 == 2 for i in rows])
vnull = [((i % 4) == 2 and i < 8) or (i % 4) == 3 for i in rows]
sums, cnts = {}, {}
for i in rows:
    cnts.setdefault(i % 4, 0)
    if not vnull[i]:
        sums[i % 4] = sums.get(i % 4, 0) + 2
        cnts[i % 4] += 1
single("GroupByNullValueSum", DNT + ":1090", "sum", [i % 4 for i in rows], [2] * 32,
       [(k, sums.get(k)) for k in range(4)], block=8, value_nulls=vnull)
single("GroupByNullValueAvg", DNT + ":1191", "avg", [i % 4 for i in rows], [2] * 32,
       [(k, 2 if k in sums else None) for k in range(4)], block=8, value_nulls=vnull)
single("GroupByNullValueCount", DNT + ":1288", "count", [i % 4 for i in rows], [2] * 32,
       [(k, cnts[k]) for k in range(4)], block=8, value_nulls=vnull)


def gbmk(name, line, agg, ka, kan, kb, kbn, vals, vn, ea, ean, eb, ebn, ev, evn):
    expected = []
    for a, an, b, bn, v, n in zip(ea, ean, eb, ebn, ev, evn):
        expected.append(((None if an else a, None if bn else b), None if n else v))
    multi(name, DNT + f":{line}", agg, ka, kb, vals, expected, block=8, ka_nulls=kan, kb_nulls=kbn,
          value_nulls=vn if any(vn) else None)


T, F = True, False
KA = [-1, 0, -1, 0, 5, 1, -1, -1]
KAN = [T, F, T, F, F, F, T, T]
KB = [-1, -1, 0, 0, 3, -1, 3, -1]
KBN = [T, T, F, F, F, T, F, T]
EA = [-1, -1, -1, 0, 1, 0, 5]
EAN = [T, T, T, F, F, F, F]
EB = [-1, 0, 3, -1, -1, 0, 3]
EBN = [T, F, F, T, T, F, F]
gbmk("GroupByMultiKeyNullKeySum", 2053, "sum", KA, KAN, KB, KBN, [10] * 8, [F] * 8, EA, EAN, EB, EBN,
     [20, 10, 10, 10, 10, 10, 10], [F] * 7)
gbmk("GroupByMultiKeyNullKeyMin", 2063, "min", KA, KAN, KB, KBN, [-5, 80, 10, 10, 10, 10, 10, 30], [F] * 8, EA, EAN,
     EB, EBN, [-5, 10, 10, 80, 10, 10, 10], [F] * 7)
gbmk("GroupByMultiKeyNullKeyMax", 2073, "max", KA, KAN, KB, KBN, [-5, 80, 1, 2, 3, 4, 5, 30], [F] * 8, EA, EAN, EB,
     EBN, [30, 1, 5, 80, 4, 2, 3], [F] * 7)
gbmk("GroupByMultiKeyNullKeyAvg", 2083, "avg", KA, KAN, KB, KBN, [10, 80, 10, 10, 10, 10, 10, 20], [F] * 8, EA, EAN,
     EB, EBN, [15, 10, 10, 80, 10, 10, 10], [F] * 7)
gbmk("GroupByMultiKeyNullKeyCount", 2093, "count", KA, KAN, KB, KBN, [10, 80, 10, 10, 10, 10, 10, 20], [F] * 8, EA,
     EAN, EB, EBN, [2, 1, 1, 1, 1, 1, 1], [F] * 7)
VA = [0, -1, 1, -1, 2, 2, 1, 0, -1, 2, 1, 2, -1, 0]
VB = [0, -1, -1, 1, 0, 0, 7, 0, -1, 0, 7, 0, 1, 0]
VV = [2, -21, -1, -1, 2, -1, -1, 2, 5, -1, 1, 7, -1, 2]
VN = [F, F, T, F, F, T, T, F, F, T, F, F, F, F]
EA2 = [0, -1, 1, -1, 2, 1]
EB2 = [0, -1, -1, 1, 0, 7]
gbmk("GroupByMultiKeyNullValueSum", 2104, "sum", VA, [F] * 14, VB, [F] * 14, VV, VN, EA2, [F] * 6, EB2, [F] * 6,
     [6, -16, -1, -2, 9, 1], [F, F, T, F, F, F])
gbmk("GroupByMultiKeyNullValueMin", 2117, "min", VA, [F] * 14, VB, [F] * 14, VV, VN, EA2, [F] * 6, EB2, [F] * 6,
     [2, -21, -1, -1, 2, 1], [F, F, T, F, F, F])
gbmk("GroupByMultiKeyNullValueMax", 2130, "max", VA, [F] * 14, VB, [F] * 14, VV, VN, EA2, [F] * 6, EB2, [F] * 6,
     [2, 5, -1, -1, 7, 1], [F, F, T, F, F, F])
gbmk("GroupByMultiKeyNullValueAvg", 2143, "avg", VA, [F] * 14, VB, [F] * 14, VV, VN, EA2, [F] * 6, EB2, [F] * 6,
     [2, -8, -1, -1, 4, 1], [F, F, T, F, F, F])
gbmk("GroupByMultiKeyNullValueCount", 2156, "count", VA, [F] * 14, VB, [F] * 14,
     [2, -21, -1, -1, 2, -1, -1, 2, 5, -1, 2, 7, -1, 2], VN, EA2, [F] * 6, EB2, [F] * 6, [3, 2, 0, 2, 2, 1], [F] * 6)

# Hash-table growth (DispatcherGroupByTests.cpp:1746-1802): 262144 * 3 / 2 unique keys, AVG of a constant 7,
# processed in blocks of 131072 rows through a table that first holds GroupByBuckets = 262144 keys.
buckets = 262144
unique = buckets * 3 // 2
cases.append({
    "name": "UnlimitedNumberOfKeysAverage", "source": DGB + ":1746", "agg": "avg", "n_key_cols": 1,
    "key_type": "int32", "value_type": "int32", "generator": {"kind": "modulo", "n": unique * 9 // 8,
                                                              "modulus": unique, "value": 7},
    "block": buckets // 2, "table_size": buckets, "grow_on_full": True,
    "expected_groups": unique, "expected_value_all": 7,
})

# GROUP BY + ORDER BY (DispatcherGroupByTests.cpp:1551-1588): SELECT colInteger, SUM(colID) ... GROUP BY colInteger
# ORDER BY colInteger (resp. ORDER BY SUM(colID) - 2, the same order as SUM(colID)), colID the row number; the
# expected rows in the order the tests assert.
order_cases = []
OBK = [10, 10, 2, 2, 6, 6, 4, 4, 8, 8]
order_cases.append({"name": "IntegerSimpleSumOrderByKeys", "source": DGB + ":1551", "agg": "sum", "keys": OBK,
                    "values": list(range(len(OBK))), "order_by": "key", "descending": False,
                    "expected": [[2, 5], [4, 13], [6, 9], [8, 17], [10, 1]]})
order_cases.append({"name": "IntegerSimpleSumOrderByValues", "source": DGB + ":1569", "agg": "sum", "keys": OBK,
                    "values": list(range(len(OBK))), "order_by": "value", "descending": False,
                    "expected": [[10, 1], [2, 5], [6, 9], [4, 13], [8, 17]]})

# GROUP BY over string keys.  blocks: the row blocks the test processes one ProcessBlock each; keys None = NULL;
# values None = NULL (values absent: COUNT of the key column, i.e. of rows); expected: (key or None, value or None).
string_cases = []


def gbs(name, src, agg, blocks_keys, blocks_vals, expected, pred_gt=None):
    string_cases.append({"name": name, "source": src, "agg": agg, "blocks_keys": blocks_keys,
                         "blocks_values": blocks_vals, "pred_values_greater": pred_gt,
                         "expected": [{"key": k, "value": v} for k, v in expected]})


gbs("StringUnique", GGB + ":474", "sum", [["Apple", "Abcd", "XYZ"]], [[1, 2, -1]],
    [("Apple", 1), ("Abcd", 2), ("XYZ", -1)])
gbs("StringSimple", GGB + ":480", "sum", [["Apple", "Abcd", "XYZ", "Abcd", "ZYX", "XYZ"]], [[1, 2, -1, 3, 7, 5]],
    [("Apple", 1), ("Abcd", 5), ("XYZ", 4), ("ZYX", 7)])
gbs("StringMultiBlockSimple", GGB + ":487", "sum",
    [["Apple", "Abcd"], ["XYZ", "Abcd"], ["ZYX", "XYZ"], ["Apple", "Apple"]], [[1, 1], [1, 2], [1, 2], [2, 4]],
    [("Apple", 7), ("Abcd", 3), ("XYZ", 3), ("ZYX", 1)])
MBK = [["Apple", "Abcd", "Apple", "XYZ"], ["Banana", "XYZ", "Abcd", "0"], ["XYZ", "XYZ"]]
MBV = [[1, 2, 3, 4], [5, 6, 7, 10], [13, 15]]
gbs("StringMultiBlockMediumSum", GGB + ":494", "sum", MBK, MBV,
    [("Apple", 4), ("Abcd", 9), ("Banana", 5), ("XYZ", 38), ("0", 10)])
gbs("StringMultiBlockMediumMin", GGB + ":502", "min", MBK, MBV,
    [("Apple", 1), ("Abcd", 2), ("Banana", 5), ("XYZ", 4), ("0", 10)])
gbs("StringMultiBlockMediumMax", GGB + ":510", "max", MBK, MBV,
    [("Apple", 3), ("Abcd", 7), ("Banana", 5), ("XYZ", 15), ("0", 10)])
SK = ["Apple", "Abcd", "Apple", "XYZ", "Banana", "XYZ", "Abcd", "0", "XYZ", "XYZ"]
SV = [1, 2, 3, 4, 5, 6, 7, 10, 13, 15]
gbs("StringSimpleSum", DGB + ":1422", "sum", [SK], [SV],
    [("Apple", 4), ("Abcd", 9), ("Banana", 5), ("XYZ", 38), ("0", 10)])
gbs("StringSimpleMin", DGB + ":1429", "min", [SK], [SV],
    [("Apple", 1), ("Abcd", 2), ("Banana", 5), ("XYZ", 4), ("0", 10)])
gbs("StringSimpleMax", DGB + ":1436", "max", [SK], [SV],
    [("Apple", 3), ("Abcd", 7), ("Banana", 5), ("XYZ", 15), ("0", 10)])
gbs("StringSimpleAvg", DGB + ":1443", "avg", [SK], [SV],
    [("Apple", 2), ("Abcd", 4), ("Banana", 5), ("XYZ", 9), ("0", 10)])
gbs("StringSimpleCount", DGB + ":1450", "count", [SK], [SV],
    [("Apple", 2), ("Abcd", 2), ("Banana", 1), ("XYZ", 4), ("0", 1)])
gbs("StringSimpleCountStringWhere", DGB + ":1457", "count", [SK], None, [("Abcd", 1), ("XYZ", 3), ("0", 1)],
    pred_gt={"values": [SV], "const": 5})
gbs("StringSimpleCountString", DGB + ":1463", "count", [SK], None,
    [("Apple", 2), ("Abcd", 2), ("Banana", 1), ("XYZ", 4), ("0", 1)])


def null_rows(n, key_of, null_key, null_val):
    keys = [None if null_key(i) else key_of(i) for i in range(n)]
    vals = [None if null_val(i) else 2 for i in range(n)]
    return [keys[b:b + 8] for b in range(0, n, 8)], [vals[b:b + 8] for b in range(0, n, 8)]


# DispatcherNullTests.cpp:1372-1456: 32 rows in blocks of 8, key i%4 (2: NULL), value 2.
nk, nv = null_rows(32, lambda i: ["Apple", "Nut", None, "XYZ"][i % 4], lambda i: i % 4 == 2, lambda i: False)
gbs("GroupByStringNullKeySum", DNT + ":1372", "sum", nk, nv, [(None, 16), ("Apple", 16), ("Nut", 16), ("XYZ", 16)])
# DispatcherNullTests.cpp:1458-1750: 24 rows in blocks of 8, value NULL where (i%4 == 2 and i < 8) or i%4 == 3.
vk, vv = null_rows(24, lambda i: ["Apple", "Nut", "Straw", "car0"][i % 4], lambda i: False,
                   lambda i: (i % 4 == 2 and i < 8) or i % 4 == 3)
gbs("GroupByStringNullValueSum", DNT + ":1458", "sum", vk, vv, [("Apple", 12), ("Nut", 12), ("Straw", 8), ("car0", None)])
gbs("GroupByStringNullValueAvg", DNT + ":1558", "avg", vk, vv, [("Apple", 2), ("Nut", 2), ("Straw", 2), ("car0", None)])
gbs("GroupByStringNullValueCount", DNT + ":1654", "count", vk, vv, [("Apple", 6), ("Nut", 6), ("Straw", 4), ("car0", 0)])

# AAFL compressed blocks (qikkDB_test/GPUCompressionTests.cpp:27-50 fixtures, 1024-row block, assertions at the line
# given): the first eight 32-bit words of the compressed block as the test asserts them on Linux (an 8-byte unsigned
# long), or "plain" when the block stays uncompressed (the test then only checks that the data is unchanged).
GCT = "qikkDB_test/GPUCompressionTests.cpp"
compression_cases = [
    {"name": "CompressionInt", "source": GCT + ":79", "column": "int32 i - 512",
     "head32": [1024, 0, 398, 0, 32, 0, 0, 0]},
    {"name": "CompressionIntLarge", "source": GCT + ":108", "column": "int32 (i - 512) * 100000000 (wrapping)",
     "head32": "plain"},
    {"name": "CompressionLong", "source": GCT + ":122", "column": "int64 (i - 512) * 100000",
     "head64": [1024, 487, 32, 0, 0, 0, 0, 0]},
    {"name": "CompressionFloatPositive", "source": GCT + ":151", "column": "float32 i / 100.0 + 10",
     "head32": [1024, 0, 846, 0, 32, 0, 0, 0]},
    {"name": "CompressionFloatNegative", "source": GCT + ":183", "column": "float32 -(i / 1000.0 + 10)",
     "head32": [1024, 0, 750, 0, 32, 0, 0, 0]},
    {"name": "CompressionFloatMixed", "source": GCT + ":229", "column": "float32 (i - 512) / 100.0",
     "head32": "plain"},
]

with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
    json.dump({"generated_by": "tests/golden/make_kats.py", "cases": cases, "order_by_cases": order_cases,
               "string_cases": string_cases, "compression_cases": compression_cases}, f, indent=1)
print(len(cases), "cases,", len(order_cases), "ORDER BY cases,", len(string_cases), "string cases")
