"""The reference's known-answer GROUP BY cases on the GPU, through the operator mirror (C ABI underneath).

Each case runs the way qikkDB's dispatcher drives the operators (GpuSqlDispatcherAggregationFunctions.h:377-553):
block by block, the WHERE mask from GPUBinary<OP> (filter kernel), keys and values compacted with
GPUReconstruct::reconstructColKeep, then GPUGroupBy::ProcessBlock; GetResults at the end.  The same case also
runs through the fused path (predicate evaluated inside the aggregation pass, whole column at once).
"""
import numpy as np
import pytest
import torch

from kat_util import OPS, expected_map, kat_inputs, load_kats, result_map
from qikkdb_b200.groupby import (GPU_HASH_TABLE_FULL, GPUBinary, GPUGroupBy, GPUReconstruct, GroupByTable,
                                 QueryEngineError, device_nullmask, make_pred, unpack_nullmask)

pytestmark = pytest.mark.gpu
CASES = load_kats()
BUCKETS = 262144  # GroupByBuckets default (configuration/main_config.default:18)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _gpu_result(gb, n_key_cols, agg):
    keys, vals, n, knull, vnull = gb.GetResults()
    if n_key_cols == 1:
        keys, knull = [keys], [knull]
    hk = [k.numpy() for k in keys]
    hkn = [unpack_nullmask(x.numpy(), n) for x in knull]
    hv = vals.numpy() if vals is not None else None
    hvn = unpack_nullmask(vnull.numpy(), n) if (vnull is not None and agg not in ("count", "none")) else None
    return result_map(hk, hkn, hv, hvn), n


def _run_blocks(case, multiplier=1):
    keys, kn, vals, vn = kat_inputs(case)
    agg = case["agg"]
    n = len(keys[0])
    K = [8, 8] if case["n_key_cols"] == 2 else np.int32
    O = np.int64 if agg == "count" else np.int32
    gb = GPUGroupBy(agg, O, K, np.int32, case.get("table_size") or BUCKETS, multiplier)
    block = case["block"] or n
    pred = case.get("pred")
    for b0 in range(0, n, block):
        b1 = min(n, b0 + block)
        nb = b1 - b0
        kcols = [_dev(k[b0:b1]) for k in keys]
        kmasks = [device_nullmask(x[b0:b1]) for x in kn] if kn is not None else [None] * len(kcols)
        vcol = _dev(vals[b0:b1]) if vals is not None else None
        vmask = device_nullmask(vn[b0:b1]) if vn is not None else None
        if pred:
            pcol = _dev(np.asarray(pred["col"], dtype=np.int32)[b0:b1])
            mask = torch.empty(nb, dtype=torch.int8, device="cuda")
            GPUBinary.Binary(OPS[pred["op"]], mask, pcol, np.int32(pred["const"]), nb)
            ck, cnt, ckm = [], 0, []
            for kc, km in zip(kcols, kmasks):
                c, cnt, m = GPUReconstruct.reconstructColKeep(kc, mask, nb, km)
                ck.append(c)
                ckm.append(m)
            cv = cvm = None
            if vcol is not None:
                cv, _, cvm = GPUReconstruct.reconstructColKeep(vcol, mask, nb, vmask)
            kcols, kmasks, vcol, vmask, nb = ck, ckm, cv, cvm, cnt
        if nb == 0:
            continue
        gb.ProcessBlock(kcols if len(kcols) > 1 else kcols[0], vcol, nb,
                        kmasks if len(kmasks) > 1 else kmasks[0], vmask)
    return _gpu_result(gb, case["n_key_cols"], agg)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_kat_operator_pipeline(cuda, case):
    if case.get("grow_on_full"):
        # GpuSqlDispatcher restarts every block with a doubled key-size multiplier on GPU_HASH_TABLE_FULL
        # (GpuSqlDispatcher.cpp:378-394).
        mult, got = 1, None
        for _ in range(6):
            try:
                got, n = _run_blocks(case, mult)
                break
            except QueryEngineError as e:
                assert e.code == GPU_HASH_TABLE_FULL
                mult *= 2
        assert mult > 1, "the first table must overflow"
        assert got is not None and n == case["expected_groups"]
        assert set(got.values()) == {case["expected_value_all"]}
        return
    got, _ = _run_blocks(case)
    assert got == expected_map(case)


@pytest.mark.parametrize("placement", [1, 2])
@pytest.mark.parametrize("case", [c for c in CASES if not c.get("grow_on_full")],
                         ids=[c["name"] for c in CASES if not c.get("grow_on_full")])
def test_kat_fused_path(cuda, case, placement):
    keys, kn, vals, vn = kat_inputs(case)
    agg = case["agg"]
    t = GroupByTable([agg], np.int32, np.int32 if agg != "none" else None, case.get("table_size") or BUCKETS,
                     case["n_key_cols"], placement)
    kd = [_dev(k) for k in keys]
    pred = None
    if case.get("pred"):
        p = case["pred"]
        pcol = _dev(np.asarray(p["col"], dtype=np.int32))
        pred = make_pred(pcol, OPS[p["op"]], p["const"], np.int32)
    t.process(kd, _dev(vals) if (vals is not None and agg != "none") else None, len(keys[0]),
              [device_nullmask(x) for x in kn] if kn is not None else None,
              device_nullmask(vn) if (vn is not None and agg != "none") else None, pred=pred)
    r = t.results_numpy()
    vals_out = r.get(agg) if agg != "none" else None
    vnull = r.get(agg + "_null") if agg not in ("count", "none") else None
    got = result_map(r["keys"], r["key_nulls"], vals_out, vnull)
    assert got == expected_map(case)
