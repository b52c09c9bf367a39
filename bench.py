#!/usr/bin/env python
"""Filtered GROUP BY benchmark (one JSON line on rank 0).

Headline workload (the filtered GROUP BY at scale): 256M rows per GPU; float32 predicate column uniform in [0, 1)
with WHERE p < 0.5; int64 keys Zipf(s = 1.1) over 1M distinct values; float32 lognormal(mu = 2, sigma = 1) values;
SUM and AVG (FP64 accumulation) in one global hash table.  Inputs are seeded synthetic columns generated on the
host; 16 bytes per row (4.3 GB per GPU), larger than L2, so no flush is needed between steps.

A step = one whole query on device-resident columns: table reset, the fused filter + aggregation pass, and
GetResults (result compaction, count read back).  With --gpus N (torchrun, one rank per GPU) every rank
aggregates its own 256M-row shard, then the partial tables are exchanged by key owner with NCCL all-to-all and
merged (weak scaling).  `e2e` measures the same query through the C ABI from pinned HOST columns
(qdb_gb_process_host: chunked H2D overlapped with aggregation) including the D2H of the result columns.
`cpu_baseline` runs the oracle over every row of the workload and its result checks the GPU's (`parity`).

On one GPU the same line also carries the other configurations, each measured after the headline:
`plain_1m` (2^20 rows, int32 keys over 1000 values, cold and warm), `composite_128m` (2^27 rows, 4096 x 4096
composite keys), `batched` (4096 instances in one CUDA graph against the plain path looped in C), `served`
(continuous batching over 2^30 resident rows at four Poisson rates), and the operators next to the path:
`scalar_256m` (the filtered workload's WHERE and values without GROUP BY), `string_32m` (GROUP BY over 2^25 string
keys), `order_by_groups` (ORDER BY SUM DESC of the string GROUP BY's groups) and `compressed_keys_256m` (the
headline workload with its keys as an AAFL-compressed block); --headline-only skips them.

--impl reference times the reference's CPU-side GROUP BY (the hash-map aggregation its tests check against,
restated in oracle/) on all host threads over the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

ROWS = 1 << 28
N_DISTINCT = 1_000_000
BYTES_PER_ROW = 16  # 4 (predicate) + 8 (key) + 4 (value)
FLOAT_RTOL = 1e-5  # float SUM/AVG against the FP64 oracle
SEED = 20240601
METRIC = "filtered GROUP BY rows/s"
BATCH_INSTANCES = 4096
BATCH_SEED = 20240602
BATCH_METRIC = "batched GROUP BY queries/s"
BATCH_WORKLOAD = ("batched-4096: 4096 independent GROUP BY instances, rows log-uniform in [1K, 4M], cardinality "
                  "log-uniform in [4, 64K], int32 keys uniform over the cardinality, int64 or f32 values (50/50), "
                  "aggregates SUM+MIN+MAX+COUNT | SUM+AVG | SUM+COUNT+MAX")
WORKLOAD = "filtered-groupby-256M: f32 pred p<0.5, int64 Zipf(1.1) keys over 1M, f32 lognormal(2,1) values, SUM+AVG"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--cpu-sample-rows", type=int, default=0,
                    help="rows of the CPU baseline (0 = every row; then its result also checks the GPU's)")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the plain, composite, batched and served sub-workloads of the default run")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="filtered",
                    choices=["filtered", "batched", "served", "plain", "composite", "scalar", "string", "compressed"])
    ap.add_argument("--composite-rows", type=int, default=1 << 27)
    ap.add_argument("--string-rows", type=int, default=1 << 25)
    ap.add_argument("--no-oracle", action="store_true",
                    help="plain / composite / scalar / string / compressed on their own: skip the oracle leg")
    ap.add_argument("--instances", type=int, default=BATCH_INSTANCES)
    ap.add_argument("--plain-sample", type=int, default=0,
                    help="batched / served: queries of the one-by-one plain-path comparison (0 = all / 24)")
    ap.add_argument("--served-rows", type=int, default=1 << 30)
    ap.add_argument("--served-queries", type=int, default=128)
    ap.add_argument("--served-batch", type=int, default=32)
    ap.add_argument("--served-plain-rows", type=int, default=None,
                    help="served: row count from which a query runs alone through the single-query fast pass "
                         "(<= 0: off; default: the library's, 2^22)")
    ap.add_argument("--served-plain-groups", type=int, default=None,
                    help="served: table capacity from which a query runs alone through the single-query fast pass "
                         "(<= 0: off, the library's default)")
    return ap.parse_args()


def gen_columns(n: int, shard: int, pinned: bool):
    """Host columns of the workload (shard selects the RNG streams, so every rank holds different rows)."""
    import torch

    from qikkdb_b200 import datagen as dg
    cols = {}
    for name, dt in (("pred", torch.float32), ("key", torch.int64), ("val", torch.float32)):
        cols[name] = torch.empty(n, dtype=dt, pin_memory=pinned)
    dg.uniform_f32(SEED, 3 * shard + 0, n, out=cols["pred"].numpy())
    dg.zipf_i64(SEED, 3 * shard + 1, n, N_DISTINCT, 1.1, out=cols["key"].numpy())
    dg.lognormal_f32(SEED, 3 * shard + 2, n, 2.0, 1.0, out=cols["val"].numpy())
    return cols


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms; `summary()` keeps the samples taken while the
    timed region ran (from `__enter__` to `__exit__`).  `__enter__` waits for the sampler's first line before it
    returns, so a short timed region still falls between samples that exist."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
            deadline = time.time() + 5.0
            while time.time() < deadline and os.path.getsize(self.file.name) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        self.t0 = time.time()
        return self

    def __exit__(self, *exc):
        self.t1 = time.time()
        if self.proc is not None:
            time.sleep(0.12)  # one more sample after the region
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import datetime
        if self.file is None:
            return None
        try:
            rows = [[c.strip() for c in r.split(",")] for r in open(self.file.name).read().strip().splitlines()
                    if r.strip()]
            os.unlink(self.file.name)
        except Exception:
            return None
        rows = [r for r in rows if len(r) > 9]
        if not rows:
            return None

        def stamp(r):
            try:
                return datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except Exception:
                return None

        inside = [r for r in rows if stamp(r) is not None and self.t0 - 0.05 <= stamp(r) <= self.t1 + 0.1]
        use = inside or rows
        sm = [float(r[2]) for r in use]
        mx = max(float(r[3]) for r in use)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in use for i in range(4) if r[6 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(use),
                "window": "timed region" if inside else "whole sampler run (no sample inside the timed region)"}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the aggregation kernel from the committed ncu summary, if present."""
    try:
        with open(os.path.join(ROOT, "profiles", "gb_fast_kernel_filtered_256M.json")) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch_256M")
    except Exception:
        return None


def cpu_baseline_and_parity(cols, table, sample_rows: int):
    """The cpu_baseline leg: the oracle (the hash-map GROUP BY the reference's tests check against, all host threads)
    over the first sample_rows rows of the workload (every row by default), timed.  When it covered every row its
    result is also the checker of this run's GPU result: keys and COUNT exactly, SUM and AVG as the largest relative
    error over the groups (the per-query error), against the 1e-5 bound."""
    import oracle
    n = min(sample_rows, cols["key"].numel()) if sample_rows > 0 else cols["key"].numel()
    p = cols["pred"].numpy()[:n]
    k = cols["key"].numpy()[:n]
    v = cols["val"].numpy()[:n]
    full = n == cols["key"].numel()
    r = oracle.groupby(k, v, pred=(p, 2, 0.5, np.float32, None), threads=0, sort=full, timing_only=not full)
    cpu = {"value": n / r["seconds"], "unit": "rows/s", "cores": r["threads"], "kind": "port",
           "sample": f"{'all' if full else 'first'} {n} rows of the workload (same columns), hash-map GROUP BY, "
                     f"{r['threads']} threads, {r['seconds']:.3f} s"}
    if not full:
        return cpu, None
    g = table.results_numpy(["sum", "avg", "count"])
    order = np.argsort(g["keys"][0], kind="stable")
    same_groups = g["n_groups"] == r["count"]
    keys_equal = bool(same_groups and (g["keys"][0][order] == r["keys"][0]).all())
    count_equal = bool(keys_equal and (g["count"][order] == r["cnt"]).all())
    rel = {}
    if keys_equal:
        for a in ("sum", "avg"):
            rel[a] = float((np.abs(g[a][order] - r[a]) / np.abs(r[a])).max())
    ok = keys_equal and count_equal and max(rel.values(), default=1.0) <= FLOAT_RTOL
    parity = {"checked_against": "oracle (FP64 hash-map GROUP BY) over every row", "groups": int(g["n_groups"]),
              "keys_equal": keys_equal, "count_equal": count_equal, "max_rel_err": rel, "rtol": FLOAT_RTOL,
              "parity": bool(ok)}
    return cpu, parity


def run_reference(args):
    """The reference arm: the reference's CPU-side GROUP BY (the hash-map aggregation its tests check against,
    restated in oracle/) on all host threads over the same 256M-row workload.  A step aggregates every row; only if
    K + W such steps would take more than four minutes does a step take a leading sample of the rows instead."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    n_all = args.rows
    cols = gen_columns(n_all, 0, pinned=False)
    p, k, v = cols["pred"].numpy(), cols["key"].numpy(), cols["val"].numpy()

    def one(n):
        return oracle.groupby(k[:n], v[:n], pred=(p[:n], 2, 0.5, np.float32, None), threads=0, sort=False,
                              timing_only=True)

    first = one(n_all)
    n = n_all
    if (args.warmup + args.steps) * first["seconds"] > 240.0:
        n = max(1 << 20, int(n_all * 240.0 / ((args.warmup + args.steps) * first["seconds"])))
    secs = []
    threads = first["threads"]
    for i in range(args.warmup + args.steps):
        r = first if (i == 0 and n == n_all) else one(n)
        if i >= args.warmup:
            secs.append(r["seconds"])
    t = statistics.mean(secs)
    value = n / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rows_per_step": n, "rows_of_workload": n_all,
                       "same_config": n == n_all},
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                             "sample": f"{'all' if n == n_all else 'first'} {n} rows of the workload per step, "
                                       f"all host threads"},
            "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    from qikkdb_b200 import _capi
    from qikkdb_b200.groupby import FilterConditions, GroupByTable, make_pred

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    lib = _capi.lib()
    n = args.rows
    cols = gen_columns(n, rank, pinned=True)
    dcols = {k: v.to(dev, non_blocking=False) for k, v in cols.items()}
    torch.cuda.synchronize()
    aggs = ["sum", "avg", "count"]
    cap = 1 << 20
    table = GroupByTable(aggs, np.int64, np.float32, cap)
    pred = make_pred(dcols["pred"], FilterConditions.less, 0.5, np.float32)
    stream = torch.cuda.current_stream()
    owner_ops = None
    if world > 1:
        from qikkdb_b200.dist import CudaOps
        owner_ops = CudaOps(aggs, np.int64, np.float32, cap)

    agg_ms = []

    def step(timed: bool):
        table.reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        table.process([dcols["key"]], dcols["val"], n, pred=pred, sync=False)
        e1.record(stream)
        out = table
        if world > 1:
            from qikkdb_b200.dist import exchange_and_merge
            out = exchange_and_merge(table, owner_ops, device=dev)
        keys, knulls, vals, g = out.results(["sum", "avg"])
        table.check()
        if timed:
            agg_ms.append(e0.elapsed_time(e1))
        return g

    for _ in range(args.warmup):
        groups = step(False)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.qdb_launch_count()
    sampler = ClockSampler(local)
    with sampler:
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(args.steps):
            groups = step(True)
        end.record(stream)
        torch.cuda.synchronize()
    launches = lib.qdb_launch_count() - launches0
    clocks = sampler.summary()
    ms = start.elapsed_time(end) / args.steps
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n / (ms / 1e3)

    # end to end through the C ABI from pinned host columns, result columns read back to host
    e2e = None
    if not args.no_e2e:
        host_out = {}
        e2e_ms = []
        h2d = n * BYTES_PER_ROW
        d2h = 0
        for i in range(args.warmup + args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            table.reset()
            table.process_host([cols["key"]], cols["val"],
                               pred=(cols["pred"], FilterConditions.less, 0.5, np.float32), chunk_rows=1 << 24)
            keys, knulls, vals, g = table.results(["sum", "avg"])
            host = [keys[0], vals["sum"][0], vals["avg"][0], vals["sum"][1]]
            d2h = 0
            for j, b in enumerate(host):
                if j not in host_out or host_out[j].numel() * host_out[j].element_size() < b.nbytes:
                    host_out[j] = torch.empty(max(b.nbytes, 8), dtype=torch.uint8, pin_memory=True)
                if b.nbytes:
                    _capi.check(lib.qdb_memcpy_d2h(host_out[j].data_ptr(), b.ptr, b.nbytes, stream.cuda_stream))
                d2h += b.nbytes
            e1.record(stream)
            torch.cuda.synchronize()
            table.check()
            if i >= args.warmup:
                e2e_ms.append(e0.elapsed_time(e1))
        em = statistics.mean(e2e_ms)
        if world > 1:
            t = torch.tensor([em], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            em = float(t.item())
        e2e = {"value": world * n / (em / 1e3), "unit": "rows/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": em,
               "path": "qdb_gb_process_host (pinned host columns, 16M-row chunks) + qdb_gb_results_multi + D2H"}

    peak, peak_kind = measured_peak()
    t_agg = statistics.mean(agg_ms) / 1e3
    achieved = n * BYTES_PER_ROW / t_agg / 1e9
    traffic = profiled_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "gb_fast_kernel + gb_fspill_kernel (fused filter + shared-table aggregate, spill pass)",
                "kernel_ms": t_agg * 1e3, "algorithmic_bytes_per_launch": n * BYTES_PER_ROW,
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, copy bandwidth)"}
    cpu, parity = (cpu_baseline_and_parity(cols, table, args.cpu_sample_rows) if (rank == 0 and world == 1)
                   else (None, None))
    subs = {}
    if world == 1 and not args.headline_only:
        # The other configurations of the workload family, each measured on its own after the headline's columns
        # are released: plain 1M-row GROUP BY (cold and warm), the 128M-row composite key, batched and served.
        del dcols, table, pred
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        subs["plain_1m"] = c0_measure(args, dev)
        subs["composite_128m"] = c2_measure(args, dev)
        torch.cuda.empty_cache()
        subs["batched"] = batched_measure(args, dev, sub=True)
        torch.cuda.empty_cache()
        subs["served"] = served_measure(args, dev, sub=True)
        torch.cuda.empty_cache()
        subs["scalar_256m"] = scalar_measure(args, dev)
        torch.cuda.empty_cache()
        subs["string_32m"], subs["order_by_groups"] = string_and_order_measure(args, dev)
        torch.cuda.empty_cache()
        subs["compressed_keys_256m"] = compressed_measure(args, dev)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "rows_per_gpu": n, "global_rows": world * n, "groups": int(groups),
                           "parallelism": f"dp{world}" if world > 1 else "single", "l2": "inputs (4.3 GB) > L2, no flush",
                           "step": "reset + fused filter/aggregate + exchange (N>1) + GetResults"},
                "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "e2e": e2e, "clocks": clocks,
                "gpu_launches": int(launches), **subs}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------------------------
# The plain 1M-row GROUP BY (cold and warm) and the 128M-row composite-key GROUP BY, measured after the headline.
# ---------------------------------------------------------------------------------------------------------------
C0_SEED = 20240604
C0_WORKLOAD = ("plain-groupby-1M: 2^20 rows, int32 key uniform in [0,1000), int32 value uniform in [-1000,1000]; "
               "SUM+MIN+MAX+COUNT in one table, one block")
C2_SEED = 20240605
C2_WORKLOAD = ("composite-groupby-128M: 2^27 rows, (int32 uniform in [0,4096), int32 uniform in [0,4096)) keys "
               "(~16.8M groups), int64 value uniform in [0,2^31); SUM+COUNT+MAX")


def _event_steps(fn, steps: int, warmup: int, before=None):
    """Device time (ms) of each of `steps` calls of fn after `warmup` untimed ones; `before` runs outside the timed
    region ahead of every call (an L2 flush)."""
    import torch
    for _ in range(warmup):
        if before:
            before()
        fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(steps):
        if before:
            before()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def _exact_parity(g: dict, r: dict, aggs) -> dict:
    """Integer GROUP BY results against the oracle's: group count, keys and every aggregate bit for bit."""
    ok = g["n_groups"] == r["count"]
    if ok:
        order = np.lexsort([np.asarray(k, np.int64) for k in reversed(g["keys"])])
        ok = all((np.asarray(gk, np.int64)[order] == rk).all() for gk, rk in zip(g["keys"], r["keys"]))
        for a in aggs:
            ok = ok and bool((np.asarray(g[a], np.int64)[order] == r["cnt" if a == "count" else a]).all())
    return {"checked_against": "oracle (hash-map GROUP BY) over every row", "groups": int(g["n_groups"]),
            "exact": bool(ok), "parity": bool(ok)}


def c0_measure(args, dev) -> dict:
    import torch

    import oracle
    from qikkdb_b200 import datagen as dg
    from qikkdb_b200.groupby import GroupByTable
    n = 1 << 20
    aggs = ["sum", "min", "max", "count"]
    k = dg.uniform_i32(C0_SEED, 0, n, 0, 999)
    v = dg.uniform_i32(C0_SEED, 1, n, -1000, 1000)
    dk, dv = torch.from_numpy(k).to(dev), torch.from_numpy(v).to(dev)
    t = GroupByTable(aggs, np.int32, np.int32, 1000)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # twice the L2

    def step():
        t.reset()
        t.process([dk], dv, n, sync=False)
        t.results(aggs)

    warm = _event_steps(step, args.steps, args.warmup)
    cold = _event_steps(step, args.steps, args.warmup, before=lambda: flush.fill_(1))
    g = t.results_numpy(aggs)
    # cpu_baseline leg: the oracle over the same 1M rows, timed; its result checks the GPU result bit for bit
    r = oracle.groupby(k, v, threads=0)
    wm, cm = statistics.median(warm), statistics.median(cold)
    return {"workload": C0_WORKLOAD, "metric": "plain GROUP BY rows/s", "unit": "rows/s",
            "warm": {"value": n / (wm / 1e3), "ms_per_step": wm},
            "cold": {"value": n / (cm / 1e3), "ms_per_step": cm, "l2": "256 MB written before every step"},
            "step": "reset + fused aggregate + GetResults (4 aggregates, one pass)",
            "bytes_per_row": 8,
            "cpu_baseline": {"value": n / r["seconds"], "unit": "rows/s", "cores": r["threads"], "kind": "port",
                             "sample": f"all {n} rows, hash-map GROUP BY, {r['threads']} threads"},
            "parity": _exact_parity(g, r, aggs)}


def c2_measure(args, dev) -> dict:
    import torch

    from qikkdb_b200 import datagen as dg
    from qikkdb_b200.groupby import GroupByTable
    n = args.composite_rows
    aggs = ["sum", "count", "max"]
    a = dg.uniform_i32(C2_SEED, 0, n, 0, 4095)
    b = dg.uniform_i32(C2_SEED, 1, n, 0, 4095)
    v = dg.uniform_i64(C2_SEED, 2, n, 0, (1 << 31) - 1)
    da, db, dv = (torch.from_numpy(x).to(dev) for x in (a, b, v))
    t = GroupByTable(aggs, np.int32, np.int64, 1 << 24, n_key_cols=2)
    agg_ms = []

    def step():
        t.reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        t.process([da, db], dv, n, sync=False)
        e1.record()
        t.results(aggs)
        agg_ms.append((e0, e1))

    ms = _event_steps(step, args.steps, args.warmup)
    kms = statistics.median(x.elapsed_time(z) for x, z in agg_ms[args.warmup:])
    t.check()
    g = t.results_numpy(aggs)
    del da, db, dv
    peak, peak_kind = measured_peak()
    out = {"workload": C2_WORKLOAD, "metric": "composite GROUP BY rows/s", "unit": "rows/s",
           "value": n / (statistics.median(ms) / 1e3), "ms_per_step": statistics.median(ms),
           "step": "reset + aggregation (partition pass + spill pass) + GetResults", "groups": int(g["n_groups"]),
           "roofline": {"bound": "hbm", "achieved": n * 16 / (kms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": n * 16 / (kms / 1e3) / 1e9 / peak, "kernel_ms": kms,
                        "algorithmic_bytes_per_launch": n * 16, "peak_kind": peak_kind},
           "global_updates_per_s": n / (kms / 1e3)}
    if getattr(args, "no_oracle", False):
        return out
    # cpu_baseline leg: the oracle over every row, timed; its result checks the GPU result bit for bit
    import oracle
    r = oracle.groupby([a, b], v, threads=0)
    out["cpu_baseline"] = {"value": n / r["seconds"], "unit": "rows/s", "cores": r["threads"], "kind": "port",
                           "sample": f"all {n} rows, hash-map GROUP BY, {r['threads']} threads, {r['seconds']:.1f} s"}
    out["parity"] = _exact_parity(g, r, aggs)
    return out


# ---------------------------------------------------------------------------------------------------------------
# The operators next to the path: scalar aggregation, GROUP BY over string keys, ORDER BY of GROUP BY results.
# ---------------------------------------------------------------------------------------------------------------
SCALAR_WORKLOAD = ("scalar-256M: 2^28 rows, SUM+COUNT+MIN+MAX of f32 lognormal(2,1) values WHERE f32 U[0,1) < 0.5 "
                   "(the filtered workload's predicate and value columns, no GROUP BY)")
STR_SEED = 20240606
STR_WORKLOAD = ("string-groupby-32M: 2^25 rows, string keys Zipf(1.1) over 1M distinct strings of 8-24 bytes "
                "('c' + 7 digits + '#' padding; GPUString layout: characters + int64 end offsets), int32 value "
                "uniform in [-1000,1000]; SUM+COUNT")
OB_WORKLOAD = "order-by-sum-desc: ORDER BY SUM(value) DESC of the string GROUP BY's groups (int32 column, no NULLs)"


def scalar_measure(args, dev) -> dict:
    import torch

    from qikkdb_b200 import datagen as dg
    from qikkdb_b200.groupby import FilterConditions, ScalarAggregate, make_pred
    n = args.rows
    p = dg.uniform_f32(SEED, 0, n)
    v = dg.lognormal_f32(SEED, 2, n, 2.0, 1.0)
    dp, dv = torch.from_numpy(p).to(dev), torch.from_numpy(v).to(dev)
    pred = make_pred(dp, FilterConditions.less, 0.5, np.float32)
    acc = ScalarAggregate(np.float32)

    def step():
        acc.reset()
        acc.process(dv, n, pred=pred)

    ms = statistics.median(_event_steps(step, args.steps, args.warmup))
    got = {a: acc.result(a) for a in ("sum", "count", "min", "max")}
    peak, peak_kind = measured_peak()
    out = {"workload": SCALAR_WORKLOAD, "metric": "scalar aggregation rows/s", "unit": "rows/s",
           "value": n / (ms / 1e3), "ms_per_step": ms, "step": "reset + one fused filter/reduce launch",
           "l2": "inputs (2.1 GB) > L2, no flush",
           "roofline": {"bound": "hbm", "achieved": n * 8 / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": n * 8 / (ms / 1e3) / 1e9 / peak, "kernel": "scalar_kernel",
                        "algorithmic_bytes_per_launch": n * 8, "peak_kind": peak_kind}}
    del dp, dv, pred
    if getattr(args, "no_oracle", False):
        return out
    # cpu_baseline leg: the oracle (a GROUP BY whose keys are all equal has one group) over every row
    import oracle
    r = oracle.groupby(np.zeros(n, np.int32), v, pred=(p, FilterConditions.less, 0.5, np.float32, None), threads=0)
    err = abs(got["sum"] - r["sum"][0]) / abs(r["sum"][0])
    exact = got["count"] == r["cnt"][0] and got["min"] == r["min"][0] and got["max"] == r["max"][0]
    out["cpu_baseline"] = {"value": n / r["seconds"], "unit": "rows/s", "cores": r["threads"], "kind": "port",
                           "sample": f"all {n} rows, {r['threads']} threads, {r['seconds']:.2f} s"}
    out["parity"] = {"checked_against": "oracle over every row", "count_min_max_exact": bool(exact),
                     "sum_rel_err": err, "parity": bool(exact and err <= FLOAT_RTOL)}
    return out


def string_columns(n: int, n_distinct: int, dev):
    """Device GPUString columns (characters, end offsets) of n rows whose keys are Zipf(1.1) picks from a vocabulary
    of n_distinct strings of 8-24 bytes, assembled on the device from the vocabulary."""
    import torch

    from qikkdb_b200 import datagen as dg
    ids = np.arange(n_distinct, dtype=np.int64)
    lens = 8 + (ids * 7919) % 17
    full = np.full((n_distinct, 24), ord("#"), dtype=np.uint8)
    full[:, 0] = ord("c")
    for j in range(7):
        full[:, 1 + j] = ord("0") + (ids // 10 ** (6 - j)) % 10
    vchars = full[np.arange(24)[None, :] < lens[:, None]]
    vends = np.cumsum(lens)
    pick = dg.zipf_i64(STR_SEED, 0, n, n_distinct, 1.1, map_keys=False) - 1
    dvc = torch.from_numpy(vchars).to(dev)
    dstart = torch.from_numpy(vends - lens).to(dev)
    dlen = torch.from_numpy(lens).to(dev)
    dpick = torch.from_numpy(pick).to(dev)
    rl = dlen[dpick]
    ends = torch.cumsum(rl, 0)
    row = torch.repeat_interleave(torch.arange(n, device=dev), rl)
    pos = torch.arange(int(ends[-1]), device=dev) - (ends - rl)[row]
    chars = dvc[dstart[dpick][row] + pos].contiguous()
    del row, pos, rl
    return chars, ends.contiguous()


def string_and_order_measure(args, dev) -> tuple:
    import torch

    from qikkdb_b200 import datagen as dg
    from qikkdb_b200.groupby import GPUString, StringGroupByTable, order_by
    n, d = args.string_rows, 1 << 20
    chars, ends = string_columns(n, d, dev)
    vals_h = dg.uniform_i32(STR_SEED, 1, n, -1000, 1000)
    vals = torch.from_numpy(vals_h).to(dev)
    nchars = int(chars.numel())
    torch.cuda.empty_cache()
    tab = StringGroupByTable(["sum", "count"], np.int32, d)
    keys = GPUString(chars, ends)
    agg_ms = []

    def step():
        tab.reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        tab.process(keys, vals, n, sync=False)
        e1.record()
        tab.results(["sum", "count"])
        agg_ms.append((e0, e1))

    ms = statistics.median(_event_steps(step, args.steps, args.warmup))
    kms = statistics.median(x.elapsed_time(z) for x, z in agg_ms[args.warmup:])
    tab.check()
    alg = nchars + 12 * n
    peak, peak_kind = measured_peak()
    s_out = {"workload": STR_WORKLOAD, "metric": "string GROUP BY rows/s", "unit": "rows/s",
             "value": n / (ms / 1e3), "ms_per_step": ms,
             "step": "reset + dictionary pass + aggregation pass over slot numbers + GetResults",
             "roofline": {"bound": "hbm", "achieved": alg / (kms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                          "frac": alg / (kms / 1e3) / 1e9 / peak, "kernel": "gbs_map_kernel + aggregation pass",
                          "kernel_ms": kms, "algorithmic_bytes_per_launch": alg,
                          "bytes_per_row": "key characters + 8 (end offset) + 4 (value)", "peak_kind": peak_kind}}

    # ORDER BY SUM DESC of the groups (the step after the GROUP BY), timed alone
    _, _, rv, g = tab.results(["sum"])
    sums = rv["sum"][0].torch()
    perm_box = []
    ob_ms = statistics.median(_event_steps(lambda: perm_box.append(order_by([sums], [True])), args.steps,
                                           args.warmup))
    perm = perm_box[-1].cpu().numpy()
    o_out = {"workload": OB_WORKLOAD, "metric": "ORDER BY rows/s", "unit": "rows/s", "rows": int(g),
             "value": g / (ob_ms / 1e3), "ms_per_step": ob_ms,
             "step": "qdb_order_by: key encoding, 4 stable radix passes (8-bit digits), permutation",
             "roofline": {"bound": "hbm", "achieved": g * 4 * 16 / (ob_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                          "frac": g * 4 * 16 / (ob_ms / 1e3) / 1e9 / peak,
                          "algorithmic_bytes_per_launch": g * 4 * 16,
                          "note": "4 passes x (key + index read and written) per row; at 1M rows launch-bound",
                          "peak_kind": peak_kind}}
    if getattr(args, "no_oracle", False):
        return s_out, o_out
    # cpu_baseline legs: the oracle over every row (string ids by first occurrence + hash-map GROUP BY), and its
    # ORDER BY of the GPU's SUM column; the results check the GPU's bit for bit
    import oracle
    hc, he = chars.cpu().numpy(), ends.cpu().numpy()
    del chars, ends, keys
    t0 = time.perf_counter()
    r = oracle.groupby_string(hc, he, vals_h, threads=0)
    cpu_s = time.perf_counter() - t0
    got = tab.results_host(["sum", "count"])
    ok = len(got) == len(r) and all(k in got and got[k]["sum"] == int(st["sum"]) and got[k]["count"] == int(st["cnt"])
                                    for k, st in r.items())
    s_out["cpu_baseline"] = {"value": n / cpu_s, "unit": "rows/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"all {n} rows: string ids (1 thread) + hash-map GROUP BY, {cpu_s:.1f} s"}
    s_out["parity"] = {"checked_against": "oracle over every row", "groups": len(r), "exact": bool(ok),
                       "parity": bool(ok)}
    hs = sums.cpu().numpy()
    t0 = time.perf_counter()
    operm = oracle.order_by([hs], [True])
    ob_cpu = time.perf_counter() - t0
    same = bool((perm == operm).all())
    o_out["cpu_baseline"] = {"value": g / ob_cpu, "unit": "rows/s", "cores": 1, "kind": "port",
                             "sample": f"all {g} rows, stable sort, {ob_cpu * 1e3:.1f} ms"}
    o_out["parity"] = {"checked_against": "oracle stable ORDER BY of the same column", "exact": same, "parity": same}
    return s_out, o_out


AAFL_WORKLOAD = ("filtered-groupby-256M-aafl-keys: the filtered workload (2^28 rows, f32 pred p<0.5, f32 lognormal(2,1) "
                 "values, SUM+AVG) with int64 Zipf(1.1) keys as ranks 1..1M stored as an AAFL-compressed block "
                 "(20 bits per key); keys unpacked inside the aggregation pass")


def compressed_measure(args, dev) -> dict:
    import torch

    from qikkdb_b200 import datagen as dg
    from qikkdb_b200.groupby import AaflBlock, FilterConditions, GroupByTable, make_pred, process_aafl
    n = args.rows
    k = dg.zipf_i64(SEED, 1, n, N_DISTINCT, 1.1, map_keys=False)
    p = dg.uniform_f32(SEED, 0, n)
    v = dg.lognormal_f32(SEED, 2, n, 2.0, 1.0)
    dk, dp, dv = (torch.from_numpy(x).to(dev) for x in (k, p, v))
    blk = AaflBlock.compress(dk, 1, N_DISTINCT)
    block_bytes = blk.elements * 8
    pred = make_pred(dp, FilterConditions.less, 0.5, np.float32)
    t = GroupByTable(["sum", "avg"], np.int64, np.float32, 1 << 20)
    agg = {"aafl": [], "plain": []}

    def step(kind):
        t.reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        if kind == "aafl":
            process_aafl(t, blk, dv, pred, sync=False)
        else:
            t.process([dk], dv, n, pred=pred, sync=False)
        e1.record()
        t.results(["sum", "avg"])
        agg[kind].append((e0, e1))

    ms = statistics.median(_event_steps(lambda: step("aafl"), args.steps, args.warmup))
    t.check()
    kms = statistics.median(x.elapsed_time(z) for x, z in agg["aafl"][args.warmup:])
    g = t.results_numpy(["sum", "avg"])
    _event_steps(lambda: step("plain"), args.steps, args.warmup)
    pkms = statistics.median(x.elapsed_time(z) for x, z in agg["plain"][args.warmup:])
    alg = n * 8 + block_bytes
    peak, peak_kind = measured_peak()
    out = {"workload": AAFL_WORKLOAD, "metric": "filtered GROUP BY rows/s", "unit": "rows/s",
           "value": n / (ms / 1e3), "ms_per_step": ms, "block_bytes": block_bytes,
           "key_bytes_per_row": block_bytes / n,
           "step": "reset + aggregation pass unpacking the key block + spill pass + GetResults",
           "roofline": {"bound": "hbm", "achieved": alg / (kms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": alg / (kms / 1e3) / 1e9 / peak, "kernel_ms": kms,
                        "kernel": "gb_fast_kernel (keys unpacked in the consumer warps) + gb_fspill_kernel",
                        "algorithmic_bytes_per_launch": alg, "peak_kind": peak_kind},
           "plain_keys_kernel_ms": pkms}
    del dk, dp, dv, pred, blk
    if getattr(args, "no_oracle", False):
        return out
    # cpu_baseline leg: the oracle over every row of the plain columns; its result checks the GPU's
    import oracle
    r = oracle.groupby(k, v, pred=(p, FilterConditions.less, 0.5, np.float32, None), threads=0)
    order = np.argsort(g["keys"][0], kind="stable")
    ok = g["n_groups"] == r["count"] and bool(np.array_equal(g["keys"][0][order], r["keys"][0]))
    err = 0.0
    if ok:
        for a in ("sum", "avg"):
            e = np.abs(g[a][order].astype(np.float64) - r[a]) / np.maximum(np.abs(r[a]), 1e-30)
            err = max(err, float(e.max()))
    out["cpu_baseline"] = {"value": n / r["seconds"], "unit": "rows/s", "cores": r["threads"], "kind": "port",
                           "sample": f"all {n} rows (plain columns), {r['threads']} threads, {r['seconds']:.2f} s"}
    out["parity"] = {"checked_against": "oracle over every row of the plain columns", "groups": int(r["count"]),
                     "keys_exact": bool(ok), "max_rel_err": err, "parity": bool(ok and err <= FLOAT_RTOL)}
    return out


# ---------------------------------------------------------------------------------------------------------------
# Batched workload: many independent GROUP BY queries in one persistent launch (CUDA graph) against the same
# queries issued one by one through the plain path.
# ---------------------------------------------------------------------------------------------------------------
AGG_SHAPES = (("sum", "min", "max", "count"), ("sum", "avg"), ("sum", "count", "max"))


def batched_instances(n_inst: int):
    """Per-instance shape: (rows, cardinality, value dtype, aggregates); seeded."""
    from qikkdb_b200 import datagen as dg
    rows = dg.loguniform_i64(BATCH_SEED, 0, n_inst, 1000, 4_000_000)
    card = dg.loguniform_i64(BATCH_SEED, 1, n_inst, 4, 65536)
    pick = dg.uniform_i32(BATCH_SEED, 2, n_inst, 0, 5)
    out = []
    for i in range(n_inst):
        vdt = np.int64 if pick[i] % 2 == 0 else np.float32
        out.append((int(rows[i]), int(card[i]), vdt, AGG_SHAPES[int(pick[i]) // 2]))
    return out


def batched_columns(shapes, dev, host: bool = False):
    """Keys and values of every instance (seeded per instance), 16-byte aligned slices of three device buffers."""
    import torch

    from qikkdb_b200 import datagen as dg
    pad = lambda n: (n + 3) // 4 * 4  # noqa: E731
    tot_k = sum(pad(r) for r, _, _, _ in shapes)
    tot_i64 = sum(pad(r) for r, _, v, _ in shapes if v == np.int64)
    tot_f32 = sum(pad(r) for r, _, v, _ in shapes if v == np.float32)
    keys = torch.empty(tot_k, dtype=torch.int32, device=dev)
    vi = torch.empty(max(tot_i64, 4), dtype=torch.int64, device=dev)
    vf = torch.empty(max(tot_f32, 4), dtype=torch.float32, device=dev)
    stage_k = torch.empty(4_000_004, dtype=torch.int32, pin_memory=True)
    stage_v = torch.empty(4_000_004, dtype=torch.int64, pin_memory=True)
    views, ok, oi, of = [], 0, 0, 0
    hosts = []
    for i, (r, c, vdt, _) in enumerate(shapes):
        kh = stage_k.numpy()[:r]
        dg.uniform_i32(BATCH_SEED + 1, i, r, 0, c - 1, out=kh)
        kd = keys[ok:ok + r]
        kd.copy_(stage_k[:r])
        ok += pad(r)
        if vdt == np.int64:
            vh = stage_v.numpy()[:r]
            dg.uniform_i64(BATCH_SEED + 2, i, r, -(1 << 40), 1 << 40, out=vh)
            vd = vi[oi:oi + r]
            vd.copy_(stage_v[:r])
            oi += pad(r)
        else:
            vh = stage_v.numpy().view(np.float32)[:r]
            dg.lognormal_f32(BATCH_SEED + 2, i, r, 2.0, 1.0, out=vh)
            vd = vf[of:of + r]
            vd.copy_(stage_v.view(torch.float32)[:r])
            of += pad(r)
        if host:
            hosts.append((kh.copy(), vh.copy()))
        views.append((kd, vd))
        torch.cuda.synchronize(dev)
    return views, hosts, (keys, vi, vf)


def run_batched(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    line = batched_measure(args, torch.device("cuda", local))
    if int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps(line), flush=True)


def batched_measure(args, dev, sub: bool = False) -> dict:
    """The batched workload on `dev`: every instance in one CUDA graph (value: queries/s, device-timed), end to end
    with the results copied to host, against the same queries one by one through the plain path looped in C."""
    import ctypes as C

    import torch

    from qikkdb_b200 import _capi
    from qikkdb_b200.batch import GroupByBatch, Query, plain_run, required_bytes

    lib = _capi.lib()
    shapes = batched_instances(args.instances)
    views, _, bufs = batched_columns(shapes, dev)
    rows_total = sum(r for r, _, _, _ in shapes)
    bytes_total = sum(r * (4 + (8 if v == np.int64 else 4)) for r, _, v, _ in shapes)
    queries = [Query(k, v, list(a), c) for (k, v), (r, c, _, a) in zip(views, shapes)]
    table_bytes, result_bytes = required_bytes(queries)
    b = GroupByBatch(len(queries), table_bytes, result_bytes)
    st = torch.cuda.Stream(dev)
    t0 = time.perf_counter()
    b.set(queries, stream=st.cuda_stream)
    torch.cuda.synchronize(dev)
    set_ms = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    b.autotune(stream=st.cuda_stream)
    tune_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        b.run(graph=True, stream=st.cuda_stream)
    counts, status = b.fetch(stream=st.cuda_stream)
    assert (status == 0).all(), "batched run reported an error status"
    launches0 = lib.qdb_launch_count()
    sampler = ClockSampler(dev.index or 0)
    ev = []
    with sampler:
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            b.run(graph=True, stream=st.cuda_stream)
            e1.record(st)
            ev.append((e0, e1))
        torch.cuda.synchronize(dev)
    launches = lib.qdb_launch_count() - launches0
    step_ms = [x.elapsed_time(z) for x, z in ev]
    ms = statistics.median(step_ms)
    value = len(queries) / (ms / 1e3)
    groups = int(counts.sum())

    # end to end through the C ABI: run + per-query counts/status + every result copied to host
    need = C.c_int64()
    _capi.check(lib.qdb_gb_batch_copy_results(b.handle, 0, len(queries), None, 0, C.byref(need), st.cuda_stream))
    host_res = torch.empty(max(need.value, 8), dtype=torch.uint8, pin_memory=True)
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        b.run(graph=True, stream=st.cuda_stream)
        b.fetch(stream=st.cuda_stream)
        _capi.check(lib.qdb_gb_batch_copy_results(b.handle, 0, len(queries), host_res.data_ptr(), need.value,
                                                  C.byref(need), st.cuda_stream))
        if i >= args.warmup:
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    em = statistics.median(e2e_ms)

    # the same queries one by one through the plain path, the loop in C (no per-query Python): results to host
    sample = queries if args.plain_sample <= 0 else queries[:args.plain_sample]
    plain_run(sample[:8], stream=st.cuda_stream)  # warm-up (pool allocations, module load)
    t0 = time.perf_counter()
    pg = plain_run(sample, results_to_host=True, stream=st.cuda_stream)
    plain_s = time.perf_counter() - t0
    plain_qps = len(sample) / plain_s
    if len(sample) == len(queries):
        assert int(pg.sum()) == groups, f"plain path groups {int(pg.sum())} != batched {groups}"

    peak, peak_kind = measured_peak()
    achieved = bytes_total / (ms / 1e3) / 1e9
    cpu = batched_cpu_baseline(shapes, args, budget_s=5.0 if sub else 15.0)
    del b, views, bufs
    line = {"metric": BATCH_METRIC, "value": value, "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "replicas only",
            "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
            "config": {"workload": BATCH_WORKLOAD, "instances": len(queries), "rows_total": rows_total,
                       "bytes_total": bytes_total, "groups_total": groups,
                       "l2": f"inputs ({bytes_total / 1e9:.1f} GB) > L2, no flush",
                       "step": "one CUDA graph: table init (skipped after the first run) + persistent aggregation "
                               "kernel + result kernel, all instances"},
            "plain_one_by_one": {"value": plain_qps, "unit": "queries/s", "queries": len(sample),
                                 "seconds": plain_s, "groups": int(pg.sum()),
                                 "path": "qdb_gb_plain_run: per query qdb_gb_create, qdb_gb_process_sync, "
                                         "qdb_gb_results_multi, results to host, qdb_free, qdb_gb_destroy (loop in C)"},
            "speedup_vs_plain": value / plain_qps,
            "e2e_speedup_vs_plain": (len(queries) / (em / 1e3)) / plain_qps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "kernel": "whole graph (init + gb_batch_agg_kernel + results)",
                         "algorithmic_bytes_per_launch": bytes_total, "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": len(queries) / (em / 1e3), "unit": "queries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(need.value + len(queries) * 12), "ms_per_step": em,
                    "path": "qdb_gb_batch_run (graph) + qdb_gb_batch_fetch + qdb_gb_batch_copy_results to pinned host; "
                            "inputs device-resident"},
            "set_ms": set_ms, "autotune_s": tune_s, "clocks": sampler.summary(), "gpu_launches": int(launches),
            "step_ms_min_max": [min(step_ms), max(step_ms)]}
    return line


def batched_cpu_baseline(shapes, args, budget_s: float = 15.0) -> dict:
    """The oracle (hash-map GROUP BY, all host threads) on instances in workload order until budget_s."""
    import oracle
    from qikkdb_b200 import datagen as dg
    done, secs, rows = 0, 0.0, 0
    threads = 0
    for i, (r, c, vdt, _) in enumerate(shapes):
        k = dg.uniform_i32(BATCH_SEED + 1, i, r, 0, c - 1)
        v = (dg.uniform_i64(BATCH_SEED + 2, i, r, -(1 << 40), 1 << 40) if vdt == np.int64
             else dg.lognormal_f32(BATCH_SEED + 2, i, r, 2.0, 1.0))
        res = oracle.groupby(k, v, threads=0, sort=False, timing_only=True)
        secs += res["seconds"]
        threads = res["threads"]
        done += 1
        rows += r
        if secs >= budget_s:
            break
    return {"value": done / secs, "unit": "queries/s", "cores": threads, "kind": "port",
            "sample": f"first {done} of {len(shapes)} instances ({rows} rows), hash-map GROUP BY per query, "
                      f"{threads} threads, {secs:.2f} s"}


def run_batched_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    shapes = batched_instances(args.instances)
    secs = []
    cb = None
    for i in range(args.warmup + args.steps):
        cb = batched_cpu_baseline(shapes, args, budget_s=max(2.0, 20.0 / (args.warmup + args.steps)))
        if i >= args.warmup:
            secs.append(cb["value"])
    value = statistics.mean(secs)
    line = {"impl": "reference", "metric": BATCH_METRIC, "value": value, "unit": "queries/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "replicas only", "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
            "config": {"workload": BATCH_WORKLOAD, "instances": len(shapes)},
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cb["cores"], "kind": "port",
                             "sample": cb["sample"]},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------------------------
# Served workload: an open-loop Poisson stream of GROUP BY queries against 1B device-resident rows, continuously
# batched by the serving loop, against the same queries issued one by one through the plain path.
# ---------------------------------------------------------------------------------------------------------------
SERVE_SEED = 20240603
SERVE_METRIC = "served GROUP BY queries/s"
SERVE_WORKLOAD = ("served-1B: open-loop Poisson query stream at 4 rates against 2^30 device-resident rows (int32 key "
                  "uniform, int64 key uniform, f32 predicate U[0,1), f32 lognormal(2,1) value; 20 GB); queries of "
                  "the shapes GROUP BY k32 % c: SUM+MIN+MAX+COUNT | k64 % c: SUM+AVG | k64 % c: SUM+COUNT+MAX, "
                  "WHERE p < s with s uniform in [0.01, 1], c log-uniform in [10, 1M]; table admission budget 40 GB")
SERVE_SHAPES = (("k32", ("sum", "min", "max", "count")), ("k64", ("sum", "avg")), ("k64", ("sum", "count", "max")))


def served_columns(n: int, dev):
    """The resident columns, generated in chunks on the host (seeded) and copied into device buffers."""
    import torch

    from qikkdb_b200 import datagen as dg
    cols = {"k32": torch.empty(n, dtype=torch.int32, device=dev), "k64": torch.empty(n, dtype=torch.int64, device=dev),
            "p": torch.empty(n, dtype=torch.float32, device=dev), "v": torch.empty(n, dtype=torch.float32, device=dev)}
    chunk = 1 << 26
    st = {k: torch.empty(chunk, dtype=v.dtype, pin_memory=True) for k, v in cols.items()}
    for c0 in range(0, n, chunk):
        m = min(chunk, n - c0)
        part = c0 // chunk
        dg.uniform_i32(SERVE_SEED, 4 * part + 0, m, 0, (1 << 31) - 1, out=st["k32"].numpy())
        dg.uniform_i64(SERVE_SEED, 4 * part + 1, m, 0, 1 << 62, out=st["k64"].numpy())
        dg.uniform_f32(SERVE_SEED, 4 * part + 2, m, out=st["p"].numpy())
        dg.lognormal_f32(SERVE_SEED, 4 * part + 3, m, 2.0, 1.0, out=st["v"].numpy())
        for k in cols:
            cols[k][c0:c0 + m].copy_(st[k][:m])
        torch.cuda.synchronize(dev)
    return cols


def served_queries(cols, n_q: int, seed: int):
    from qikkdb_b200.batch import Query
    from qikkdb_b200.groupby import FilterConditions
    from qikkdb_b200 import datagen as dg
    card = dg.loguniform_i64(seed, 0, n_q, 10, 1_000_000)
    sel = dg.uniform_f32(seed, 1, n_q, 0.01, 1.0)
    shape = dg.uniform_i32(seed, 2, n_q, 0, len(SERVE_SHAPES) - 1)
    out = []
    for i in range(n_q):
        kc, aggs = SERVE_SHAPES[int(shape[i])]
        out.append(Query(cols[kc], cols["v"], list(aggs), 0, key_mod=int(card[i]),
                         pred=(cols["p"], FilterConditions.less, float(sel[i]), np.float32)))
    return out


def run_served(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    print(json.dumps(served_measure(args, torch.device("cuda", local))), flush=True)


def served_measure(args, dev, sub: bool = False) -> dict:
    """The served workload on `dev`: closed-burst capacity and four open-loop Poisson rates through the serving loop
    (latencies from arrival to results on the host), against the same kind of queries one by one through the plain
    path looped in C (results to host)."""
    import dataclasses

    import torch

    from qikkdb_b200 import _capi
    from qikkdb_b200.batch import plain_run
    from qikkdb_b200.serve import Server, percentile_ms, poisson_arrivals

    lib = _capi.lib()
    n = args.served_rows
    cols = served_columns(n, dev)
    srv = Server(max_batch=args.served_batch, in_flight=2, table_budget=40 << 30, result_budget=4 << 30,
                 plain_rows=args.served_plain_rows, plain_groups=args.served_plain_groups)
    n_q = args.served_queries
    # warm-up, then capacity: every query of a closed burst submitted at once
    warm = served_queries(cols, 16, SERVE_SEED + 99)
    srv.run_open_loop(warm, np.zeros(len(warm), np.int64))
    burst = served_queries(cols, n_q, SERVE_SEED + 1)
    launches0 = lib.qdb_launch_count()
    sampler = ClockSampler(dev.index or 0)
    with sampler:
        lat, stat, wall = srv.run_open_loop(burst, np.zeros(n_q, np.int64))
    launches = lib.qdb_launch_count() - launches0
    assert (stat == 0).all(), f"served queries failed: {np.unique(stat)}"
    capacity = n_q / (wall / 1e9)
    burst_p50, burst_p99 = percentile_ms(lat, 50), percentile_ms(lat, 99)
    rates = []
    for k, frac in enumerate((0.25, 0.5, 0.75, 0.95)):
        rate = capacity * frac
        qs = served_queries(cols, n_q, SERVE_SEED + 10 + k)
        lat, stat, wall = srv.run_open_loop(qs, poisson_arrivals(rate, n_q, SERVE_SEED + 20 + k))
        assert (stat == 0).all()
        rates.append({"offered_qps": rate, "achieved_qps": n_q / (wall / 1e9), "p50_ms": percentile_ms(lat, 50),
                      "p99_ms": percentile_ms(lat, 99), "queries": n_q})
    st = srv.stats()
    srv.close()

    # the same queries one by one through the plain path (loop in C): key % c column, a table with the query's true
    # group bound, ProcessBlock with the fused WHERE, GetResults, results to host, everything freed
    plain = [dataclasses.replace(q, max_groups=min(q.key_mod, n)) for q in burst[:args.plain_sample or 32]]
    s0 = torch.cuda.current_stream().cuda_stream
    plain_run(plain[:2], stream=s0)
    t0 = time.perf_counter()
    plain_run(plain, results_to_host=True, stream=s0)
    plain_s = time.perf_counter() - t0
    plain_qps = len(plain) / plain_s
    del cols
    line = {"metric": SERVE_METRIC, "value": capacity, "unit": "queries/s", "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "replicas only",
            "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
            "config": {"workload": SERVE_WORKLOAD, "rows": n, "queries_per_rate": n_q, "max_batch": args.served_batch,
                       "in_flight_batches": 2, "table_budget_bytes": 40 << 30,
                       "single_query_route": {
                           "min_rows": args.served_plain_rows if args.served_plain_rows is not None else 1 << 22,
                           "min_groups": args.served_plain_groups or 0},
                       "tables": "sized by the server's cardinality estimate (sampled GEE, capped by the modulus)"},
            "value_is": "closed-burst capacity: all queries submitted at t=0, queries / (first arrival to last result)",
            "burst_p50_ms": burst_p50, "burst_p99_ms": burst_p99,
            "rates": rates,
            "plain_one_by_one": {"value": plain_qps, "unit": "queries/s", "queries": len(plain), "seconds": plain_s,
                                 "path": "qdb_gb_plain_run: per query qdb_arith_mod (key % c column), qdb_gb_create "
                                         "(true bound), qdb_gb_process_sync (fused WHERE), qdb_gb_results_multi, "
                                         "results to host, qdb_free (loop in C)"},
            "speedup_vs_plain": capacity / plain_qps, "server_stats": st,
            "e2e": {"value": capacity, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": None,
                    "path": "qdb_server_run_open_loop: results on the host per query; columns device-resident"},
            "clocks": sampler.summary(), "gpu_launches": int(launches)}
    return line


def run_served_reference(args):
    """The oracle on a bounded sample of the served query stream (rows sampled from the same columns)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    import oracle
    from qikkdb_b200 import datagen as dg
    rows = min(args.served_rows, 1 << 24)
    k32 = dg.uniform_i32(SERVE_SEED, 0, rows, 0, (1 << 31) - 1)
    k64 = dg.uniform_i64(SERVE_SEED, 1, rows, 0, 1 << 62)
    p = dg.uniform_f32(SERVE_SEED, 2, rows)
    v = dg.lognormal_f32(SERVE_SEED, 3, rows, 2.0, 1.0)
    card = dg.loguniform_i64(SERVE_SEED + 1, 0, 64, 10, 1_000_000)
    sel = dg.uniform_f32(SERVE_SEED + 1, 1, 64, 0.01, 1.0)
    shape = dg.uniform_i32(SERVE_SEED + 1, 2, 64, 0, len(SERVE_SHAPES) - 1)
    secs, done, threads = 0.0, 0, 0
    for i in range(64):
        k = k32 if SERVE_SHAPES[int(shape[i])][0] == "k32" else k64
        r = oracle.groupby(np.fmod(k, int(card[i])), v, pred=(p, 2, float(sel[i]), np.float32, None), threads=0,
                           sort=False, timing_only=True)
        secs += r["seconds"]
        threads = r["threads"]
        done += 1
        if secs > 20:
            break
    # scale the sampled rows to the full column length
    value = done / (secs * args.served_rows / rows)
    line = {"impl": "reference", "metric": SERVE_METRIC, "value": value, "unit": "queries/s", "n_gpus": args.gpus,
            "steps": 1, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "replicas only",
            "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
            "config": {"workload": SERVE_WORKLOAD, "rows": args.served_rows},
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "port",
                             "sample": f"{done} queries of the stream over {rows} rows each (time scaled to "
                                       f"{args.served_rows} rows), hash-map GROUP BY, {threads} threads, {secs:.1f} s"},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_sub(args, fn):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps(fn(args, torch.device("cuda", local))), flush=True)


def main():
    args = parse_args()
    if args.workload in ("plain", "composite", "scalar", "string", "compressed"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the headline workload"}))
            return
        fn = {"plain": c0_measure, "composite": c2_measure, "scalar": scalar_measure, "compressed": compressed_measure,
              "string": lambda a, d: dict(zip(("string_32m", "order_by_groups"), string_and_order_measure(a, d)))}
        run_sub(args, fn[args.workload])
        return
    if args.workload == "batched":
        if args.impl == "reference":
            run_batched_reference(args)
        else:
            run_batched(args)
        return
    if args.workload == "served":
        if args.impl == "reference":
            run_served_reference(args)
        else:
            run_served(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
