#!/usr/bin/env python
"""Filtered GROUP BY benchmark (one JSON line on rank 0).

Workload (the filtered GROUP BY at scale): 256M rows per GPU; float32 predicate column uniform in [0, 1) with
WHERE p < 0.5; int64 keys Zipf(s = 1.1) over 1M distinct values; float32 lognormal(mu = 2, sigma = 1) values;
SUM and AVG (FP64 accumulation) in one global hash table.  Inputs are seeded synthetic columns generated on
the host; 16 bytes per row (4.3 GB per GPU), larger than L2, so no flush is needed between steps.

A step = one whole query on device-resident columns: table reset, the fused filter + aggregation pass, and
GetResults (result compaction, count read back).  With --gpus N (torchrun, one rank per GPU) every rank
aggregates its own 256M-row shard, then the partial tables are exchanged by key owner with NCCL all-to-all and
merged (weak scaling).  `e2e` measures the same query through the C ABI from pinned HOST columns
(qdb_gb_process_host: chunked H2D overlapped with aggregation) including the D2H of the result columns.

--impl reference times the reference's CPU-side GROUP BY (the hash-map aggregation its tests check against,
restated in oracle/) on all host threads over a bounded sample of the same workload.
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
SEED = 20240601
METRIC = "filtered GROUP BY rows/s"
WORKLOAD = "filtered-groupby-256M: f32 pred p<0.5, int64 Zipf(1.1) keys over 1M, f32 lognormal(2,1) values, SUM+AVG"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--cpu-sample-rows", type=int, default=1 << 25)
    ap.add_argument("--no-e2e", action="store_true")
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
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.file is None:
            return None
        try:
            rows = [r.split(",") for r in open(self.file.name).read().strip().splitlines() if r.strip()]
            os.unlink(self.file.name)
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if len(r) > 8]
        mx = max(float(r[2]) for r in rows if len(r) > 8)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) > 8 for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the aggregation kernel from the committed ncu summary, if present."""
    try:
        with open(os.path.join(ROOT, "profiles", "gb_agg_kernel_filtered_256M.json")) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch_256M")
    except Exception:
        return None


def cpu_baseline(cols, sample_rows: int) -> dict:
    import oracle
    n = min(sample_rows, cols["key"].numel())
    p = cols["pred"].numpy()[:n]
    k = cols["key"].numpy()[:n]
    v = cols["val"].numpy()[:n]
    r = oracle.groupby(k, v, pred=(p, 2, 0.5, np.float32, None), threads=0, sort=False, timing_only=True)
    return {"value": n / r["seconds"], "unit": "rows/s", "cores": r["threads"], "kind": "port",
            "sample": f"first {n} rows of the workload (same columns), hash-map GROUP BY, {r['threads']} threads, "
                      f"{r['seconds']:.3f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    n = args.cpu_sample_rows
    cols = gen_columns(n, 0, pinned=False)
    p, k, v = cols["pred"].numpy(), cols["key"].numpy(), cols["val"].numpy()
    secs = []
    threads = 0
    for i in range(args.warmup + args.steps):
        r = oracle.groupby(k, v, pred=(p, 2, 0.5, np.float32, None), threads=0, sort=False, timing_only=True)
        threads = r["threads"]
        if i >= args.warmup:
            secs.append(r["seconds"])
    t = statistics.mean(secs)
    value = n / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rows_per_step": n, "sample_of_rows": args.rows},
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                             "sample": f"{n} rows of the workload per step, all host threads"},
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
                "traffic": traffic, "kernel": "gb_agg_kernel (fused filter + hash aggregate)",
                "kernel_ms": t_agg * 1e3, "algorithmic_bytes_per_launch": n * BYTES_PER_ROW,
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, copy bandwidth)"}
    cpu = cpu_baseline(cols, args.cpu_sample_rows) if (rank == 0 and world == 1) else None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "rows_per_gpu": n, "global_rows": world * n, "groups": int(groups),
                           "parallelism": f"dp{world}" if world > 1 else "single", "l2": "inputs (4.3 GB) > L2, no flush",
                           "step": "reset + fused filter/aggregate + exchange (N>1) + GetResults"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": sampler.summary(),
                "gpu_launches": int(launches)}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
