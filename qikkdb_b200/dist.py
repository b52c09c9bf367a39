"""Multi-GPU GROUP BY: row shards on every rank, one exchange of partial states, owner-side merge.

The reference shards row blocks round-robin over GPUs (qikkDB/GpuSqlParser/GpuSqlDispatcher.cpp:364, :1167)
and merges the per-GPU tables through host memory on device 0 (GPUGroupBy.cuh:594-790).  Here:

1. every rank aggregates its contiguous row range into its own table (no communication);
2. every rank exports its occupied slots bucketed by owner = hash(key) mod world (``export_partitioned``);
3. one all-to-all moves bucket r of every rank to rank r (NCCL over NVLink in production; any
   torch.distributed backend works, which is how the gloo tests on CPU drive the same protocol);
4. every owner merges what it received into a fresh owner table (``merge_partial``); results stay sharded by
   key (each rank returns its owned groups) and can be gathered if needed.

The exchange protocol is written against an ``ops`` object (export / merge / empty-table) so the same host
logic runs with the CUDA library (``CudaOps``) or with any other implementation of the three steps.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import torch

from . import _capi as capi
from .groupby import DeviceBuffer, GroupByTable, _stream


@dataclass
class Partial:
    """Exported partial records of one owner bucket: key words, state words (W-1 per record), flags."""
    keys: torch.Tensor   # int64 [m]
    state: torch.Tensor  # int64 [m * state_words]
    flags: torch.Tensor  # uint8 [m]
    state_words: int

    @property
    def count(self) -> int:
        return int(self.keys.numel())


def export_partitioned(table: GroupByTable, n_parts: int, stream=None) -> List[Partial]:
    """qdb_gb_export_partitioned: the table's occupied slots bucketed by owner, as CUDA tensors."""
    L = capi.lib()
    sw = C.c_int32()
    capi.check(L.qdb_gb_state_words(table.handle, C.byref(sw)))
    ok, osv, of = C.c_void_p(), C.c_void_p(), C.c_void_p()
    counts = (C.c_int64 * n_parts)()
    capi.check(L.qdb_gb_export_partitioned(table.handle, n_parts, C.byref(ok), C.byref(osv), C.byref(of), counts,
                                           _stream(stream)))
    total = sum(counts)
    kb = DeviceBuffer(ok.value, total, np.int64).torch(stream)
    sb = DeviceBuffer(osv.value, total * sw.value, np.int64).torch(stream)
    fb = DeviceBuffer(of.value, total, np.uint8).torch(stream)
    out, off = [], 0
    for p in range(n_parts):
        c = counts[p]
        out.append(Partial(kb[off:off + c], sb[off * sw.value:(off + c) * sw.value], fb[off:off + c], sw.value))
        off += c
    return out


def merge_partial(table: GroupByTable, part: Partial, stream=None) -> None:
    """qdb_gb_merge_partial: merges exported records into `table` (asynchronous on `stream`)."""
    if part.count == 0:
        return
    capi.check(capi.lib().qdb_gb_merge_partial(table.handle, part.keys.data_ptr(),
                                               part.state.data_ptr() if part.state.numel() else None,
                                               part.flags.data_ptr(), part.count, _stream(stream)))


class CudaOps:
    """The three exchange steps on the CUDA library."""

    def __init__(self, aggs, key_dtype, val_dtype, max_groups: int, n_key_cols: int = 1):
        self.aggs, self.key_dtype, self.val_dtype = aggs, key_dtype, val_dtype
        self.max_groups, self.n_key_cols = max_groups, n_key_cols

    def new_table(self) -> GroupByTable:
        return GroupByTable(self.aggs, self.key_dtype, self.val_dtype, self.max_groups, self.n_key_cols)

    def export(self, table, n_parts: int) -> List[Partial]:
        return export_partitioned(table, n_parts)

    def merge(self, table, part: Partial) -> None:
        merge_partial(table, part)


def exchange_and_merge(local_table, ops, group=None, device: Optional[torch.device] = None):
    """Steps 2-4 over torch.distributed: returns this rank's owner table.  Every rank takes the same collective
    steps in the same order (two all-to-alls: counts, then the three record arrays)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts = ops.export(local_table, world)
    dev = device or (parts[0].keys.device if parts else torch.device("cpu"))
    sw = parts[0].state_words if parts else 0
    send_counts = torch.tensor([p.count for p in parts], dtype=torch.int64, device=dev)
    recv_counts = torch.empty_like(send_counts)
    dist.all_to_all_single(recv_counts, send_counts, group=group)
    sc = send_counts.tolist()
    rc = recv_counts.tolist()
    keys_out = torch.cat([p.keys for p in parts]) if parts else torch.empty(0, dtype=torch.int64, device=dev)
    flags_out = torch.cat([p.flags for p in parts]) if parts else torch.empty(0, dtype=torch.uint8, device=dev)
    state_out = torch.cat([p.state for p in parts]) if parts else torch.empty(0, dtype=torch.int64, device=dev)
    keys_in = torch.empty(sum(rc), dtype=torch.int64, device=dev)
    flags_in = torch.empty(sum(rc), dtype=torch.uint8, device=dev)
    state_in = torch.empty(sum(rc) * sw, dtype=torch.int64, device=dev)
    dist.all_to_all_single(keys_in, keys_out, rc, sc, group=group)
    dist.all_to_all_single(flags_in, flags_out, rc, sc, group=group)
    dist.all_to_all_single(state_in, state_out, [c * sw for c in rc], [c * sw for c in sc], group=group)
    owner = ops.new_table()
    ops.merge(owner, Partial(keys_in, state_in, flags_in, sw))
    return owner
