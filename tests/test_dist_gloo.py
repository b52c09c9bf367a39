"""The multi-GPU merge protocol of qikkdb_b200.dist on CPU ranks (gloo, world sizes 2 and 3).

Each rank aggregates its own row shard, exports its partial states bucketed by key owner, takes part in the
all-to-all exchange and merges what it receives.  The three table steps run on a small CPU stand-in here (the
GPU path supplies the CUDA library's export/merge); the exchange itself is the product code.  The union of the
owner tables must equal one GROUP BY over all rows, and every key must live on exactly one rank.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from qikkdb_b200.dist import Partial, exchange_and_merge


class CpuTable:
    def __init__(self):
        self.state = {}  # key -> [count, sum]

    def add(self, k, c, s):
        st = self.state.setdefault(int(k), [0, 0])
        st[0] += int(c)
        st[1] += int(s)


class CpuOps:
    """Stand-in for the three table steps: state words are (count, sum) of integer values."""

    def new_table(self):
        return CpuTable()

    def export(self, table, n_parts):
        buckets = [[] for _ in range(n_parts)]
        for k, (c, s) in table.state.items():
            buckets[(k * 0x9E3779B1 & 0xFFFFFFFF) % n_parts].append((k, c, s))
        parts = []
        for b in buckets:
            keys = torch.tensor([x[0] for x in b], dtype=torch.int64)
            state = torch.tensor([v for x in b for v in (x[1], x[2])], dtype=torch.int64)
            flags = torch.zeros(len(b), dtype=torch.uint8)
            parts.append(Partial(keys, state, flags, 2))
        return parts

    def merge(self, table, part):
        st = part.state.view(-1, 2) if part.count else part.state.view(0, 2)
        for k, row in zip(part.keys.tolist(), st.tolist()):
            table.add(k, row[0], row[1])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, keys, vals, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shard = np.array_split(np.arange(len(keys)), world)[rank]
        local = CpuTable()
        for i in shard:
            local.add(keys[i], 1, vals[i])
        owner = exchange_and_merge(local, CpuOps(), device=torch.device("cpu"))
        gathered = [None] * world
        dist.all_gather_object(gathered, owner.state)
        if rank == 0:
            out.put(gathered)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_and_merge_gloo(world):
    rng = np.random.default_rng(world)
    n = 5000
    keys = rng.integers(0, 700, n).astype(np.int64)
    vals = rng.integers(-50, 50, n).astype(np.int64)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, keys, vals, q)) for r in range(world)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seen = {}
    for r, st in enumerate(gathered):
        for k, v in st.items():
            assert k not in seen, f"key {k} owned by two ranks"
            seen[k] = v
    ref = {}
    for k, v in zip(keys.tolist(), vals.tolist()):
        st = ref.setdefault(k, [0, 0])
        st[0] += 1
        st[1] += v
    assert seen == ref
