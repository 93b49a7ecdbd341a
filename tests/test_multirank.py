"""Multi-GPU host logic on CPU ranks (gloo, world size 2): each rank labels
its own absolute super-chunk range (the labels here come from the CPU
oracle), the ranges tile one region byte-for-byte, and the step time is the
max over ranks.  No data-path collective exists; the all_gather below is only
the check."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import load_workloads


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q) -> None:
    import sys
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__))))
    from conftest import load_workloads as lw
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    from oracle import Oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        wl = lw()
        w = {"key": wl.splitmix64_key(7), "chunk_blocks": 16, "chunks": 3, "rbo": 16 * 5}
        rbo, n = wl.rank_region(w, rank, world)
        mine = Oracle().label_region(w["key"], w["chunk_blocks"], n, rbo)
        got = [torch.zeros(len(mine), dtype=torch.uint8) for _ in range(world)]
        dist.all_gather(got, torch.from_numpy(mine.copy()))
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            whole = Oracle().label_region(w["key"], w["chunk_blocks"], n * world, w["rbo"])
            q.put((np.concatenate([g.numpy() for g in got]).tobytes() == whole.tobytes(), float(t[0])))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_shards_tile_the_region():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    same, tmax = q.get(timeout=5)
    assert same and tmax == 2.0


def test_rank_region_is_disjoint_and_contiguous():
    wl = load_workloads()
    w = wl.plain_2e17()
    spans = [wl.rank_region(w, r, 8) for r in range(8)]
    for r in range(7):
        assert spans[r][0] + spans[r][1] * w["chunk_blocks"] == spans[r + 1][0]
    with pytest.raises(ValueError):
        wl.rank_region(w, 8, 8)
