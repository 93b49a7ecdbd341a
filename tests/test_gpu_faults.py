"""Failure handling, with the failures made on the host.

POSE_B200_FAIL_ALLOC=n makes the library's next n device allocations fail as
if the device were out of memory (dev_alloc.h); nothing faults the GPU.  The
labeling call must react as the reference does to a failed scratch
allocation: halve the batch and carry on (common/src/cuda/label_gpu_warp.cu:
165-175), and, when even one team's scratch cannot be had, return -1 with
the CUDA error in the message (label_gpu_common.cu:237-243) and leave the
topology usable.  The other entry points return their error codes
(NULL / -1) and work again once memory is back."""
from __future__ import annotations

import contextlib
import hashlib
import os

import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def failing_allocs(n: int):
    os.environ.pop("POSE_B200_FAIL_ALLOC", None)
    os.environ["POSE_B200_FAIL_ALLOC"] = str(n)
    try:
        yield
    finally:
        os.environ.pop("POSE_B200_FAIL_ALLOC", None)


def small(wl):
    c = wl.plain_small()
    return c, c["chunks"] * c["chunk_blocks"] * 32


def test_scratch_failure_halves_the_schedule_and_keeps_the_bytes(pkg, cuda, wl):
    g = golden("configs.json")["plain_small"]
    c, n = small(wl)
    buf = cuda.zeros(n, dtype=cuda.uint8, device="cuda")
    with pkg.Topology(c["chunk_blocks"]) as topo:
        full = topo.plan(c["chunks"])
        assert full is not None and full.max_teams > 4
        sched = pkg.Sched(kernel=1, team_warps=1, units_per_team=1)
        with failing_allocs(2):
            rc, st = topo.label(c["key"], buf.data_ptr(), n, c["rbo"], sched=sched, stats=True)
        assert rc == 0, pkg.last_error()
        assert 0 < st["teams"] <= topo.plan(c["chunks"], sched).max_teams // 4
        assert hashlib.sha256(buf.cpu().numpy().tobytes()).hexdigest() == g["region_sha256"]


def test_scratch_that_cannot_be_had_fails_cleanly(pkg, cuda, wl):
    g = golden("configs.json")["plain_small"]
    c, n = small(wl)
    buf = cuda.zeros(n, dtype=cuda.uint8, device="cuda")
    with pkg.Topology(c["chunk_blocks"]) as topo:
        with failing_allocs(1 << 20):
            rc = topo.label(c["key"], buf.data_ptr(), n, c["rbo"])
        assert rc == -1
        assert "alloc" in pkg.last_error() and "memory" in pkg.last_error().lower()
        # memory is back: the same topology labels correctly
        rc = topo.label(c["key"], buf.data_ptr(), n, c["rbo"])
        assert rc == 0, pkg.last_error()
        assert hashlib.sha256(buf.cpu().numpy().tobytes()).hexdigest() == g["region_sha256"]


def test_topology_build_failure_returns_null(pkg, cuda):
    with failing_allocs(1):
        with pytest.raises(RuntimeError):
            pkg.Topology(1024)
    with pkg.Topology(1024) as topo:
        assert topo.info()["chunk_blocks"] == 1024


def test_batch_and_stream_failures_return_errors(pkg, cuda, wl):
    c, n = small(wl)
    buf = cuda.zeros(n, dtype=cuda.uint8, device="cuda")
    with pkg.Topology(c["chunk_blocks"]) as topo:
        reqs = [(topo, c["key"], buf.data_ptr(), n, c["rbo"])]
        with failing_allocs(1 << 20):
            with pytest.raises(RuntimeError):
                pkg.Batch(reqs)
            rc, _ = topo.label_stream(c["key"], n, lambda view, off: 0, c["rbo"],
                                      window_bytes=n // 4)
            assert rc == -1
        with pkg.Batch(reqs) as b:
            rc, _ = b.run()
            assert rc == 0
