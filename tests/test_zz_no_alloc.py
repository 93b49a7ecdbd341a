"""The labeling entry point that allocates no device memory.

Some callers cannot allocate while they label: a wipe worker that reserved
the device's free memory for its label window up front must not risk an
allocation failing half-way through a disk, and a host whose own memory pool
already holds the device's memory has none left for the library to take.
pose_b200_topo_label_noalloc serves them from the library's own static device
arrays.  These tests call it through the C ABI and check that it writes
exactly the bytes of the allocating entry point, pose_graph_hbm_topo_label,
on two calls in a row (the second call sees the first call's leftovers in the
shared arrays), while every device allocation the library attempts is made
to fail, and that it leaves no device memory allocated.
"""
from __future__ import annotations

import contextlib
import os

import pytest

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def every_library_allocation_fails():
    """Make each device allocation the library attempts fail on the host
    (POSE_B200_FAIL_ALLOC, the library's allocation-failure injector), so a
    call that succeeds under it allocated nothing through the library."""
    os.environ.pop("POSE_B200_FAIL_ALLOC", None)
    os.environ["POSE_B200_FAIL_ALLOC"] = str(1 << 20)
    try:
        yield
    finally:
        os.environ.pop("POSE_B200_FAIL_ALLOC", None)


def _label_both_ways(pkg, torch, cb, nsup, rbo, key):
    nbytes = nsup * cb * 32
    with pkg.Topology(cb) as topo:
        want = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
        assert topo.label(key, want.data_ptr(), nbytes, rbo) == 0, pkg.last_error()
        torch.cuda.synchronize()
        outs = [torch.full((nbytes,), 0x5A, dtype=torch.uint8, device="cuda") for _ in range(2)]
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        with every_library_allocation_fails():
            rcs = [topo.label_noalloc(key, got.data_ptr(), nbytes, rbo) for got in outs]
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        for call, (rc, got) in enumerate(zip(rcs, outs)):
            assert rc == 0, f"call {call}: {pkg.last_error()}"
            assert torch.equal(got, want), f"call {call}: bytes differ from pose_graph_hbm_topo_label"
        assert free_after >= free_before, "the calls left device memory allocated"


@pytest.mark.parametrize("cb,nsup,rbo", [
    (1024, 8, 0),            # small chunks, one launch
    (16, 9000, 16 * 7),      # more super-chunks than the static seed table: several launches
    (1 << 17, 20, 5 << 17),  # 40 chunk copies through a 64 MiB pool (16 at a time)
])
def test_no_alloc_matches_allocating_entry_point(pkg, cuda, cb, nsup, rbo):
    _label_both_ways(pkg, cuda, cb, nsup, rbo, bytes(range(7, 39)))


def test_no_alloc_rejects_oversized_seed(pkg, cuda):
    with pkg.Topology(16) as topo:
        buf = cuda.zeros(16 * 32, dtype=cuda.uint8, device="cuda")
        assert topo.label_noalloc(b"x" * 1017, buf.data_ptr(), 16 * 32, 0) == -1
        assert "1016" in pkg.last_error() and "seed" in pkg.last_error()
        assert topo.label_noalloc(b"x" * 1016, buf.data_ptr(), 16 * 32, 0) == 0
