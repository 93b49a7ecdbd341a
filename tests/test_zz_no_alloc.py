"""The labeling entry point that allocates no device memory.

Some callers cannot allocate while they label: a wipe worker that reserved
the device's free memory for its label window up front must not risk an
allocation failing half-way through a disk, and a host whose allocator (or an
active stream capture) forbids new device allocations cannot let the library
call cudaMalloc.  pose_b200_topo_label_noalloc serves them from the library's
own static device arrays.  These tests call it through the C ABI and check it
writes exactly the bytes of the allocating entry point,
pose_graph_hbm_topo_label, on two calls in a row (the second call sees the
first call's leftovers in the shared arrays).
"""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def _label_both_ways(pkg, torch, cb, nsup, rbo, key):
    nbytes = nsup * cb * 32
    with pkg.Topology(cb) as topo:
        want = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
        assert topo.label(key, want.data_ptr(), nbytes, rbo) == 0, pkg.last_error()
        torch.cuda.synchronize()
        for call in range(2):
            got = torch.full((nbytes,), 0x5A, dtype=torch.uint8, device="cuda")
            rc = topo.label_noalloc(key, got.data_ptr(), nbytes, rbo)
            torch.cuda.synchronize()
            assert rc == 0, f"call {call}"
            assert torch.equal(got, want), f"call {call}: bytes differ from pose_graph_hbm_topo_label"


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
        assert topo.label_noalloc(b"x" * 1016, buf.data_ptr(), 16 * 32, 0) == 0
