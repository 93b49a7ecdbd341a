"""No label, chunk seed or session key of a call stays on the device.

The reference zeroes its scratch before it frees it (common/src/cuda/
label_gpu_warp.cu:236-238).  This library keeps its workspace (scratch pool,
chunk-seed table, session seed copy) on the topology across calls, and the
allocation-free entry point keeps its own in static device arrays, so each
call clears all of it before it returns, failed calls included.
pose_b200_topo_residue counts the nonzero bytes left there; these tests
check the count itself against torch, then that it reads 0 after every kind
of call."""
from __future__ import annotations

import contextlib
import os

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nbytes", [0, 1, 15, 16, 17, 4096 + 9, (3 << 20) + 5])
def test_count_nonzero_matches_torch(pkg, cuda, nbytes):
    g = cuda.Generator(device="cpu").manual_seed(nbytes)
    host = cuda.randint(0, 4, (nbytes,), generator=g, dtype=cuda.uint8)  # about a quarter zeros
    buf = host.to("cuda")
    assert pkg.count_nonzero(buf.data_ptr(), nbytes) == int(cuda.count_nonzero(host))


def test_count_nonzero_of_a_zeroed_buffer_is_zero(pkg, cuda):
    buf = cuda.zeros(1 << 20, dtype=cuda.uint8, device="cuda")
    assert pkg.count_nonzero(buf.data_ptr(), buf.numel()) == 0
    buf[-1] = 1
    buf[0] = 255
    assert pkg.count_nonzero(buf.data_ptr(), buf.numel()) == 2


def _buf(cuda, topo, nsup):
    n = nsup * topo.info()["chunk_blocks"] * 32
    return cuda.zeros(n, dtype=cuda.uint8, device="cuda"), n


def test_workspace_is_clear_after_each_kind_of_call(pkg, cuda):
    key = bytes(range(1, 33))
    with pkg.Topology(1024) as topo:
        assert topo.residue() == 0
        buf, n = _buf(cuda, topo, 24)
        assert topo.label(key, buf.data_ptr(), n, 0) == 0, pkg.last_error()
        assert cuda.count_nonzero(buf) > 0          # labels were written to the caller's buffer
        assert topo.residue() == 0                  # and nothing else stayed behind
        for kernel in (1, 3):
            sched = pkg.Sched(kernel=kernel)
            assert topo.label(key, buf.data_ptr(), n, 1024 * 5, sched=sched) == 0, pkg.last_error()
            assert topo.residue() == 0, f"kernel {kernel}"
        # a session seed longer than the device derivation takes (host path)
        assert topo.label(b"s" * 2000, buf.data_ptr(), n, 0) == 0
        assert topo.residue() == 0
        rc, _, _ = topo.autotune(key, buf.data_ptr(), n, 0, trials=3)
        assert rc == 0, pkg.last_error()
        assert topo.residue() == 0
        assert topo.label_noalloc(key, buf.data_ptr(), n, 0) == 0
        assert topo.residue() == 0                  # the static arrays are counted too


@contextlib.contextmanager
def _failing_allocs(n: int):
    os.environ["POSE_B200_FAIL_ALLOC"] = str(n)
    try:
        yield
    finally:
        os.environ.pop("POSE_B200_FAIL_ALLOC", None)


def test_workspace_is_clear_after_a_failed_call(pkg, cuda):
    key = bytes(range(3, 35))
    with pkg.Topology(1024) as topo:
        small, ns = _buf(cuda, topo, 2)
        assert topo.label(key, small.data_ptr(), ns, 0) == 0
        big, nb = _buf(cuda, topo, 256)
        with _failing_allocs(1 << 20):
            assert topo.label(key, big.data_ptr(), nb, 0) == -1
        assert topo.residue() == 0
        assert topo.label(key, big.data_ptr(), nb, 0) == 0, pkg.last_error()
        assert topo.residue() == 0
