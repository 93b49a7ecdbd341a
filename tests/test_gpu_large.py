"""Full-size parity: the workloads at their real sizes, every persisted byte
checked through per-super-chunk SHA-256 digests that the reference CPU path
(compiled from source) produced for the same seeds and positions
(tests/golden/configs.json, made by tests/golden/gen_golden.py)."""
from __future__ import annotations

import hashlib

import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def digests(torch, buf, sb, n):
    host = buf.cpu().numpy()
    return [hashlib.sha256(host[j * sb:(j + 1) * sb].tobytes()).hexdigest() for j in range(n)]


def test_plain_2e17_every_super_chunk(pkg, cuda, wl):
    g = golden("configs.json")["plain_2e17"]
    c = wl.plain_2e17()
    cb, n = c["chunk_blocks"], c["chunks"]
    buf = cuda.zeros(n * cb * 32, dtype=cuda.uint8, device="cuda")
    with pkg.Topology(cb) as topo:
        # the depth kernel alone and with a cluster of 2 CTAs per copy, and the lockstep kernel
        for kernel, cl in ((3, 1), (3, 2), (1, 0)):
            rc, st = topo.label(c["key"], buf.data_ptr(), n * cb * 32, c["rbo"],
                                sched=pkg.Sched(kernel=kernel, cluster_ctas=cl), stats=True)
            assert rc == 0, pkg.last_error()
            assert st["kernel"] == kernel and st["cluster_ctas"] == cl
            assert digests(cuda, buf, cb * 32, n) == g["super_chunk_sha256"], (kernel, cl)
            buf.zero_()
        # the block-0 table and in-register block 0 give the same bytes
    with pkg.Topology(cb, cv0_table=False) as topo:
        assert topo.label(c["key"], buf.data_ptr(), n * cb * 32, c["rbo"]) == 0
        assert digests(cuda, buf, cb * 32, n) == g["super_chunk_sha256"]


def test_deep_2e20_every_super_chunk_under_40GiB_cap(pkg, cuda, wl):
    g = golden("configs.json")["deep_2e20"]
    c = wl.deep_2e20()
    cb, n = c["chunk_blocks"], c["chunks"]
    buf = cuda.zeros(n * cb * 32, dtype=cuda.uint8, device="cuda")
    with pkg.Topology(cb) as topo:
        # the automatic schedule, and the depth kernel with clusters of 8 CTAs per copy
        for cl in (0, 8):
            s = pkg.Sched(scratch_cap_bytes=c["scratch_cap_bytes"], cluster_ctas=cl, kernel=3 if cl else 0)
            rc, st = topo.label(c["key"], buf.data_ptr(), n * cb * 32, c["rbo"], sched=s, stats=True)
            assert rc == 0, pkg.last_error()
            assert st["scratch_bytes"] <= c["scratch_cap_bytes"]
            assert digests(cuda, buf, cb * 32, n) == g["super_chunk_sha256"], st
            buf.zero_()


def test_batched_sessions_sampled_chunks(pkg, cuda, wl):
    rows = {r["session"]: r for r in golden("configs.json")["batched_sampled"]}
    sessions = wl.batched()
    by_cb = {}
    for s in sessions[:48]:
        by_cb.setdefault(s["chunk_blocks"], []).append(s)
    for cb, group in by_cb.items():
        buf = cuda.zeros(cb * 32, dtype=cuda.uint8, device="cuda")
        with pkg.Topology(cb) as topo:
            for s in group:
                r = rows[s["session"]]
                assert r["chunk_blocks"] == cb
                assert topo.label(s["key"], buf.data_ptr(), cb * 32, r["chunk_index"] * cb) == 0
                assert digests(cuda, buf, cb * 32, 1)[0] == r["sha256"], s["session"]
