"""GPU parity: every label the B200 path persists must be byte-identical to
the reference CPU path on the same seed and positions.

Oracles: the golden fixtures made by the reference compiled from source
(tests/golden/), and the C restatement in oracle/ for randomised cases.
All calls go through the C ABI (libpose_b200.so)."""
from __future__ import annotations

import hashlib
import random

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def dev_buffer(torch, nbytes: int, fill: int = 0xA5):
    return torch.full((max(1, nbytes),), fill, dtype=torch.uint8, device="cuda")


def host_bytes(t) -> bytes:
    return t.cpu().numpy().tobytes()


def label_region(pkg, torch, key, cb, nsuper, rbo, sched=None, cv0=True, extra=0):
    buf = dev_buffer(torch, nsuper * cb * 32 + extra)
    with pkg.Topology(cb, cv0_table=cv0) as topo:
        rc = topo.label(key, buf.data_ptr(), nsuper * cb * 32 + extra, rbo, sched=sched)
    torch.cuda.synchronize()
    assert rc == 0, pkg.last_error()
    return host_bytes(buf)


def test_kat_single_node(pkg, cuda, oracle):
    k = golden("hash_kats.json")
    for c in k["labels"]:
        p0 = bytes.fromhex(c["p0"]) if c["p0"] else None
        p1 = bytes.fromhex(c["p1"]) if c["p1"] else None
        got = pkg.label_node_single(c["is_source"], c["index"], p0, p1, bytes.fromhex(c["seed"]),
                                    bytes.fromhex(c["desc"]), k["key_src"], k["key_int"])
        assert got is not None and got.hex() == c["hex"]
    rnd = random.Random(7)
    for _ in range(16):
        idx = rnd.randrange(1 << 64)
        p0 = rnd.randbytes(32)
        seed, desc = rnd.randbytes(32), rnd.randbytes(32)
        got = pkg.label_node_single(0, idx, p0, None, seed, desc, k["key_src"], k["key_int"])
        assert got == oracle.label_node(0, idx, p0, None, seed, desc)


def test_small_regions_all_bytes(pkg, cuda):
    for r in golden("small_regions.json"):
        key = bytes.fromhex(r["key"])
        for cv0 in (True, False):
            got = label_region(pkg, cuda, key, r["chunk_blocks"], r["super_chunks"], r["rbo"], cv0=cv0)
            assert got.hex() == r["hex"], (r["chunk_blocks"], r["rbo"], cv0)


def test_plain_small_config(pkg, cuda, wl):
    g = golden("configs.json")["plain_small"]
    c = wl.plain_small()
    got = label_region(pkg, cuda, c["key"], c["chunk_blocks"], c["chunks"], c["rbo"])
    sb = c["chunk_blocks"] * 32
    for j in range(c["chunks"]):
        assert hashlib.sha256(got[j * sb:(j + 1) * sb]).hexdigest() == g["super_chunk_sha256"][j], j
    assert hashlib.sha256(got).hexdigest() == g["region_sha256"]


@pytest.mark.parametrize("T,G", [(1, 1), (1, 2), (1, 4), (1, 8), (1, 32), (2, 1), (4, 4), (8, 2), (16, 1), (16, 32)])
def test_every_schedule_gives_the_same_bytes(pkg, cuda, wl, T, G):
    g = golden("configs.json")["plain_small"]
    c = wl.plain_small()
    s = pkg.Sched(team_warps=T, units_per_team=G, kernel=1)
    got = label_region(pkg, cuda, c["key"], c["chunk_blocks"], c["chunks"], c["rbo"], sched=s,
                       cv0=(G % 2 == 0))
    assert hashlib.sha256(got).hexdigest() == g["region_sha256"]


@pytest.mark.parametrize("nc", [7, 15])
def test_warp_specialised_kernel_gives_the_same_bytes(pkg, cuda, wl, oracle, nc):
    g = golden("configs.json")["plain_small"]
    c = wl.plain_small()
    s = pkg.Sched(team_warps=nc, kernel=3)
    got = label_region(pkg, cuda, c["key"], c["chunk_blocks"], c["chunks"], c["rbo"], sched=s)
    assert hashlib.sha256(got).hexdigest() == g["region_sha256"]
    for r in golden("small_regions.json"):
        got = label_region(pkg, cuda, bytes.fromhex(r["key"]), r["chunk_blocks"], r["super_chunks"],
                           r["rbo"], sched=s)
        assert got.hex() == r["hex"], (r["chunk_blocks"], r["rbo"])
    # wide levels (more items than hashing threads) and few resident CTAs
    rnd = random.Random(nc)
    for cb in (4096, 3000):
        key = rnd.randbytes(32)
        s2 = pkg.Sched(team_warps=nc, kernel=3, max_teams=2)
        got = label_region(pkg, cuda, key, cb, 5, cb * 3, sched=s2)
        assert got == oracle.label_region(key, cb, 5, cb * 3, threads=8).tobytes(), cb


@pytest.mark.parametrize("C,split", [(2, None), (4, None), (8, None), (2, "0"), (4, "100"), (8, "0")])
def test_cluster_depth_kernel_gives_the_same_bytes(pkg, cuda, oracle, monkeypatch, C, split):
    """The depth kernel with a cluster of C CTAs per chunk copy sharing the
    levels wider than the split width: the default width, every level
    shared (width 0), and a narrow width; power-of-two and other
    chunk_blocks, unaligned positions."""
    if split is not None:
        monkeypatch.setenv("POSE_B200_SPLIT_WIDTH", split)  # read when the topology is built
    rnd = random.Random(C * 31 + (int(split) if split else 7))
    for cb, nsup in ((1024, 8), (4096, 4), (3000, 3)):
        nsup = min(nsup, 16 // C)  # one wave of clusters: at most 8 C-CTA clusters of 2 copies
        key = rnd.randbytes(32)
        rbo = cb * rnd.randrange(1 << 20) + rnd.randrange(cb)
        s = pkg.Sched(kernel=3, cluster_ctas=C)
        buf = dev_buffer(cuda, nsup * cb * 32)
        with pkg.Topology(cb) as topo:
            rc, st = topo.label(key, buf.data_ptr(), nsup * cb * 32, rbo, sched=s, stats=True)
        cuda.cuda.synchronize()
        assert rc == 0, pkg.last_error()
        assert st["kernel"] == 3 and st["cluster_ctas"] == C
        assert host_bytes(buf) == oracle.label_region(key, cb, nsup, rbo, threads=8).tobytes(), (cb, C, split)


def test_cluster_schedule_is_validated(pkg, cuda):
    with pkg.Topology(1024) as topo:
        buf = cuda.zeros(1024 * 32, dtype=cuda.uint8, device="cuda")
        for bad in (pkg.Sched(kernel=1, cluster_ctas=2), pkg.Sched(kernel=3, cluster_ctas=3),
                    pkg.Sched(kernel=3, cluster_ctas=32)):
            assert topo.label(bytes(32), buf.data_ptr(), 1024 * 32, 0, sched=bad) == -1
            assert "cluster_ctas" in pkg.last_error()


def test_retired_kernel_number_is_refused(pkg, cuda):
    with pkg.Topology(1024) as topo:
        buf = cuda.zeros(1024 * 32, dtype=cuda.uint8, device="cuda")
        assert topo.label(bytes(32), buf.data_ptr(), 1024 * 32, 0, sched=pkg.Sched(kernel=2)) == -1
        assert "kernel 2" in pkg.last_error()


def test_autotune_keeps_the_bytes_and_its_schedule(pkg, cuda, wl):
    g = golden("configs.json")["plain_small"]
    c = wl.plain_small()
    n = c["chunks"] * c["chunk_blocks"] * 32
    buf = dev_buffer(cuda, n)
    with pkg.Topology(c["chunk_blocks"]) as topo:
        rc, chosen, st = topo.autotune(c["key"], buf.data_ptr(), n, c["rbo"], trials=6)
        assert rc == 0, pkg.last_error()
        cuda.cuda.synchronize()
        assert hashlib.sha256(host_bytes(buf)).hexdigest() == g["region_sha256"]
        assert st["kernel"] == chosen["kernel"] and st["team_warps"] == chosen["team_warps"]
        buf.fill_(0)
        rc, st2 = topo.label(c["key"], buf.data_ptr(), n, c["rbo"], stats=True)
        assert rc == 0, pkg.last_error()
        assert (st2["kernel"], st2["team_warps"], st2["units_per_team"]) == \
            (chosen["kernel"], chosen["team_warps"], chosen["units_per_team"])
        assert hashlib.sha256(host_bytes(buf)).hexdigest() == g["region_sha256"]
        # another call size keeps the automatic policy and the same bytes
        buf.fill_(0)
        half, sb = c["chunks"] // 2, c["chunk_blocks"] * 32
        rc, st3 = topo.label(c["key"], buf.data_ptr(), half * sb, c["rbo"], stats=True)
        assert rc == 0, pkg.last_error()
        got = host_bytes(buf)
        for j in range(half):
            assert hashlib.sha256(got[j * sb:(j + 1) * sb]).hexdigest() == g["super_chunk_sha256"][j], j


def test_few_resident_teams_loop_over_the_queue(pkg, cuda, wl):
    # 128 units through 3 resident teams: every team pulls many batches
    g = golden("configs.json")["plain_small"]
    c = wl.plain_small()
    s = pkg.Sched(team_warps=1, units_per_team=2, max_teams=3)
    got = label_region(pkg, cuda, c["key"], c["chunk_blocks"], c["chunks"], c["rbo"], sched=s)
    assert hashlib.sha256(got).hexdigest() == g["region_sha256"]


def test_random_regions_vs_oracle(pkg, cuda, oracle):
    rnd = random.Random(11)
    for _ in range(12):
        cb = rnd.choice([1, 2, 3, 6, 8, 33, 64, 255, 256, 1000, 2048])
        nsup = rnd.randint(1, 9)
        rbo = rnd.choice([0, rnd.randrange(1 << 40), cb * rnd.randrange(1 << 20)])
        key = rnd.randbytes(rnd.choice([32, 0, 7, 64]))
        got = label_region(pkg, cuda, key, cb, nsup, rbo)
        want = oracle.label_region(key, cb, nsup, rbo, threads=8).tobytes()
        assert got == want, (cb, nsup, rbo, len(key))


def test_tail_and_short_buffers_are_untouched(pkg, cuda, oracle):
    key = b"\x11" * 32
    cb, nsup, extra = 16, 3, 16 * 32 - 32
    got = label_region(pkg, cuda, key, cb, nsup, 5, extra=extra)
    assert got[: nsup * cb * 32] == oracle.label_region(key, cb, nsup, 5).tobytes()
    assert got[nsup * cb * 32:] == b"\xa5" * extra
    buf = dev_buffer(cuda, cb * 32)
    with pkg.Topology(cb) as topo:
        assert topo.label(key, buf.data_ptr(), cb * 32 - 1, 0) == 0
    assert host_bytes(buf) == b"\xa5" * (cb * 32)


def test_one_shot_entry_point_and_defaults(pkg, cuda, oracle):
    key = b"\x22" * 32
    buf = dev_buffer(cuda, 2 * 4096 * 32)
    assert pkg.label_hbm(key, 0, buf.data_ptr(), 2 * 4096 * 32, 4096) == 0  # 0 -> 4096
    cuda.cuda.synchronize()
    assert host_bytes(buf) == oracle.label_region(key, 4096, 2, 4096, threads=2).tobytes()
    assert pkg.label_hbm(key, 16, buf.data_ptr(), 64, 0, pkg.POSE_HASH_SHA256) == -1


def test_topology_reused_across_calls_and_seeds(pkg, cuda, oracle):
    with pkg.Topology(100) as topo:
        for i in range(3):
            key = bytes([i]) * 32
            buf = dev_buffer(cuda, 4 * 100 * 32)
            assert topo.label(key, buf.data_ptr(), 4 * 100 * 32, 100 * i) == 0
            assert host_bytes(buf) == oracle.label_region(key, 100, 4, 100 * i, threads=4).tobytes()


def test_stats_report_the_work(pkg, cuda):
    buf = dev_buffer(cuda, 8 * 1024 * 32)
    with pkg.Topology(1024) as topo:
        rc, st = topo.label(b"s" * 32, buf.data_ptr(), 8 * 1024 * 32, 0, stats=True)
        assert st["kernel"] in (1, 3)
    assert rc == 0
    assert st["super_chunks"] == 8 and st["units"] == 16
    assert st["nodes"] == 8 * 96254
    assert st["kernel_ms"] > 0 and st["kernel_launches"] == 1


@pytest.mark.parametrize("team_warps,per_sm", [(16, 1), (1, 3), (4, 7)])
def test_teams_per_sm_cap_keeps_the_bytes(pkg, cuda, oracle, team_warps, per_sm):
    # k teams on every SM, held there by padding each CTA's shared memory:
    # every SM gets the same number of teams, and the bytes do not change
    import os
    key, cb, nsup, rbo = b"\x5a" * 32, 64, 1200, 64 * 17
    sms = cuda.cuda.get_device_properties(0).multi_processor_count
    s = pkg.Sched(kernel=1, team_warps=team_warps, units_per_team=1)
    os.environ["POSE_B200_TEAMS_PER_SM"] = str(per_sm)
    try:
        buf = dev_buffer(cuda, nsup * cb * 32)
        with pkg.Topology(cb) as topo:
            rc, st = topo.label(key, buf.data_ptr(), nsup * cb * 32, rbo, sched=s, stats=True)
        cuda.cuda.synchronize()
    finally:
        os.environ.pop("POSE_B200_TEAMS_PER_SM", None)
    assert rc == 0, pkg.last_error()
    assert st["teams"] == per_sm * sms
    assert host_bytes(buf) == oracle.label_region(key, cb, nsup, rbo, threads=8).tobytes()
