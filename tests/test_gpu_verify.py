"""GPU verifier: challenge recompute and the sampled verify, through the C ABI.

pose_b200_challenge answers the reference's pose_graph_challenge
(common/src/graph.c:1019-1042); pose_b200_challenge_blocks answers absolute
region blocks of a session; pose_b200_verify_sampled is disk-wipe-bench's
verify_disk (tools/disk-wipe-bench/disk_wipe_bench.cu:300-366) with the
recompute and compare on the GPU.  All checked bit-exact against the fixtures
made by the reference and against the oracle.
"""
from __future__ import annotations

import random

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def topos(pkg):
    cache = {}

    def get(cb):
        if cb not in cache:
            cache[cb] = pkg.Topology(cb)
        return cache[cb]

    yield get
    for t in cache.values():
        t.free()


def test_challenge_matches_reference(topos):
    for c in golden("challenges.json")["graph"]:
        got = topos(c["m"]).challenge(bytes.fromhex(c["seed"]), c["index"])
        assert got is not None and got.hex() == c["hex"], (c["m"], c["index"])


def test_challenge_out_of_range_and_short_seed(topos):
    t = topos(100)
    assert t.challenge(bytes(32), 100) is None  # challenge_idx >= m (graph.c:1023)
    assert t.challenge(bytes(31), 0) is None    # the graph seed is 32 bytes


def test_challenge_blocks_match_reference(topos):
    ch = golden("challenges.json")
    key = bytes.fromhex(ch["region_key"])
    by_cb = {}
    for c in ch["region"]:
        by_cb.setdefault(c["chunk_blocks"], []).append(c)
    for cb, rows in by_cb.items():
        blocks = [r["block"] for r in rows]
        rc, out, st = topos(cb).challenge_blocks(key, blocks)
        assert rc == 0
        for k, r in enumerate(rows):
            assert out[32 * k:32 * k + 32].hex() == r["hex"], (cb, r["block"])
        assert st["super_chunks"] == len({b // cb for b in blocks})


def test_challenge_blocks_random_against_labeling(pkg, topos, cuda):
    """Random blocks (duplicates, unsorted, one chunk repeated) against the
    labels of the same region written by the labeling path."""
    torch = cuda
    rnd = random.Random(11)
    cb, nsup, rbo_chunk = 4096, 12, 777
    key = bytes(rnd.randrange(256) for _ in range(48))
    t = topos(cb)
    buf = torch.zeros(nsup * cb * 32, dtype=torch.uint8, device="cuda")
    assert t.label(key, buf.data_ptr(), nsup * cb * 32, rbo_chunk * cb) == 0
    region = buf.cpu().numpy()
    blocks = [rbo_chunk * cb + rnd.randrange(nsup * cb) for _ in range(300)]
    blocks += blocks[:20]
    rc, out, _ = t.challenge_blocks(key, blocks)
    assert rc == 0
    for k, b in enumerate(blocks):
        off = (b - rbo_chunk * cb) * 32
        assert out[32 * k:32 * k + 32] == region[off:off + 32].tobytes(), k


def _region(pkg, t, key, nsup, torch):
    buf = torch.zeros(nsup * t.super_bytes, dtype=torch.uint8, device="cuda")
    assert t.label(key, buf.data_ptr(), nsup * t.super_bytes, 0) == 0
    return bytearray(buf.cpu().numpy().tobytes())


def test_verify_sampled_clean_and_planted(pkg, topos, cuda):
    torch = cuda
    cb, nsup = 1024, 40
    key = bytes(range(32))
    t = topos(cb)
    disk = _region(pkg, t, key, nsup, torch)
    sb = t.super_bytes

    def read(n, off):
        return disk[off:off + n]

    r = t.verify_sampled(key, len(disk), 16, read)
    assert r["rc"] == 0 and r["checked"] == 16 and r["mismatched"] == 0
    assert r["first_bad"] == [None] * 16
    # sample k reads super-chunk k*(n-1)/(samples-1); plant a flipped byte in
    # sample 5's super-chunk at block 77 and in the last one at block 0
    J5 = 5 * (nsup - 1) // 15
    disk[J5 * sb + 77 * 32 + 3] ^= 0x40
    disk[(nsup - 1) * sb] ^= 1
    r = t.verify_sampled(key, len(disk), 16, read)
    assert r["rc"] == 0 and r["checked"] == 16 and r["mismatched"] == 2
    assert r["first_bad"][5] == 77 and r["first_bad"][15] == 0
    assert all(v is None for i, v in enumerate(r["first_bad"]) if i not in (5, 15))


def test_verify_sampled_edges(pkg, topos, cuda):
    torch = cuda
    cb = 64
    key = b"k" * 40
    t = topos(cb)
    disk = _region(pkg, t, key, 3, torch)
    read = lambda n, off: disk[off:off + n]
    # samples clamp to n_super; samples 0 means one (super-chunk 0)
    r = t.verify_sampled(key, len(disk), 100, read)
    assert r["rc"] == 0 and r["checked"] == 3 and r["mismatched"] == 0
    r = t.verify_sampled(key, len(disk), 0, read)
    assert r["rc"] == 0 and r["checked"] == 1
    # a wrong session seed mismatches every sample at block 0
    r = t.verify_sampled(b"x" * 40, len(disk), 3, read)
    assert r["rc"] == 0 and r["mismatched"] == 3 and r["first_bad"] == [0, 0, 0]
    # nothing labelled, and a failing read, are errors
    assert t.verify_sampled(key, t.super_bytes - 1, 4, read)["rc"] == -1
    assert t.verify_sampled(key, len(disk), 3, lambda n, off: None)["rc"] == -1


def test_verify_sampled_2e17_config(pkg, cuda):
    """The 2^17 workload's 16 sampled super-chunks re-verified on the GPU
    against the stored region (the check disk-wipe-bench runs on the CPU)."""
    import hashlib
    torch = cuda
    cfg = golden("configs.json")["plain_2e17"]
    key = bytes.fromhex(cfg["key"])
    cb, n = cfg["chunk_blocks"], cfg["chunks"]
    with pkg.Topology(cb) as t:
        disk = _region(pkg, t, key, n, torch)
        sb = t.super_bytes
        for j in (0, n - 1):
            assert hashlib.sha256(disk[j * sb:(j + 1) * sb]).hexdigest() == cfg["super_chunk_sha256"][j]
        r = t.verify_sampled(key, len(disk), 16, lambda m, off: disk[off:off + m])
        assert r["rc"] == 0 and r["checked"] == 16 and r["mismatched"] == 0
