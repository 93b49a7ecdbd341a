"""Batched labeling (one persistent launch over many sessions and chunk
sizes, replayed from a captured CUDA graph) writes exactly the bytes each
request gets from pose_graph_hbm_topo_label alone, and the 256-session
workload's sampled chunks equal the reference CPU path's digests."""
from __future__ import annotations

import hashlib
import random

import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_batch_equals_individual_calls(pkg, cuda, oracle):
    rnd = random.Random(3)
    cbs = [1, 3, 16, 100, 1024, 4096]
    topos = {cb: pkg.Topology(cb) for cb in cbs}
    try:
        reqs, bufs, want = [], [], []
        for i in range(40):
            cb = rnd.choice(cbs)
            ns = rnd.randint(1, 6)
            extra = rnd.choice([0, 0, 32 * rnd.randint(1, cb)]) if cb > 1 else 0
            rbo = rnd.choice([0, cb * rnd.randrange(1 << 30), rnd.randrange(1 << 40)])
            key = rnd.randbytes(rnd.choice([32, 32, 0, 9, 200]))
            nbytes = ns * cb * 32 + extra
            buf = cuda.full((nbytes,), 0x5C, dtype=cuda.uint8, device="cuda")
            ref = cuda.full((nbytes,), 0x5C, dtype=cuda.uint8, device="cuda")
            assert topos[cb].label(key, ref.data_ptr(), nbytes, rbo) == 0
            reqs.append((topos[cb], key, buf.data_ptr(), nbytes, rbo))
            bufs.append(buf)
            want.append(ref)
        with pkg.Batch(reqs) as b:
            for _ in range(2):  # the captured graph replays identically
                for t in bufs:
                    t.fill_(0x5C)
                rc, st = b.run()
                assert rc == 0
                cuda.cuda.synchronize()
                for i, (t, r) in enumerate(zip(bufs, want)):
                    assert cuda.equal(t, r), i
        assert st["kernel"] == 4 and st["super_chunks"] == sum(r[3] // (r[0].chunk_blocks * 32) for r in reqs)
        # spot-check against the CPU oracle
        topo, key, _, nbytes, rbo = reqs[0]
        ns = nbytes // (topo.chunk_blocks * 32)
        assert bufs[0].cpu().numpy().tobytes()[: ns * topo.chunk_blocks * 32] == \
            oracle.label_region(key, topo.chunk_blocks, ns, rbo, threads=4).tobytes()
    finally:
        for t in topos.values():
            t.free()


@pytest.mark.parametrize("sched", [None, {"team_warps": 2, "units_per_team": 4}, {"max_teams": 5},
                                   {"team_warps": 8, "lane_efficiency": 255}, {"team_warps": 1, "lane_efficiency": 70},
                                   {"team_warps": 4, "units_per_team": 1}, {"flags": 1}, "autotune"])
def test_batch_schedules(pkg, cuda, oracle, sched):
    topos = {cb: pkg.Topology(cb) for cb in (64, 512)}
    try:
        reqs, bufs = [], []
        for i in range(12):
            cb = 64 if i % 2 else 512
            buf = cuda.zeros(3 * cb * 32, dtype=cuda.uint8, device="cuda")
            reqs.append((topos[cb], bytes([i]) * 32, buf.data_ptr(), 3 * cb * 32, i * cb))
            bufs.append(buf)
        s = pkg.Sched(**sched) if isinstance(sched, dict) else None
        with pkg.Batch(reqs, s, autotune=3 if sched == "autotune" else 0) as b:
            if sched == "autotune":
                assert b.chosen["team_warps"] in (1, 2, 4, 8)
                assert b.chosen["lane_efficiency"] in (50, 70, 85, pkg.PACK_CHAIN)
                for t in bufs:
                    t.zero_()
            rc, _ = b.run()
            assert rc == 0
        for (topo, key, _, nbytes, rbo), buf in zip(reqs, bufs):
            want = oracle.label_region(key, topo.chunk_blocks, 3, rbo, threads=4).tobytes()
            assert buf.cpu().numpy().tobytes() == want
    finally:
        for t in topos.values():
            t.free()


def test_deep_requests_run_as_a_second_launch(pkg, cuda):
    """Requests of a much deeper topology run as their own concurrent launch;
    POSE_B200_BATCH_ONE_LAUNCH keeps one launch; both write the same bytes."""
    topos = {cb: pkg.Topology(cb) for cb in (256, 4096)}
    try:
        reqs, bufs = [], []
        for i in range(11):
            cb = 4096 if i < 3 or i == 10 else 256
            n = 2 * cb * 32 if i != 10 else 32  # the last: shorter than one super-chunk, labels nothing
            buf = cuda.zeros(n, dtype=cuda.uint8, device="cuda")
            reqs.append((topos[cb], bytes([i + 7]) * 32, buf.data_ptr(), n, (5 + i) * cb))
            bufs.append(buf)
        got = {}
        for flags, launches in ((0, 4), (pkg.BATCH_ONE_LAUNCH, 2)):
            for t in bufs:
                t.fill_(0x33)
            with pkg.Batch(reqs, pkg.Sched(flags=flags)) as b:
                rc, st = b.run()
            assert rc == 0 and st["kernel_launches"] == launches, (flags, st)
            got[flags] = [t.cpu().numpy().tobytes() for t in bufs]
        assert got[0] == got[pkg.BATCH_ONE_LAUNCH]
        for (topo, key, ptr, nbytes, rbo), data in zip(reqs, got[0]):
            ref = cuda.full((nbytes,), 0x33, dtype=cuda.uint8, device="cuda")
            assert topo.label(key, ref.data_ptr(), nbytes, rbo) == 0
            assert ref.cpu().numpy().tobytes() == data
        # only short deep requests: no deep part, nothing to label there
        with pkg.Batch([reqs[10], reqs[5]]) as b:
            rc, st = b.run()
            assert rc == 0 and st["kernel_launches"] == 2
    finally:
        for t in topos.values():
            t.free()


@pytest.mark.parametrize("deep_cb,shallow_cb,units", [(4096, 256, "1"), (4096, 256, "2"), (4096, 256, "3"),
                                                     (4096, 256, "4"), (3000, 100, "4"), (3000, 100, "3")])
def test_multi_unit_depth_kernel_writes_the_same_bytes(pkg, cuda, monkeypatch, deep_cb, shallow_cb, units):
    """The deep part on the multi-unit depth kernel with 1 to 4 units per
    CTA (a ragged last batch, levels wider than the staged slots, session
    seeds of several lengths) writes what single calls and the lockstep
    kernel write."""
    rnd = random.Random(deep_cb + int(units))
    topos = {cb: pkg.Topology(cb) for cb in (deep_cb, shallow_cb)}
    try:
        reqs, bufs = [], []
        for i, ns in enumerate([1, 2, 1, 3, 2, 2, 1]):  # 9 deep chunks = 18 units
            cb = deep_cb if i < 5 else shallow_cb
            key = rnd.randbytes([32, 0, 9, 200, 32, 32, 5][i])
            nbytes = ns * cb * 32 + (17 if i == 2 else 0)
            buf = cuda.zeros(nbytes, dtype=cuda.uint8, device="cuda")
            reqs.append((topos[cb], key, buf.data_ptr(), nbytes, cb * rnd.randrange(1 << 20)))
            bufs.append(buf)
        got = {}
        for kernel in ("1", "0"):
            monkeypatch.setenv("POSE_B200_DEEP_UNITS", units)
            monkeypatch.setenv("POSE_B200_DEEP_KERNEL", kernel)
            for t in bufs:
                t.fill_(0x6B)
            with pkg.Batch(reqs) as b:
                rc, st = b.run()
            assert rc == 0 and st["kernel_launches"] == 4, (kernel, st)
            got[kernel] = [t.cpu().numpy().tobytes() for t in bufs]
        assert got["1"] == got["0"]
        for (topo, key, ptr, nbytes, rbo), data in zip(reqs, got["1"]):
            ref = cuda.full((nbytes,), 0x6B, dtype=cuda.uint8, device="cuda")
            assert topo.label(key, ref.data_ptr(), nbytes, rbo) == 0
            assert ref.cpu().numpy().tobytes() == data
    finally:
        for t in topos.values():
            t.free()


def test_next_deepest_topology_runs_as_a_third_launch(pkg, cuda, monkeypatch):
    """With three topologies, the deepest one's requests and those of the
    next-deepest (its chain at least a third as long) each run on the
    multi-unit depth kernel (the second on the SMs the first leaves, three
    copies per CTA, a ragged last batch); the rest in the lockstep launch.
    The bytes equal single calls and the two-launch form
    (POSE_B200_DEEP2=0).  The 256-session workload below runs the second
    part's CTAs over more batches than CTAs."""
    rnd = random.Random(23)
    cbs = (4096, 2048, 256)
    topos = {cb: pkg.Topology(cb) for cb in cbs}
    try:
        reqs, bufs = [], []
        for i, (cb, ns) in enumerate([(4096, 2), (2048, 3), (256, 2), (2048, 2), (4096, 1), (256, 1), (2048, 2)]):
            key = rnd.randbytes([32, 7, 32, 100, 32, 1, 32][i])
            buf = cuda.zeros(ns * cb * 32, dtype=cuda.uint8, device="cuda")
            reqs.append((topos[cb], key, buf.data_ptr(), ns * cb * 32, cb * rnd.randrange(1 << 20)))
            bufs.append(buf)
        got = {}
        for deep2, launches in (("1", 6), ("0", 4)):
            monkeypatch.setenv("POSE_B200_DEEP2", deep2)
            for t in bufs:
                t.fill_(0x4D)
            with pkg.Batch(reqs) as b:
                rc, st = b.run()
            assert rc == 0 and st["kernel_launches"] == launches, (deep2, st)
            got[deep2] = [t.cpu().numpy().tobytes() for t in bufs]
        assert got["1"] == got["0"]
        for (topo, key, ptr, nbytes, rbo), data in zip(reqs, got["1"]):
            ref = cuda.full((nbytes,), 0x4D, dtype=cuda.uint8, device="cuda")
            assert topo.label(key, ref.data_ptr(), nbytes, rbo) == 0
            assert ref.cpu().numpy().tobytes() == data
    finally:
        for t in topos.values():
            t.free()


def test_batched_256_sessions_sampled_vs_reference(pkg, cuda, wl):
    rows = {r["session"]: r for r in golden("configs.json")["batched_sampled"]}
    sessions = wl.batched()
    cbs = sorted({s["chunk_blocks"] for s in sessions})
    topos = {cb: pkg.Topology(cb) for cb in cbs}
    try:
        total = sum(s["chunk_blocks"] * 32 * len(s["chunk_indices"]) for s in sessions)
        big = cuda.zeros(total, dtype=cuda.uint8, device="cuda")
        reqs, first_off = [], {}
        off = 0
        for s in sessions:
            cb = s["chunk_blocks"]
            for k, idx in enumerate(s["chunk_indices"]):
                if k == 0:
                    first_off[s["session"]] = off
                reqs.append((topos[cb], s["key"], big.data_ptr() + off, cb * 32, idx * cb))
                off += cb * 32
        with pkg.Batch(reqs) as b:
            rc, st = b.run()
        assert rc == 0
        host = big.cpu().numpy()
        for s in sessions:
            r = rows[s["session"]]
            o = first_off[s["session"]]
            got = hashlib.sha256(host[o:o + r["chunk_blocks"] * 32].tobytes()).hexdigest()
            assert got == r["sha256"], s["session"]
    finally:
        for t in topos.values():
            t.free()


def test_batch_rejects_bad_schedules(pkg, cuda):
    with pkg.Topology(64) as t:
        buf = cuda.zeros(64 * 32, dtype=cuda.uint8, device="cuda")
        for bad in ({"team_warps": 3}, {"team_warps": 16}, {"lane_efficiency": 101}):
            with pytest.raises(RuntimeError):
                pkg.Batch([(t, b"k" * 32, buf.data_ptr(), 64 * 32, 0)], pkg.Sched(**bad))
