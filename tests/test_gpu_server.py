"""Continuous-batching server: requests submitted from several threads while
other work runs are admitted into concurrent waves, and every result is
byte-identical to labelling that request alone."""
from __future__ import annotations

import random
import threading
import time

import pytest

pytestmark = pytest.mark.gpu


def test_results_alone_equal_results_in_the_mix(pkg, cuda):
    rnd = random.Random(9)
    cbs = [64, 1024, 4096, 1 << 14]
    topos = {cb: pkg.Topology(cb) for cb in cbs}
    try:
        seed_list = [rnd.randbytes(32) for _ in range(6)]
        reqs = []
        for i in range(48):
            cb = rnd.choice(cbs)
            ns = rnd.randint(1, 6)
            reqs.append((cb, ns, cb * rnd.randrange(1 << 20), rnd.randrange(6),
                         cuda.full((ns * cb * 32,), 0x33, dtype=cuda.uint8, device="cuda")))
        cuda.cuda.synchronize()
        with pkg.Server(scratch_bytes=1 << 30, max_waves=4) as srv:
            sessions = [srv.session(k) for k in seed_list]
            tickets = [None] * len(reqs)

            def submitter(lo, hi, r):
                for i in range(lo, hi):
                    cb, ns, rbo, sid, buf = reqs[i]
                    tickets[i] = srv.submit(topos[cb], sessions[sid], buf.data_ptr(), ns * cb * 32, rbo)
                    time.sleep(r.random() * 0.004)

            th = [threading.Thread(target=submitter, args=(k * 24, (k + 1) * 24, random.Random(k)))
                  for k in range(2)]
            for t in th:
                t.start()
            for t in th:
                t.join()
            assert all(t is not None and t >= 0 for t in tickets)
            for t in tickets:
                rc, q, tot = srv.wait(t)
                assert rc == 0 and tot >= q >= 0
            st = srv.stats()
            assert st["submitted"] == len(reqs) and st["waves"] >= 2
        # the same requests alone, through the drop-in entry point
        for cb, ns, rbo, sid, buf in reqs:
            alone = cuda.zeros(ns * cb * 32, dtype=cuda.uint8, device="cuda")
            assert topos[cb].label(seed_list[sid], alone.data_ptr(), ns * cb * 32, rbo) == 0
            cuda.cuda.synchronize()
            assert cuda.equal(alone, buf), (cb, ns, rbo, sid)
    finally:
        for t in topos.values():
            t.free()


def test_oversized_request_is_rejected(pkg, cuda):
    with pkg.Topology(1 << 12) as topo, pkg.Server(scratch_bytes=64 << 10, max_waves=1) as srv:
        sid = srv.session(b"s" * 32)
        buf = cuda.zeros(4096 * 32, dtype=cuda.uint8, device="cuda")
        assert srv.submit(topo, sid, buf.data_ptr(), 4096 * 32, 0) == -1  # one copy needs 128 KiB
        assert srv.submit(topo, 99, buf.data_ptr(), 4096 * 32, 0) == -1  # unknown session


@pytest.mark.parametrize("deep_sms,units", [(0, None), (8, "0"), (8, "1")])
def test_deep_requests_run_on_the_depth_kernel_and_match_alone(pkg, cuda, monkeypatch, deep_sms, units):
    """Requests at chunk_blocks 2^17 run on the depth kernel: three chunk
    copies per CTA with the SM held alone (the default: 2 and 5 chunks make
    ragged last batches); with units "0", the fewest copies per CTA that fit
    an idle GPU; with the depth kernel held to 8 SMs, a request that does
    not fit the free SMs waits for them, and one larger than all 8 (units
    "1": 10 copies) runs its CTAs over the batches in turn.  Shallow
    requests in waves run beside them.  Every result equals labelling that
    request alone."""
    if deep_sms:
        monkeypatch.setenv("POSE_B200_SERVER_DEEP_SMS", str(deep_sms))
    if units is not None:
        monkeypatch.setenv("POSE_B200_SERVER_DEEP_UNITS", units)
    rnd = random.Random(17)
    deep_cb, cbs = 1 << 17, [1024, 1 << 14]
    topos = {cb: pkg.Topology(cb) for cb in [deep_cb] + cbs}
    try:
        seed_list = [rnd.randbytes(32) for _ in range(3)]
        plan = [(deep_cb, 2), (1024, 3), (1 << 14, 2), (deep_cb, 5), (1024, 5), (1 << 14, 1), (1024, 2)]
        reqs = []
        for cb, ns in plan:
            reqs.append((cb, ns, cb * rnd.randrange(1 << 16), rnd.randrange(3),
                         cuda.full((ns * cb * 32,), 0x5A, dtype=cuda.uint8, device="cuda")))
        cuda.cuda.synchronize()
        with pkg.Server(scratch_bytes=2 << 30, max_waves=2) as srv:
            sessions = [srv.session(k) for k in seed_list]
            for t in topos.values():
                srv.prepare(t)
            # the first deep request alone (an idle GPU), then the rest in a burst
            cb, ns, rbo, sid, buf = reqs[0]
            first = srv.submit(topos[cb], sessions[sid], buf.data_ptr(), ns * cb * 32, rbo)
            assert srv.wait(first)[0] == 0
            tickets = [first] + [srv.submit(topos[cb], sessions[sid], buf.data_ptr(), ns * cb * 32, rbo)
                                 for cb, ns, rbo, sid, buf in reqs[1:]]
            assert all(t >= 0 for t in tickets)
            for t in tickets:
                rc, q, tot = srv.wait(t)
                assert rc == 0 and tot >= q >= 0
        for cb, ns, rbo, sid, buf in reqs:
            alone = cuda.zeros(ns * cb * 32, dtype=cuda.uint8, device="cuda")
            assert topos[cb].label(seed_list[sid], alone.data_ptr(), ns * cb * 32, rbo) == 0
            cuda.cuda.synchronize()
            assert cuda.equal(alone, buf), (cb, ns, rbo, sid)
    finally:
        for t in topos.values():
            t.free()
