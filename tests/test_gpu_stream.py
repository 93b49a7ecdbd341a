"""Streaming to a host sink: the labels delivered window by window (labelling
of window k+1 overlapped with the copy and sink of window k) are the bytes of
labelling the whole region at once, at the right absolute offsets."""
from __future__ import annotations

import threading

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cb,nsuper,window_chunks", [(1024, 10, 3), (4096, 5, 1), (16, 100, 7), (1024, 4, 64)])
def test_stream_matches_region(pkg, cuda, oracle, cb, nsuper, window_chunks):
    key = bytes(range(100, 132))
    rbo, base = cb * 9, 1 << 20
    out = bytearray(nsuper * cb * 32)
    calls = []
    lock = threading.Lock()

    def sink(buf, off):
        with lock:
            calls.append((off, len(buf), threading.get_ident()))
            out[off - base: off - base + len(buf)] = bytes(buf)
        return 0

    with pkg.Topology(cb) as topo:
        rc, st = topo.label_stream(key, nsuper * cb * 32 + 17, sink, rbo, base, window_chunks * cb * 32)
    assert rc == 0
    assert bytes(out) == oracle.label_region(key, cb, nsuper, rbo, threads=8).tobytes()
    w = min(window_chunks, nsuper) * cb * 32
    assert [c[0] for c in calls] == [base + i * w for i in range((nsuper * cb * 32 + w - 1) // w)]
    assert st["super_chunks"] == nsuper


def test_failing_sink_aborts(pkg, cuda):
    seen = []

    def sink(buf, off):
        seen.append(off)
        return 1 if len(seen) == 2 else 0

    with pkg.Topology(64) as topo:
        rc, _ = topo.label_stream(b"k" * 32, 20 * 64 * 32, sink, 0, 0, 2 * 64 * 32)
    assert rc == -1
    assert 2 <= len(seen) <= 3
