"""Host threads labeling at the same time, each with its own topology.

disk-wipe-bench drives its GPUs from one process, one host thread per GPU,
each thread building its own topology and labeling its own windows
(tools/disk-wipe-bench/disk_wipe_bench.cu:563-708, threads started at
:1014-1033).  Here two threads do that on device 0 at once through the
drop-in C ABI (pose_graph_hbm_topo_build / _label / _free), with different
chunk sizes, and every super-chunk they persist is checked against the
reference CPU labeler's digests (tests/golden/configs.json).  The library's
process-wide state (the allocation-failure injector's counter, the kernels'
shared-memory attributes, the per-device tables) is touched by both threads.
ctypes releases the GIL for the duration of each call, so the two threads'
calls overlap on the host and on the device."""
from __future__ import annotations

import ctypes as C
import hashlib
import threading

import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_two_threads_two_topologies_label_concurrently(pkg, cuda, wl):
    L = pkg.load()
    g = golden("configs.json")
    jobs = []
    for name, work, nsup in (("plain_small", wl.plain_small(), 64), ("plain_2e17", wl.plain_2e17(), 8)):
        cb = work["chunk_blocks"]
        buf = cuda.zeros(nsup * cb * 32, dtype=cuda.uint8, device="cuda")
        jobs.append({"name": name, "cb": cb, "nsup": nsup, "key": work["key"], "rbo": work["rbo"],
                     "buf": buf, "want": g[name]["super_chunk_sha256"][:nsup], "got": [], "err": None})
    cuda.cuda.synchronize()
    start = threading.Barrier(len(jobs))

    def worker(job):
        try:
            topo = L.pose_graph_hbm_topo_build(job["cb"], pkg.POSE_HASH_BLAKE3)
            assert topo, pkg.last_error()
            key = C.cast(C.create_string_buffer(job["key"], len(job["key"])), C.POINTER(C.c_uint8))
            nbytes = job["nsup"] * job["cb"] * 32
            start.wait(timeout=120)
            for _ in range(3):
                rc = L.pose_graph_hbm_topo_label(topo, key, len(job["key"]), C.c_void_p(job["buf"].data_ptr()),
                                                 nbytes, job["rbo"])
                job["got"].append(rc)
            L.pose_graph_hbm_topo_free(topo)
        except BaseException as exc:  # reported by the main thread
            job["err"] = exc
            start.abort()

    threads = [threading.Thread(target=worker, args=(j,)) for j in jobs]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
        assert not t.is_alive(), "a labeling thread did not finish"
    cuda.cuda.synchronize()
    for job in jobs:
        assert job["err"] is None, f"{job['name']}: {job['err']!r}"
        assert job["got"] == [0, 0, 0], job["name"]
        host = job["buf"].cpu().numpy()
        sb = job["cb"] * 32
        got = [hashlib.sha256(host[j * sb:(j + 1) * sb].tobytes()).hexdigest() for j in range(job["nsup"])]
        assert got == job["want"], job["name"]
