#!/usr/bin/env python3
"""COMPARATOR ONLY: time the reference's own CUDA "warp" strategy on this GPU.

Loads oracle/_ref/libposeref_warp.so — the reference's common/src/cuda/
label_gpu_common.cu + label_gpu_warp.cu + blake3_node.cu and its CPU path,
compiled from the reference sources for sm_100 by `make -C oracle ref_gpu`,
exactly as -DPOSE_CUDA_ARCH=100 -DPOSE_GPU_LABEL_STRATEGY=warp
-DPOSE_GPU_WARP_MIN_BLOCKS=3 would build it — and drives it the way
disk-wipe-bench's worker does: pose_graph_hbm_topo_build once, then
pose_graph_hbm_topo_label on a device window (tools/disk-wipe-bench/
disk_wipe_bench.cu:590-658).  Prints one JSON line per workload.

It runs in its own process: the reference library exports the same C symbol
names as libpose_b200.so.  With --check it also compares the window's bytes to
the digests in tests/golden/configs.json.

    python oracle/ref_gpu_bench.py [--chunks 32] [--chunk-blocks 131072] [--reps 2] [--check]
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SO = os.path.join(HERE, "_ref", "libposeref_warp.so")


def splitmix_key(state: int) -> bytes:
    mask = (1 << 64) - 1
    s, out = state & mask, b""
    for _ in range(4):
        s = (s + 0x9E3779B97F4A7C15) & mask
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        out += (z ^ (z >> 31)).to_bytes(8, "little")
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--chunks", type=int, default=32)
    ap.add_argument("--chunk-blocks", type=int, default=1 << 17)
    ap.add_argument("--key-state", type=int, default=1)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--check", action="store_true")
    args = ap.parse_args()
    os.environ.setdefault("POSE_GPU_QUIET", "1")
    import torch
    torch.cuda.init()
    L = C.CDLL(SO)
    L.pose_graph_hbm_topo_build.argtypes = [C.c_uint32, C.c_int]
    L.pose_graph_hbm_topo_build.restype = C.c_void_p
    L.pose_graph_hbm_topo_label.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_uint64]
    L.pose_graph_hbm_topo_label.restype = C.c_int
    L.pose_graph_hbm_topo_free.argtypes = [C.c_void_p]
    cb, n = args.chunk_blocks, args.chunks
    key = splitmix_key(args.key_state)
    nbytes = n * cb * 32
    t0 = time.perf_counter()
    topo = L.pose_graph_hbm_topo_build(cb, 0)
    build_s = time.perf_counter() - t0
    assert topo, "reference topology build failed"
    buf = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    times = []
    for _ in range(args.reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = L.pose_graph_hbm_topo_label(topo, key, len(key), C.c_void_p(buf.data_ptr()), nbytes, 0)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        assert rc == 0
    best = min(times)
    line = {"impl": "reference-warp-sm100", "chunk_blocks": cb, "super_chunks": n,
            "mib_s": nbytes / float(1 << 20) / best, "seconds": best, "all_seconds": times,
            "topo_build_s": build_s}
    if args.check:
        g = json.load(open(os.path.join(ROOT, "tests", "golden", "configs.json")))
        ref = {"plain_2e17": g.get("plain_2e17"), "plain_small": g.get("plain_small")}
        host = buf.cpu().numpy()
        sb = cb * 32
        got = [hashlib.sha256(host[j * sb:(j + 1) * sb].tobytes()).hexdigest() for j in range(n)]
        for name, r in ref.items():
            if r and r["chunk_blocks"] == cb and r["key"] == key.hex():
                line["matches_golden_" + name] = got[:len(r["super_chunk_sha256"])] == r["super_chunk_sha256"][:n]
    L.pose_graph_hbm_topo_free(topo)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
