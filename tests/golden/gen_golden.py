#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in the build container (it needs the reference sources at
/root/reference and the reference CPU path compiled from them by
``make -C oracle ref``):

    python tests/golden/gen_golden.py [--skip-large]

Everything recorded here is produced by the reference's own code
(``oracle/_ref/libposeref.so``: common/src/hash.c, common/src/graph.c and the
vendored BLAKE3 1.8.5), except the three official BLAKE3 vectors, which are
read from the reference's own test (common/test/test_hash.c:47-67).

Fixtures:
  blake3_official.json  the official unkeyed BLAKE3 vectors of test_hash.c
  hash_kats.json        label keys, descriptors, chunk seeds, node labels
  edges.json            SHA-256 digests of pose_graph_edges for many m
  small_regions.json    full output bytes (hex) of small regions
  configs.json          per-super-chunk SHA-256 digests of the workloads
"""
from __future__ import annotations

import argparse
import hashlib
import importlib.util
import json
import os
import random
import re
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_ROOT = os.environ.get("POSE_REF", "/root/reference")  # the reference tree; override with POSE_REF
REF_TEST_HASH = os.path.join(REF_ROOT, "common", "test", "test_hash.c")
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import RefCPU  # noqa: E402


def _workloads():
    spec = importlib.util.spec_from_file_location(
        "pb_workloads", os.path.join(ROOT, "pose-memory-wiping_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def sha(b) -> str:
    return hashlib.sha256(bytes(b)).hexdigest()


def official_vectors() -> list[dict]:
    src = open(REF_TEST_HASH).read()
    found = re.findall(r'check_blake3\("([^"]+)",\s*([^,]+),\s*(\d+),\s*"([0-9a-f]{64})"\)', src)
    out = []
    for name, _data, length, hexd in found:
        n = int(length)
        data = bytes(i % 251 for i in range(n))  # test_hash.c:59-64 pattern; 0/1 byte cases are zeros
        if n <= 1:
            data = bytes(n)
        out.append({"name": name, "len": n, "pattern": "i % 251", "hex": hexd})
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-large", action="store_true", help="skip the 2^17 / 2^20 / batched digests")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only-challenges", action="store_true", help="write challenges.json alone")
    args = ap.parse_args()
    ref = RefCPU()
    wl = _workloads()
    if args.only_challenges:
        challenges(ref, wl)
        return
    rnd = random.Random(0xC0FFEE)

    # 1. official BLAKE3 vectors held by the reference test
    json.dump(official_vectors(), open(os.path.join(HERE, "blake3_official.json"), "w"), indent=1)

    # 2. hash KATs
    ksrc, kint = ref.label_keys()
    kats = {"key_src": [int(x) for x in ksrc], "key_int": [int(x) for x in kint],
            "descriptors": [], "chunk_seeds": [], "labels": []}
    for m in [1, 2, 3, 4, 5, 16, 17, 100, 1024, 4096, 1 << 17, 1 << 18, 1 << 20, 12345]:
        n = ref.L.pose_graph_parameter_n(m)
        kats["descriptors"].append({"m": m, "n": n, "hex": ref.descriptor(m, n).hex()})
    for seed_len in [0, 1, 16, 32, 55, 56, 64, 100, 1016, 1017, 2048, 5000]:
        seed = bytes(rnd.randrange(256) for _ in range(seed_len))
        for idx in [0, 1, 7, 1 << 32, (1 << 64) - 1]:
            kats["chunk_seeds"].append({"seed": seed.hex(), "index": idx,
                                        "hex": ref.chunk_seed(seed, idx).hex()})
    for _ in range(64):
        is_src = rnd.random() < 0.25
        idx = rnd.choice([0, 1, rnd.randrange(1 << 29), rnd.randrange(1 << 64)])
        p0 = bytes(rnd.randrange(256) for _ in range(32)) if rnd.random() < 0.8 else None
        p1 = bytes(rnd.randrange(256) for _ in range(32)) if (p0 and rnd.random() < 0.7) else None
        seed = bytes(rnd.randrange(256) for _ in range(32))
        desc = bytes(rnd.randrange(256) for _ in range(32))
        out = ref.label_node(int(is_src), idx, p0, p1, seed, desc)
        kats["labels"].append({"is_source": int(is_src), "index": idx,
                               "p0": p0.hex() if p0 else None, "p1": p1.hex() if p1 else None,
                               "seed": seed.hex(), "desc": desc.hex(), "hex": out.hex()})
    json.dump(kats, open(os.path.join(HERE, "hash_kats.json"), "w"), indent=1)

    # 3. topology digests (pose_graph_edges)
    edges = []
    for m in [1, 2, 3, 4, 5, 7, 8, 9, 15, 16, 17, 31, 32, 33, 100, 1000, 1024, 4096, 4097,
              50000, 1 << 17]:
        np_, p0, p1, rk = ref.edges(m)
        edges.append({"m": m, "count": int(len(np_)), "np": sha(np_.tobytes()),
                      "p0": sha(p0.tobytes()), "p1": sha(p1.tobytes()), "rank": sha(rk.tobytes())})
    json.dump(edges, open(os.path.join(HERE, "edges.json"), "w"), indent=1)

    # 4. small regions, full bytes
    small = []
    key = wl.splitmix64_key(42)
    for cb, nsup, rbo in [(1, 5, 0), (2, 4, 3), (3, 3, 0), (4, 3, 5), (5, 2, 0), (7, 2, 9),
                          (16, 4, 0), (16, 3, 7), (16, 2, 16 * 1000), (17, 2, 0), (100, 2, 250),
                          (1024, 2, 0), (4096, 1, 4096 * 3)]:
        out = ref.label_super_chunks(key, cb, nsup, rbo, threads=args.threads)
        small.append({"key": key.hex(), "chunk_blocks": cb, "super_chunks": nsup, "rbo": rbo,
                      "hex": out.tobytes().hex()})
    # a long session seed (host-side chunk-seed path)
    long_key = bytes(rnd.randrange(256) for _ in range(1500))
    out = ref.label_super_chunks(long_key, 16, 3, 16, threads=args.threads)
    small.append({"key": long_key.hex(), "chunk_blocks": 16, "super_chunks": 3, "rbo": 16,
                  "hex": out.tobytes().hex()})
    json.dump(small, open(os.path.join(HERE, "small_regions.json"), "w"), indent=1)

    # 5. workload digests
    cfg_path = os.path.join(HERE, "configs.json")
    cfgs = json.load(open(cfg_path)) if os.path.exists(cfg_path) else {}

    def region_digests(key, cb, n, rbo):
        t0 = time.time()
        out = ref.label_super_chunks(key, cb, n, rbo, threads=args.threads)
        sb = cb * 32
        d = [sha(out[j * sb:(j + 1) * sb]) for j in range(n)]
        print(f"  cb={cb} x{n}: {time.time() - t0:.1f}s", flush=True)
        return d, sha(out)

    c1 = wl.plain_small()
    d, whole = region_digests(c1["key"], c1["chunk_blocks"], c1["chunks"], c1["rbo"])
    cfgs["plain_small"] = {"key": c1["key"].hex(), "chunk_blocks": c1["chunk_blocks"],
                           "chunks": c1["chunks"], "rbo": c1["rbo"], "super_chunk_sha256": d,
                           "region_sha256": whole}
    if not args.skip_large:
        c2 = wl.plain_2e17()
        d, whole = region_digests(c2["key"], c2["chunk_blocks"], c2["chunks"], c2["rbo"])
        cfgs["plain_2e17"] = {"key": c2["key"].hex(), "chunk_blocks": c2["chunk_blocks"],
                              "chunks": c2["chunks"], "rbo": c2["rbo"], "super_chunk_sha256": d,
                              "region_sha256": whole}
        sess = wl.batched()
        t0 = time.time()

        def one(s):
            # one sampled chunk per session (its first), checked through its digest
            idx = s["chunk_indices"][0]
            cb = s["chunk_blocks"]
            out = ref.label_super_chunks(s["key"], cb, 1, idx * cb, threads=1)
            return {"session": s["session"], "chunk_blocks": cb, "chunk_index": idx,
                    "sha256": sha(out)}

        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(args.threads) as ex:
            rows = list(ex.map(one, sess))
        print(f"  batched sampled chunks: {time.time() - t0:.1f}s", flush=True)
        cfgs["batched_sampled"] = rows
        c4 = wl.deep_2e20()
        d, whole = region_digests(c4["key"], c4["chunk_blocks"], c4["chunks"], c4["rbo"])
        cfgs["deep_2e20"] = {"key": c4["key"].hex(), "chunk_blocks": c4["chunk_blocks"],
                             "chunks": c4["chunks"], "rbo": c4["rbo"], "super_chunk_sha256": d,
                             "region_sha256": whole}
    json.dump(cfgs, open(cfg_path, "w"), indent=1)
    challenges(ref, wl)
    print("golden fixtures written to", HERE)


def challenges(ref, wl) -> None:
    """6. verifier recompute: pose_graph_challenge on raw graph seeds, and
    absolute region blocks of one session (chunk seed from the block's chunk
    index) read out of the reference's region labeler."""
    rnd = random.Random(0xC4A11)
    graph = []
    for m in [1, 2, 3, 5, 16, 17, 100, 1000, 1024, 4097, 1 << 12, 1 << 14]:
        seed = bytes(rnd.randrange(256) for _ in range(32))
        for idx in sorted({0, m - 1, rnd.randrange(m), rnd.randrange(m)}):
            lab = ref.challenge(seed, m, idx)
            assert lab is not None
            graph.append({"seed": seed.hex(), "m": m, "index": idx, "hex": lab.hex()})
        assert ref.challenge(seed, m, m) is None  # out of range
    key = wl.splitmix64_key(7)
    region = []
    for cb in [64, 1000, 1024]:
        chunks = sorted(rnd.sample(range(1 << 20), 5))
        for J in chunks:
            out = ref.label_super_chunks(key, cb, 1, J * cb, threads=1)
            for r in sorted({0, cb - 1, rnd.randrange(cb)}):
                region.append({"chunk_blocks": cb, "block": J * cb + r, "hex": out[32 * r:32 * r + 32].tobytes().hex()})
    json.dump({"graph": graph, "region_key": key.hex(), "region": region},
              open(os.path.join(HERE, "challenges.json"), "w"), indent=1)


if __name__ == "__main__":
    main()
