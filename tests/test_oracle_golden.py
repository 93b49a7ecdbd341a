"""Pin the CPU oracle (oracle/pose_oracle.c) to the reference.

The fixtures were produced by the reference compiled from source
(tests/golden/gen_golden.py); the three unkeyed BLAKE3 vectors are the
official ones the reference's own test holds (common/test/test_hash.c:47-67).
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import golden


def test_blake3_official_vectors(oracle):
    vecs = golden("blake3_official.json")
    assert len(vecs) == 3
    for v in vecs:
        data = bytes(i % 251 for i in range(v["len"])) if v["len"] > 1 else bytes(v["len"])
        assert oracle.blake3(data).hex() == v["hex"], v["name"]


def test_label_keys(oracle):
    k = golden("hash_kats.json")
    src, intk = oracle.label_keys()
    assert [int(x) for x in src] == k["key_src"]
    assert [int(x) for x in intk] == k["key_int"]


def test_descriptors(oracle):
    for d in golden("hash_kats.json")["descriptors"]:
        assert oracle.parameter_n(d["m"]) == d["n"]
        assert oracle.descriptor(d["m"], d["n"]).hex() == d["hex"], d["m"]


def test_chunk_seeds(oracle):
    for c in golden("hash_kats.json")["chunk_seeds"]:
        assert oracle.chunk_seed(bytes.fromhex(c["seed"]), c["index"]).hex() == c["hex"]


def test_node_label_kats(oracle):
    for c in golden("hash_kats.json")["labels"]:
        p0 = bytes.fromhex(c["p0"]) if c["p0"] else None
        p1 = bytes.fromhex(c["p1"]) if c["p1"] else None
        got = oracle.label_node(c["is_source"], c["index"], p0, p1, bytes.fromhex(c["seed"]),
                                bytes.fromhex(c["desc"]))
        assert got.hex() == c["hex"]


def test_edges(oracle):
    for e in golden("edges.json"):
        if e["m"] > 50000:
            continue
        np_, p0, p1, rk = oracle.edges(e["m"])
        assert len(np_) == e["count"] == oracle.node_count(e["m"])
        assert hashlib.sha256(np_.tobytes()).hexdigest() == e["np"], e["m"]
        assert hashlib.sha256(p0.tobytes()).hexdigest() == e["p0"], e["m"]
        assert hashlib.sha256(p1.tobytes()).hexdigest() == e["p1"], e["m"]
        assert hashlib.sha256(rk.tobytes()).hexdigest() == e["rank"], e["m"]


def test_edge_invariants(oracle):
    # every predecessor id is smaller than its reader; 2-pred nodes list the
    # lower id first (common/src/graph.c:128-144); exactly m outputs
    for m in [1, 2, 3, 9, 100, 4096]:
        np_, p0, p1, rk = oracle.edges(m)
        ids = np.arange(len(np_), dtype=np.int64)
        assert (p0[np_ >= 1] < ids[np_ >= 1]).all()
        assert (p1[np_ == 2] < ids[np_ == 2]).all()
        assert (p0[np_ == 2] < p1[np_ == 2]).all()
        assert (np_ == 0).sum() == 2
        assert sorted(rk[rk >= 0].tolist()) == list(range(m))


def test_small_regions(oracle):
    for r in golden("small_regions.json"):
        key = bytes.fromhex(r["key"])
        out = oracle.label_region(key, r["chunk_blocks"], r["super_chunks"], r["rbo"], threads=4)
        assert out.tobytes().hex() == r["hex"], (r["chunk_blocks"], r["rbo"])


def test_plain_small_config(oracle, wl):
    g = golden("configs.json")["plain_small"]
    c = wl.plain_small()
    assert c["key"].hex() == g["key"]
    out = oracle.label_region(c["key"], c["chunk_blocks"], c["chunks"], c["rbo"], threads=8)
    sb = c["chunk_blocks"] * 32
    for j in range(c["chunks"]):
        assert hashlib.sha256(out[j * sb:(j + 1) * sb].tobytes()).hexdigest() == g["super_chunk_sha256"][j]


def test_scaffold_labels_match_reference_order(oracle):
    # every scaffold label (not only outputs) equals the reference's, for
    # small m, when the reference build is present in this container
    try:
        from oracle import RefCPU
        ref = RefCPU()
    except (FileNotFoundError, OSError):
        pytest.skip("reference CPU build not present")
    cs = oracle.chunk_seed(b"\x07" * 32, 5)
    for m in [1, 2, 5, 16, 64]:
        _, allb = oracle.label_chunk(cs, m, with_all=True)
        assert (allb == ref.scaffold_labels(cs, m)).all()


def test_challenges(oracle):
    """Verifier recompute: the oracle's chunk labeler answers the reference's
    pose_graph_challenge (graph.c:1019-1042) on raw graph seeds, and region
    blocks of one session (chunk seed from the block's chunk index)."""
    ch = golden("challenges.json")
    memo = {}
    for c in ch["graph"]:
        key = (c["seed"], c["m"])
        if key not in memo:
            memo[key] = oracle.label_chunk(bytes.fromhex(c["seed"]), c["m"])
        r = c["index"]
        assert memo[key][32 * r:32 * r + 32].tobytes().hex() == c["hex"], (c["m"], r)
    skey = bytes.fromhex(ch["region_key"])
    for c in ch["region"]:
        cb, b = c["chunk_blocks"], c["block"]
        out = oracle.label_region(skey, cb, 1, (b // cb) * cb)
        r = b % cb
        assert out[32 * r:32 * r + 32].tobytes().hex() == c["hex"], (cb, b)
