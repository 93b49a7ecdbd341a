"""Seeded synthetic workloads of the labeling path.

All inputs of this path are session keys and chunk positions, so every
workload is synthetic by construction.  Session keys are four successive
splitmix64 outputs from a configured state, each serialised little-endian
(32 bytes); the CPU oracle and the GPU path share this convention, so it
cannot affect parity.

  plain_small   one session, key splitmix64(0), chunk_blocks 2^10, 64
                consecutive chunks from absolute position 0
  plain_2e17    one session, key splitmix64(1), chunk_blocks 2^17, 32
                consecutive super-chunks from position 0
  batched       256 sessions, key i = splitmix64(2 + i), chunk_blocks 2^e
                with e uniform in {12..17}, 1-8 chunks each at random
                chunk-aligned absolute positions
  deep_2e20     one session, key splitmix64(3), chunk_blocks 2^20, 4 chunks,
                scratch capped at 40 GiB
  served        Poisson arrivals (200 requests/s) from 64 sessions, chunk_blocks
                2^e with e uniform in {10..18}, 1-16 consecutive chunks per
                request at a random chunk-aligned position
"""
from __future__ import annotations

import random

MASK64 = (1 << 64) - 1


def splitmix64_key(state: int) -> bytes:
    out = b""
    s = state & MASK64
    for _ in range(4):
        s = (s + 0x9E3779B97F4A7C15) & MASK64
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        z ^= z >> 31
        out += z.to_bytes(8, "little")
    return out


def plain_small() -> dict:
    return {"name": "plain_small", "key": splitmix64_key(0), "chunk_blocks": 1 << 10,
            "chunks": 64, "rbo": 0}


def plain_2e17() -> dict:
    return {"name": "plain_2e17", "key": splitmix64_key(1), "chunk_blocks": 1 << 17,
            "chunks": 32, "rbo": 0}


def deep_2e20() -> dict:
    return {"name": "deep_2e20", "key": splitmix64_key(3), "chunk_blocks": 1 << 20,
            "chunks": 4, "rbo": 0, "scratch_cap_bytes": 40 << 30}


def batched(sessions: int = 256, rng_seed: int = 0x5EED_0003) -> list[dict]:
    """One entry per session: key, chunk_blocks and absolute chunk indices
    (each chunk is one super-chunk at region_block_offset = index * cb)."""
    rng = random.Random(rng_seed)
    out = []
    for i in range(sessions):
        cb = 1 << rng.randint(12, 17)
        n = rng.randint(1, 8)
        idx = sorted(rng.sample(range(1 << 20), n))
        out.append({"session": i, "key": splitmix64_key(2 + i), "chunk_blocks": cb,
                    "chunk_indices": idx})
    return out


def served(requests: int = 2000, rate_per_s: float = 200.0, sessions: int = 64,
           rng_seed: int = 0x5EED_0005) -> list[dict]:
    """A fixed Poisson arrival trace: arrival time (s), session, key,
    chunk_blocks, first chunk index and chunk count."""
    rng = random.Random(rng_seed)
    t = 0.0
    out = []
    for r in range(requests):
        t += rng.expovariate(rate_per_s)
        s = rng.randrange(sessions)
        cb = 1 << rng.randint(10, 18)
        n = rng.randint(1, 16)
        first = rng.randrange(1 << 16)
        out.append({"request": r, "arrival_s": t, "session": s, "key": splitmix64_key(1000 + s),
                    "chunk_blocks": cb, "first_chunk": first, "chunks": n})
    return out


def copy_nodes(chunk_blocks: int) -> int:
    """Nodes in one standalone copy (half a chunk's scaffold)."""
    def b(d):
        return (d + 1) << d

    def c(level):
        return 1 if level == 0 else 2 * c(level - 1) + 2 * b(level - 1)

    def s(level):
        return 1 if level == 0 else s(level - 1) + b(level - 1) + c(level - 1)

    n = max(0, (chunk_blocks - 1).bit_length() - 1) if chunk_blocks > 1 else 0
    return s(n + 1)


def chunk_nodes(chunk_blocks: int) -> int:
    return 2 * copy_nodes(chunk_blocks)


def rank_region(workload: dict, rank: int, world: int) -> tuple[int, int]:
    """(region_block_offset, super_chunks) of one rank under weak scaling:
    every rank labels the workload's number of super-chunks, rank r taking
    the r-th consecutive range of absolute positions.  No data crosses ranks:
    a label depends only on (seed, absolute position), so the ranges are
    independent and together equal one region of world * chunks super-chunks
    (the K-GPUs-per-range split of tools/disk-wipe-bench/disk_wipe_bench.cu:
    1016-1031, with each GPU given a whole range)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    cb, n = workload["chunk_blocks"], workload["chunks"]
    return workload["rbo"] + rank * n * cb, n
