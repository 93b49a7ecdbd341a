"""Fleet wipe-time model for B200 labelers.

How long a set of disks takes to persist with G GPUs, K of them per disk, given
each stage's rate: the GPU labeler, the device-to-host copy, the disk write,
and the host's aggregate write.  The model restates the reference's planner
(tools/disk-calc/disk_calc.py:71-225: node counts 71-103, rate source
112-124, team rate 128-137, longest-processing-time assignment 140-148, the
K sweep 151-181 and 184-213) so that it gives the same numbers on the same
inputs, and adds the B200 label rate: `b200_gpu_bps` derives one GPU's
persisted-output rate at any chunk_blocks from the measured compression peak
and the fraction of it the throughput-regime labeler reaches, replacing the
reference's hand-entered `--gpu-mibs`.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from functools import lru_cache

LABEL_BYTES = 32
MIB = float(1 << 20)

# Measured on this project's B200 (bench.py): k_compress_bench's peak in the
# FMA-add form, and the throughput-regime labeler's fraction of it on a full
# 16 GiB window at chunk_blocks 2^17.
B200_COMPRESSIONS_PER_S = 36.9e9
B200_THROUGHPUT_FRACTION = 0.68
# node hashes per label: two compressions with the block-0 table (three without)
COMPRESSIONS_PER_NODE = 2


# ── node counts of one chunk (common/src/graph.c:33-54) ─────────────────────

def graph_n(cb: int) -> int:
    """The graph parameter n = bit_length(m - 1) - 1 (0 for m <= 2)."""
    return 0 if cb <= 1 else max(0, (cb - 1).bit_length() - 1)


def _butterfly(d: int) -> int:
    return (d + 1) << d


@lru_cache(maxsize=None)
def _connected(level: int) -> int:
    return 1 if level == 0 else 2 * _connected(level - 1) + 2 * _butterfly(level - 1)


@lru_cache(maxsize=None)
def _standalone(level: int) -> int:
    return 1 if level == 0 else _standalone(level - 1) + _butterfly(level - 1) + _connected(level - 1)


def chunk_nodes(cb: int) -> int:
    """Scaffold nodes hashed for one persisted super-chunk (two copies)."""
    return 2 * _standalone(graph_n(cb) + 1)


def nodes_per_label(cb: int) -> float:
    return chunk_nodes(cb) / cb


def b200_gpu_bps(cb: int, compressions_per_s: float = B200_COMPRESSIONS_PER_S,
                 fraction: float = B200_THROUGHPUT_FRACTION) -> float:
    """Persisted-output bytes per second of one B200 at chunk_blocks `cb` in
    the throughput regime (thousands of chunks in flight)."""
    labels_per_s = compressions_per_s * fraction / (COMPRESSIONS_PER_NODE * nodes_per_label(cb))
    return labels_per_s * LABEL_BYTES


# ── the schedule model ──────────────────────────────────────────────────────

@dataclass
class Fleet:
    gpus: int = 8
    gpu_mibs: float = 0.0        # one GPU's persisted-output rate; 0 = b200_gpu_bps(chunk_blocks)
    gpu_hash_rate: float = 0.0   # alternative: one GPU's node hashes per second
    chunk_blocks: int = 4096
    disk_sizes_bytes: list = field(default_factory=list)
    disk_mibs: float = 0.0       # per-disk write cap (0 = none)
    d2h_mibs: float = 0.0        # per-GPU device-to-host cap (0 = none)
    host_mibs: float = 0.0       # all disks together (0 = none)
    pool_eff: float = 1.0        # efficiency of K > 1 GPUs sharing a disk
    sector_bytes: int = 4096
    gpus_per_disk: int = 0       # 0 = report the sweep only


def gpu_rate(f: Fleet) -> tuple[float, str]:
    if f.gpu_mibs > 0:
        return f.gpu_mibs * MIB, "measured (--gpu-mibs)"
    if f.gpu_hash_rate > 0:
        return f.gpu_hash_rate * LABEL_BYTES / nodes_per_label(f.chunk_blocks), \
            "derived upper bound (--gpu-hash-rate / excess multiplier)"
    return b200_gpu_bps(f.chunk_blocks), "B200 model (measured compression peak x labeler fraction)"


def team_rate(f: Fleet, gpu_bps: float, k: int) -> tuple[float, str]:
    """Bytes per second a team of k GPUs writes into one disk, and the stage
    that sets it (the slowest of labeler, copy and disk)."""
    eff = f.pool_eff if k > 1 else 1.0
    stages = [("gpu labeler", k * gpu_bps * eff),
              ("d2h copy", k * f.d2h_mibs * MIB if f.d2h_mibs > 0 else math.inf),
              ("disk write", f.disk_mibs * MIB if f.disk_mibs > 0 else math.inf)]
    name, rate = stages[0]
    for n, r in stages[1:]:
        if r < rate:
            name, rate = n, r
    return rate, name


def assign_longest_first(sizes: list[float], teams: int, rate: float) -> tuple[float, list[float]]:
    """Give each disk, largest first, to the team that frees up first;
    returns the makespan and every team's busy time."""
    busy = [0.0] * teams
    for size in sorted(sizes, reverse=True):
        i = min(range(teams), key=lambda t: (busy[t], t))
        busy[i] += size / rate
    return max(busy), busy


def plan_k(f: Fleet, gpu_bps: float, k: int) -> dict:
    teams = f.gpus // k
    rate, stage = team_rate(f, gpu_bps, k)
    host_bound = f.host_mibs > 0 and teams * rate > f.host_mibs * MIB
    if host_bound:
        rate, stage = f.host_mibs * MIB / teams, "host aggregate write"
    super_bytes = f.chunk_blocks * LABEL_BYTES
    pad = math.ceil(super_bytes / f.sector_bytes) * f.sector_bytes / super_bytes
    makespan, busy = assign_longest_first(f.disk_sizes_bytes, teams, rate / pad)
    ideal = sum(f.disk_sizes_bytes) / (f.gpus * gpu_bps)
    return {"k": k, "teams": teams, "idle_gpus": f.gpus - teams * k, "team_rate_mibs": rate / MIB,
            "binding_stage": stage, "host_bound": host_bound, "pad_factor": pad,
            "concurrent_disks": min(teams, len(f.disk_sizes_bytes)), "makespan_s": makespan,
            "team_busy_s": busy, "gpu_utilisation": ideal / makespan if makespan > 0 else 0.0}


def plan(f: Fleet) -> dict:
    """Every K from 1 to gpus, the fastest, and the two named strategies."""
    gpu_bps, source = gpu_rate(f)
    if gpu_bps <= 0:
        raise ValueError("no GPU rate")
    if not f.disk_sizes_bytes:
        raise ValueError("no disks")
    if f.gpus < 1:
        raise ValueError("gpus must be >= 1")
    total = sum(f.disk_sizes_bytes)
    sweep = [plan_k(f, gpu_bps, k) for k in range(1, f.gpus + 1)]
    best = sweep[0]
    for r in sweep[1:]:
        if r["makespan_s"] < best["makespan_s"]:
            best = r
    by_k = {r["k"]: r for r in sweep}
    return {"rate_source": source, "gpu_mibs": gpu_bps / MIB,
            "implied_node_hashes_per_sec": gpu_bps / LABEL_BYTES * nodes_per_label(f.chunk_blocks),
            "chunk_blocks": f.chunk_blocks,
            "valid_cb": 1 <= f.chunk_blocks <= (1 << 20) and f.chunk_blocks & (f.chunk_blocks - 1) == 0,
            "excess": nodes_per_label(f.chunk_blocks), "scaffold_nodes": chunk_nodes(f.chunk_blocks),
            "super_bytes": f.chunk_blocks * LABEL_BYTES, "total_bytes": total,
            "aggregate_gpu_mibs": f.gpus * gpu_bps / MIB, "ideal_s": total / (f.gpus * gpu_bps),
            "single_gpu_s": total / gpu_bps, "sweep": sweep, "best": best,
            "gpus_per_disk": by_k[f.gpus], "disk_per_gpu": by_k[1],
            "chosen": by_k.get(f.gpus_per_disk) if f.gpus_per_disk else None}
