"""The reference arm of bench.py: the reference's own CPU labeler
(oracle/_ref) timed on this host, printed as the bench's one JSON line.
It runs the warm-up and timed steps it is given, and under torchrun only
rank 0 works and prints.  Needs the reference CPU build (oracle/_ref), so
it is skipped where that is absent."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libposeref.so")
pytestmark = pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference CPU build absent")


def _run(env_extra: dict, *args: str) -> subprocess.CompletedProcess:
    env = dict(os.environ, POSE_GPU_QUIET="1", **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, env=env, timeout=300, cwd=ROOT)


def test_reference_arm_prints_the_bench_line():
    r = _run({}, "--workload", "plain_small", "--steps", "2", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["steps"] == 2 and d["warmup"] == 3
    assert d["value"] > 0 and d["unit"] == "MiB/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == "plain_small" and d["n_gpus"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "MiB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    for key in ("metric", "ms_per_step", "scaling", "vs_baseline", "dtype", "data"):
        assert key in d, key


def test_reference_arm_is_silent_on_other_ranks():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"}, "--workload", "plain_small", "--steps", "1", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_bench_parity_check_against_reference_digests():
    """bench.py hashes the bytes it timed against the reference's digests:
    the reference CPU labeler's own output of the small plain workload reads
    bit-exact, a planted byte flip (in that host copy) reads mismatch, and a
    range no digest covers reads unchecked."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    bench.load_pkg()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefCPU
    w = bench.workload("plain_small")
    data = RefCPU().label_super_chunks(w["key"], w["chunk_blocks"], w["chunks"], w["rbo"])
    ok = bench.golden_parity(w, w["rbo"], w["chunks"], data)
    assert ok["parity"] == "bit-exact" and ok["checked_super_chunks"] == w["chunks"]
    data[5 * w["chunk_blocks"] * 32 + 17] ^= 1
    bad = bench.golden_parity(w, w["rbo"], w["chunks"], data)
    assert bad["parity"] == "mismatch" and bad["mismatched_super_chunks"] == [5]
    far = w["rbo"] + 10_000 * w["chunk_blocks"]
    assert bench.golden_parity(w, far, w["chunks"], data)["parity"] == "unchecked"
