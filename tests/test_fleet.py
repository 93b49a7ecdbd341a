"""The fleet wipe-time model (pose_b200.fleet) against the reference's own
planner (tools/disk-calc/disk_calc.py) on the fixtures of
tests/golden/gen_fleet.py, and the B200 rate model against the measured
throughput-regime rate."""
from __future__ import annotations

import math

import pytest

from conftest import golden


@pytest.fixture(scope="module")
def fleet(pkg):
    import pose_b200.fleet as fl
    return fl


def close(a, b):
    return a == b or math.isclose(a, b, rel_tol=1e-12, abs_tol=1e-12)


def test_matches_reference_planner(fleet):
    for case in golden("fleet.json"):
        r = fleet.plan(fleet.Fleet(**case["params"]))
        want = case["result"]
        for k in ("gpu_mibs", "implied_node_hashes_per_sec", "excess", "total_bytes", "ideal_s", "single_gpu_s"):
            assert close(r[k], want[k]), (k, r[k], want[k])
        assert r["scaffold_nodes"] == want["scaffold_nodes"]
        assert r["best"]["k"] == want["best_k"]
        assert (r["chosen"]["k"] if r["chosen"] else None) == want["chosen_k"]
        assert len(r["sweep"]) == len(want["sweep"])
        for got, exp in zip(r["sweep"], want["sweep"]):
            for k, v in exp.items():
                assert close(got[k], v) if isinstance(v, float) else got[k] == v, (k, got[k], v)


def test_node_counts_match_the_topology(fleet, wl):
    for cb in (1, 2, 3, 64, 1000, 1 << 12, 1 << 17):
        assert fleet.chunk_nodes(cb) == wl.chunk_nodes(cb)


def test_b200_rate_model(fleet):
    # the model reproduces the measured 16 GiB-window rate at 2^17 (1387 MiB/s)
    mibs = fleet.b200_gpu_bps(1 << 17) / fleet.MIB
    assert 1300 < mibs < 1480
    r = fleet.plan(fleet.Fleet(gpus=8, chunk_blocks=1 << 17, disk_sizes_bytes=[8e12] * 8))
    assert r["rate_source"].startswith("B200 model")
    assert r["best"]["k"] == 1 and math.isclose(r["best"]["makespan_s"], 8e12 / fleet.b200_gpu_bps(1 << 17))
