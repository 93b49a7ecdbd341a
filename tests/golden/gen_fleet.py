#!/usr/bin/env python3
"""Generate tests/golden/fleet.json: the reference's own wipe-time planner
(tools/disk-calc/disk_calc.py, imported from the reference tree in
/root/reference) run on a set of fleet configurations.  tests/test_fleet.py
checks pose_b200.fleet against these numbers.

    python tests/golden/gen_fleet.py
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("POSE_REF", "/root/reference")  # the reference tree; override with POSE_REF
REF = os.path.join(REF_ROOT, "tools", "disk-calc", "disk_calc.py")

TB = 1e12
CASES = [
    dict(gpus=4, gpu_mibs=620.0, chunk_blocks=1 << 17, disk_sizes_bytes=[8 * TB] * 4),
    dict(gpus=8, gpu_mibs=1387.0, chunk_blocks=1 << 17, disk_sizes_bytes=[16 * TB, 8 * TB, 8 * TB, 4 * TB, 2 * TB],
         disk_mibs=2500.0, d2h_mibs=20000.0, pool_eff=0.9),
    dict(gpus=8, gpu_hash_rate=1.2e10, chunk_blocks=4096, disk_sizes_bytes=[3.84 * TB] * 12,
         disk_mibs=3000.0, host_mibs=12000.0),
    dict(gpus=3, gpu_mibs=185.0, chunk_blocks=64, disk_sizes_bytes=[1 * TB, 0.5 * TB], sector_bytes=4096,
         gpus_per_disk=3),
    dict(gpus=6, gpu_mibs=900.0, chunk_blocks=1 << 20, disk_sizes_bytes=[20 * TB] * 3 + [10 * TB] * 2,
         d2h_mibs=400.0, pool_eff=0.75, gpus_per_disk=2),
    dict(gpus=1, gpu_hash_rate=5e9, chunk_blocks=1 << 10, disk_sizes_bytes=[0.25 * TB], sector_bytes=512),
]


def main() -> None:
    spec = importlib.util.spec_from_file_location("disk_calc", REF)
    dc = importlib.util.module_from_spec(spec)
    sys.modules["disk_calc"] = dc  # its dataclasses resolve their module
    spec.loader.exec_module(dc)
    out = []
    for c in CASES:
        r = dc.compute(dc.Params(**c))
        keep = {k: r[k] for k in ("gpu_mibs", "implied_node_hashes_per_sec", "excess", "scaffold_nodes",
                                  "total_bytes", "ideal_s", "single_gpu_s")}
        keep["sweep"] = [{k: s[k] for k in ("k", "teams", "idle_gpus", "team_rate_mibs", "binding_stage",
                                            "host_bound", "pad_factor", "makespan_s", "gpu_utilisation")}
                         for s in r["sweep"]]
        keep["best_k"] = r["best"]["k"]
        keep["chosen_k"] = r["chosen"]["k"] if r["chosen"] else None
        out.append({"params": c, "result": keep})
    with open(os.path.join(HERE, "fleet.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"{len(out)} cases")


if __name__ == "__main__":
    main()
