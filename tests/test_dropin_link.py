"""Drop-in check: the reference's disk-wipe-bench (tools/disk-wipe-bench/
disk_wipe_bench.cu) compiles unchanged and links against libpose_b200.so in
place of the reference's pose_common_cuda (build only; nothing is run).
Needs the reference sources, so it is skipped where they are absent."""
from __future__ import annotations

import os
import subprocess

import pytest

from conftest import PKG_DIR, ROOT

REF_ROOT = os.environ.get("POSE_REF", "/root/reference")  # the reference tree; override with POSE_REF
REF = os.path.join(REF_ROOT, "tools", "disk-wipe-bench", "disk_wipe_bench.cu")


@pytest.mark.skipif(not os.path.exists(REF), reason="reference sources not present")
def test_disk_wipe_bench_links_unchanged(pkg, tmp_path):
    pkg.load()
    refso = os.path.join(ROOT, "oracle", "_ref", "libposeref.so")
    if not os.path.exists(refso):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    r = subprocess.run(["sh", os.path.join(ROOT, "oracle", "link_disk_wipe_bench.sh"), str(tmp_path)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    undefined = subprocess.run(["nm", "-u", str(tmp_path / "disk-wipe-bench-b200")], capture_output=True,
                               text=True, check=True).stdout.split()
    used = {s for s in undefined if s.startswith(("pose_graph_hbm", "pose_graph_label_hbm", "pose_gpu"))}
    assert used == {"pose_graph_hbm_topo_build", "pose_graph_hbm_topo_label", "pose_graph_hbm_topo_free"}
    ours = subprocess.run(["nm", "-D", "--defined-only", pkg.LIB_PATH], capture_output=True, text=True,
                          check=True).stdout
    for s in used:
        assert f" T {s}" in ours
