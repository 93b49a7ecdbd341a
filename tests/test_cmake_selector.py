"""The build-time strategy selector: the reference's own CMake build of
disk-wipe-bench (tools/disk-wipe-bench/CMakeLists.txt, which adds common/ as
a subdirectory) configured with -DPOSE_GPU_LABEL_STRATEGY=b200 takes its
pose_common_cuda target from libpose_b200.so (cmake/pose_b200.cmake).

A scratch copy of the reference's common/ and tools/disk-wipe-bench/ gets the
one edit INTEGRATION.md asks a maintainer to make to common/CMakeLists.txt
(the reference's pose_common_cuda block moves into the else() branch of a
`b200` test); then CMake configures and builds the disk-wipe-bench target for
sm_100.  Build only, nothing is run.  Needs the reference sources, cmake and
nvcc, so it is skipped where any is absent."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

from conftest import PKG_DIR

REF_ROOT = os.environ.get("POSE_REF", "/root/reference")  # the reference tree; override with POSE_REF
HAVE = (os.path.isdir(os.path.join(REF_ROOT, "common")) and shutil.which("cmake") and shutil.which("nvcc"))
pytestmark = pytest.mark.skipif(not HAVE, reason="reference sources, cmake or nvcc absent")

MARK_BEGIN = "    add_library(pose_common_cuda STATIC"
MARK_END = "    target_link_libraries(pose_common_cuda PUBLIC pose_common)\n"


def add_b200_branch(cmakelists: str, cmake_file: str) -> str:
    """INTEGRATION.md's edit: the reference's pose_common_cuda block, from its
    add_library to its target_link_libraries, becomes the else() branch of a
    POSE_GPU_LABEL_STRATEGY == "b200" test that includes pose_b200.cmake."""
    a = cmakelists.index(MARK_BEGIN)
    b = cmakelists.index(MARK_END) + len(MARK_END)
    return (cmakelists[:a] + '    if(POSE_GPU_LABEL_STRATEGY STREQUAL "b200")\n'
            f"        include({cmake_file})\n" + "    else()\n" + cmakelists[a:b] + "    endif()\n"
            + cmakelists[b:])


def test_b200_strategy_builds_disk_wipe_bench(pkg, tmp_path):
    pkg.load()
    src = tmp_path / "src"
    shutil.copytree(os.path.join(REF_ROOT, "common"), src / "common",
                    ignore=shutil.ignore_patterns("build"))  # the reference's prebuilt tree is never used
    shutil.copytree(os.path.join(REF_ROOT, "tools", "disk-wipe-bench"), src / "tools" / "disk-wipe-bench")
    cm = src / "common" / "CMakeLists.txt"
    cm.write_text(add_b200_branch(cm.read_text(), os.path.join(PKG_DIR, "cmake", "pose_b200.cmake")))
    bld = tmp_path / "build"
    cfg = subprocess.run(["cmake", "-S", str(src / "tools" / "disk-wipe-bench"), "-B", str(bld),
                          "-DPOSE_GPU_LABEL_STRATEGY=b200", "-DPOSE_CUDA_ARCH=100", "-DCMAKE_BUILD_TYPE=Release"],
                         capture_output=True, text=True, timeout=300)
    assert cfg.returncode == 0, cfg.stdout[-2000:] + cfg.stderr[-2000:]
    assert "labeling strategy b200" in cfg.stdout
    mk = subprocess.run(["cmake", "--build", str(bld), "--target", "disk-wipe-bench", "-j", "8"],
                        capture_output=True, text=True, timeout=600)
    assert mk.returncode == 0, mk.stdout[-3000:] + mk.stderr[-2000:]
    exe = bld / "disk-wipe-bench"
    assert exe.exists()
    # none of the reference's GPU labeler sources was compiled ...
    built = [os.path.join(d, f) for d, _, fs in os.walk(bld) for f in fs]
    assert not [f for f in built if "label_gpu_" in f or "blake3_node" in f]
    # ... the labeler symbols come from libpose_b200.so at run time
    und = subprocess.run(["nm", "-u", str(exe)], capture_output=True, text=True, check=True).stdout
    for s in ("pose_graph_hbm_topo_build", "pose_graph_hbm_topo_label", "pose_graph_hbm_topo_free"):
        assert s in und
    dyn = subprocess.run(["readelf", "-d", str(exe)], capture_output=True, text=True, check=True).stdout
    assert "[libpose_b200.so]" in dyn
