"""The C-ABI library loads on a machine without a GPU and exports every
function include/*.h declares; argument errors that need no device are
rejected with the reference's return codes (common/src/cuda/
label_gpu_common.cu:75-78, 262-264, 344-357)."""
from __future__ import annotations

import ctypes as C
import subprocess

from conftest import PKG_DIR


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.load()
    declared = pkg.exported_symbols()
    for name in ["pose_graph_label_hbm", "pose_graph_hbm_topo_build", "pose_graph_hbm_topo_label",
                 "pose_graph_hbm_topo_free", "pose_gpu_label_node_single"]:
        assert name in declared
    for name in declared:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", pkg.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert exported == set(declared), exported ^ set(declared)


def test_bad_algo_is_rejected(pkg):
    L = pkg.load()
    for algo in (pkg.POSE_HASH_SHA256, pkg.POSE_HASH_AES_PRF):
        assert L.pose_graph_hbm_topo_build(1024, algo) is None
        assert pkg.label_hbm(b"k" * 32, 1024, 0x1000, 1 << 20, 0, algo) == -1


def test_chunk_blocks_out_of_range(pkg):
    L = pkg.load()
    assert L.pose_graph_hbm_topo_build((1 << 20) + 1, pkg.POSE_HASH_BLAKE3) is None
    assert pkg.label_hbm(b"k" * 32, (1 << 20) + 1, 0x1000, 1 << 30, 0) == -1


def test_buffer_smaller_than_one_super_chunk_labels_nothing(pkg):
    # returns 0 before touching the device (label_gpu_common.cu:356-357)
    assert pkg.label_hbm(b"k" * 32, 1024, 0x1000, 1024 * 32 - 1, 0) == 0
    assert pkg.label_hbm(b"k" * 32, 0, 0x1000, 4096 * 32 - 32, 0) == 0


def test_null_topology(pkg):
    L = pkg.load()
    assert L.pose_graph_hbm_topo_label(None, None, 0, None, 1 << 20, 0) == -1
    L.pose_graph_hbm_topo_free(None)  # no-op, as in the reference


def test_autotune_rejects_null_topology_and_short_buffer(pkg):
    L = pkg.load()
    assert L.pose_b200_topo_autotune(None, None, 0, None, 1 << 20, 0, 2, None, None) == -1


def test_kat_rejects_null_arguments(pkg):
    L = pkg.load()
    out = (C.c_uint8 * 32)()
    assert L.pose_gpu_label_node_single(C.cast(out, C.POINTER(C.c_uint8)), 1, 0, None, None,
                                        None, None, None, None) == -1


def test_headers_compile_as_c11_and_cxx():
    src = '#include "gpu_label.h"\n#include "pose_b200.h"\nint main(void){return 0;}\n'
    inc = PKG_DIR.replace("pose-memory-wiping_b200", "include")
    for compiler, std in (("gcc", "-std=c11"), ("g++", "-std=c++17")):
        lang = "c" if compiler == "gcc" else "c++"
        r = subprocess.run([compiler, std, "-Wall", "-Werror", "-fsyntax-only", "-I", inc, "-x", lang, "-"],
                           input=src, text=True, capture_output=True)
        assert r.returncode == 0, r.stderr


def test_workspace_audit_rejects_bad_arguments(pkg):
    L = pkg.load()
    n = C.c_uint64(7)
    assert L.pose_b200_topo_residue(None, C.byref(n)) == -1
    assert L.pose_b200_count_nonzero(None, 16, C.byref(n)) == -1
    assert L.pose_b200_count_nonzero(C.c_void_p(0x1001), 16, C.byref(n)) == -1  # not 16-byte aligned
    assert L.pose_b200_count_nonzero(None, 0, C.byref(n)) == 0 and n.value == 0  # nothing to count
