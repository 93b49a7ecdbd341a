#!/bin/sh
# Drop-in check (build only, nothing is run): compile the reference's
# tools/disk-wipe-bench/disk_wipe_bench.cu UNCHANGED and link it against
# libpose_b200.so (in place of the reference's pose_common_cuda) plus the
# reference's own CPU library (oracle/_ref/libposeref.so, built from
# common/src by oracle/Makefile).  Success means every GPU labeler symbol the
# bench calls resolves to this library and nothing clashes.
# Usage: oracle/link_disk_wipe_bench.sh <out-dir>
set -e
REF=${POSE_REF:-${REF:-/root/reference}}
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=$(dirname "$HERE")
OUT=${1:-$HERE/_ref}
mkdir -p "$OUT"
nvcc -std=c++17 -O2 -gencode arch=compute_100a,code=sm_100a \
    -I"$REF/common/include" -c "$REF/tools/disk-wipe-bench/disk_wipe_bench.cu" -o "$OUT/disk_wipe_bench.o"
nvcc -gencode arch=compute_100a,code=sm_100a -o "$OUT/disk-wipe-bench-b200" "$OUT/disk_wipe_bench.o" \
    -L"$ROOT/pose-memory-wiping_b200" -lpose_b200 \
    -L"$HERE/_ref" -lposeref \
    -Xlinker -rpath -Xlinker "$ROOT/pose-memory-wiping_b200" -Xlinker -rpath -Xlinker "$HERE/_ref" \
    -lcudart -lpthread
nm -u "$OUT/disk-wipe-bench-b200" | grep -E "pose_graph_hbm|pose_graph_label_hbm|pose_gpu" || true
