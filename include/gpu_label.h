/*
 * gpu_label.h — drop-in C ABI of the B200 labeler (libpose_b200.so).
 *
 * These five entry points have the signatures, argument meaning, return
 * conventions and synchronous behaviour of the reference's CUDA labeler API
 * (Amodo-Design/PoSE-Memory-Wiping, common/include/gpu_label.h:40-100), so a
 * caller such as tools/disk-wipe-bench links this library in place of the
 * reference's pose_common_cuda without source changes.  Labels are
 * byte-identical to the reference CPU in-place labeler
 * (common/src/graph.c:1604, pose_graph_label_region_pooled_inplace).
 *
 * Conventions (as in the reference):
 *   - 0 on success, -1 on error (bad algo, allocation failure, CUDA error),
 *     with a message on stderr; NULL from pose_graph_hbm_topo_build on error.
 *   - algo must be POSE_HASH_BLAKE3; chunk_blocks 0 means 4096; chunk_blocks
 *     must be in [1, 2^20].
 *   - hbm_dev_ptr is device memory of the CURRENT device; a topology is bound
 *     to the device current when it was built.
 *   - Calls are synchronous: they return after the device work finished.
 *     A topology may be used by one host thread at a time.
 *   - Layout: super-chunk j of chunk_blocks*32 bytes at hbm[j*chunk_blocks*32]
 *     holds output rank r's label at +32r; its chunk index is
 *     (region_block_offset + j*chunk_blocks) / chunk_blocks.  Tail bytes
 *     smaller than one super-chunk are left untouched (a buffer smaller than
 *     one super-chunk labels nothing and returns 0).
 *   - Progress lines go to stdout unless POSE_GPU_QUIET is set (non-empty,
 *     not "0").
 */
#ifndef POSE_B200_GPU_LABEL_H
#define POSE_B200_GPU_LABEL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef POSE_HASH_H
/* Hash selector, numerically identical to the reference's pose_hash_algo_t
 * (common/include/hash.h:31-35).  Only BLAKE3 runs on the GPU.  When the
 * reference's hash.h is included first its definition is used instead. */
typedef enum {
    POSE_HASH_BLAKE3 = 0,
    POSE_HASH_SHA256 = 1,
    POSE_HASH_AES_PRF = 2,
} pose_hash_algo_t;
#endif

/* Opaque resident topology (seed-independent; depends only on chunk_blocks). */
typedef struct pose_hbm_topo pose_hbm_topo_t;

/* Replaces common/include/gpu_label.h:40-45 (pose_graph_label_hbm,
 * implemented in common/src/cuda/label_gpu_common.cu:338-365): build, label,
 * free in one call. */
int pose_graph_label_hbm(const uint8_t *session_seed, size_t seed_len,
                         uint32_t chunk_blocks,
                         void *hbm_dev_ptr, size_t hbm_len,
                         uint64_t region_block_offset,
                         pose_hash_algo_t algo);

/* Replaces common/include/gpu_label.h:77-78 (pose_graph_hbm_topo_build,
 * label_gpu_common.cu:72-254): builds the schedule on the host, uploads it,
 * and builds the block-0 chaining-value table on the device. */
pose_hbm_topo_t *pose_graph_hbm_topo_build(uint32_t chunk_blocks,
                                           pose_hash_algo_t algo);

/* Replaces common/include/gpu_label.h:80-83 (pose_graph_hbm_topo_label,
 * label_gpu_common.cu:256-319). */
int pose_graph_hbm_topo_label(const pose_hbm_topo_t *topo,
                              const uint8_t *session_seed, size_t seed_len,
                              void *hbm_dev_ptr, size_t hbm_len,
                              uint64_t region_block_offset);

/* Replaces common/include/gpu_label.h:85 (pose_graph_hbm_topo_free,
 * label_gpu_common.cu:321-331).  Zeroes the topology's scratch pool before
 * releasing it. */
void pose_graph_hbm_topo_free(pose_hbm_topo_t *topo);

/* Replaces common/include/gpu_label.h:95-100 (pose_gpu_label_node_single,
 * common/src/cuda/blake3_node.cu:33-73): one node label on the GPU for a
 * known-answer test.  pred0/pred1 may be NULL (zero blocks). */
int pose_gpu_label_node_single(uint8_t out[32], int is_source,
                               uint64_t node_index,
                               const uint8_t *pred0, const uint8_t *pred1,
                               const uint8_t *seed, const uint8_t *descriptor,
                               const uint32_t key_src[8],
                               const uint32_t key_int[8]);

#ifdef __cplusplus
}
#endif

#endif /* POSE_B200_GPU_LABEL_H */
