/*
 * pose_b200.h — additive C ABI of the B200 labeler (libpose_b200.so).
 *
 * New symbols next to the drop-in ones in gpu_label.h; none of them changes
 * the behaviour of the drop-in entry points.  The reference has no
 * counterpart for the schedule/statistics structs; each function below names
 * the reference interface it extends.
 */
#ifndef POSE_B200_H
#define POSE_B200_H

#include "gpu_label.h"

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Schedule of one labeling launch.  Zero fields mean "choose automatically". */
typedef struct {
    uint32_t team_warps;        /* T: warps that cooperate on one batch (1..16, power of 2) */
    uint32_t units_per_team;    /* G: chunk copies run in lockstep by one team (1..32, power of 2) */
    uint32_t max_teams;         /* cap on resident teams (0 = occupancy and memory bound) */
    uint32_t kernel;            /* 0 = automatic, 1 = basic lockstep kernel, 2 = pipelined kernel */
    uint64_t scratch_cap_bytes; /* cap on the scratch pool (0 = free HBM less a margin) */
} pose_b200_sched_t;

/* What one call did (device times from CUDA events on the labeler's stream). */
typedef struct {
    double kernel_ms;           /* labeling kernel(s) */
    double total_ms;            /* whole call on the device stream (seeds, kernel, zeroing) */
    uint64_t super_chunks;      /* super-chunks labelled */
    uint64_t units;             /* chunk copies (2 per super-chunk unless chunk_blocks == 1) */
    uint64_t nodes;             /* node labels computed */
    uint64_t scratch_bytes;     /* scratch pool bytes used */
    uint32_t team_warps, units_per_team, teams, kernel_launches;
    uint32_t used_cv0_table;    /* 1 when block 0 came from the precomputed table */
    uint32_t kernel;            /* 1 = basic lockstep kernel, 2 = pipelined kernel */
} pose_b200_stats_t;

/* Extends pose_graph_hbm_topo_build (common/include/gpu_label.h:77-78).
 * with_cv0_table: 1 = also build the block-0 chaining-value table
 * (copies * nodes * 32 bytes of HBM), 0 = hash block 0 in every label call. */
pose_hbm_topo_t *pose_b200_topo_build(uint32_t chunk_blocks, int with_cv0_table);

/* Extends pose_graph_hbm_topo_label (common/include/gpu_label.h:80-83) with an
 * explicit schedule (NULL = automatic) and statistics (NULL = none).  Same
 * bytes, same return convention, synchronous. */
int pose_b200_topo_label(const pose_hbm_topo_t *topo, const uint8_t *session_seed,
                         size_t seed_len, void *hbm_dev_ptr, size_t hbm_len,
                         uint64_t region_block_offset, const pose_b200_sched_t *sched,
                         pose_b200_stats_t *stats);

/* Topology facts (any pointer may be NULL). */
void pose_b200_topo_info(const pose_hbm_topo_t *topo, uint32_t *chunk_blocks,
                         uint64_t *nodes_per_chunk, uint32_t *levels, uint32_t *pool_slots,
                         uint64_t *device_bytes);

/* The schedule the automatic policy would pick for `units` chunk copies. */
int pose_b200_plan(const pose_hbm_topo_t *topo, uint64_t super_chunks,
                   const pose_b200_sched_t *hint, pose_b200_sched_t *out);

/* Sustained compression rate of this GPU for the labeler's instruction mix:
 * every SM full of threads chaining register-resident compressions.  Returns
 * compressions per second (0 on error); *latency_cycles gets the dependent
 * latency of one compression in SM clocks (NULL to skip). */
double pose_b200_compress_rate(uint32_t iters, double *latency_cycles);

/* Labeling that allocates no device memory during the call.
 *
 * No counterpart in the reference: it is an addition of this library.  Same
 * arguments, bytes and return convention as pose_graph_hbm_topo_label, for
 * callers that must not call cudaMalloc while they label — e.g. a wipe worker
 * that reserved the device's free memory for its label window before
 * starting (a late allocation could fail half-way through a disk), or a host
 * whose own allocator or an active stream capture forbids new device
 * allocations.  The topology, seed and output buffer are still the caller's.
 *
 * Its scratch pool (64 MiB), chunk-seed table (8192 seeds) and work counter
 * are static device arrays inside the library: a device holds them from when
 * it loads them (at the latest, this function's first call on that device)
 * until the process exits.  The schedule shrinks to fit 64 MiB, so every
 * chunk_blocks in [1, 2^20] works; session seeds longer than 1016 bytes are
 * rejected with an error, and buffers of more than 8192 super-chunks are
 * labelled in several launches.
 *
 * The first call on a device looks up the arrays' device addresses
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the same arrays: the work counter is cleared by each launch
 * and the scratch and seed table are zeroed before the call returns, but
 * calls whose device work overlaps (from several host threads, or on several
 * topologies of one device at once) race on them and must be serialised by
 * the caller. */
int pose_b200_topo_label_noalloc(const pose_hbm_topo_t *topo, const uint8_t *session_seed,
                                 size_t seed_len, void *hbm_dev_ptr, size_t hbm_len,
                                 uint64_t region_block_offset);

/* Last error message of the calling thread ("" when none). */
const char *pose_b200_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* POSE_B200_H */
