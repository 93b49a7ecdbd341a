/* topo_internal.h — read-only access to a topology handle for code outside
 * label_api.c (internal). */
#ifndef PB_TOPO_INTERNAL_H
#define PB_TOPO_INTERNAL_H

#include "kernels.h"
#include "gpu_label.h"
#include "pose_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int device;
    uint32_t cb, copies;
    uint64_t super_bytes;
    pb_topo_view_t view;
    cudaStream_t stream;
    int sms;
} pb_topo_internal_t;

typedef struct {
    uint32_t T, G, teams, grid, cta;
    uint64_t team_scratch, scratch_bytes;
} pb_plan_out_t;

int pb_topo_internal(const pose_hbm_topo_t *t, pb_topo_internal_t *out);
/* Record a calling thread's error message for pose_b200_last_error() and
 * print it to stderr, as every public entry point does on failure. */
void pb_set_err(const char *fmt, ...);
/* The automatic schedule for nunits chunk copies within a fixed scratch budget. */
int pb_plan_for_budget(const pose_hbm_topo_t *t, uint64_t nunits, uint64_t budget, pb_plan_out_t *out);

/* Label the whole super-chunks of a device buffer with the given chunk seeds
 * (32 bytes each, host memory) instead of seeds derived from a session seed. */
int pb_topo_label_raw(const pose_hbm_topo_t *t, const uint8_t *chunk_seeds, void *hbm_dev_ptr,
                      size_t hbm_len, const pose_b200_sched_t *sched, pose_b200_stats_t *stats);

/* The pipelined records for a 512-slot shared pool per unit (built on the
 * first call and kept with the topology), for the multi-unit depth kernel.
 * Needs a topology built with its block-0 table.  Returns 0 or -1. */
int pb_topo_view2_small(const pose_hbm_topo_t *t, pb_topo_view2_t *out);

/* Passes a team of T warps makes over all levels running G units in lockstep. */
uint64_t pb_topo_passes(const pose_hbm_topo_t *t, uint32_t T, uint32_t G);
/* Free device memory usable for scratch under an optional cap (the topology's
 * own scratch pool counts as free). */
uint64_t pb_topo_scratch_budget(const pose_hbm_topo_t *t, uint64_t cap);

#ifdef __cplusplus
}
#endif
#endif
