/* topo_internal.h — read-only access to a topology handle for code outside
 * label_api.c (internal). */
#ifndef PB_TOPO_INTERNAL_H
#define PB_TOPO_INTERNAL_H

#include "kernels.h"
#include "gpu_label.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int device;
    uint32_t cb, copies;
    uint64_t super_bytes;
    pb_topo_view_t view;
    cudaStream_t stream;
} pb_topo_internal_t;

typedef struct {
    uint32_t T, G, teams, grid, cta;
    uint64_t team_scratch, scratch_bytes;
} pb_plan_out_t;

int pb_topo_internal(const pose_hbm_topo_t *t, pb_topo_internal_t *out);
/* The automatic schedule for nunits chunk copies within a fixed scratch budget. */
int pb_plan_for_budget(const pose_hbm_topo_t *t, uint64_t nunits, uint64_t budget, pb_plan_out_t *out);

#ifdef __cplusplus
}
#endif
#endif
