/* batch_internal.h — planning shared by batched labeling and the server
 * (internal). */
#ifndef PB_BATCH_INTERNAL_H
#define PB_BATCH_INTERNAL_H

#include "kernels.h"
#include "topo_internal.h"
#include "pose_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One request as the planner sees it: the session seed is already in a
 * device blob at seed_off. */
typedef struct {
    const pose_hbm_topo_t *topo;
    void *dev_ptr;
    size_t len;
    uint64_t rbo;
    uint32_t seed_off, seed_len;
} pb_req_t;

/* Host tables of one multi-topology launch. */
typedef struct {
    size_t ntopo;
    pb_topo_view_t *views;  /* [ntopo] */
    pb_munit_t *units;      /* [nunits], grouped by topology */
    uint32_t *unit_req;     /* [nunits] request index of each unit */
    pb_seedjob_t *jobs;     /* [njobs], one per super-chunk */
    pb_mbatch_t *batches;   /* [nbatches], longest first */
    uint64_t nunits, njobs, nbatches, nodes, team_scratch;
    uint64_t max_chain;  /* passes of the longest batch */
    double warp_passes;  /* one-warp passes of all batches (ALU work; idle warps skip a level) */
    uint32_t Gmax, all_cv0, sms;
} pb_plan_tables_t;

/* Plan n requests for teams of T warps with at most gcap units per team;
 * eff_min > 0 packs units per topology up to that lane efficiency, eff_min
 * <= 0 packs them while their chain stays within the launch's longest.
 * Unit i's seed index is its job's index.  Returns 0, or -1 with a message on
 * stderr (bad request, devices differ, out of host memory). */
int pb_plan_requests(const pb_req_t *reqs, size_t n, uint32_t T, uint32_t gcap, double eff_min,
                     pb_plan_tables_t *out);
/* Estimated makespan (SM clocks) of a plan run by R resident teams of T warps:
 * the longest batch chain (passes x latency per pass) against the ALU time of
 * all nodes spread over the SMs. */
double pb_plan_makespan(const pb_plan_tables_t *p, uint32_t T, uint64_t R);
void pb_plan_free(pb_plan_tables_t *p);
/* A schedule candidate: team size, packing rule (eff_min of
 * pb_plan_requests) and its estimated makespan. */
typedef struct {
    uint32_t T;
    double eff;
    double est;
} pb_cand_t;
/* The candidates sched leaves open (T in 1, 2, 4, 8; four packing rules),
 * best estimate first; returns their number (at most cap) or -1. */
int pb_plan_rank(const pb_req_t *reqs, size_t n, const pose_b200_sched_t *sched, pb_cand_t *out, int cap);
/* Team size T (1, 2, 4 or 8, unless sched fixes it) and packing rule for
 * pb_plan_requests with the lowest estimated makespan. */
int pb_plan_choose(const pb_req_t *reqs, size_t n, const pose_b200_sched_t *sched, uint32_t *T, double *eff_min);

#ifdef __cplusplus
}
#endif
#endif
