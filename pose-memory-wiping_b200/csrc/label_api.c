/*
 * label_api.c — C11 host side of the B200 labeler: the drop-in C ABI of
 * include/gpu_label.h and the additive ABI of include/pose_b200.h.
 *
 * Mirrors the reference host driver (common/src/cuda/label_gpu_common.cu and
 * the warp strategy's label_gpu_run, common/src/cuda/label_gpu_warp.cu:
 * 125-248) in behaviour: same entry points, same validation and return
 * codes, synchronous calls, a topology bound to the device current at build
 * time, scratch zeroed before the call returns.  The machinery differs:
 *   - the schedule is this library's own (topology.c) and is uploaded once;
 *   - per-chunk seeds are derived on the device (k_chunk_seeds) instead of a
 *     host loop plus copy per batch;
 *   - one persistent launch covers up to PB_MAX_CHUNKS_PER_LAUNCH chunks;
 *     its schedule (team warps T, units per team G, resident teams) comes
 *     from a throughput model over the topology's level widths;
 *   - the workspace (scratch pool, chunk seeds, session seed copy) is kept
 *     on the topology across calls (grown on demand) and zeroed at the end
 *     of every call, failed calls included, and before it is freed.
 */
#include "b3_host.h"
#include "dev_alloc.h"
#include "kernels.h"
#include "topology.h"

#include "gpu_label.h"
#include "pose_b200.h"

#include <nvtx3/nvToolsExt.h>
#include <cuda_runtime_api.h>
#include <math.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define PB_DEFAULT_CHUNK_BLOCKS 4096u
#define PB_MAX_CHUNKS_PER_LAUNCH (1u << 20)
#define PB_DEVICE_SEED_MAX 1016u /* seed_len + 8 must fit one BLAKE3 chunk */
#define PB_SCRATCH_MARGIN ((uint64_t)2 << 30)

static _Thread_local char g_err[512];

static void set_err(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    fprintf(stderr, "%s\n", g_err);
}

const char *pose_b200_last_error(void) { return g_err; }

void pb_set_err(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    fprintf(stderr, "%s\n", g_err);
}

static int quiet(void)
{
    const char *e = getenv("POSE_GPU_QUIET");
    return (e && e[0] && e[0] != '0') ? 1 : 0;
}

static double now_sec(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

struct pose_hbm_topo {
    int device;
    uint32_t cb;
    uint64_t super_bytes;
    uint32_t copies;
    uint32_t S, L, pool, half_w, retained, max_width;
    uint8_t desc[32];
    /* distinct level widths and how many levels have each (schedule model) */
    uint32_t nw;
    uint32_t *wval;
    uint64_t *wcnt;
    /* device schedule */
    void *d_recs, *d_cv0, *d_orank, *d_lstart, *d_recs2;
    uint64_t dev_bytes;
    pb_topo_view_t view;
    pb_topo_view2_t view2; /* pipelined records (d_recs2 != NULL) */
    int occ_ws[2];         /* warp-specialised kernel CTAs/SM for 7 and 15 hashing warps */
    /* levels wider than split_width (ascending), shared by a cluster's CTAs */
    uint32_t *d_split, nsplit, split_width;
    int occ_wsc[4];        /* clusters of 2, 4, 8, 16 CTAs (15 hashing warps) the device holds */
    /* per-topology workspace, reused across calls (one caller thread at a time) */
    cudaStream_t stream;
    cudaEvent_t ev[4];
    uint8_t *d_scratch;
    uint64_t scratch_alloc;
    uint32_t *d_seeds;
    uint64_t seeds_alloc; /* chunks */
    uint8_t *d_sess;
    size_t sess_alloc;
    unsigned int *d_queue;
    int occ_team[5], sms; /* k_label CTAs (one team of 2^i warps each) per SM */
    /* pipelined records for a PB_CSM_MULTI-slot shared pool per unit (the
     * multi-unit depth kernel's), built on first use */
    void *d_recs2s;
    pb_topo_view2_t view2s;
    pthread_mutex_t lazy_mu; /* guards the first-use build of d_recs2s / view2s */
    /* schedule chosen by pose_b200_topo_autotune for calls of tuned_units chunk copies */
    int tuned_ok;
    uint64_t tuned_units;
    pose_b200_sched_t tuned;
};

/* ── schedule model ──────────────────────────────────────────────────────── */

/* Model constants: integer lanes an SM retires per clock for this
 * instruction mix, and the dependent latency of one node label in SM clocks.
 * Defaults come from the compression microbenchmark; POSE_B200_INT_LANES and
 * POSE_B200_LABEL_LATENCY override them. */
static double model_lanes(void)
{
    const char *e = getenv("POSE_B200_INT_LANES");
    double v = e ? atof(e) : 0.0;
    return v > 0 ? v : 72.0;
}

static double model_latency(int cv0)
{
    const char *e = getenv("POSE_B200_LABEL_LATENCY");
    double v = e ? atof(e) : 0.0;
    return v > 0 ? v : (cv0 ? 6000.0 : 7000.0);
}

typedef struct {
    uint32_t T, G, teams, grid, cta, kernel, smem, fma;
    uint32_t per_sm; /* lockstep kernel: teams per SM to cap residency at (0 = no cap) */
    uint32_t cluster; /* depth kernel: CTAs per chunk copy (1 = k_label_ws, >1 = k_label_wsc) */
    uint64_t team_scratch, scratch_bytes;
    double cost;
} plan_t;

#define PB_CSM_LATENCY 2048u /* shared-memory label slots per copy in the pipelined records */
#define PB_CSM_MULTI 512u    /* the same for the multi-unit depth kernel (four pools per CTA) */
#define PB_SPLIT_WIDTH 480u  /* levels a depth-kernel cluster shares: wider than one pass of its hashing threads */

static double model_ws_latency(void)
{
    const char *e = getenv("POSE_B200_WS_LATENCY");
    double v = e ? atof(e) : 0.0;
    return v > 0 ? v : 2700.0;
}

static uint32_t ws_smem_bytes(const pose_hbm_topo_t *t, uint32_t nc)
{
    return (2u * t->view2.csm + 18u * 32u * nc + 3u) * 16u;
}

static int ws_occupancy(pose_hbm_topo_t *t, uint32_t nc)
{
    int i = nc == 7 ? 0 : 1;
    if (t->occ_ws[i] < 0) {
        int occ = 0;
        uint32_t smem = ws_smem_bytes(t, nc);
        if (smem > 227u * 1024u || pb_dev_label_ws_occupancy(32 * (nc + 1), smem, &occ) != 0) occ = 0;
        cudaGetLastError();
        t->occ_ws[i] = occ;
    }
    return t->occ_ws[i];
}

/* SM clocks a cluster barrier adds to a level (POSE_B200_CLUSTER_SYNC overrides). */
static double model_cluster_sync(void)
{
    const char *e = getenv("POSE_B200_CLUSTER_SYNC");
    double v = e ? atof(e) : 0.0;
    return v > 0 ? v : 1500.0;
}

/* Clusters of C CTAs of the depth kernel (15 hashing warps) the device holds
 * at once (0 when C is not 2, 4, 8 or 16, or the kernel cannot run so). */
static int wsc_clusters(pose_hbm_topo_t *t, uint32_t C)
{
    const int i = C == 2 ? 0 : C == 4 ? 1 : C == 8 ? 2 : C == 16 ? 3 : -1;
    if (i < 0 || !t->d_split) return 0;
    if (t->occ_wsc[i] < 0) {
        int n = 0;
        const uint32_t smem = ws_smem_bytes(t, 15);
        if (smem > 227u * 1024u || pb_dev_label_wsc_max_clusters(C, 15, smem, &n) != 0) n = 0;
        cudaGetLastError();
        t->occ_wsc[i] = n;
    }
    return t->occ_wsc[i];
}

static uint64_t passes_lanes(const pose_hbm_topo_t *t, uint64_t lanes)
{
    uint64_t passes = 0;
    for (uint32_t k = 0; k < t->nw; k++) passes += t->wcnt[k] * ((t->wval[k] + lanes - 1) / lanes);
    return passes;
}

static uint64_t passes_for(const pose_hbm_topo_t *t, uint32_t T, uint32_t G)
{
    uint64_t lanes = 32ull * T, passes = 0;
    for (uint32_t k = 0; k < t->nw; k++) {
        uint64_t items = (uint64_t)G * t->wval[k];
        passes += t->wcnt[k] * ((items + lanes - 1) / lanes);
    }
    return passes;
}

static int is_pow2(uint32_t v) { return v && !(v & (v - 1)); }

/* One-warp passes of a batch of G units: sum over levels of ceil(G w / 32).
 * Warps without a node of a level skip it, so this is the batch's ALU work
 * in warp-wide node hashes, idle lanes of partly filled warps included. */
static uint64_t warp_passes(const pose_hbm_topo_t *t, uint32_t G)
{
    uint64_t passes = 0;
    for (uint32_t k = 0; k < t->nw; k++) passes += t->wcnt[k] * (((uint64_t)G * t->wval[k] + 31) / 32);
    return passes;
}

/* Throughput model of one launch.  A team's batch takes at least its
 * latency-bound time (every pass of every level waits for a label: t_lat per
 * pass for the basic kernel; the depth kernel's levels cost its per-level
 * time, further passes of a wide level t_lat), and an SM needs at least its
 * ALU time (the warp passes of the teams resident on it, 32 lanes each, at
 * lanes_clk lane-operations per clock).  A launch runs its full waves of the
 * larger of the two, then the rest of the batches spread over the SMs. */
static int make_plan(const pose_hbm_topo_t *ct, uint64_t nunits, const pose_b200_sched_t *hint,
                     uint64_t budget, plan_t *best)
{
    pose_hbm_topo_t *t = (pose_hbm_topo_t *)ct; /* occupancy cache */
    const double lanes_clk = model_lanes();
    const double t_lat = model_latency(t->d_cv0 != NULL);
    const double item_instr = t->d_cv0 ? 1400.0 : 2080.0;
    const int want = hint ? (int)hint->kernel : 0;
    memset(best, 0, sizeof(*best));
    best->cost = -1;
    for (int kernel = 1; kernel <= 1; kernel++) {
        if (want && want != kernel) continue;
        /* One team per CTA (its barrier is the CTA's, so a CTA reserves one
         * hardware barrier and the SM's barriers never cap residency), so
         * that any number k of teams per SM can be resident.  Teams pull
         * batches until the queue is empty, and a batch's time is set by
         * the ALU share of its SM.  Every k is costed; a k below the
         * occupancy limit is enforced by padding the CTA's shared memory
         * (pb_dev_label_balance_smem), so that no SM takes k + 1. */
        const char *fk = getenv("POSE_B200_TEAMS_PER_SM"); /* forces k (tests, sweeps) */
        const int force_k = fk ? atoi(fk) : 0;
        for (uint32_t T = 1, ti = 0; T <= 16; T <<= 1, ti++) {
            if (hint && hint->team_warps && hint->team_warps != T) continue;
            const uint32_t cta = 32 * T;
            const int occ = t->occ_team[ti];
            if (occ <= 0) continue;
            for (uint32_t G = 1; G <= 32 && G <= 32 * T; G <<= 1) {
                if (hint && hint->units_per_team && hint->units_per_team != G) continue;
                uint64_t slots = t->pool;
                uint64_t team_scratch = (uint64_t)G * slots * 32;
                uint64_t batches = (nunits + G - 1) / G;
                uint64_t memcap = budget / team_scratch;
                uint64_t passes = passes_for(t, T, G);
                double lat = (double)passes * t_lat;
                /* one batch's ALU clocks on an SM of its own: its warp passes
                 * of 32 lanes, idle lanes included */
                const double alu1 = (double)warp_passes(t, G) * 32.0 * item_instr / lanes_clk;
                for (int k = occ; k >= 1; k--) {
                    if (force_k && k != force_k) continue;
                    uint64_t R = (uint64_t)t->sms * (uint64_t)k;
                    if (R > memcap) R = memcap;
                    if (R > batches) R = batches;
                    if (hint && hint->max_teams && R > hint->max_teams) R = hint->max_teams;
                    if (R == 0) continue;
                    uint64_t sbytes = R * team_scratch;
                    if (sbytes > budget) continue;
                    /* full waves of R teams, then the rest, spread over the SMs */
                    const uint64_t full = batches / R, rest = batches - full * R;
                    const uint64_t teams_sm = (R + t->sms - 1) / t->sms, rest_sm = (rest + t->sms - 1) / t->sms;
                    const double alu = (double)teams_sm * alu1, alu_rest = (double)rest_sm * alu1;
                    double cost = (double)full * (lat > alu ? lat : alu);
                    if (rest) cost += lat > alu_rest ? lat : alu_rest;
                    if (best->cost < 0 || cost < best->cost * 0.999 ||
                        (cost <= best->cost * 1.001 && sbytes < best->scratch_bytes)) {
                        best->T = T; best->G = G; best->teams = (uint32_t)R;
                        best->grid = (uint32_t)R; best->cta = cta;
                        best->team_scratch = team_scratch; best->scratch_bytes = sbytes;
                        best->cost = cost; best->kernel = (uint32_t)kernel;
                        /* residency cap when fewer than the occupancy limit
                         * of teams go on every SM */
                        best->smem = 0;
                        best->per_sm = R % t->sms == 0 && R / t->sms < (uint64_t)occ ? (uint32_t)(R / t->sms) : 0;
                        best->fma = kernel == 1 && alu >= lat; /* ALU-bound: move adds to the FMA pipe */
                    }
                }
            }
        }
    }
    /* warp-specialised kernel with a cluster of C CTAs per chunk copy: one
     * wave of nunits clusters, the levels wider than split_width shared by
     * the cluster (their extra passes divided by C, two cluster barriers
     * each at most) */
    for (uint32_t C = 2; C <= 16 && t->d_split && (!want || want == 3); C <<= 1) {
        const uint32_t nc = 15;
        if (hint && hint->team_warps && hint->team_warps != nc) continue;
        if (hint && hint->units_per_team > 1) continue;
        if (hint && hint->cluster_ctas && hint->cluster_ctas != C) continue;
        if (!(hint && hint->cluster_ctas == C) && C > 8) continue; /* 16 only on request */
        const int ncl = wsc_clusters(t, C);
        if (ncl <= 0 || nunits > (uint64_t)ncl) continue;
        if (hint && hint->max_teams && nunits > hint->max_teams) continue;
        uint64_t team_scratch = (uint64_t)(t->view2.gpool ? t->view2.gpool : 1) * 32;
        uint64_t sbytes = nunits * team_scratch;
        if (sbytes > budget) continue;
        uint64_t passes = passes_lanes(t, 32ull * nc);
        /* the cluster form runs every level ~250 clocks slower than the
         * one-CTA kernel (measured at 2^17: 742 ms against 693 ms with only
         * 169 shared levels), so it pays only where wide levels dominate */
        double lat = (double)t->L * (model_ws_latency() + 250.0) + (double)(passes - t->L) * t_lat / C +
                     2.0 * t->nsplit * model_cluster_sync();
        double cost = lat;
        if (best->cost < 0 || cost < best->cost * 0.999) {
            best->T = nc; best->G = 1; best->teams = (uint32_t)nunits;
            best->grid = (uint32_t)(nunits * C); best->cta = 32 * (nc + 1);
            best->team_scratch = team_scratch; best->scratch_bytes = sbytes;
            best->cost = cost; best->kernel = 3; best->smem = ws_smem_bytes(t, nc); best->fma = 0;
            best->per_sm = 0;
            best->cluster = C;
        }
    }
    /* warp-specialised kernel: one chunk copy per CTA, NC hashing warps */
    for (uint32_t nc = 7; nc <= 15 && t->d_recs2 && (!want || want == 3); nc += 8) {
        if (hint && hint->team_warps && hint->team_warps != nc) continue;
        if (hint && hint->units_per_team > 1) continue;
        if (hint && hint->cluster_ctas > 1) continue;
        int occ = ws_occupancy(t, nc);
        if (occ <= 0) continue;
        uint64_t team_scratch = (uint64_t)(t->view2.gpool ? t->view2.gpool : 1) * 32;
        uint64_t batches = nunits;
        uint64_t cap = (uint64_t)t->sms * occ;
        uint64_t memcap = budget / team_scratch;
        uint64_t R = cap < memcap ? cap : memcap;
        if (R > batches) R = batches;
        if (hint && hint->max_teams && R > hint->max_teams) R = hint->max_teams;
        if (R == 0) continue;
        uint64_t waves = (batches + R - 1) / R;
        uint64_t passes = passes_lanes(t, 32ull * nc);
        double lat = (double)t->L * model_ws_latency() + (double)(passes - t->L) * t_lat;
        double teams_sm = (double)((R + t->sms - 1) / t->sms);
        double alu = teams_sm * (double)t->S * item_instr / lanes_clk;
        double cost = (double)waves * (lat > alu ? lat : alu);
        uint64_t sbytes = R * team_scratch;
        if (sbytes > budget) continue;
        if (best->cost < 0 || cost < best->cost * 0.999) {
            best->T = nc; best->G = 1; best->teams = (uint32_t)R;
            best->grid = (uint32_t)R; best->cta = 32 * (nc + 1);
            best->team_scratch = team_scratch; best->scratch_bytes = sbytes;
            best->cost = cost; best->kernel = 3; best->smem = ws_smem_bytes(t, nc); best->fma = 0;
            best->per_sm = 0;
            best->cluster = 1;
        }
    }
    return best->cost < 0 ? -1 : 0;
}

/* ── helpers ─────────────────────────────────────────────────────────────── */

#define CK(call, what)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            set_err("pose_b200: %s: CUDA error: %s", what, cudaGetErrorString(e_));      \
            goto fail;                                                                   \
        }                                                                                \
    } while (0)

static pthread_mutex_t g_fail_mu = PTHREAD_MUTEX_INITIALIZER;
static char g_fail_seen[32];
static long g_fail_left;

cudaError_t pb_dev_malloc(void **ptr, size_t bytes)
{
    const char *e = getenv("POSE_B200_FAIL_ALLOC");
    pthread_mutex_lock(&g_fail_mu);
    if (!e) e = "";
    if (strncmp(e, g_fail_seen, sizeof(g_fail_seen) - 1) != 0) {
        snprintf(g_fail_seen, sizeof(g_fail_seen), "%s", e);
        g_fail_left = atol(e);
    }
    const int fail = g_fail_left > 0;
    if (fail) g_fail_left--;
    pthread_mutex_unlock(&g_fail_mu);
    if (fail) {
        *ptr = NULL;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(ptr, bytes);
}

static _Thread_local cudaError_t g_last_alloc_err; /* this thread's last failed grow() */

static int grow(void **p, uint64_t *have, uint64_t need, size_t elem)
{
    if (*have >= need) return 0;
    if (*p) cudaFree(*p);
    *p = NULL;
    *have = 0;
    const cudaError_t e = pb_dev_malloc(p, need * elem);
    if (e != cudaSuccess) { *p = NULL; g_last_alloc_err = e; return -1; }
    *have = need;
    return 0;
}

/* Zero the whole workspace (scratch labels, chunk seeds, the session seed),
 * best effort: after a failed call the context may refuse the memsets, and
 * then there is nothing more a host can do. */
static void wipe_workspace(pose_hbm_topo_t *t)
{
    if (t->d_scratch) cudaMemsetAsync(t->d_scratch, 0, t->scratch_alloc, t->stream);
    if (t->d_seeds) cudaMemsetAsync(t->d_seeds, 0, t->seeds_alloc * 32, t->stream);
    if (t->d_sess) cudaMemsetAsync(t->d_sess, 0, t->sess_alloc, t->stream);
    cudaStreamSynchronize(t->stream);
    cudaGetLastError();
}

static void free_workspace(pose_hbm_topo_t *t)
{
    wipe_workspace(t);
    cudaFree(t->d_scratch);
    t->d_scratch = NULL;
    t->scratch_alloc = 0;
    cudaFree(t->d_seeds);
    t->d_seeds = NULL;
    t->seeds_alloc = 0;
    cudaFree(t->d_sess);
    t->d_sess = NULL;
    t->sess_alloc = 0;
}

/* ── build / free ────────────────────────────────────────────────────────── */

void pose_graph_hbm_topo_free(pose_hbm_topo_t *t)
{
    if (!t) return;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != t->device) cudaSetDevice(t->device);
    if (t->stream) free_workspace(t);
    cudaFree(t->d_recs);
    cudaFree(t->d_recs2);
    cudaFree(t->d_recs2s);
    cudaFree(t->d_split);
    cudaFree(t->d_cv0);
    cudaFree(t->d_orank);
    cudaFree(t->d_lstart);
    cudaFree(t->d_queue);
    for (int i = 0; i < 4; i++) if (t->ev[i]) cudaEventDestroy(t->ev[i]);
    if (t->stream) cudaStreamDestroy(t->stream);
    if (prev >= 0 && prev != t->device) cudaSetDevice(prev);
    free(t->wval);
    free(t->wcnt);
    pthread_mutex_destroy(&t->lazy_mu);
    free(t);
}

static int cmp_u32(const void *a, const void *b)
{
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}

static pose_hbm_topo_t *pose_b200_topo_build_impl(uint32_t chunk_blocks, int with_cv0_table)
{
    uint32_t cb = chunk_blocks ? chunk_blocks : PB_DEFAULT_CHUNK_BLOCKS;
    if (cb > PB_MAX_CHUNK_BLOCKS) {
        set_err("pose_graph_hbm_topo_build: chunk_blocks %u out of range [1, %u]", cb,
                PB_MAX_CHUNK_BLOCKS);
        return NULL;
    }
    pb_topo_host_t h;
    if (pb_topo_host_build_ex(cb, with_cv0_table ? PB_CSM_LATENCY : 0, &h) != 0) {
        set_err("pose_graph_hbm_topo_build: schedule build failed for chunk_blocks %u", cb);
        return NULL;
    }
    pose_hbm_topo_t *t = (pose_hbm_topo_t *)calloc(1, sizeof(*t));
    uint32_t *ws = NULL;
    if (!t) { set_err("pose_graph_hbm_topo_build: out of host memory"); goto fail_host; }
    pthread_mutex_init(&t->lazy_mu, NULL);
    cudaGetDevice(&t->device);
    t->cb = cb;
    t->super_bytes = (uint64_t)cb * 32;
    t->copies = h.retained ? 2 : 1;
    t->S = h.S; t->L = h.L; t->pool = h.pool; t->half_w = h.half_w;
    t->retained = h.retained; t->max_width = h.max_width;
    memcpy(t->desc, h.desc, 32);

    /* width histogram */
    ws = (uint32_t *)malloc((size_t)h.L * 4);
    if (!ws) { set_err("pose_graph_hbm_topo_build: out of host memory"); goto fail_host; }
    for (uint32_t l = 0; l < h.L; l++) ws[l] = h.lstart[l + 1] - h.lstart[l];
    qsort(ws, h.L, 4, cmp_u32);
    t->wval = (uint32_t *)malloc((size_t)h.L * 4);
    t->wcnt = (uint64_t *)malloc((size_t)h.L * 8);
    if (!t->wval || !t->wcnt) { set_err("pose_graph_hbm_topo_build: out of host memory"); goto fail_host; }
    for (uint32_t l = 0; l < h.L; l++) {
        if (t->nw && t->wval[t->nw - 1] == ws[l]) t->wcnt[t->nw - 1]++;
        else { t->wval[t->nw] = ws[l]; t->wcnt[t->nw] = 1; t->nw++; }
    }
    free(ws);
    ws = NULL;

    {
        CK(cudaStreamCreate(&t->stream), "stream");
        for (int i = 0; i < 4; i++) CK(cudaEventCreate(&t->ev[i]), "event");
        CK(pb_dev_malloc(&t->d_recs, (size_t)h.S * 16), "topology records");
        CK(pb_dev_malloc(&t->d_orank, (size_t)h.S * 4), "output ranks");
        CK(pb_dev_malloc(&t->d_lstart, ((size_t)h.L + 1) * 4), "level offsets");
        CK(pb_dev_malloc((void **)&t->d_queue, 64), "work counter");
        t->dev_bytes = (uint64_t)h.S * 20 + ((uint64_t)h.L + 1) * 4;
        CK(cudaMemcpyAsync(t->d_recs, h.recs, (size_t)h.S * 16, cudaMemcpyHostToDevice, t->stream),
           "upload records");
        CK(cudaMemcpyAsync(t->d_orank, h.orank, (size_t)h.S * 4, cudaMemcpyHostToDevice, t->stream),
           "upload ranks");
        CK(cudaMemcpyAsync(t->d_lstart, h.lstart, ((size_t)h.L + 1) * 4, cudaMemcpyHostToDevice,
                           t->stream),
           "upload levels");
        uint32_t ksrc[8], kint[8], kseed[8];
        pb_label_keys(ksrc, kint);
        pb_context_key("pose-db/chunk-seed", kseed);
        if (pb_dev_set_keys(ksrc, kint, kseed) != 0) {
            set_err("pose_graph_hbm_topo_build: key upload failed");
            goto fail;
        }
        if (with_cv0_table && h.recs2) {
            CK(pb_dev_malloc(&t->d_recs2, (size_t)h.S * 32), "pipelined records");
            CK(cudaMemcpyAsync(t->d_recs2, h.recs2, (size_t)h.S * 32, cudaMemcpyHostToDevice, t->stream),
               "upload pipelined records");
            t->dev_bytes += (uint64_t)h.S * 32;
        }
        if (with_cv0_table) {
            uint64_t bytes = (uint64_t)t->copies * h.S * 32;
            CK(pb_dev_malloc(&t->d_cv0, bytes), "block-0 table");
            t->dev_bytes += bytes;
            if (pb_dev_cv0_table(t->d_recs, h.S, t->copies, t->d_cv0, t->stream) != 0) {
                set_err("pose_graph_hbm_topo_build: block-0 table kernel failed");
                goto fail;
            }
        }
        CK(cudaStreamSynchronize(t->stream), "build");
        for (int i = 0; i < 5; i++)
            if (pb_dev_label_occupancy(32u << i, &t->occ_team[i]) != 0) {
                set_err("pose_graph_hbm_topo_build: occupancy query failed");
                goto fail;
            }
        CK(cudaDeviceGetAttribute(&t->sms, cudaDevAttrMultiProcessorCount, t->device), "SM count");
        t->view.recs = (const pb_u4 *)t->d_recs;
        t->view.cv0 = (const pb_u4 *)t->d_cv0;
        t->view.orank = (const uint32_t *)t->d_orank;
        t->view.lstart = (const uint32_t *)t->d_lstart;
        t->view.S = h.S; t->view.L = h.L; t->view.pool = h.pool;
        t->view.half_w = h.half_w; t->view.retained = h.retained;
        for (int i = 0; i < 8; i++)
            t->view.desc[i] = (uint32_t)h.desc[4 * i] | ((uint32_t)h.desc[4 * i + 1] << 8) |
                              ((uint32_t)h.desc[4 * i + 2] << 16) | ((uint32_t)h.desc[4 * i + 3] << 24);
        t->view2.recs2 = (const pb_u4 *)t->d_recs2;
        t->view2.cv0 = (const pb_u4 *)t->d_cv0;
        t->view2.lstart = (const uint32_t *)t->d_lstart;
        t->view2.S = h.S; t->view2.L = h.L; t->view2.half_w = h.half_w;
        t->view2.retained = h.retained; t->view2.csm = h.csm; t->view2.gpool = h.gpool2;
        memcpy(t->view2.desc, t->view.desc, sizeof(t->view2.desc));
        memset(t->occ_ws, 0xFF, sizeof(t->occ_ws));
        memset(t->occ_wsc, 0xFF, sizeof(t->occ_wsc));
        if (t->d_recs2) {
            /* the levels a cluster of the depth kernel shares: wider than
             * split_width (POSE_B200_SPLIT_WIDTH overrides the default, the
             * depth kernel's hashing threads) */
            const char *e = getenv("POSE_B200_SPLIT_WIDTH");
            t->split_width = e && e[0] ? (uint32_t)strtoul(e, NULL, 10) : PB_SPLIT_WIDTH;
            uint32_t n = 0;
            for (uint32_t l = 0; l < h.L; l++) n += h.lstart[l + 1] - h.lstart[l] > t->split_width;
            if (n) {
                uint32_t *hs = (uint32_t *)malloc((size_t)n * 4);
                if (!hs) { set_err("pose_graph_hbm_topo_build: out of host memory"); goto fail; }
                n = 0;
                for (uint32_t l = 0; l < h.L; l++)
                    if (h.lstart[l + 1] - h.lstart[l] > t->split_width) hs[n++] = l;
                cudaError_t e1 = pb_dev_malloc((void **)&t->d_split, (size_t)n * 4);
                if (e1 == cudaSuccess) e1 = cudaMemcpy(t->d_split, hs, (size_t)n * 4, cudaMemcpyHostToDevice);
                free(hs);
                CK(e1, "split levels");
                t->nsplit = n;
                t->dev_bytes += (uint64_t)n * 4;
            }
        }
    }
    pb_topo_host_free(&h);
    return t;

fail:
    pb_topo_host_free(&h);
    pose_graph_hbm_topo_free(t);
    return NULL;
fail_host:
    free(ws);
    pb_topo_host_free(&h);
    if (t) { free(t->wval); free(t->wcnt); pthread_mutex_destroy(&t->lazy_mu); free(t); }
    return NULL;
}

pose_hbm_topo_t *pose_b200_topo_build(uint32_t chunk_blocks, int with_cv0_table)
{
    nvtxRangePushA("pose_b200: topology build");
    pose_hbm_topo_t *rc = pose_b200_topo_build_impl(chunk_blocks, with_cv0_table);
    nvtxRangePop();
    return rc;
}

pose_hbm_topo_t *pose_graph_hbm_topo_build(uint32_t chunk_blocks, pose_hash_algo_t algo)
{
    if (algo != POSE_HASH_BLAKE3) {
        set_err("pose_graph_hbm_topo_build: only BLAKE3 supported on GPU");
        return NULL;
    }
    return pose_b200_topo_build(chunk_blocks, 1);
}

void pose_b200_topo_info(const pose_hbm_topo_t *t, uint32_t *chunk_blocks, uint64_t *nodes_per_chunk,
                         uint32_t *levels, uint32_t *pool_slots, uint64_t *device_bytes)
{
    if (!t) return;
    if (chunk_blocks) *chunk_blocks = t->cb;
    if (nodes_per_chunk) *nodes_per_chunk = 2ull * t->S;
    if (levels) *levels = t->L;
    if (pool_slots) *pool_slots = t->pool;
    if (device_bytes) *device_bytes = t->dev_bytes;
}

/* ── labeling ────────────────────────────────────────────────────────────── */

static uint64_t scratch_budget(const pose_hbm_topo_t *t, const pose_b200_sched_t *s)
{
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    uint64_t avail = (uint64_t)fr + t->scratch_alloc;
    avail = avail > PB_SCRATCH_MARGIN ? avail - PB_SCRATCH_MARGIN : avail / 2;
    if (s && s->scratch_cap_bytes && s->scratch_cap_bytes < avail) avail = s->scratch_cap_bytes;
    return avail;
}

int pose_b200_plan(const pose_hbm_topo_t *t, uint64_t super_chunks, const pose_b200_sched_t *hint,
                   pose_b200_sched_t *out)
{
    if (!t || !out) return -1;
    uint64_t chunks = super_chunks < PB_MAX_CHUNKS_PER_LAUNCH ? super_chunks : PB_MAX_CHUNKS_PER_LAUNCH;
    plan_t p;
    if (chunks == 0 || make_plan(t, chunks * t->copies, hint, scratch_budget(t, hint), &p) != 0)
        return -1;
    memset(out, 0, sizeof(*out));
    out->team_warps = p.T;
    out->units_per_team = p.G;
    out->max_teams = p.teams;
    out->kernel = p.kernel;
    out->scratch_cap_bytes = p.scratch_bytes;
    out->cluster_ctas = p.kernel == 3 ? p.cluster : 0;
    return 0;
}

static int topo_label_core(const pose_hbm_topo_t *ct, const uint8_t *session_seed, size_t seed_len,
                           const uint8_t *raw_seeds, void *hbm_dev_ptr, size_t hbm_len, uint64_t rbo,
                           const pose_b200_sched_t *sched, pose_b200_stats_t *stats);

/* Candidates of the autotuner: every (team size, units per team) of the
 * basic kernel, and the depth kernel, as planned by the schedule model;
 * group g = team size (0 = the depth kernel), cost = modelled cost. */
#define PB_TUNE_MAX 40
typedef struct {
    pose_b200_sched_t s;
    double cost;
    uint32_t group;
} tune_cand_t;

static int autotune_candidates(pose_hbm_topo_t *t, uint64_t nunits, uint64_t budget, tune_cand_t *c)
{
    int n = 0;
    for (uint32_t T = 1; T <= 16; T <<= 1)
        for (uint32_t G = 1; G <= 32 && n < PB_TUNE_MAX - 1; G <<= 1) {
            pose_b200_sched_t h;
            memset(&h, 0, sizeof(h));
            h.kernel = 1; h.team_warps = T; h.units_per_team = G;
            plan_t p;
            if (make_plan(t, nunits, &h, budget, &p) != 0) continue;
            memset(&c[n], 0, sizeof(c[n]));
            c[n].s.kernel = 1; c[n].s.team_warps = p.T; c[n].s.units_per_team = p.G; c[n].s.max_teams = p.teams;
            c[n].cost = p.cost; c[n].group = T; n++;
        }
    /* the depth kernel alone and with a cluster of 2, 4 or 8 CTAs per copy */
    for (uint32_t cl = 1; cl <= 8 && n < PB_TUNE_MAX; cl <<= 1) {
        pose_b200_sched_t h;
        memset(&h, 0, sizeof(h));
        h.kernel = 3;
        h.cluster_ctas = cl;
        plan_t p;
        if (make_plan(t, nunits, &h, budget, &p) != 0) continue;
        memset(&c[n], 0, sizeof(c[n]));
        c[n].s.kernel = 3; c[n].s.team_warps = p.T; c[n].s.units_per_team = 1; c[n].s.max_teams = p.teams;
        c[n].s.cluster_ctas = p.cluster;
        c[n].cost = p.cost; c[n].group = 0; n++;
    }
    /* by modelled cost */
    for (int i = 1; i < n; i++) {
        tune_cand_t v = c[i];
        int j = i;
        while (j > 0 && c[j - 1].cost > v.cost) { c[j] = c[j - 1]; j--; }
        c[j] = v;
    }
    return n;
}

int pose_b200_topo_autotune(pose_hbm_topo_t *t, const uint8_t *session_seed, size_t seed_len, void *hbm_dev_ptr,
                            size_t hbm_len, uint64_t region_block_offset, uint32_t trials,
                            pose_b200_sched_t *chosen, pose_b200_stats_t *stats)
{
    if (stats) memset(stats, 0, sizeof(*stats));
    if (!t) { set_err("pose_b200_topo_autotune: NULL topology"); return -1; }
    const uint64_t num_super = hbm_len / t->super_bytes;
    if (num_super == 0) { set_err("pose_b200_topo_autotune: buffer smaller than one super-chunk"); return -1; }
    const uint64_t per_launch = num_super < PB_MAX_CHUNKS_PER_LAUNCH ? num_super : PB_MAX_CHUNKS_PER_LAUNCH;
    const uint64_t nunits = per_launch * t->copies;
    tune_cand_t c[PB_TUNE_MAX];
    int tried[PB_TUNE_MAX];
    t->tuned_ok = 0;
    const int n = autotune_candidates(t, nunits, scratch_budget(t, NULL), c);
    if (n <= 0) { set_err("pose_b200_topo_autotune: no schedule fits the scratch budget"); return -1; }
    memset(tried, 0, sizeof(tried));
    int budget_trials = (int)(trials == 0 ? 4u : trials);
    int best = -1;
    pose_b200_stats_t bst;
    memset(&bst, 0, sizeof(bst));
    /* stage 1: the cheapest candidate of each group (team size or the depth
     * kernel), cheapest first; stage 2: the other candidates of the winning
     * group, cheapest first, with the trials left */
    for (int stage = 0; stage < 2 && budget_trials > 0; stage++) {
        uint32_t seen = 0; /* bit per group in stage 1 */
        const uint32_t win = best >= 0 ? c[best].group : 0xFFFFFFFFu;
        for (int i = 0; i < n && budget_trials > 0; i++) {
            if (tried[i]) continue;
            if (c[i].cost > 2.0 * c[0].cost) break; /* the model is good to well within 2x */
            if (stage == 0) {
                const uint32_t bit = 1u << (c[i].group ? __builtin_ctz(c[i].group) + 1 : 0);
                if (seen & bit) continue;
                seen |= bit;
            } else if (c[i].group != win) {
                continue;
            }
            tried[i] = 1;
            budget_trials--;
            pose_b200_stats_t st;
            if (topo_label_core(t, session_seed, seed_len, NULL, hbm_dev_ptr, hbm_len, region_block_offset,
                                &c[i].s, &st) != 0)
                continue;
            if (best < 0 || st.total_ms < bst.total_ms) { best = i; bst = st; }
        }
    }
    if (best < 0) return -1; /* the error of the last trial is kept */
    t->tuned = c[best].s;
    t->tuned_units = nunits;
    t->tuned_ok = 1;
    if (chosen) *chosen = c[best].s;
    if (stats) *stats = bst;
    /* the buffer holds the labels of the last trial: every trial writes the same bytes */
    return 0;
}

/* The labeling call.  Chunk seeds come either from the session seed (derived
 * per super-chunk from its absolute position), or, when raw_seeds is set, are
 * taken as given: raw_seeds holds 32 bytes per super-chunk of the buffer. */
static int topo_label_core_impl(const pose_hbm_topo_t *ct, const uint8_t *session_seed, size_t seed_len,
                           const uint8_t *raw_seeds, void *hbm_dev_ptr, size_t hbm_len, uint64_t rbo,
                           const pose_b200_sched_t *sched, pose_b200_stats_t *stats)
{
    pose_hbm_topo_t *t = (pose_hbm_topo_t *)ct; /* workspace is mutable state */
    if (stats) memset(stats, 0, sizeof(*stats));
    if (!t) { set_err("pose_graph_hbm_topo_label: NULL topology"); return -1; }
    uint64_t num_super = hbm_len / t->super_bytes;
    if (num_super == 0) return 0; /* smaller than one super-chunk: nothing to label */
    if (!hbm_dev_ptr) { set_err("pose_graph_hbm_topo_label: NULL buffer"); return -1; }
    if (!raw_seeds && !session_seed && seed_len) { set_err("pose_graph_hbm_topo_label: NULL seed"); return -1; }
    if (sched && sched->kernel != 0 && sched->kernel != 1 && sched->kernel != 3) {
        set_err("pose_b200_topo_label: kernel %u is not one of 0 (automatic), 1 (lockstep) and 3 (depth)",
                sched->kernel);
        return -1;
    }
    if (sched && sched->kernel == 3 && sched->team_warps && sched->team_warps != 7 && sched->team_warps != 15) {
        set_err("pose_b200_topo_label: the warp-specialised kernel takes 7 or 15 hashing warps");
        return -1;
    }
    if (sched && sched->kernel != 3 && ((sched->team_warps && (!is_pow2(sched->team_warps) || sched->team_warps > 16)) ||
                  (sched->units_per_team &&
                   (!is_pow2(sched->units_per_team) || sched->units_per_team > 32)))) {
        set_err("pose_b200_topo_label: schedule must use powers of two (T <= 16, G <= 32)");
        return -1;
    }
    if (sched && sched->cluster_ctas > 1 &&
        ((sched->kernel != 0 && sched->kernel != 3) || !is_pow2(sched->cluster_ctas) || sched->cluster_ctas > 16)) {
        set_err("pose_b200_topo_label: cluster_ctas must be 0, 1, 2, 4, 8 or 16, with the depth kernel");
        return -1;
    }
    if (sched && sched->kernel > 3) {
        set_err("pose_b200_topo_label: kernel must be 0 (automatic), 1, 2 or 3");
        return -1;
    }
    int prev = -1, rc = -1;
    uint32_t *h_seeds = NULL;
    cudaGetDevice(&prev);
    if (prev != t->device && cudaSetDevice(t->device) != cudaSuccess) {
        set_err("pose_graph_hbm_topo_label: cannot select the topology's device");
        return -1;
    }

    const uint64_t per_launch = num_super < PB_MAX_CHUNKS_PER_LAUNCH ? num_super : PB_MAX_CHUNKS_PER_LAUNCH;
    plan_t plan;
    if (!sched && t->tuned_ok && t->tuned_units == per_launch * t->copies) sched = &t->tuned;
    uint64_t budget = scratch_budget(t, sched);
    if (make_plan(t, per_launch * t->copies, sched, budget, &plan) != 0) {
        set_err("pose_graph_hbm_topo_label: no schedule fits the scratch budget "
                "(one copy needs %llu bytes)", (unsigned long long)t->pool * 32ull);
        goto out;
    }
    /* scratch: when the allocation fails, halve the budget and re-plan, down
     * to a single team, as the reference halves its chunk batch on an
     * allocation failure (common/src/cuda/label_gpu_warp.cu:165-175) */
    while (grow((void **)&t->d_scratch, &t->scratch_alloc, plan.scratch_bytes, 1) != 0) {
        cudaGetLastError();
        if (plan.scratch_bytes <= plan.team_scratch || plan.teams <= 1) {
            set_err("pose_graph_hbm_topo_label: scratch alloc of %llu bytes failed: %s",
                    (unsigned long long)plan.scratch_bytes, cudaGetErrorString(g_last_alloc_err));
            goto out;
        }
        budget = plan.scratch_bytes / 2;
        if (budget < plan.team_scratch) budget = plan.team_scratch;
        if (make_plan(t, per_launch * t->copies, sched, budget, &plan) != 0) {
            set_err("pose_graph_hbm_topo_label: no schedule fits %llu bytes of scratch",
                    (unsigned long long)budget);
            goto out;
        }
    }
    if (!quiet()) {
        printf("  GPU label: strategy=b200  %llu super-chunks  scaffold=%llu nodes  "
               "T=%u G=%u teams=%u\n",
               (unsigned long long)num_super, 2ull * t->S, plan.T, plan.G, plan.teams);
        fflush(stdout);
    }
    {
        double t0 = now_sec();
        if (grow((void **)&t->d_seeds, &t->seeds_alloc, per_launch, 32) != 0) {
            set_err("pose_graph_hbm_topo_label: seed buffer alloc failed");
            goto out;
        }
        const int dev_seeds = !raw_seeds && seed_len <= PB_DEVICE_SEED_MAX;
        if (dev_seeds && seed_len) {
            uint64_t have = t->sess_alloc;
            if (grow((void **)&t->d_sess, &have, seed_len, 1) != 0) {
                set_err("pose_graph_hbm_topo_label: seed alloc failed");
                goto out;
            }
            t->sess_alloc = (size_t)have;
            CK(cudaMemcpyAsync(t->d_sess, session_seed, seed_len, cudaMemcpyHostToDevice, t->stream),
               "seed upload");
        }
        CK(cudaEventRecord(t->ev[0], t->stream), "event");
        float kms = 0;
        uint32_t launches = 0;
        for (uint64_t first = 0; first < num_super; first += per_launch) {
            uint64_t n = num_super - first < per_launch ? num_super - first : per_launch;
            if (raw_seeds) {
                CK(cudaMemcpyAsync(t->d_seeds, raw_seeds + 32 * first, n * 32, cudaMemcpyHostToDevice, t->stream),
                   "seed upload");
                CK(cudaStreamSynchronize(t->stream), "seed upload");
            } else if (dev_seeds) {
                if (pb_dev_chunk_seeds(t->d_sess, (uint32_t)seed_len, rbo, t->cb, (uint32_t)n, first,
                                       t->d_seeds, t->stream) != 0) {
                    set_err("pose_graph_hbm_topo_label: chunk-seed kernel failed");
                    goto out;
                }
            } else {
                /* long session seeds: derive on the host */
                if (!h_seeds) h_seeds = (uint32_t *)malloc(per_launch * 32);
                if (!h_seeds) { set_err("pose_graph_hbm_topo_label: out of host memory"); goto out; }
                for (uint64_t j = 0; j < n; j++) {
                    uint8_t cs[32];
                    pb_chunk_seed(cs, session_seed, seed_len, (rbo + (first + j) * (uint64_t)t->cb) / t->cb);
                    memcpy(h_seeds + 8 * j, cs, 32);
                }
                CK(cudaMemcpyAsync(t->d_seeds, h_seeds, n * 32, cudaMemcpyHostToDevice, t->stream),
                   "seed upload");
                CK(cudaStreamSynchronize(t->stream), "seed upload");
            }
            CK(cudaMemsetAsync(t->d_queue, 0, 64, t->stream), "queue reset");
            pb_label_params_t p;
            memset(&p, 0, sizeof(p));
            p.topo = t->view;
            p.seeds = t->d_seeds;
            p.persist = (uint8_t *)hbm_dev_ptr;
            p.super_bytes = t->super_bytes;
            p.first_super = first;
            p.scratch = t->d_scratch;
            p.team_scratch_bytes = plan.team_scratch;
            p.nunits = (uint32_t)(n * t->copies);
            p.copies_log2 = t->copies == 2 ? 1 : 0;
            p.g_log2 = (uint32_t)__builtin_ctz(plan.G);
            p.team_warps = plan.T;
            p.nbatches = (uint32_t)((p.nunits + plan.G - 1) / plan.G);
            p.queue = t->d_queue;
            p.fma_adds = plan.fma;
            p.one = 1;
            { const char *e = getenv("POSE_B200_FMA_ADDS"); if (e && e[0]) p.fma_adds = (uint32_t)atoi(e); }
            CK(cudaEventRecord(t->ev[1], t->stream), "event");
            int lrc;
            if (plan.kernel == 3) {
                pb_pipe_params_t pp;
                memset(&pp, 0, sizeof(pp));
                pp.topo = t->view2;
                pp.seeds = p.seeds; pp.persist = p.persist; pp.super_bytes = p.super_bytes;
                pp.first_super = p.first_super; pp.scratch = p.scratch;
                pp.team_scratch_bytes = plan.team_scratch; pp.nunits = p.nunits;
                pp.copies_log2 = p.copies_log2; pp.g_log2 = p.g_log2; pp.team_warps = p.team_warps;
                pp.nbatches = p.nbatches; pp.queue = p.queue;
                if (plan.cluster > 1) {
                    pp.cluster = plan.cluster;
                    pp.split_width = t->split_width;
                    pp.split_levels = t->d_split;
                    pp.nsplit = t->nsplit;
                    lrc = pb_dev_label_wsc(&pp, plan.smem, t->stream);
                } else {
                    lrc = pb_dev_label_ws(&pp, plan.grid, plan.cta, plan.smem, t->stream);
                }
            } else {
                uint32_t smem = 0;
                const char *pad = getenv("POSE_B200_BALANCE_SMEM");
                if (plan.per_sm && !(pad && pad[0] == '0') &&
                    pb_dev_label_balance_smem(plan.cta, plan.per_sm, &smem) != 0)
                    smem = 0;
                cudaGetLastError();
                lrc = pb_dev_label(&p, plan.grid, plan.cta, smem, t->stream);
            }
            if (lrc != 0) {
                set_err("pose_graph_hbm_topo_label: label kernel launch failed: %s",
                        cudaGetErrorString(cudaGetLastError()));
                goto out;
            }
            CK(cudaEventRecord(t->ev[2], t->stream), "event");
            launches++;
            CK(cudaEventSynchronize(t->ev[2]), "label kernel");
            float ms = 0;
            if (cudaEventElapsedTime(&ms, t->ev[1], t->ev[2]) != cudaSuccess) { cudaGetLastError(); ms = 0; }
            kms += ms;
        }
        /* scratch labels, chunk seeds and the session seed never outlive the
         * call (the reference zeroes its scratch before freeing it,
         * label_gpu_warp.cu:236-238) */
        CK(cudaMemsetAsync(t->d_scratch, 0, plan.scratch_bytes, t->stream), "scratch zero");
        CK(cudaMemsetAsync(t->d_seeds, 0, per_launch * 32, t->stream), "seed zero");
        if (dev_seeds && seed_len) CK(cudaMemsetAsync(t->d_sess, 0, seed_len, t->stream), "seed zero");
        CK(cudaEventRecord(t->ev[3], t->stream), "event");
        CK(cudaStreamSynchronize(t->stream), "label");
        float tms = 0;
        if (cudaEventElapsedTime(&tms, t->ev[0], t->ev[3]) != cudaSuccess) { cudaGetLastError(); tms = 0; }
        double elapsed = now_sec() - t0;
        if (stats) {
            stats->kernel_ms = kms;
            stats->total_ms = tms;
            stats->super_chunks = num_super;
            stats->units = num_super * t->copies;
            stats->nodes = num_super * t->copies * (uint64_t)t->S;
            stats->scratch_bytes = plan.scratch_bytes;
            stats->team_warps = plan.T;
            stats->units_per_team = plan.G;
            stats->teams = plan.teams;
            stats->kernel_launches = launches;
            stats->used_cv0_table = t->d_cv0 != NULL;
            stats->kernel = plan.kernel;
            stats->cluster_ctas = plan.kernel == 3 ? (plan.cluster ? plan.cluster : 1) : 0;
        }
        if (!quiet() && elapsed > 0) {
            double mib = (double)(num_super * t->super_bytes) / (double)(1u << 20);
            printf("  GPU wipe: %.0f MiB in %.3f s = %.1f MiB/s\n", mib, elapsed, mib / elapsed);
            fflush(stdout);
        }
        rc = 0;
    }
fail:
out:
    free(h_seeds);
    if (rc != 0) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) fprintf(stderr, "pose_graph_hbm_topo_label: CUDA error: %s\n", cudaGetErrorString(e));
        /* a call that stopped part way clears whatever it got to write */
        wipe_workspace(t);
    }
    if (prev >= 0 && prev != t->device) cudaSetDevice(prev);
    return rc;
}

static int topo_label_core(const pose_hbm_topo_t *ct, const uint8_t *session_seed, size_t seed_len,
                           const uint8_t *raw_seeds, void *hbm_dev_ptr, size_t hbm_len, uint64_t rbo,
                           const pose_b200_sched_t *sched, pose_b200_stats_t *stats)
{
    nvtxRangePushA("pose_b200: label call");
    int rc = topo_label_core_impl(ct, session_seed, seed_len, raw_seeds, hbm_dev_ptr, hbm_len, rbo, sched, stats);
    nvtxRangePop();
    return rc;
}

int pose_b200_topo_label(const pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                         void *hbm_dev_ptr, size_t hbm_len, uint64_t rbo,
                         const pose_b200_sched_t *sched, pose_b200_stats_t *stats)
{
    return topo_label_core(topo, session_seed, seed_len, NULL, hbm_dev_ptr, hbm_len, rbo, sched, stats);
}

int pb_topo_label_raw(const pose_hbm_topo_t *topo, const uint8_t *chunk_seeds, void *hbm_dev_ptr,
                      size_t hbm_len, const pose_b200_sched_t *sched, pose_b200_stats_t *stats)
{
    if (!chunk_seeds) { set_err("pose_b200: NULL chunk seeds"); return -1; }
    return topo_label_core(topo, NULL, 0, chunk_seeds, hbm_dev_ptr, hbm_len, 0, sched, stats);
}

int pose_graph_hbm_topo_label(const pose_hbm_topo_t *topo, const uint8_t *session_seed,
                              size_t seed_len, void *hbm_dev_ptr, size_t hbm_len,
                              uint64_t region_block_offset)
{
    return pose_b200_topo_label(topo, session_seed, seed_len, hbm_dev_ptr, hbm_len,
                                region_block_offset, NULL, NULL);
}

int pose_graph_label_hbm(const uint8_t *session_seed, size_t seed_len, uint32_t chunk_blocks,
                         void *hbm_dev_ptr, size_t hbm_len, uint64_t region_block_offset,
                         pose_hash_algo_t algo)
{
    if (algo != POSE_HASH_BLAKE3) {
        set_err("pose_graph_label_hbm: only BLAKE3 supported on GPU");
        return -1;
    }
    uint32_t cb = chunk_blocks ? chunk_blocks : PB_DEFAULT_CHUNK_BLOCKS;
    if (cb > PB_MAX_CHUNK_BLOCKS) {
        set_err("pose_graph_label_hbm: super_blocks out of range");
        return -1;
    }
    if (hbm_len / ((size_t)cb * 32) == 0) return 0;
    pose_hbm_topo_t *t = pose_graph_hbm_topo_build(cb, algo);
    if (!t) return -1;
    int rc = pose_graph_hbm_topo_label(t, session_seed, seed_len, hbm_dev_ptr, hbm_len,
                                       region_block_offset);
    pose_graph_hbm_topo_free(t);
    return rc;
}

/* ── known-answer helper ─────────────────────────────────────────────────── */

static void le_words(uint32_t *w, const uint8_t *p)
{
    for (int i = 0; i < 8; i++)
        w[i] = (uint32_t)p[4 * i] | ((uint32_t)p[4 * i + 1] << 8) | ((uint32_t)p[4 * i + 2] << 16) |
               ((uint32_t)p[4 * i + 3] << 24);
}

int pose_gpu_label_node_single(uint8_t out[32], int is_source, uint64_t node_index,
                               const uint8_t *pred0, const uint8_t *pred1, const uint8_t *seed,
                               const uint8_t *descriptor, const uint32_t key_src[8],
                               const uint32_t key_int[8])
{
    if (!out || !seed || !descriptor || !key_src || !key_int) {
        set_err("pose_gpu_label_node_single: NULL argument");
        return -1;
    }
    uint32_t in[56];
    memset(in, 0, sizeof(in));
    if (pred0) le_words(in, pred0);
    if (pred1) le_words(in + 8, pred1);
    le_words(in + 16, seed);
    le_words(in + 24, descriptor);
    memcpy(in + 32, key_src, 32);
    memcpy(in + 40, key_int, 32);
    uint32_t *d = NULL, res[8];
    int rc = -1;
    CK(pb_dev_malloc((void **)&d, sizeof(in)), "KAT alloc");
    CK(cudaMemcpy(d, in, sizeof(in), cudaMemcpyHostToDevice), "KAT upload");
    if (pb_dev_label_single(d + 48, is_source, node_index, d, pred0 != NULL, pred1 != NULL, 0) != 0) {
        set_err("pose_gpu_label_node_single: launch failed");
        goto fail;
    }
    CK(cudaDeviceSynchronize(), "KAT kernel");
    CK(cudaMemcpy(res, d + 48, 32, cudaMemcpyDeviceToHost), "KAT download");
    for (int i = 0; i < 8; i++) {
        out[4 * i] = (uint8_t)res[i];
        out[4 * i + 1] = (uint8_t)(res[i] >> 8);
        out[4 * i + 2] = (uint8_t)(res[i] >> 16);
        out[4 * i + 3] = (uint8_t)(res[i] >> 24);
    }
    rc = 0;
fail:
    cudaFree(d);
    return rc;
}

/* ── compression-rate microbenchmark ─────────────────────────────────────── */

double pose_b200_compress_rate(uint32_t iters, double *latency_cycles)
{
    int dev = 0, sms = 0;
    uint32_t *d_sink = NULL;
    unsigned long long *d_cyc = NULL, cyc = 0;
    cudaEvent_t a = NULL, b = NULL;
    double rate = 0;
    cudaGetDevice(&dev);
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    CK(pb_dev_malloc((void **)&d_sink, 4096 * 4), "sink");
    CK(pb_dev_malloc((void **)&d_cyc, 8), "cycles");
    CK(cudaEventCreate(&a), "event");
    CK(cudaEventCreate(&b), "event");
    {
        uint32_t grid = (uint32_t)sms * 8; /* 8 CTAs x 256 threads per SM */
        for (int fma = 0; fma <= 1; fma++) {
            if (pb_dev_compress_bench(grid, iters / 8 + 1, 1, d_sink, fma, 0) != 0) goto fail; /* warm-up */
            CK(cudaEventRecord(a, 0), "event");
            if (pb_dev_compress_bench(grid, iters, 2, d_sink, fma, 0) != 0) goto fail;
            CK(cudaEventRecord(b, 0), "event");
            CK(cudaEventSynchronize(b), "bench");
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            double r = (double)grid * 256.0 * iters / (ms * 1e-3);
            if (r > rate) rate = r;
        }
        if (latency_cycles) {
            if (pb_dev_compress_latency(iters, d_cyc, d_sink, 0) != 0) goto fail;
            CK(cudaMemcpy(&cyc, d_cyc, 8, cudaMemcpyDeviceToHost), "cycles");
            *latency_cycles = (double)cyc / iters;
        }
    }
fail:
    cudaFree(d_sink);
    cudaFree(d_cyc);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    return rate;
}

/* ── workspace audit ─────────────────────────────────────────────────────── */

int pb_noalloc_residue(int device, unsigned long long *d_count, uint32_t grid, cudaStream_t s);

int pose_b200_topo_residue(const pose_hbm_topo_t *ct, uint64_t *nonzero_bytes)
{
    pose_hbm_topo_t *t = (pose_hbm_topo_t *)ct;
    if (!t || !nonzero_bytes) { set_err("pose_b200_topo_residue: NULL argument"); return -1; }
    *nonzero_bytes = 0;
    int prev = -1, rc = -1;
    cudaGetDevice(&prev);
    if (prev != t->device && cudaSetDevice(t->device) != cudaSuccess) {
        set_err("pose_b200_topo_residue: cannot select the topology's device");
        return -1;
    }
    unsigned long long *d_count = NULL, h_count = 0;
    const uint32_t grid = (uint32_t)(t->sms > 0 ? t->sms : 1) * 8u;
    if (pb_dev_malloc((void **)&d_count, sizeof(*d_count)) != cudaSuccess) {
        set_err("pose_b200_topo_residue: alloc failed");
        goto out;
    }
    if (cudaMemsetAsync(d_count, 0, sizeof(*d_count), t->stream) != cudaSuccess ||
        (t->d_scratch && pb_dev_count_nonzero(t->d_scratch, t->scratch_alloc, d_count, grid, t->stream) != 0) ||
        (t->d_seeds && pb_dev_count_nonzero(t->d_seeds, t->seeds_alloc * 32, d_count, grid, t->stream) != 0) ||
        (t->d_sess && pb_dev_count_nonzero(t->d_sess, t->sess_alloc, d_count, grid, t->stream) != 0) ||
        pb_noalloc_residue(t->device, d_count, grid, t->stream) != 0 ||
        cudaMemcpyAsync(&h_count, d_count, sizeof(h_count), cudaMemcpyDeviceToHost, t->stream) != cudaSuccess ||
        cudaStreamSynchronize(t->stream) != cudaSuccess) {
        set_err("pose_b200_topo_residue: CUDA error: %s", cudaGetErrorString(cudaGetLastError()));
        goto out;
    }
    *nonzero_bytes = h_count;
    rc = 0;
out:
    cudaFree(d_count);
    if (prev >= 0 && prev != t->device) cudaSetDevice(prev);
    return rc;
}

int pose_b200_count_nonzero(const void *dev_ptr, size_t bytes, uint64_t *nonzero_bytes)
{
    if (!nonzero_bytes || (bytes && !dev_ptr)) { set_err("pose_b200_count_nonzero: NULL argument"); return -1; }
    *nonzero_bytes = 0;
    if (bytes == 0) return 0;
    if ((uintptr_t)dev_ptr & 15u) { set_err("pose_b200_count_nonzero: buffer not 16-byte aligned"); return -1; }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 1;
    unsigned long long *d_count = NULL, h_count = 0;
    cudaStream_t st = NULL;
    int rc = -1;
    if (pb_dev_malloc((void **)&d_count, sizeof(*d_count)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMemsetAsync(d_count, 0, sizeof(*d_count), st) != cudaSuccess ||
        pb_dev_count_nonzero(dev_ptr, bytes, d_count, (uint32_t)sms * 8u, st) != 0 ||
        cudaMemcpyAsync(&h_count, d_count, sizeof(h_count), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        set_err("pose_b200_count_nonzero: CUDA error: %s", cudaGetErrorString(cudaGetLastError()));
    } else {
        *nonzero_bytes = h_count;
        rc = 0;
    }
    if (st) cudaStreamDestroy(st);
    cudaFree(d_count);
    return rc;
}

/* ── read-only access for the other translation units ────────────────────── */

#include "topo_internal.h"

int pb_topo_internal(const pose_hbm_topo_t *t, pb_topo_internal_t *out)
{
    if (!t || !out) return -1;
    out->device = t->device;
    out->cb = t->cb;
    out->copies = t->copies;
    out->super_bytes = t->super_bytes;
    out->view = t->view;
    out->stream = t->stream;
    out->sms = t->sms;
    return 0;
}

int pb_topo_view2_small(const pose_hbm_topo_t *ct, pb_topo_view2_t *out)
{
    pose_hbm_topo_t *t = (pose_hbm_topo_t *)ct; /* the record set is built once and kept */
    if (!t || !out || !t->d_cv0 || !t->d_recs2) return -1;
    /* several host threads may create batches on one topology at once: the
     * first one builds the records, the others wait for it and reuse them */
    pthread_mutex_lock(&t->lazy_mu);
    if (!t->d_recs2s) {
        pb_topo_host_t h;
        if (pb_topo_host_build_ex(t->cb, PB_CSM_MULTI, &h) != 0) {
            pthread_mutex_unlock(&t->lazy_mu);
            return -1;
        }
        /* the same levels and node order as the default records; only the
         * pool slots differ */
        int ok = h.recs2 && h.S == t->S && h.L == t->L;
        int prev = -1;
        cudaGetDevice(&prev);
        if (ok && prev != t->device) ok = cudaSetDevice(t->device) == cudaSuccess;
        if (ok) ok = pb_dev_malloc(&t->d_recs2s, (size_t)h.S * 32) == cudaSuccess;
        if (ok) ok = cudaMemcpy(t->d_recs2s, h.recs2, (size_t)h.S * 32, cudaMemcpyHostToDevice) == cudaSuccess;
        if (ok) {
            t->view2s = t->view2;
            t->view2s.recs2 = (const pb_u4 *)t->d_recs2s;
            t->view2s.csm = h.csm;
            t->view2s.gpool = h.gpool2;
            t->dev_bytes += (uint64_t)h.S * 32;
        } else {
            cudaFree(t->d_recs2s);
            t->d_recs2s = NULL;
            cudaGetLastError();
        }
        if (prev >= 0 && prev != t->device) cudaSetDevice(prev);
        pb_topo_host_free(&h);
        if (!ok) {
            pthread_mutex_unlock(&t->lazy_mu);
            return -1;
        }
    }
    *out = t->view2s;
    pthread_mutex_unlock(&t->lazy_mu);
    return 0;
}

uint64_t pb_topo_passes(const pose_hbm_topo_t *t, uint32_t T, uint32_t G)
{
    return t ? passes_for(t, T, G) : 0;
}

uint64_t pb_topo_scratch_budget(const pose_hbm_topo_t *t, uint64_t cap)
{
    pose_b200_sched_t s;
    memset(&s, 0, sizeof(s));
    s.scratch_cap_bytes = cap;
    return scratch_budget(t, &s);
}

int pb_plan_for_budget(const pose_hbm_topo_t *t, uint64_t nunits, uint64_t budget, pb_plan_out_t *out)
{
    /* the caller launches the basic lockstep kernel (k_label) with this plan */
    pose_b200_sched_t basic;
    memset(&basic, 0, sizeof(basic));
    basic.kernel = 1;
    plan_t p;
    if (!t || !out || nunits == 0 || make_plan(t, nunits, &basic, budget, &p) != 0) return -1;
    out->T = p.T; out->G = p.G; out->teams = p.teams; out->grid = p.grid; out->cta = p.cta;
    out->team_scratch = p.team_scratch;
    out->scratch_bytes = p.scratch_bytes;
    return 0;
}
