/*
 * label_server.c — a continuous-batching labeling server (C11 + pthreads).
 *
 * Requests (topology, session, device buffer, region_block_offset — the
 * arguments of pose_graph_hbm_topo_label with the session seed kept on the
 * device) are submitted from any thread.  A dispatcher thread owns the GPU
 * side:
 *   - sessions: every session seed lives in one device blob; seed jobs of a
 *     launch point into it (chunk seeds are derived on the device);
 *   - admission: pending requests are taken, oldest first, into a "wave" as
 *     soon as a wave slot (stream) is free and the scratch arena has room for
 *     at least one team; a wave's teams are as many as the arena's free space,
 *     the GPU's residency and the wave's batches allow;
 *   - a wave is one persistent multi-topology launch (k_label_multi) on its
 *     own stream with its own arena range; waves run concurrently, and a
 *     wave's teams leave as its queue drains, so newly admitted work fills the
 *     GPU behind it;
 *   - completion, per request: when a team finishes a batch, each of its
 *     units adds 1 to its request's counter in mapped host memory (after a
 *     system-scope fence), and the dispatcher marks a request done as soon as
 *     all its chunk copies are in, while the rest of its wave still runs;
 *   - finished waves are reaped and their arena range is zeroed on the device
 *     before it is reused;
 *   - deep requests (topologies of at least PB_SERVER_DEEP_LEVELS levels,
 *     chunk_blocks 2^17 and up) do not join waves: the pending deep requests
 *     of one topology run together on the multi-unit depth kernel
 *     (k_label_wsg: a producer warp and 15 hashing warps per CTA, three chunk
 *     copies per CTA) in a slot of their own, on a high-priority stream.
 *     Each depth CTA holds its SM alone (its shared memory is raised to the
 *     limit), so no lockstep warp slows its chain, and at most one depth CTA
 *     per SM is in flight: a deep request that does not fit the free SMs
 *     waits for them, without holding back the shallow requests behind it.
 *     Their scratch comes from the same arena;
 *   - the dispatcher never waits for the GPU: launch tables go up from
 *     pinned per-slot staging, and every slot's buffers are allocated when
 *     the server is created (an allocation, or a copy from pageable memory,
 *     can wait behind the kernels already running);
 *   - streams share the device's host-to-device work queues
 *     (CUDA_DEVICE_MAX_CONNECTIONS, 8 unless the environment raises it), and
 *     a stream's work that waits behind its own long kernel holds back every
 *     other stream of the same queue; a launch takes a slot whose queue no
 *     running launch uses.  With 32 queues every slot has its own.
 * Every request's bytes are those of labelling it alone.
 */
#include "batch_internal.h"
#include "dev_alloc.h"
#include "kernels.h"
#include "pose_b200.h"

#include <cuda_runtime_api.h>
#include <errno.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define PB_SERVER_MAX_WAVES 16
/* Concurrent launches of the depth kernel. */
#define PB_SERVER_MAX_DEEP 16
/* Requests whose topology has at least this many levels (chunk_blocks 2^17
 * and up) run on the depth kernel instead of joining a wave.  On the
 * 120-request Poisson trace (200 requests/s, chunk_blocks 2^10..2^18), with
 * three chunk copies per depth CTA: 603 MiB/s, against 549 with only 2^18 on
 * the depth kernel and 448 with every request in waves. */
#define PB_SERVER_DEEP_LEVELS 300000u
/* Chunk copies per depth CTA under the default policy (measured on the same
 * trace: 3 copies 549-603 MiB/s, 4 copies 515-548, 2 copies 520). */
#define PB_SERVER_DEEP_UNITS 3u
/* Hashing warps of a depth-kernel CTA. */
#define PB_SERVER_DEEP_WARPS 15u
/* A deep request joins a wave instead when more than this many requests
 * are pending (tuning; by default never). */
#define PB_SERVER_DEEP_QUEUE 0xffffffffu

typedef struct {
    const pose_hbm_topo_t *topo;
    void *dev_ptr;
    size_t len;
    uint64_t rbo;
    int session;
    int deep;  /* runs on the depth kernel */
    int state; /* 0 pending, 1 running, 2 done, 3 failed */
    double t_submit, t_start, t_done;
} sreq_t;

typedef struct {
    int busy;
    cudaStream_t stream;
    cudaEvent_t done;
    uint64_t arena_off, arena_len;
    void *d_tables;
    size_t tables_cap;
    uint8_t *h_stage;          /* pinned host copy of the launch tables, the uploads' source */
    size_t stage_cap;
    uint64_t *reqs;
    uint32_t *need;            /* chunk copies of each request of the wave */
    size_t nreqs, reqs_cap;
    unsigned int *h_done;      /* mapped host counters, one per request */
    unsigned int *d_done;
    size_t done_cap;
    int deep;                  /* deep requests on the depth kernel (complete with the launch) */
    uint32_t chan;             /* the host-to-device work queue its stream maps to (creation order) */
    uint32_t ctas;             /* its CTAs, one SM each */
} wave_t;

struct pose_b200_server {
    int device, running;
    pthread_t thread;
    pthread_mutex_t mu;
    pthread_cond_t cv;
    /* sessions */
    uint8_t *d_sessions;
    size_t sess_bytes, sess_cap;
    uint32_t *sess_off, *sess_len;
    size_t nsess, sess_arr_cap;
    /* requests */
    sreq_t *reqs;
    size_t nreqs, reqs_cap, next_pending;
    /* scratch arena: free ranges */
    uint8_t *d_arena;
    uint64_t arena_bytes;
    uint64_t free_off[2 * PB_SERVER_MAX_WAVES + 2], free_len[2 * PB_SERVER_MAX_WAVES + 2];
    int nfree;
    wave_t waves[PB_SERVER_MAX_WAVES];
    wave_t deeps[PB_SERVER_MAX_DEEP]; /* depth-kernel launches, high-priority streams */
    uint32_t max_waves;        /* concurrent multi-topology waves */
    uint32_t deep_ctas;        /* depth-kernel CTAs in flight */
    uint32_t deep_queue;       /* deep requests take the depth kernel while at most this many requests wait */
    uint32_t deep_units;       /* units per depth CTA: 0 = the fewest of 1, 2, 4 that fit the free SMs */
    uint32_t deep_gmax;        /* most units per depth CTA */
    int deep_wait;             /* a deep request that does not fit waits for SMs instead of joining a wave */
    int deep_excl;             /* a depth CTA holds its SM alone (shared memory raised to the limit) */
    uint32_t deep_levels;      /* requests of topologies with at least this many levels are deep */
    uint32_t sms;
    uint32_t conns;            /* host-to-device work queues (CUDA_DEVICE_MAX_CONNECTIONS, default 8) */
    uint32_t wsg_smem_max;     /* the depth kernel's shared-memory limit (0: no depth kernel) */
    int occ;
    uint64_t waves_launched;
    double busy_ms;
};

static double now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return 1e3 * (double)ts.tv_sec + 1e-6 * (double)ts.tv_nsec;
}

/* first fit, keeping the free list sorted by offset */
static int arena_take(pose_b200_server_t *s, uint64_t want, uint64_t *off)
{
    for (int i = 0; i < s->nfree; i++) {
        if (s->free_len[i] >= want) {
            *off = s->free_off[i];
            s->free_off[i] += want;
            s->free_len[i] -= want;
            if (s->free_len[i] == 0) {
                memmove(&s->free_off[i], &s->free_off[i + 1], (size_t)(s->nfree - i - 1) * 8);
                memmove(&s->free_len[i], &s->free_len[i + 1], (size_t)(s->nfree - i - 1) * 8);
                s->nfree--;
            }
            return 0;
        }
    }
    return -1;
}

static uint64_t arena_largest(const pose_b200_server_t *s)
{
    uint64_t m = 0;
    for (int i = 0; i < s->nfree; i++) if (s->free_len[i] > m) m = s->free_len[i];
    return m;
}

static void arena_give(pose_b200_server_t *s, uint64_t off, uint64_t len)
{
    int i = 0;
    while (i < s->nfree && s->free_off[i] < off) i++;
    memmove(&s->free_off[i + 1], &s->free_off[i], (size_t)(s->nfree - i) * 8);
    memmove(&s->free_len[i + 1], &s->free_len[i], (size_t)(s->nfree - i) * 8);
    s->free_off[i] = off;
    s->free_len[i] = len;
    s->nfree++;
    /* merge neighbours */
    for (int k = 0; k + 1 < s->nfree;) {
        if (s->free_off[k] + s->free_len[k] == s->free_off[k + 1]) {
            s->free_len[k] += s->free_len[k + 1];
            memmove(&s->free_off[k + 1], &s->free_off[k + 2], (size_t)(s->nfree - k - 2) * 8);
            memmove(&s->free_len[k + 1], &s->free_len[k + 2], (size_t)(s->nfree - k - 2) * 8);
            s->nfree--;
        } else {
            k++;
        }
    }
}

/* Whether a request runs on the depth kernel: a deep topology whose 512-slot
 * records the multi-unit depth kernel has (built here on first use: call
 * without the server lock held), on a GPU whose CTAs hold the kernel's
 * shared memory, with one chunk copy's scratch fitting the arena
 * (otherwise it joins a wave like the others). */
static int req_is_deep(const pose_b200_server_t *s, const pose_hbm_topo_t *topo)
{
    pb_topo_internal_t ti;
    pb_topo_view2_t v2;
    if (!s->wsg_smem_max || pb_topo_internal(topo, &ti) != 0 || ti.view.L < s->deep_levels) return 0;
    if (pb_topo_view2_small(topo, &v2) != 0) {
        cudaGetLastError();
        return 0;
    }
    return pb_wsg_smem_bytes(v2.csm, 4, PB_SERVER_DEEP_WARPS) <= s->wsg_smem_max &&
           (uint64_t)v2.gpool * 32 <= s->arena_bytes;
}

/* Device tables of one launch in a slot's buffer, grown on demand. */
static int slot_tables(wave_t *wv, size_t total)
{
    if (wv->tables_cap >= total) return 0;
    cudaFree(wv->d_tables);
    wv->d_tables = NULL;
    wv->tables_cap = 0;
    if (pb_dev_malloc(&wv->d_tables, total * 2) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    wv->tables_cap = total * 2;
    return 0;
}

/* Pinned host staging of one launch's tables, grown on demand.  The uploads
 * from it are asynchronous, so the dispatcher never waits for the GPU: the
 * slot's staging stays untouched until the slot is reaped. */
static int slot_stage(wave_t *wv, size_t total)
{
    if (wv->stage_cap >= total) return 0;
    if (wv->h_stage) cudaFreeHost(wv->h_stage);
    wv->h_stage = NULL;
    wv->stage_cap = 0;
    if (cudaHostAlloc((void **)&wv->h_stage, total * 2, cudaHostAllocDefault) != cudaSuccess) {
        wv->h_stage = NULL;
        cudaGetLastError();
        return -1;
    }
    wv->stage_cap = total * 2;
    return 0;
}

static int slot_reqs(wave_t *wv, size_t n)
{
    if (wv->reqs_cap >= n) return 0;
    uint64_t *nr = (uint64_t *)realloc(wv->reqs, n * sizeof(uint64_t));
    if (nr) wv->reqs = nr;
    uint32_t *nn = nr ? (uint32_t *)realloc(wv->need, n * sizeof(uint32_t)) : NULL;
    if (nn) wv->need = nn;
    if (!nr || !nn) return -1;
    wv->reqs_cap = n;
    return 0;
}

/* Streams share the device's host-to-device work queues, assigned in
 * creation order; work that waits behind a long kernel in one stream holds
 * back every stream of its queue.  A launch therefore takes a free slot whose
 * queue no busy slot uses. */
static int chan_busy(const pose_b200_server_t *s, uint32_t chan)
{
    for (uint32_t i = 0; i < PB_SERVER_MAX_WAVES; i++)
        if (s->waves[i].busy && s->waves[i].chan == chan) return 1;
    for (uint32_t i = 0; i < PB_SERVER_MAX_DEEP; i++)
        if (s->deeps[i].busy && s->deeps[i].chan == chan) return 1;
    return 0;
}

/* With the lock held: launch the pending deep requests of the oldest pending
 * deep request's topology, oldest first, on the multi-unit depth kernel in a
 * free deep slot, one chunk copy per CTA and CTA per SM (the CTAs in flight
 * count against the SMs): the shortest chains.  Requests are taken while
 * their copies fit the free SMs.  When the oldest one does not fit, or more
 * than PB_SERVER_DEEP_QUEUE requests are pending, the GPU is loaded: it joins
 * the next wave instead, where the lockstep kernel packs many copies per SM
 * (on a loaded GPU the depth kernel's one SM per copy costs more throughput
 * than its shorter chain saves).  The requests complete with the launch.  Returns 1 when something was launched, failed
 * or moved to the waves, 0 when nothing could be done. */
static int admit_deep(pose_b200_server_t *s)
{
    size_t i0 = s->next_pending;
    while (i0 < s->nreqs && !(s->reqs[i0].state == 0 && s->reqs[i0].deep)) i0++;
    if (i0 >= s->nreqs) return 0;
    int w = -1;
    for (uint32_t i = 0; i < PB_SERVER_MAX_DEEP && w < 0; i++)
        if (!s->deeps[i].busy && !chan_busy(s, s->deeps[i].chan)) w = (int)i;
    const pose_hbm_topo_t *topo = s->reqs[i0].topo;
    pb_topo_internal_t ti;
    pb_topo_view2_t v2;
    if (pb_topo_internal(topo, &ti) != 0 || pb_topo_view2_small(topo, &v2) != 0) return 0;
    const uint32_t free_sms = s->deep_ctas < s->sms ? s->sms - s->deep_ctas : 0;
    const uint64_t units0 = (s->reqs[i0].len / ti.super_bytes) * ti.copies;
    size_t pending = 0;
    for (size_t i = s->next_pending; i < s->nreqs; i++) pending += s->reqs[i].state == 0;
    const uint32_t gmax = s->deep_units ? s->deep_units : s->deep_gmax;
    uint64_t ctas0 = (units0 + gmax - 1) / gmax;
    if (ctas0 > s->sms) ctas0 = s->sms; /* larger than the GPU: its CTAs loop over the batches */
    if (pending > s->deep_queue || (!s->deep_wait && (w < 0 || ctas0 > free_sms))) {
        s->reqs[i0].deep = 0; /* to the waves */
        return 1;
    }
    if (w < 0 || ctas0 > free_sms) return 0; /* waits for a slot or SMs */
    /* the group: same topology, oldest first, while its CTAs fit the free SMs */
    size_t n = 0;
    uint64_t units = 0, nsuper = 0;
    for (size_t i = i0; i < s->nreqs; i++) {
        const sreq_t *r = &s->reqs[i];
        if (r->state != 0 || !r->deep || r->topo != topo) continue;
        const uint64_t ns = r->len / ti.super_bytes;
        if (n > 0 && (units + ns * ti.copies + gmax - 1) / gmax > free_sms) break;
        units += ns * ti.copies;
        nsuper += ns;
        n++;
    }
    wave_t *wv = &s->deeps[w];
    if (slot_reqs(wv, n) != 0) return 0;
    {
        size_t k = 0;
        for (size_t i = i0; i < s->nreqs && k < n; i++) {
            const sreq_t *r = &s->reqs[i];
            if (r->state == 0 && r->deep && r->topo == topo) wv->reqs[k++] = i;
        }
    }
    const double t = now_ms();
    if (units == 0) { /* nothing to label */
        for (size_t k = 0; k < n; k++) {
            sreq_t *r = &s->reqs[wv->reqs[k]];
            r->state = 2;
            r->t_start = r->t_done = t;
        }
        pthread_cond_broadcast(&s->cv);
        return 1;
    }
    /* units per CTA: on an otherwise idle depth kernel (nothing of it in
     * flight, no other deep request waiting) the fewest that fit the free
     * SMs, for the shortest chains; under load the most, for the most chains
     * per SM (a narrow level of G units is still one warp pass) */
    uint32_t G = s->deep_units;
    if (!G) {
        size_t others = 0;
        for (size_t i = i0; i < s->nreqs; i++) {
            const sreq_t *r = &s->reqs[i];
            others += r->state == 0 && r->deep;
        }
        others -= n;
        if (s->deep_ctas > 0 || others > 0) {
            G = gmax;
        } else {
            G = 1;
            while (G < gmax && (units + G - 1) / G > free_sms) G *= 2;
            if (G > gmax) G = gmax;
        }
    }
    const uint64_t nbatches = (units + G - 1) / G;
    uint32_t grid = (uint32_t)(nbatches < free_sms ? nbatches : free_sms);
    const uint64_t per = (uint64_t)v2.gpool * 32 * G;
    const uint64_t fit = arena_largest(s) / per;
    if (fit < grid) grid = (uint32_t)fit;
    if (grid == 0) return 0; /* wait for scratch */
    const uint64_t scratch = (uint64_t)grid * per;
    uint64_t off = 0;
    if (arena_take(s, scratch, &off) != 0) return 0;
    /* tables: units | jobs | seeds | queue, 256-byte aligned */
#define AL(x) (((x) + 255) & ~(size_t)255)
    const size_t o_units = 0, o_jobs = AL(units * sizeof(pb_munit_t));
    const size_t o_seeds = AL(o_jobs + nsuper * sizeof(pb_seedjob_t)), o_queue = AL(o_seeds + nsuper * 32);
    const size_t total = AL(o_queue + 64);
#undef AL
    if (slot_tables(wv, total) != 0 || slot_stage(wv, o_seeds) != 0) {
        arena_give(s, off, scratch);
        return 0;
    }
    pb_munit_t *hu = (pb_munit_t *)(wv->h_stage + o_units);
    pb_seedjob_t *hj = (pb_seedjob_t *)(wv->h_stage + o_jobs);
    {
        uint64_t u = 0, j = 0;
        for (size_t k = 0; k < n; k++) {
            const sreq_t *r = &s->reqs[wv->reqs[k]];
            const uint64_t ns = r->len / ti.super_bytes;
            for (uint64_t c = 0; c < ns; c++, j++) {
                hj[j].chunk_index = (r->rbo + c * (uint64_t)ti.cb) / ti.cb;
                hj[j].seed_off = s->sess_off[r->session];
                hj[j].seed_len = s->sess_len[r->session];
                for (uint32_t cp = 0; cp < ti.copies; cp++, u++) {
                    hu[u].out = (uint64_t)(uintptr_t)r->dev_ptr + c * ti.super_bytes;
                    hu[u].seed = (uint32_t)j;
                    hu[u].copy = cp;
                }
            }
        }
    }
    uint8_t *T = (uint8_t *)wv->d_tables;
    int ok = cudaMemcpyAsync(T, wv->h_stage, o_seeds, cudaMemcpyHostToDevice, wv->stream) == cudaSuccess;
    ok = ok && pb_dev_seed_jobs(T + o_jobs, (uint32_t)nsuper, s->d_sessions, (uint32_t *)(T + o_seeds), wv->stream) == 0;
    ok = ok && cudaMemsetAsync(T + o_queue, 0, 64, wv->stream) == cudaSuccess;
    if (ok) {
        pb_wsg_params_t p;
        memset(&p, 0, sizeof(p));
        p.topo = v2;
        p.units = (const pb_munit_t *)(T + o_units);
        p.seeds = (const uint32_t *)(T + o_seeds);
        p.scratch = s->d_arena + off;
        p.unit_scratch_bytes = (uint64_t)v2.gpool * 32;
        p.nunits = (uint32_t)units;
        p.units_per_cta = G;
        p.team_warps = PB_SERVER_DEEP_WARPS;
        p.nbatches = (uint32_t)nbatches;
        p.queue = (unsigned int *)(T + o_queue);
        const uint32_t need = pb_wsg_smem_bytes(v2.csm, G, PB_SERVER_DEEP_WARPS);
        ok = pb_dev_label_wsg(&p, grid, 32 * (PB_SERVER_DEEP_WARPS + 1),
                              s->deep_excl && s->wsg_smem_max > need ? s->wsg_smem_max : need, wv->stream) == 0;
    }
    /* scratch and chunk seeds are zeroed before the requests count as done */
    ok = ok && cudaMemsetAsync(s->d_arena + off, 0, scratch, wv->stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(T + o_seeds, 0, nsuper * 32, wv->stream) == cudaSuccess;
    ok = ok && cudaEventRecord(wv->done, wv->stream) == cudaSuccess;
    if (!ok) {
        fprintf(stderr, "pose_b200_server: deep launch failed: %s\n", cudaGetErrorString(cudaGetLastError()));
        cudaStreamSynchronize(wv->stream);
        cudaMemsetAsync(s->d_arena + off, 0, scratch, wv->stream);
        cudaMemsetAsync(T + o_seeds, 0, nsuper * 32, wv->stream);
        cudaStreamSynchronize(wv->stream);
        cudaGetLastError();
        arena_give(s, off, scratch);
        for (size_t k = 0; k < n; k++) {
            s->reqs[wv->reqs[k]].state = 3;
            s->reqs[wv->reqs[k]].t_done = t;
        }
    } else {
        wv->busy = 1;
        wv->deep = 1;
        wv->ctas = grid;
        wv->arena_off = off;
        wv->arena_len = scratch;
        wv->nreqs = n;
        s->deep_ctas += grid;
        for (size_t k = 0; k < n; k++) {
            s->reqs[wv->reqs[k]].state = 1;
            s->reqs[wv->reqs[k]].t_start = t;
        }
        s->waves_launched++;
    }
    pthread_cond_broadcast(&s->cv);
    return 1;
}

/* With the lock held: launch one wave from every pending request that does
 * not run on the depth kernel.  Returns 1 when a wave was launched (or its
 * requests failed), 0 when nothing could be admitted. */
static int admit_wave(pose_b200_server_t *s)
{
    int w = -1;
    uint32_t multi = 0;
    for (uint32_t i = 0; i < PB_SERVER_MAX_WAVES; i++) {
        if (s->waves[i].busy) multi++;
        else if (w < 0 && !chan_busy(s, s->waves[i].chan)) w = (int)i;
    }
    if (w < 0 || multi >= s->max_waves) return 0;
    wave_t *wv = &s->waves[w];
    wv->deep = 0;
    wv->ctas = 0;
    size_t n = 0;
    for (size_t i = s->next_pending; i < s->nreqs; i++) n += s->reqs[i].state == 0 && !s->reqs[i].deep;
    if (n == 0) return 0;
    if (slot_reqs(wv, n) != 0) return 0;
    {
        size_t k = 0;
        for (size_t i = s->next_pending; i < s->nreqs && k < n; i++)
            if (s->reqs[i].state == 0 && !s->reqs[i].deep) wv->reqs[k++] = i;
    }
    pb_req_t *pr = (pb_req_t *)calloc(n, sizeof(*pr));
    if (!pr) return 0;
    for (size_t i = 0; i < n; i++) {
        const sreq_t *r = &s->reqs[wv->reqs[i]];
        pr[i].topo = r->topo;
        pr[i].dev_ptr = r->dev_ptr;
        pr[i].len = r->len;
        pr[i].rbo = r->rbo;
        pr[i].seed_off = s->sess_off[r->session];
        pr[i].seed_len = s->sess_len[r->session];
    }
    pb_plan_tables_t pl;
    uint32_t Tw = 4;
    double eff = 0.0;
    if (pb_plan_choose(pr, n, NULL, &Tw, &eff) != 0 || pb_plan_requests(pr, n, Tw, 32, eff, &pl) != 0) {
        free(pr);
        for (size_t i = 0; i < n; i++) { s->reqs[wv->reqs[i]].state = 3; s->reqs[wv->reqs[i]].t_done = now_ms(); }
        pthread_cond_broadcast(&s->cv);
        return 1;
    }
    free(pr);
    int launched = 0;
    if (pl.nunits == 0) { /* nothing to label: done at once */
        for (size_t i = 0; i < n; i++) {
            sreq_t *r = &s->reqs[wv->reqs[i]];
            r->state = 2;
            r->t_start = r->t_done = now_ms();
        }
        pthread_cond_broadcast(&s->cv);
        pb_plan_free(&pl);
        return 1;
    }
    /* teams: as many as fit in the largest free arena range, the GPU and the
     * batches; one team per CTA, every team with its scratch */
    const uint32_t tpc_max = 256 / (32 * Tw);
    uint64_t cap = (uint64_t)pl.sms * (s->occ > 0 ? s->occ : 1) * tpc_max;
    uint64_t R = arena_largest(s) / pl.team_scratch;
    if (R > cap) R = cap;
    if (R > pl.nbatches) R = pl.nbatches;
    if (R == 0) { pb_plan_free(&pl); return 0; } /* wait for scratch to free up */
    const uint32_t g2 = (uint32_t)R; /* one team per CTA */
    const uint64_t scratch = R * pl.team_scratch;
    uint64_t off = 0;
    if (arena_take(s, scratch, &off) != 0) { pb_plan_free(&pl); return 0; }
    /* per-request completion counters (mapped host memory) */
    if (wv->done_cap < n) {
        if (wv->h_done) cudaFreeHost(wv->h_done);
        wv->h_done = NULL;
        wv->d_done = NULL;
        wv->done_cap = 0;
        size_t cap = n < 1024 ? 1024 : 2 * n;
        if (cudaHostAlloc((void **)&wv->h_done, cap * sizeof(unsigned int), cudaHostAllocMapped) != cudaSuccess ||
            cudaHostGetDevicePointer((void **)&wv->d_done, wv->h_done, 0) != cudaSuccess) {
            if (wv->h_done) cudaFreeHost(wv->h_done);
            wv->h_done = NULL;
            cudaGetLastError();
            arena_give(s, off, scratch);
            pb_plan_free(&pl);
            return 0;
        }
        wv->done_cap = cap;
    }
    memset((void *)wv->h_done, 0, n * sizeof(unsigned int));
    memset(wv->need, 0, n * sizeof(uint32_t));
    for (uint64_t u = 0; u < pl.nunits; u++) wv->need[pl.unit_req[u]]++;
    /* tables: views | batches | units | unit_req | jobs | seeds | queue, 256-byte aligned */
    size_t o_views = 0, o_batches, o_units, o_ureq, o_jobs, o_seeds, o_queue, total;
#define AL(x) (((x) + 255) & ~(size_t)255)
    o_batches = AL(o_views + pl.ntopo * sizeof(pb_topo_view_t));
    o_units = AL(o_batches + pl.nbatches * sizeof(pb_mbatch_t));
    o_ureq = AL(o_units + pl.nunits * sizeof(pb_munit_t));
    o_jobs = AL(o_ureq + pl.nunits * sizeof(uint32_t));
    o_seeds = AL(o_jobs + pl.njobs * sizeof(pb_seedjob_t));
    o_queue = AL(o_seeds + pl.njobs * 32);
    total = AL(o_queue + 64);
#undef AL
    if (slot_tables(wv, total) != 0 || slot_stage(wv, o_seeds) != 0) {
        arena_give(s, off, scratch);
        pb_plan_free(&pl);
        return 0;
    }
    uint8_t *T = (uint8_t *)wv->d_tables;
    memcpy(wv->h_stage + o_views, pl.views, pl.ntopo * sizeof(pb_topo_view_t));
    memcpy(wv->h_stage + o_batches, pl.batches, pl.nbatches * sizeof(pb_mbatch_t));
    memcpy(wv->h_stage + o_units, pl.units, pl.nunits * sizeof(pb_munit_t));
    memcpy(wv->h_stage + o_ureq, pl.unit_req, pl.nunits * sizeof(uint32_t));
    memcpy(wv->h_stage + o_jobs, pl.jobs, pl.njobs * sizeof(pb_seedjob_t));
    int ok = cudaMemcpyAsync(T, wv->h_stage, o_seeds, cudaMemcpyHostToDevice, wv->stream) == cudaSuccess;
    ok &= pb_dev_seed_jobs(T + o_jobs, (uint32_t)pl.njobs, s->d_sessions, (uint32_t *)(T + o_seeds), wv->stream) == 0;
    ok &= cudaMemsetAsync(T + o_queue, 0, 64, wv->stream) == cudaSuccess;
    pb_multi_params_t p;
    memset(&p, 0, sizeof(p));
    p.topos = (const pb_topo_view_t *)(T + o_views);
    p.batches = (const pb_mbatch_t *)(T + o_batches);
    p.units = (const pb_munit_t *)(T + o_units);
    p.seeds = (const uint32_t *)(T + o_seeds);
    p.scratch = s->d_arena + off;
    p.team_scratch_bytes = pl.team_scratch;
    p.nbatches = (uint32_t)pl.nbatches;
    p.team_warps = Tw;
    p.queue = (unsigned int *)(T + o_queue);
    p.fma_adds = (double)R * Tw / pl.sms >= 8.0;
    p.one = 1;
    p.unit_req = (const uint32_t *)(T + o_ureq);
    p.req_done = wv->d_done;
    if (ok) ok = pb_dev_label_multi(&p, g2, 32 * Tw, wv->stream) == 0;
    /* the scratch range and the chunk seeds are zeroed before the wave
     * counts as done */
    if (ok) ok = cudaMemsetAsync(s->d_arena + off, 0, scratch, wv->stream) == cudaSuccess;
    if (ok) ok = cudaMemsetAsync(T + o_seeds, 0, pl.njobs * 32, wv->stream) == cudaSuccess;
    if (ok) ok = cudaEventRecord(wv->done, wv->stream) == cudaSuccess;
    double t = now_ms();
    if (!ok) {
        fprintf(stderr, "pose_b200_server: wave launch failed: %s\n", cudaGetErrorString(cudaGetLastError()));
        cudaStreamSynchronize(wv->stream);
        /* whatever the wave got to write goes, best effort */
        cudaMemsetAsync(s->d_arena + off, 0, scratch, wv->stream);
        cudaMemsetAsync(T + o_seeds, 0, pl.njobs * 32, wv->stream);
        cudaStreamSynchronize(wv->stream);
        cudaGetLastError();
        arena_give(s, off, scratch);
        for (size_t i = 0; i < n; i++) { s->reqs[wv->reqs[i]].state = 3; s->reqs[wv->reqs[i]].t_done = t; }
    } else {
        wv->busy = 1;
        wv->arena_off = off;
        wv->arena_len = scratch;
        wv->nreqs = n;
        for (size_t i = 0; i < n; i++) {
            s->reqs[wv->reqs[i]].state = 1;
            s->reqs[wv->reqs[i]].t_start = t;
        }
        s->waves_launched++;
        launched = 1;
    }
    pb_plan_free(&pl);
    pthread_cond_broadcast(&s->cv);
    return launched || !ok;
}

/* With the lock held: one round of admission — deep requests first (their
 * chains are the long poles), then a wave of the rest.  Returns 1 when
 * anything changed. */
static int admit(pose_b200_server_t *s)
{
    while (s->next_pending < s->nreqs && s->reqs[s->next_pending].state != 0) s->next_pending++;
    if (s->next_pending >= s->nreqs) return 0;
    const int d = admit_deep(s);
    const int w = admit_wave(s);
    return d || w;
}

/* With the lock held: complete the requests whose chunk copies are all in,
 * and retire finished waves.  Returns how many requests or waves changed. */
static int reap(pose_b200_server_t *s)
{
    int k = 0;
    for (uint32_t i = 0; i < PB_SERVER_MAX_WAVES + PB_SERVER_MAX_DEEP; i++) {
        wave_t *wv = i < PB_SERVER_MAX_WAVES ? &s->waves[i] : &s->deeps[i - PB_SERVER_MAX_WAVES];
        if (!wv->busy) continue;
        double t = now_ms();
        for (size_t r = 0; r < wv->nreqs && !wv->deep; r++) {
            sreq_t *q = &s->reqs[wv->reqs[r]];
            if (q->state == 1 && ((volatile unsigned int *)wv->h_done)[r] >= wv->need[r]) {
                q->state = 2;
                q->t_done = t;
                k++;
            }
        }
        cudaError_t e = cudaEventQuery(wv->done);
        if (e == cudaErrorNotReady) continue;
        t = now_ms();
        for (size_t r = 0; r < wv->nreqs; r++) {
            sreq_t *q = &s->reqs[wv->reqs[r]];
            if (q->state == 1 || e != cudaSuccess) {
                q->state = e == cudaSuccess ? 2 : 3;
                q->t_done = t;
            }
        }
        if (e != cudaSuccess) {
            fprintf(stderr, "pose_b200_server: wave failed: %s\n", cudaGetErrorString(e));
            cudaGetLastError();
        }
        arena_give(s, wv->arena_off, wv->arena_len);
        if (wv->deep) s->deep_ctas -= wv->ctas;
        wv->busy = 0;
        k++;
    }
    if (k) pthread_cond_broadcast(&s->cv);
    return k;
}

static int any_busy(const pose_b200_server_t *s)
{
    int busy = 0;
    for (uint32_t i = 0; i < PB_SERVER_MAX_WAVES; i++) busy |= s->waves[i].busy;
    for (uint32_t i = 0; i < PB_SERVER_MAX_DEEP; i++) busy |= s->deeps[i].busy;
    return busy;
}

static void *dispatcher(void *arg)
{
    pose_b200_server_t *s = (pose_b200_server_t *)arg;
    cudaSetDevice(s->device);
    pthread_mutex_lock(&s->mu);
    for (;;) {
        while (s->next_pending < s->nreqs && s->reqs[s->next_pending].state != 0) s->next_pending++;
        if (!s->running && !any_busy(s) && s->next_pending >= s->nreqs) break;
        int progress = reap(s);
        while (admit(s)) progress = 1;
        if (!progress) {
            const int busy = any_busy(s);
            struct timespec ts;
            clock_gettime(CLOCK_REALTIME, &ts);
            long ns = busy ? 50000 : 2000000; /* poll running waves every 50 us */
            ts.tv_nsec += ns;
            if (ts.tv_nsec >= 1000000000L) { ts.tv_sec++; ts.tv_nsec -= 1000000000L; }
            pthread_cond_timedwait(&s->cv, &s->mu, &ts);
        }
    }
    pthread_mutex_unlock(&s->mu);
    return NULL;
}

pose_b200_server_t *pose_b200_server_create(uint64_t scratch_bytes, uint32_t max_waves)
{
    pose_b200_server_t *s = (pose_b200_server_t *)calloc(1, sizeof(*s));
    if (!s) return NULL;
    cudaGetDevice(&s->device);
    {
        const char *ec = getenv("CUDA_DEVICE_MAX_CONNECTIONS");
        s->conns = ec && atoi(ec) > 0 ? (uint32_t)atoi(ec) : 8;
        if (s->conns > 32) s->conns = 32;
    }
    /* By default 5 waves with 16 or more work queues, 3 with fewer: on the
     * 120-request Poisson trace (200 requests/s, chunk_blocks 2^10..2^18,
     * deep requests on the depth kernel, 32 queues) 3 waves served 589-603
     * MiB/s (p50 1.43-1.48 s), 5 waves 593-594 (p50 1.25-1.35 s) and 8 waves
     * 578 (p50 1.15 s); with the default 8 queues every wave slot in use is
     * one fewer concurrent depth-kernel launch */
    s->max_waves = max_waves ? (max_waves < PB_SERVER_MAX_WAVES ? max_waves : PB_SERVER_MAX_WAVES)
                             : (s->conns >= 16 ? 5 : 3);
    pthread_mutex_init(&s->mu, NULL);
    pthread_cond_init(&s->cv, NULL);
    if (scratch_bytes == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        scratch_bytes = fr > ((uint64_t)8 << 30) ? (uint64_t)(fr / 2) : (uint64_t)(fr / 4);
    }
    scratch_bytes &= ~(uint64_t)255;
    if (pb_dev_malloc((void **)&s->d_arena, scratch_bytes) != cudaSuccess) {
        fprintf(stderr, "pose_b200_server_create: scratch arena of %llu bytes failed\n", (unsigned long long)scratch_bytes);
        goto fail;
    }
    s->arena_bytes = scratch_bytes;
    s->free_off[0] = 0;
    s->free_len[0] = scratch_bytes;
    s->nfree = 1;
    /* the slots' streams are created back to back: waves, then deep slots */
    for (uint32_t i = 0; i < PB_SERVER_MAX_WAVES; i++) s->waves[i].chan = i % s->conns;
    for (uint32_t i = 0; i < PB_SERVER_MAX_DEEP; i++) s->deeps[i].chan = (PB_SERVER_MAX_WAVES + i) % s->conns;
    for (uint32_t i = 0; i < PB_SERVER_MAX_WAVES; i++) {
        if (cudaStreamCreateWithFlags(&s->waves[i].stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s->waves[i].done, cudaEventDisableTiming) != cudaSuccess)
            goto fail;
    }
    {
        /* depth-kernel launches get the highest stream priority: when a
         * wave's CTA leaves an SM, a waiting depth CTA takes it first */
        int lo = 0, hi = 0;
        if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) lo = hi = 0;
        for (uint32_t i = 0; i < PB_SERVER_MAX_DEEP; i++) {
            if (cudaStreamCreateWithPriority(&s->deeps[i].stream, cudaStreamNonBlocking, hi) != cudaSuccess ||
                cudaEventCreateWithFlags(&s->deeps[i].done, cudaEventDisableTiming) != cudaSuccess)
                goto fail;
        }
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess || sms <= 0) sms = 1;
        /* POSE_B200_SERVER_DEEP_SMS caps the SMs the depth kernel may hold (tests, tuning) */
        const char *e = getenv("POSE_B200_SERVER_DEEP_SMS");
        if (e && atoi(e) > 0 && atoi(e) < sms) sms = atoi(e);
        s->sms = (uint32_t)sms;
        uint32_t mx = 0;
        if (pb_dev_label_wsg_prepare(&mx) != 0) mx = 0; /* no depth kernel: deep requests join waves */
        cudaGetLastError();
        const char *ed = getenv("POSE_B200_SERVER_DEEP"); /* 0: every request joins the waves */
        s->wsg_smem_max = ed && ed[0] == '0' ? 0 : mx;
        /* deep-request policy (tuning): queue threshold, units per CTA, wait or join a wave, SM held alone */
        s->deep_queue = PB_SERVER_DEEP_QUEUE;
        s->deep_units = PB_SERVER_DEEP_UNITS;
        s->deep_gmax = 4;
        s->deep_wait = 1;
        s->deep_excl = 1;
        s->deep_levels = PB_SERVER_DEEP_LEVELS;
        const char *e0 = getenv("POSE_B200_SERVER_DEEP_LEVELS");
        if (e0 && atoi(e0) > 0) s->deep_levels = (uint32_t)atoi(e0);
        const char *e1 = getenv("POSE_B200_SERVER_DEEP_QUEUE");
        if (e1 && e1[0]) s->deep_queue = (uint32_t)atoi(e1);
        const char *e2 = getenv("POSE_B200_SERVER_DEEP_UNITS");
        if (e2 && atoi(e2) >= 0 && atoi(e2) <= 4) s->deep_units = (uint32_t)atoi(e2);
        const char *e3 = getenv("POSE_B200_SERVER_DEEP_GMAX");
        if (e3 && atoi(e3) >= 1 && atoi(e3) <= 4) s->deep_gmax = (uint32_t)atoi(e3);
        const char *e4 = getenv("POSE_B200_SERVER_DEEP_WAIT");
        if (e4 && e4[0]) s->deep_wait = atoi(e4) != 0;
        const char *e5 = getenv("POSE_B200_SERVER_DEEP_EXCL");
        if (e5 && e5[0]) s->deep_excl = atoi(e5) != 0;
    }
    if (pb_dev_label_multi_occupancy(256, &s->occ) != 0) s->occ = 1;
    /* Launch tables and completion counters of every slot, allocated up
     * front: the dispatcher then makes no allocation while kernels run (a
     * cudaFree there waits for the whole device, and the submitters and
     * waiters wait on the dispatcher's lock meanwhile).  Best effort: a slot
     * whose buffers could not be had grows them on first use. */
    for (uint32_t i = 0; i < PB_SERVER_MAX_WAVES; i++) {
        wave_t *wv = &s->waves[i];
        if (slot_tables(wv, (size_t)512 << 10) != 0) cudaGetLastError();
        if (slot_stage(wv, (size_t)512 << 10) != 0) cudaGetLastError();
        if (cudaHostAlloc((void **)&wv->h_done, 4096 * sizeof(unsigned int), cudaHostAllocMapped) == cudaSuccess &&
            cudaHostGetDevicePointer((void **)&wv->d_done, wv->h_done, 0) == cudaSuccess) {
            wv->done_cap = 4096;
        } else {
            if (wv->h_done) cudaFreeHost(wv->h_done);
            wv->h_done = NULL;
            wv->d_done = NULL;
            cudaGetLastError();
        }
    }
    for (uint32_t i = 0; i < PB_SERVER_MAX_DEEP; i++) {
        if (slot_tables(&s->deeps[i], (size_t)64 << 10) != 0) cudaGetLastError();
        if (slot_stage(&s->deeps[i], (size_t)64 << 10) != 0) cudaGetLastError();
    }
    s->running = 1;
    if (pthread_create(&s->thread, NULL, dispatcher, s) != 0) { s->running = 0; goto fail; }
    return s;
fail:
    cudaGetLastError();
    for (uint32_t i = 0; i < PB_SERVER_MAX_WAVES; i++) {
        if (s->waves[i].stream) cudaStreamDestroy(s->waves[i].stream);
        if (s->waves[i].done) cudaEventDestroy(s->waves[i].done);
        cudaFree(s->waves[i].d_tables);
        if (s->waves[i].h_done) cudaFreeHost(s->waves[i].h_done);
        if (s->waves[i].h_stage) cudaFreeHost(s->waves[i].h_stage);
    }
    for (uint32_t i = 0; i < PB_SERVER_MAX_DEEP; i++) {
        if (s->deeps[i].stream) cudaStreamDestroy(s->deeps[i].stream);
        if (s->deeps[i].done) cudaEventDestroy(s->deeps[i].done);
        cudaFree(s->deeps[i].d_tables);
        if (s->deeps[i].h_stage) cudaFreeHost(s->deeps[i].h_stage);
    }
    cudaFree(s->d_arena);
    pthread_mutex_destroy(&s->mu);
    pthread_cond_destroy(&s->cv);
    free(s);
    return NULL;
}

int pose_b200_server_session(pose_b200_server_t *s, const uint8_t *seed, size_t seed_len)
{
    if (!s || (!seed && seed_len) || seed_len > 1016) {
        fprintf(stderr, "pose_b200_server_session: bad seed\n");
        return -1;
    }
    pthread_mutex_lock(&s->mu);
    int id = -1;
    /* sessions are appended; the blob grows by copy (in-flight waves keep
     * reading their own copy until they finish, so growth waits for idle) */
    if (s->sess_bytes + seed_len > s->sess_cap) {
        for (;;) {
            while (s->next_pending < s->nreqs && s->reqs[s->next_pending].state != 0) s->next_pending++;
            if (!any_busy(s) && s->next_pending >= s->nreqs) break;
            pthread_cond_wait(&s->cv, &s->mu);
        }
        size_t ncap = (s->sess_cap ? s->sess_cap * 2 : 4096);
        while (ncap < s->sess_bytes + seed_len) ncap *= 2;
        uint8_t *nb = NULL;
        if (pb_dev_malloc((void **)&nb, ncap) != cudaSuccess) goto out;
        if (s->sess_bytes && cudaMemcpy(nb, s->d_sessions, s->sess_bytes, cudaMemcpyDeviceToDevice) != cudaSuccess) {
            cudaFree(nb);
            goto out;
        }
        if (s->d_sessions) {
            cudaMemset(s->d_sessions, 0, s->sess_cap);
            cudaFree(s->d_sessions);
        }
        s->d_sessions = nb;
        s->sess_cap = ncap;
    }
    if (s->nsess == s->sess_arr_cap) {
        size_t nc = s->sess_arr_cap ? 2 * s->sess_arr_cap : 64;
        uint32_t *a = (uint32_t *)realloc(s->sess_off, nc * 4), *b = a ? (uint32_t *)realloc(s->sess_len, nc * 4) : NULL;
        if (!a || !b) { if (a) s->sess_off = a; goto out; }
        s->sess_off = a;
        s->sess_len = b;
        s->sess_arr_cap = nc;
    }
    if (seed_len && cudaMemcpy(s->d_sessions + s->sess_bytes, seed, seed_len, cudaMemcpyHostToDevice) != cudaSuccess)
        goto out;
    s->sess_off[s->nsess] = (uint32_t)s->sess_bytes;
    s->sess_len[s->nsess] = (uint32_t)seed_len;
    s->sess_bytes += seed_len;
    id = (int)s->nsess++;
out:
    pthread_mutex_unlock(&s->mu);
    return id;
}

int pose_b200_server_prepare(pose_b200_server_t *s, const pose_hbm_topo_t *topo)
{
    if (!s || !topo) return -1;
    (void)req_is_deep(s, topo); /* builds the depth kernel's records of a deep topology */
    return 0;
}

int64_t pose_b200_server_submit(pose_b200_server_t *s, const pose_hbm_topo_t *topo, int session, void *dev_ptr,
                                size_t len, uint64_t region_block_offset)
{
    if (!s || !topo) return -1;
    const double t_submit = now_ms(); /* latency counts from the call, lock wait included */
    /* before the lock: a deep topology's first request builds its records */
    const int deep = req_is_deep(s, topo);
    pthread_mutex_lock(&s->mu);
    int64_t id = -1;
    if (session < 0 || (size_t)session >= s->nsess) {
        fprintf(stderr, "pose_b200_server_submit: unknown session %d\n", session);
        goto out;
    }
    {
        pb_topo_internal_t ti;
        if (pb_topo_internal(topo, &ti) != 0 || ti.device != s->device) {
            fprintf(stderr, "pose_b200_server_submit: topology of another device\n");
            goto out;
        }
        if ((uint64_t)ti.view.pool * 32 > s->arena_bytes) {
            fprintf(stderr, "pose_b200_server_submit: one chunk copy needs %llu bytes of scratch, the arena has %llu\n",
                    (unsigned long long)ti.view.pool * 32, (unsigned long long)s->arena_bytes);
            goto out;
        }
        if (len / ti.super_bytes && !dev_ptr) {
            fprintf(stderr, "pose_b200_server_submit: NULL buffer\n");
            goto out;
        }
    }
    if (s->nreqs == s->reqs_cap) {
        size_t nc = s->reqs_cap ? 2 * s->reqs_cap : 1024;
        sreq_t *nr = (sreq_t *)realloc(s->reqs, nc * sizeof(sreq_t));
        if (!nr) goto out;
        s->reqs = nr;
        s->reqs_cap = nc;
    }
    sreq_t *r = &s->reqs[s->nreqs];
    memset(r, 0, sizeof(*r));
    r->topo = topo;
    r->dev_ptr = dev_ptr;
    r->len = len;
    r->rbo = region_block_offset;
    r->session = session;
    r->deep = deep;
    r->t_submit = t_submit;
    id = (int64_t)s->nreqs++;
    pthread_cond_broadcast(&s->cv);
out:
    pthread_mutex_unlock(&s->mu);
    return id;
}

int pose_b200_server_wait(pose_b200_server_t *s, int64_t ticket, double *queue_ms, double *total_ms)
{
    if (!s || ticket < 0) return -1;
    pthread_mutex_lock(&s->mu);
    if ((size_t)ticket >= s->nreqs) { pthread_mutex_unlock(&s->mu); return -1; }
    while (s->reqs[ticket].state < 2) pthread_cond_wait(&s->cv, &s->mu);
    sreq_t r = s->reqs[ticket];
    pthread_mutex_unlock(&s->mu);
    if (queue_ms) *queue_ms = r.t_start - r.t_submit;
    if (total_ms) *total_ms = r.t_done - r.t_submit;
    return r.state == 2 ? 0 : -1;
}

int pose_b200_server_query(pose_b200_server_t *s, int64_t ticket)
{
    if (!s || ticket < 0) return -1;
    pthread_mutex_lock(&s->mu);
    int st = (size_t)ticket < s->nreqs ? s->reqs[ticket].state : 3;
    pthread_mutex_unlock(&s->mu);
    return st == 2 ? 1 : st == 3 ? -1 : 0;
}

void pose_b200_server_stats(pose_b200_server_t *s, uint64_t *submitted, uint64_t *waves, uint64_t *scratch_bytes)
{
    if (!s) return;
    pthread_mutex_lock(&s->mu);
    if (submitted) *submitted = s->nreqs;
    if (waves) *waves = s->waves_launched;
    if (scratch_bytes) *scratch_bytes = s->arena_bytes;
    pthread_mutex_unlock(&s->mu);
}

void pose_b200_server_destroy(pose_b200_server_t *s)
{
    if (!s) return;
    pthread_mutex_lock(&s->mu);
    s->running = 0;
    pthread_cond_broadcast(&s->cv);
    pthread_mutex_unlock(&s->mu);
    pthread_join(s->thread, NULL);
    for (uint32_t i = 0; i < PB_SERVER_MAX_WAVES + PB_SERVER_MAX_DEEP; i++) {
        wave_t *wv = i < PB_SERVER_MAX_WAVES ? &s->waves[i] : &s->deeps[i - PB_SERVER_MAX_WAVES];
        cudaStreamSynchronize(wv->stream);
        cudaStreamDestroy(wv->stream);
        cudaEventDestroy(wv->done);
        cudaFree(wv->d_tables);
        if (wv->h_done) cudaFreeHost(wv->h_done);
        if (wv->h_stage) cudaFreeHost(wv->h_stage);
        free(wv->reqs);
        free(wv->need);
    }
    if (s->d_arena) {
        cudaMemset(s->d_arena, 0, s->arena_bytes);
        cudaFree(s->d_arena);
    }
    if (s->d_sessions) {
        cudaMemset(s->d_sessions, 0, s->sess_cap);
        cudaFree(s->d_sessions);
    }
    free(s->sess_off);
    free(s->sess_len);
    free(s->reqs);
    pthread_mutex_destroy(&s->mu);
    pthread_cond_destroy(&s->cv);
    free(s);
}
