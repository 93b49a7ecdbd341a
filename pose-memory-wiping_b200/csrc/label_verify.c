/*
 * label_verify.c — the verifier's recompute on the GPU.
 *
 * A PoSE verifier checks a prover's stored labels by recomputing them.  The
 * reference does this on the CPU: pose_graph_challenge labels the whole
 * graph for one challenged rank (common/src/graph.c:1019-1042), and
 * disk-wipe-bench's sampled verify recomputes whole super-chunks with the
 * in-place CPU labeler, one after the other, at tens of seconds each at
 * chunk_blocks = 2^17 (tools/disk-wipe-bench/disk_wipe_bench.cu:300-366).
 * Here every recompute runs on the labeling kernels: one challenge through
 * the topology's single-call path with its chunk seed taken as given, many
 * challenges or samples as one batched launch per group of distinct chunks,
 * and the comparison of a sample against what was read back happens on the
 * device while the next group's reads are already done.
 */
#include "kernels.h"
#include "dev_alloc.h"
#include "pose_b200.h"
#include "topo_internal.h"

#include <nvtx3/nvToolsExt.h>
#include <cuda_runtime_api.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define PB_CHALLENGE_GROUP_BYTES ((uint64_t)4 << 30) /* labels recomputed per batched launch */
#define PB_VERIFY_GROUP_BYTES ((uint64_t)1 << 30)    /* samples read and recomputed per group */

static double now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return 1e3 * (double)ts.tv_sec + 1e-6 * (double)ts.tv_nsec;
}

static void add_stats(pose_b200_stats_t *acc, const pose_b200_stats_t *st)
{
    acc->kernel_ms += st->kernel_ms;
    acc->super_chunks += st->super_chunks;
    acc->units += st->units;
    acc->nodes += st->nodes;
    acc->kernel_launches += st->kernel_launches ? st->kernel_launches : 1;
    if (st->scratch_bytes > acc->scratch_bytes) acc->scratch_bytes = st->scratch_bytes;
    acc->team_warps = st->team_warps;
    acc->units_per_team = st->units_per_team;
    acc->teams = st->teams;
    acc->used_cv0_table = st->used_cv0_table;
    acc->kernel = st->kernel;
}

int pose_b200_challenge(const pose_hbm_topo_t *topo, const uint8_t *seed, size_t seed_len,
                        uint64_t challenge_idx, uint8_t out[32])
{
    pb_topo_internal_t ti;
    if (!topo || pb_topo_internal(topo, &ti) != 0) { fprintf(stderr, "pose_b200_challenge: NULL topology\n"); return -1; }
    if (!seed || seed_len < 32 || !out) {
        fprintf(stderr, "pose_b200_challenge: the graph seed must be 32 bytes\n");
        return -1;
    }
    if (challenge_idx >= ti.cb) return -1; /* graph.c:1023 */
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != ti.device && cudaSetDevice(ti.device) != cudaSuccess) return -1;
    int rc = -1;
    void *buf = NULL;
    if (pb_dev_malloc(&buf, ti.super_bytes) != cudaSuccess) {
        fprintf(stderr, "pose_b200_challenge: %s\n", cudaGetErrorString(cudaGetLastError()));
        goto out;
    }
    if (pb_topo_label_raw(topo, seed, buf, ti.super_bytes, NULL, NULL) != 0) goto out;
    if (cudaMemcpy(out, (const uint8_t *)buf + 32 * challenge_idx, 32, cudaMemcpyDeviceToHost) != cudaSuccess) {
        fprintf(stderr, "pose_b200_challenge: %s\n", cudaGetErrorString(cudaGetLastError()));
        goto out;
    }
    rc = 0;
out:
    if (buf) {
        cudaMemset(buf, 0, ti.super_bytes);
        cudaFree(buf);
    }
    if (prev >= 0 && prev != ti.device) cudaSetDevice(prev);
    return rc;
}

typedef struct {
    uint64_t chunk; /* chunk index */
    uint64_t k;     /* position in the caller's list */
} chal_t;

static int cmp_chal(const void *a, const void *b)
{
    const chal_t *x = (const chal_t *)a, *y = (const chal_t *)b;
    if (x->chunk != y->chunk) return x->chunk < y->chunk ? -1 : 1;
    return x->k < y->k ? -1 : x->k > y->k;
}

/* Recompute chunks[0..n) of one session into consecutive super-chunks of
 * d_work (one batched launch). */
static int recompute(const pose_hbm_topo_t *topo, const pb_topo_internal_t *ti, const uint8_t *seed, size_t seed_len,
                     const uint64_t *chunks, size_t n, uint8_t *d_work, const pose_b200_sched_t *sched,
                     pose_b200_stats_t *st)
{
    pose_b200_request_t *r = (pose_b200_request_t *)calloc(n, sizeof(*r));
    if (!r) return -1;
    for (size_t i = 0; i < n; i++) {
        r[i].topo = topo;
        r[i].session_seed = seed;
        r[i].seed_len = seed_len;
        r[i].hbm_dev_ptr = d_work + i * ti->super_bytes;
        r[i].hbm_len = ti->super_bytes;
        r[i].region_block_offset = chunks[i] * (uint64_t)ti->cb;
    }
    int rc = pose_b200_label_batch(r, n, sched, st);
    free(r);
    return rc;
}

static int pose_b200_challenge_blocks_impl(const pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                               const uint64_t *blocks, size_t n, uint8_t *out,
                               const pose_b200_sched_t *sched, pose_b200_stats_t *stats)
{
    if (stats) memset(stats, 0, sizeof(*stats));
    pb_topo_internal_t ti;
    if (!topo || pb_topo_internal(topo, &ti) != 0) { fprintf(stderr, "pose_b200_challenge_blocks: NULL topology\n"); return -1; }
    if (n == 0) return 0;
    if (!blocks || !out || (!session_seed && seed_len)) {
        fprintf(stderr, "pose_b200_challenge_blocks: NULL argument\n");
        return -1;
    }
    if (n > 0xFFFFFFFFull) { fprintf(stderr, "pose_b200_challenge_blocks: too many challenges\n"); return -1; }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != ti.device && cudaSetDevice(ti.device) != cudaSuccess) return -1;

    const double t0 = now_ms();
    int rc = -1;
    chal_t *c = (chal_t *)malloc(n * sizeof(*c));
    uint64_t *chunks = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint64_t *src = (uint64_t *)malloc(n * sizeof(uint64_t));
    uint64_t *slot_of = (uint64_t *)malloc(n * sizeof(uint64_t)); /* group-local super-chunk of each sorted entry */
    uint8_t *d_work = NULL, *d_out = NULL;
    uint64_t *d_src = NULL;
    uint8_t *h_out = NULL;
    uint64_t group_cap = PB_CHALLENGE_GROUP_BYTES / ti.super_bytes;
    if (group_cap == 0) group_cap = 1;
    pose_b200_stats_t acc;
    memset(&acc, 0, sizeof(acc));
    if (!c || !chunks || !src || !slot_of) { fprintf(stderr, "pose_b200_challenge_blocks: out of host memory\n"); goto out; }
    for (size_t k = 0; k < n; k++) {
        c[k].chunk = blocks[k] / ti.cb;
        c[k].k = k;
    }
    qsort(c, n, sizeof(*c), cmp_chal);
    {
        uint64_t distinct = 0;
        for (size_t i = 0; i < n; i++)
            if (i == 0 || c[i].chunk != c[i - 1].chunk) distinct++;
        const uint64_t wchunks = distinct < group_cap ? distinct : group_cap;
        if (pb_dev_malloc((void **)&d_work, wchunks * ti.super_bytes) != cudaSuccess ||
            pb_dev_malloc((void **)&d_out, n * 32) != cudaSuccess ||
            pb_dev_malloc((void **)&d_src, n * sizeof(uint64_t)) != cudaSuccess) {
            fprintf(stderr, "pose_b200_challenge_blocks: device allocation failed: %s\n",
                    cudaGetErrorString(cudaGetLastError()));
            goto out;
        }
    }
    /* walk the sorted challenges in groups of at most group_cap distinct chunks */
    for (size_t i = 0; i < n;) {
        size_t j = i, nch = 0;
        while (j < n) {
            if (j == i || c[j].chunk != c[j - 1].chunk) {
                if (nch == group_cap) break;
                chunks[nch++] = c[j].chunk;
            }
            slot_of[j] = nch - 1;
            j++;
        }
        pose_b200_stats_t st;
        if (recompute(topo, &ti, session_seed, seed_len, chunks, nch, d_work, sched, &st) != 0) goto out;
        add_stats(&acc, &st);
        /* gather the group's labels into their final positions */
        for (size_t q = i; q < j; q++) src[q - i] = slot_of[q] * ti.cb + blocks[c[q].k] % ti.cb;
        if (cudaMemcpy(d_src, src, (j - i) * sizeof(uint64_t), cudaMemcpyHostToDevice) != cudaSuccess ||
            pb_dev_gather_labels(d_work, d_src, (uint32_t)(j - i), d_out + 32 * i, 0) != 0 ||
            cudaDeviceSynchronize() != cudaSuccess) {
            fprintf(stderr, "pose_b200_challenge_blocks: gather failed: %s\n", cudaGetErrorString(cudaGetLastError()));
            goto out;
        }
        i = j;
    }
    h_out = (uint8_t *)malloc(n * 32);
    if (!h_out || cudaMemcpy(h_out, d_out, n * 32, cudaMemcpyDeviceToHost) != cudaSuccess) {
        fprintf(stderr, "pose_b200_challenge_blocks: read-back failed\n");
        goto out;
    }
    for (size_t i = 0; i < n; i++) memcpy(out + 32 * c[i].k, h_out + 32 * i, 32);
    rc = 0;
out:
    if (d_work) {
        uint64_t distinct = 0;
        for (size_t i = 0; c && i < n; i++)
            if (i == 0 || c[i].chunk != c[i - 1].chunk) distinct++;
        cudaMemset(d_work, 0, (distinct < group_cap ? distinct : group_cap) * ti.super_bytes);
    }
    if (d_out) cudaMemset(d_out, 0, n * 32);
    cudaDeviceSynchronize();
    cudaFree(d_work);
    cudaFree(d_out);
    cudaFree(d_src);
    free(c); free(chunks); free(src); free(slot_of); free(h_out);
    if (stats) {
        *stats = acc;
        stats->total_ms = now_ms() - t0;
    }
    if (prev >= 0 && prev != ti.device) cudaSetDevice(prev);
    return rc;
}

int pose_b200_challenge_blocks(const pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                               const uint64_t *blocks, size_t n, uint8_t *out,
                               const pose_b200_sched_t *sched, pose_b200_stats_t *stats)
{
    nvtxRangePushA("pose_b200: challenge blocks");
    int rc = pose_b200_challenge_blocks_impl(topo, session_seed, seed_len, blocks, n, out, sched, stats);
    nvtxRangePop();
    return rc;
}

/* ── sampled verify ──────────────────────────────────────────────────────── */

typedef struct {
    const pose_hbm_topo_t *topo;
    const pb_topo_internal_t *ti;
    const uint8_t *seed;
    size_t seed_len;
    const uint64_t *chunks;
    size_t n;
    uint8_t *d_work;
    const pose_b200_sched_t *sched;
    pose_b200_stats_t st;
    int rc;
} recompute_job_t;

static void *recompute_thread(void *arg)
{
    recompute_job_t *j = (recompute_job_t *)arg;
    cudaSetDevice(j->ti->device);
    j->rc = recompute(j->topo, j->ti, j->seed, j->seed_len, j->chunks, j->n, j->d_work, j->sched, &j->st);
    return NULL;
}

static int pose_b200_verify_sampled_impl(const pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                             uint64_t wipe_len, uint64_t samples, pose_b200_read_fn read, void *read_ctx,
                             uint64_t *checked_out, uint64_t *mism_out, uint64_t *first_bad,
                             const pose_b200_sched_t *sched, pose_b200_stats_t *stats)
{
    if (stats) memset(stats, 0, sizeof(*stats));
    if (checked_out) *checked_out = 0;
    if (mism_out) *mism_out = 0;
    pb_topo_internal_t ti;
    if (!topo || pb_topo_internal(topo, &ti) != 0 || !read) {
        fprintf(stderr, "pose_b200_verify_sampled: NULL topology or read function\n");
        return -1;
    }
    if (!session_seed && seed_len) { fprintf(stderr, "pose_b200_verify_sampled: NULL seed\n"); return -1; }
    const uint64_t sb = ti.super_bytes;
    const uint64_t n_super = wipe_len / sb;
    if (n_super == 0) { fprintf(stderr, "pose_b200_verify_sampled: nothing labeled to verify\n"); return -1; }
    const uint64_t samples_in = samples;
    if (samples == 0) samples = 1;
    if (samples > n_super) samples = n_super;
    if (first_bad)
        for (uint64_t k = 0; k < samples_in && k < samples; k++) first_bad[k] = UINT64_MAX;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != ti.device && cudaSetDevice(ti.device) != cudaSuccess) return -1;

    const double t0 = now_ms();
    uint64_t group = PB_VERIFY_GROUP_BYTES / sb;
    if (group == 0) group = 1;
    if (group > samples) group = samples;
    int rc = -1;
    uint64_t checked = 0, mism = 0;
    uint64_t *chunks = (uint64_t *)malloc(group * sizeof(uint64_t));
    unsigned long long *h_bad = NULL, *d_bad = NULL;
    uint8_t *h_disk = NULL, *d_disk = NULL, *d_ref = NULL;
    cudaStream_t s = NULL;
    pose_b200_stats_t acc;
    memset(&acc, 0, sizeof(acc));
    if (!chunks) goto out;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost((void **)&h_disk, group * sb) != cudaSuccess ||
        cudaMallocHost((void **)&h_bad, group * sizeof(unsigned long long)) != cudaSuccess ||
        pb_dev_malloc((void **)&d_disk, group * sb) != cudaSuccess ||
        pb_dev_malloc((void **)&d_ref, group * sb) != cudaSuccess ||
        pb_dev_malloc((void **)&d_bad, group * sizeof(unsigned long long)) != cudaSuccess) {
        fprintf(stderr, "pose_b200_verify_sampled: buffers of %llu bytes failed: %s\n",
                (unsigned long long)(group * sb), cudaGetErrorString(cudaGetLastError()));
        goto out;
    }
    for (uint64_t k0 = 0; k0 < samples; k0 += group) {
        const uint64_t g = samples - k0 < group ? samples - k0 : group;
        for (uint64_t i = 0; i < g; i++) {
            const uint64_t k = k0 + i;
            chunks[i] = samples == 1 ? 0 : k * (n_super - 1) / (samples - 1);
        }
        /* the GPU recomputes this group while the host reads it back */
        recompute_job_t job;
        memset(&job, 0, sizeof(job));
        job.topo = topo;
        job.ti = &ti;
        job.seed = session_seed;
        job.seed_len = seed_len;
        job.chunks = chunks;
        job.n = (size_t)g;
        job.d_work = d_ref;
        job.sched = sched;
        job.rc = -1;
        pthread_t th;
        const int threaded = pthread_create(&th, NULL, recompute_thread, &job) == 0;
        if (!threaded) recompute_thread(&job);
        int rerr = 0;
        for (uint64_t i = 0; i < g && !rerr; i++) {
            if (read(read_ctx, h_disk + i * sb, sb, chunks[i] * sb) != 0) {
                fprintf(stderr, "pose_b200_verify_sampled: read of super-chunk %llu failed\n",
                        (unsigned long long)chunks[i]);
                rerr = 1;
            }
        }
        if (!rerr && (cudaMemcpyAsync(d_disk, h_disk, g * sb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
                      cudaMemsetAsync(d_bad, 0xFF, g * sizeof(unsigned long long), s) != cudaSuccess)) {
            fprintf(stderr, "pose_b200_verify_sampled: upload failed: %s\n", cudaGetErrorString(cudaGetLastError()));
            rerr = 1;
        }
        if (threaded) pthread_join(th, NULL);
        if (rerr || job.rc != 0) goto out;
        add_stats(&acc, &job.st);
        if (pb_dev_compare_blocks(d_ref, d_disk, g * ti.cb, ti.cb, d_bad, (uint32_t)ti.sms * 8, s) != 0 ||
            cudaMemcpyAsync(h_bad, d_bad, g * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            fprintf(stderr, "pose_b200_verify_sampled: compare failed: %s\n", cudaGetErrorString(cudaGetLastError()));
            goto out;
        }
        for (uint64_t i = 0; i < g; i++) {
            checked++;
            if (first_bad && k0 + i < samples_in) first_bad[k0 + i] = h_bad[i];
            if (h_bad[i] != ~0ull) {
                mism++;
                if (mism <= 3)
                    fprintf(stderr, "  verify: MISMATCH super-chunk %llu (block %llu)\n",
                            (unsigned long long)chunks[i], (unsigned long long)h_bad[i]);
            }
        }
    }
    rc = 0;
out:
    if (checked_out) *checked_out = checked;
    if (mism_out) *mism_out = mism;
    if (d_ref) cudaMemset(d_ref, 0, group * sb);
    cudaDeviceSynchronize();
    cudaFree(d_ref); cudaFree(d_disk); cudaFree(d_bad);
    if (h_disk) cudaFreeHost(h_disk);
    if (h_bad) cudaFreeHost(h_bad);
    if (s) cudaStreamDestroy(s);
    free(chunks);
    if (stats) {
        *stats = acc;
        stats->total_ms = now_ms() - t0;
        stats->kernel_ms = acc.kernel_ms;
    }
    if (prev >= 0 && prev != ti.device) cudaSetDevice(prev);
    return rc;
}

int pose_b200_verify_sampled(const pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                             uint64_t wipe_len, uint64_t samples, pose_b200_read_fn read, void *read_ctx,
                             uint64_t *checked_out, uint64_t *mism_out, uint64_t *first_bad,
                             const pose_b200_sched_t *sched, pose_b200_stats_t *stats)
{
    nvtxRangePushA("pose_b200: sampled verify");
    int rc = pose_b200_verify_sampled_impl(topo, session_seed, seed_len, wipe_len, samples, read, read_ctx, checked_out, mism_out, first_bad, sched, stats);
    nvtxRangePop();
    return rc;
}
