/*
 * label_stream.c — labeling straight into a host sink, with the device-to-
 * host copy and the sink overlapped with the labeling of the next window.
 *
 * The reference's disk worker labels an HBM window, then copies it to a
 * pinned stage and writes it, strictly one after the other
 * (tools/disk-wipe-bench/disk_wipe_bench.cu:646-697).  Here the region is cut
 * into windows of whole super-chunks labelled alternately into two device
 * buffers; a worker thread copies each finished window into one of two pinned
 * host buffers on its own stream and hands it to the sink, while the calling
 * thread already labels the next window.  The sink has the shape of the
 * reference's pose_label_sink_fn (common/include/graph.h:244-245) and, as
 * there, may be called from a worker thread.
 */
#include "pose_b200.h"
#include "dev_alloc.h"

#include <nvtx3/nvToolsExt.h>
#include <cuda_runtime_api.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
    pthread_mutex_t mu;
    pthread_cond_t cv;
    /* job handed to the worker (valid when posted) */
    int posted, quit;
    int buf;
    size_t len;
    uint64_t off;
    /* per buffer: 1 while the worker still uses it */
    int busy[2];
    int error;
    double d2h_ms, sink_ms;
    /* resources */
    uint8_t *dev[2], *host[2];
    cudaStream_t stream;
    int device;
    pose_b200_sink_fn sink;
    void *ctx;
} stream_state_t;

static double now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return 1e3 * (double)ts.tv_sec + 1e-6 * (double)ts.tv_nsec;
}

static void *sink_worker(void *arg)
{
    stream_state_t *s = (stream_state_t *)arg;
    cudaSetDevice(s->device);
    pthread_mutex_lock(&s->mu);
    for (;;) {
        while (!s->posted && !s->quit) pthread_cond_wait(&s->cv, &s->mu);
        if (!s->posted && s->quit) break;
        int i = s->buf;
        size_t len = s->len;
        uint64_t off = s->off;
        s->posted = 0;
        pthread_cond_broadcast(&s->cv);
        pthread_mutex_unlock(&s->mu);

        int err = 0;
        double t0 = now_ms();
        if (cudaMemcpyAsync(s->host[i], s->dev[i], len, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess) {
            fprintf(stderr, "pose_b200_label_stream: D2H copy failed: %s\n", cudaGetErrorString(cudaGetLastError()));
            err = -1;
        }
        double t1 = now_ms();
        if (!err && s->sink(s->ctx, s->host[i], len, off) != 0) {
            fprintf(stderr, "pose_b200_label_stream: sink failed at offset %llu\n", (unsigned long long)off);
            err = -1;
        }
        double t2 = now_ms();

        pthread_mutex_lock(&s->mu);
        s->d2h_ms += t1 - t0;
        s->sink_ms += t2 - t1;
        if (err) s->error = 1;
        s->busy[i] = 0;
        pthread_cond_broadcast(&s->cv);
    }
    pthread_mutex_unlock(&s->mu);
    return NULL;
}

static int pose_b200_label_stream_impl(const pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                           uint64_t region_bytes, uint64_t region_block_offset, uint64_t byte_offset,
                           size_t window_bytes, pose_b200_sink_fn sink, void *sink_ctx,
                           const pose_b200_sched_t *sched, pose_b200_stats_t *stats)
{
    if (stats) memset(stats, 0, sizeof(*stats));
    if (!topo || !sink) {
        fprintf(stderr, "pose_b200_label_stream: NULL topology or sink\n");
        return -1;
    }
    uint32_t cb = 0;
    pose_b200_topo_info(topo, &cb, NULL, NULL, NULL, NULL);
    const uint64_t sb = (uint64_t)cb * 32;
    const uint64_t nsuper = region_bytes / sb;
    if (nsuper == 0) return 0;
    uint64_t W = window_bytes / sb;
    if (W == 0) W = 1;
    if (W > nsuper) W = nsuper;
    const uint64_t wbytes = W * sb;

    stream_state_t s;
    memset(&s, 0, sizeof(s));
    pthread_mutex_init(&s.mu, NULL);
    pthread_cond_init(&s.cv, NULL);
    s.sink = sink;
    s.ctx = sink_ctx;
    cudaGetDevice(&s.device);
    int rc = -1, started = 0;
    pthread_t th;
    double t0 = now_ms(), kernel_ms = 0, label_ms = 0;
    uint64_t nodes = 0;
    uint32_t launches = 0;
    pose_b200_stats_t last;
    memset(&last, 0, sizeof(last));

    for (int i = 0; i < 2; i++) {
        if (pb_dev_malloc((void **)&s.dev[i], wbytes) != cudaSuccess ||
            cudaMallocHost((void **)&s.host[i], wbytes) != cudaSuccess) {
            fprintf(stderr, "pose_b200_label_stream: window buffers of %llu bytes failed\n",
                    (unsigned long long)wbytes);
            goto out;
        }
    }
    if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess) goto out;
    if (pthread_create(&th, NULL, sink_worker, &s) != 0) goto out;
    started = 1;

    for (uint64_t k = 0, first = 0; first < nsuper; k++, first += W) {
        const int i = (int)(k & 1);
        const uint64_t n = nsuper - first < W ? nsuper - first : W;
        pthread_mutex_lock(&s.mu);
        while (s.busy[i] && !s.error) pthread_cond_wait(&s.cv, &s.mu);
        int err = s.error;
        pthread_mutex_unlock(&s.mu);
        if (err) goto out;
        double l0 = now_ms();
        pose_b200_stats_t st;
        if (pose_b200_topo_label(topo, session_seed, seed_len, s.dev[i], n * sb,
                                 region_block_offset + first * (uint64_t)cb, sched, &st) != 0)
            goto out;
        label_ms += now_ms() - l0;
        kernel_ms += st.kernel_ms;
        nodes += st.nodes;
        launches += st.kernel_launches;
        last = st;
        pthread_mutex_lock(&s.mu);
        while (s.posted) pthread_cond_wait(&s.cv, &s.mu);
        s.busy[i] = 1;
        s.buf = i;
        s.len = n * sb;
        s.off = byte_offset + first * sb;
        s.posted = 1;
        pthread_cond_broadcast(&s.cv);
        pthread_mutex_unlock(&s.mu);
    }
    pthread_mutex_lock(&s.mu);
    while ((s.posted || s.busy[0] || s.busy[1]) && !s.error) pthread_cond_wait(&s.cv, &s.mu);
    rc = s.error ? -1 : 0;
    pthread_mutex_unlock(&s.mu);

out:
    if (started) {
        pthread_mutex_lock(&s.mu);
        while (s.posted || s.busy[0] || s.busy[1]) {
            if (s.error && !s.posted) break;
            pthread_cond_wait(&s.cv, &s.mu);
        }
        s.quit = 1;
        pthread_cond_broadcast(&s.cv);
        pthread_mutex_unlock(&s.mu);
        pthread_join(th, NULL);
    }
    if (stats) {
        *stats = last;
        stats->kernel_ms = kernel_ms;
        stats->total_ms = now_ms() - t0;
        stats->super_chunks = nsuper;
        stats->units = nsuper * (last.units && last.super_chunks ? last.units / last.super_chunks : 2);
        stats->nodes = nodes;
        stats->kernel_launches = launches;
    }
    for (int i = 0; i < 2; i++) {
        cudaFree(s.dev[i]);
        if (s.host[i]) cudaFreeHost(s.host[i]);
    }
    if (s.stream) cudaStreamDestroy(s.stream);
    pthread_mutex_destroy(&s.mu);
    pthread_cond_destroy(&s.cv);
    (void)label_ms;
    return rc;
}

int pose_b200_label_stream(const pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                           uint64_t region_bytes, uint64_t region_block_offset, uint64_t byte_offset,
                           size_t window_bytes, pose_b200_sink_fn sink, void *sink_ctx,
                           const pose_b200_sched_t *sched, pose_b200_stats_t *stats)
{
    nvtxRangePushA("pose_b200: streamed labeling");
    int rc = pose_b200_label_stream_impl(topo, session_seed, seed_len, region_bytes, region_block_offset, byte_offset, window_bytes, sink, sink_ctx, sched, stats);
    nvtxRangePop();
    return rc;
}
