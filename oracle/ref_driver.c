/*
 * ref_driver.c — TEST INFRASTRUCTURE ONLY (part of the oracle).
 *
 * A thin multi-threaded driver around the reference's own CPU in-place
 * labeler, compiled together with the reference sources (common/src/hash.c,
 * common/src/graph.c, common/vendor/blake3/) into oracle/_ref/libposeref.so
 * by oracle/Makefile.  It adds no labeling logic of its own: every super-chunk
 * is produced by the reference's pose_graph_label_region_pooled_inplace
 * (common/src/graph.c:1604-1689), one call per super-chunk, from `threads`
 * host threads.  The reference is built with POSE_REGION_THREADS=1 so each
 * call runs on the thread that made it and the thread count is chosen at run
 * time (the reference's own pool fixes it at compile time,
 * common/include/graph.h:61-63).
 *
 * The chunk index of super-chunk j is the reference's
 * (region_block_offset + j*cb) / cb (common/src/graph.c:1646-1649): calling
 * the reference on one super-chunk at block offset rbo + j*cb derives exactly
 * that index.
 *
 * Never linked into the product library.
 */
#include "graph.h"
#include "hash.h"

#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    const uint8_t *seed;
    size_t seed_len;
    uint32_t cb;
    uint8_t *out;
    uint64_t num_super;
    uint64_t rbo;
    atomic_ullong next;
    atomic_int rc;
} ref_job_t;

static void *ref_worker(void *arg)
{
    ref_job_t *job = (ref_job_t *)arg;
    size_t super_bytes = (size_t)job->cb * POSE_HASH_BYTES;
    uint8_t *scratch[POSE_REGION_THREADS];
    scratch[0] = (uint8_t *)malloc(pose_graph_scratch_bytes_inplace(job->cb));
    pose_graph_pool_t *pool = pose_graph_pool_create();
    if (!scratch[0] || !pool) {
        atomic_store(&job->rc, -1);
        free(scratch[0]);
        pose_graph_pool_destroy(pool);
        return NULL;
    }
    for (;;) {
        uint64_t j = atomic_fetch_add(&job->next, 1);
        if (j >= job->num_super || atomic_load(&job->rc) != 0) break;
        int rc = pose_graph_label_region_pooled_inplace(
            job->seed, job->seed_len, job->out + j * super_bytes, super_bytes,
            job->rbo + j * (uint64_t)job->cb, scratch, pool, POSE_HASH_BLAKE3,
            job->cb);
        if (rc != 0) atomic_store(&job->rc, rc);
    }
    free(scratch[0]);
    pose_graph_pool_destroy(pool);
    return NULL;
}

/* Label num_super consecutive super-chunks starting at block offset rbo into
 * out (num_super * cb * 32 bytes) with `threads` host threads.  Returns 0 on
 * success, non-zero on error. */
int ref_label_super_chunks(const uint8_t *seed, size_t seed_len, uint32_t cb,
                           uint8_t *out, uint64_t num_super, uint64_t rbo,
                           int threads)
{
    if (threads < 1) threads = 1;
    if ((uint64_t)threads > num_super) threads = (int)num_super;
    if (num_super == 0) return 0;
    ref_job_t job;
    job.seed = seed;
    job.seed_len = seed_len;
    job.cb = cb;
    job.out = out;
    job.num_super = num_super;
    job.rbo = rbo;
    atomic_init(&job.next, 0);
    atomic_init(&job.rc, 0);
    pthread_t *tids = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    if (!tids) return -1;
    int started = 0;
    for (int i = 0; i < threads - 1; i++) {
        if (pthread_create(&tids[i], NULL, ref_worker, &job) != 0) break;
        started++;
    }
    ref_worker(&job);
    for (int i = 0; i < started; i++) pthread_join(tids[i], NULL);
    free(tids);
    return atomic_load(&job.rc);
}

/* Per-node scaffold labels of one chunk in node-id order (count * 32 bytes),
 * produced with the reference's own pose_graph_edges topology
 * (common/src/graph.c:1044-1100) and pose_label_node (common/src/hash.c:110),
 * i.e. the label every node of do_label's scaffold buffer holds
 * (common/src/graph.c:575-645).  Returns the node count, or 0 on error. */
uint64_t ref_scaffold_labels(const uint8_t *chunk_seed, uint32_t cb,
                             uint8_t *labels, uint64_t cap_nodes)
{
    pose_node_t *nodes = NULL;
    uint64_t count = 0;
    if (pose_graph_edges(cb, &nodes, &count) != 0) return 0;
    if (count > cap_nodes) { free(nodes); return 0; }
    uint8_t desc[POSE_HASH_BYTES];
    pose_graph_descriptor(desc, cb, (uint64_t)pose_graph_parameter_n(cb));
    for (uint64_t id = 0; id < count; id++) {
        const pose_node_t *nd = &nodes[id];
        const uint8_t *p0 = nd->num_preds >= 1 ? labels + nd->pred[0] * 32 : NULL;
        const uint8_t *p1 = nd->num_preds >= 2 ? labels + nd->pred[1] * 32 : NULL;
        pose_label_node(labels + id * 32, nd->num_preds == 0, id, p0, p1,
                        chunk_seed, desc, POSE_HASH_BLAKE3);
    }
    free(nodes);
    return count;
}

/* Flattened copy of pose_graph_edges for the Python side: np[count],
 * p0[count], p1[count] (0 when absent), rank[count] (-1 = internal). */
uint64_t ref_edges(uint32_t cb, uint8_t *np, uint32_t *p0, uint32_t *p1,
                   int32_t *rank, uint64_t cap_nodes)
{
    pose_node_t *nodes = NULL;
    uint64_t count = 0;
    if (pose_graph_edges(cb, &nodes, &count) != 0) return 0;
    if (count > cap_nodes) { free(nodes); return 0; }
    for (uint64_t id = 0; id < count; id++) {
        np[id] = (uint8_t)nodes[id].num_preds;
        p0[id] = nodes[id].num_preds >= 1 ? (uint32_t)nodes[id].pred[0] : 0;
        p1[id] = nodes[id].num_preds >= 2 ? (uint32_t)nodes[id].pred[1] : 0;
        rank[id] = nodes[id].challenge_rank;
    }
    free(nodes);
    return count;
}
