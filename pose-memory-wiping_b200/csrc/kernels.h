/* kernels.h — the thin C-ABI between the C11 host code and the sm_100a
 * kernels in label_kernels.cu (internal; plain C types only). */
#ifndef PB_KERNELS_H
#define PB_KERNELS_H

#include <stdint.h>
#include <cuda_runtime_api.h>

#include "topology.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Largest CTA the labeling kernel is launched with (teams of up to 16 warps). */
#define PB_CTA_THREADS 512
/* Largest CTA of the multi-topology kernel (k_label_multi is compiled for
 * three such CTAs per SM). */
#define PB_MULTI_CTA_THREADS 256
/* Dynamic shared memory of k_label / k_label_multi per thread: two staging
 * buffers of one node's record and block-0 chaining value (48 bytes each). */
#define PB_PREF_BYTES_PER_THREAD 96u

#ifdef __CUDACC__
typedef uint4 pb_u4;
#else
typedef struct { uint32_t x, y, z, w; } pb_u4;
#endif

/* Device view of one chunk_blocks' schedule. */
typedef struct {
    const pb_u4 *recs;       /* [S] packed node records, level order */
    const pb_u4 *cv0;        /* [copies * S * 2] block-0 chaining values, or NULL */
    const uint32_t *orank;   /* [S] local output rank, PB_NO_RANK otherwise */
    const uint32_t *lstart;  /* [L + 1] */
    uint32_t S, L, pool, half_w, retained;
    uint32_t desc[8];        /* graph descriptor words */
} pb_topo_view_t;

/* One launch of the labeling kernel over `nunits` units of one topology:
 * unit k is copy (k & (2^copies_log2 - 1)) of local chunk k >> copies_log2,
 * whose seed is seeds[8*chunk..] and whose persisted super-chunk starts at
 * persist + (first_super + chunk) * super_bytes. */
typedef struct {
    pb_topo_view_t topo;
    const uint32_t *seeds;
    uint8_t *persist;
    uint64_t super_bytes;
    uint64_t first_super;
    uint8_t *scratch;            /* teams * team_scratch_bytes */
    uint64_t team_scratch_bytes; /* G * pool * 32 */
    uint32_t nunits;
    uint32_t copies_log2;
    uint32_t g_log2;             /* G = 2^g_log2 units per team */
    uint32_t team_warps;         /* T warps per team */
    uint32_t nbatches;           /* ceil(nunits / G) */
    unsigned int *queue;         /* zeroed work counter */
    uint32_t fma_adds;           /* 1: additions on the FMA pipe (throughput-bound launches) */
    uint32_t one;                /* must be 1 */
} pb_label_params_t;

/* Multi-topology launch (batched sessions): batch b runs units
 * [first_unit, first_unit + count) of topology `topo`, count <= 2^glog. */
typedef struct {
    uint32_t topo, first_unit, count, glog;
} pb_mbatch_t;

typedef struct {
    uint64_t out;   /* device address of the unit's persisted super-chunk */
    uint32_t seed;  /* index of its chunk seed in the seed table */
    uint32_t copy;  /* 0 = left copy, 1 = right copy */
} pb_munit_t;

typedef struct {
    uint64_t chunk_index;
    uint32_t seed_off, seed_len; /* session seed in the seed blob */
} pb_seedjob_t;

typedef struct {
    const pb_topo_view_t *topos;
    const pb_mbatch_t *batches;
    const pb_munit_t *units;
    const uint32_t *seeds;
    uint8_t *scratch;
    uint64_t team_scratch_bytes;
    uint32_t nbatches;
    uint32_t team_warps;
    unsigned int *queue;
    uint32_t fma_adds;
    uint32_t one;
    /* optional completion signal: when a batch finishes, each of its units
     * adds 1 to req_done[unit_req[unit]] (system-scope, after a system
     * fence), so the host sees every request end as it happens */
    const uint32_t *unit_req;
    unsigned int *req_done;
} pb_multi_params_t;

int pb_dev_label_multi(const pb_multi_params_t *params, uint32_t grid, uint32_t cta_threads, cudaStream_t stream);
int pb_dev_label_multi_occupancy(uint32_t cta_threads, int *blocks_per_sm);
int pb_dev_seed_jobs(const void *jobs, uint32_t njobs, const uint8_t *blob, uint32_t *seeds, cudaStream_t stream);

/* Device view of the pipelined records (topology.h, PB_REF_*). */
typedef struct {
    const pb_u4 *recs2;      /* [2 * S] pipelined records, level order */
    const pb_u4 *cv0;        /* [copies * S * 2] block-0 chaining values (required) */
    const uint32_t *lstart;  /* [L + 1] */
    uint32_t S, L, half_w, retained;
    uint32_t csm;            /* shared-memory label slots per chunk copy */
    uint32_t gpool;          /* global label slots per chunk copy */
    uint32_t desc[8];
} pb_topo_view2_t;

/* One launch of the depth kernel k_label_ws (label_ws.cu); fields as in
 * pb_label_params_t, with the pipelined records' view. */
typedef struct {
    pb_topo_view2_t topo;
    const uint32_t *seeds;
    uint8_t *persist;
    uint64_t super_bytes;
    uint64_t first_super;
    uint8_t *scratch;
    uint64_t team_scratch_bytes; /* G * gpool * 32 */
    uint32_t nunits;
    uint32_t copies_log2;
    uint32_t g_log2;
    uint32_t team_warps;
    uint32_t nbatches;
    unsigned int *queue;
    /* k_label_wsc only: CTAs per chunk copy (a cluster), levels wider than
     * split_width shared by them, and the indices of those levels */
    uint32_t cluster;
    uint32_t split_width;
    const uint32_t *split_levels;
    uint32_t nsplit;
} pb_pipe_params_t;

/* Warp-specialised depth-regime kernel (label_ws.cu): team_warps hashing
 * warps + 1 producer warp per CTA, one chunk copy per CTA, g_log2 = 0. */
int pb_dev_label_ws(const pb_pipe_params_t *params, uint32_t grid, uint32_t cta_threads,
                    uint32_t smem_bytes, cudaStream_t stream);
int pb_dev_label_ws_occupancy(uint32_t cta_threads, uint32_t smem_bytes, int *blocks_per_sm);
/* The depth kernel with a cluster of params->cluster CTAs per chunk copy
 * (label_ws.cu, k_label_wsc): params->nunits * cluster CTAs, one copy per
 * cluster, no work queue. */
int pb_dev_label_wsc(const pb_pipe_params_t *params, uint32_t smem_bytes, cudaStream_t stream);
int pb_dev_label_wsc_max_clusters(uint32_t C, uint32_t team_warps, uint32_t smem_bytes, int *clusters);

/* Multi-unit depth kernel (label_ws.cu): k_label_ws with G = units_per_cta
 * (1 to 4) units of one topology per CTA in lockstep.  Batch b is units
 * [b * G, min(nunits, (b + 1) * G)) of `units`; unit k's global label pool
 * is scratch + (cta * G + k % G) * unit_scratch_bytes.  The
 * topology's pipelined records are built for a pool of topo.csm slots per
 * unit, and shared memory holds G such pools (pb_wsg_smem_bytes). */
typedef struct {
    pb_topo_view2_t topo;
    const pb_munit_t *units;
    const uint32_t *seeds;       /* 8 words per seed index (pb_munit_t.seed) */
    uint8_t *scratch;
    uint64_t unit_scratch_bytes; /* topo.gpool * 32 */
    uint32_t nunits;
    uint32_t units_per_cta;      /* G: 1 to 4 */
    uint32_t team_warps;         /* hashing warps: 7 or 15 */
    uint32_t nbatches;           /* ceil(nunits / G) */
    unsigned int *queue;         /* zeroed work counter */
} pb_wsg_params_t;

uint32_t pb_wsg_smem_bytes(uint32_t csm, uint32_t units_per_cta, uint32_t team_warps);
int pb_dev_label_wsg(const pb_wsg_params_t *params, uint32_t grid, uint32_t cta_threads, uint32_t smem_bytes,
                     cudaStream_t stream);
/* Raise k_label_wsg's dynamic shared memory limit to the most a CTA can
 * have and report it; before any launch or stream capture of it. */
int pb_dev_label_wsg_prepare(uint32_t *max_smem_bytes);

/* Verifier helpers (label_verify.cu).  Compare nblocks 32-byte blocks of a
 * and b, grouped blocks_per_group to a group: first_bad[g] = min over
 * mismatching blocks of their index within group g (initialise it to all
 * ones).  Gather: out[k] = the 32-byte label at block src[k] of work. */
int pb_dev_compare_blocks(const void *a, const void *b, uint64_t nblocks, uint64_t blocks_per_group,
                          unsigned long long *first_bad, uint32_t grid, cudaStream_t stream);
int pb_dev_gather_labels(const void *work, const uint64_t *src, uint32_t n, void *out, cudaStream_t stream);
/* *d_count += the nonzero bytes of buf[0, bytes) (buf 16-byte aligned), with
 * at most `grid` CTAs of 256 threads. */
int pb_dev_count_nonzero(const void *buf, uint64_t bytes, unsigned long long *d_count, uint32_t grid,
                         cudaStream_t stream);

int pb_dev_set_keys(const uint32_t ksrc[8], const uint32_t kint[8], const uint32_t kseed[8]);
int pb_dev_cv0_table(const void *recs, uint32_t S, uint32_t copies, void *cv0, cudaStream_t stream);
int pb_dev_chunk_seeds(const uint8_t *d_session_seed, uint32_t seed_len, uint64_t rbo, uint32_t cb,
                       uint32_t nchunks, uint64_t first_super, uint32_t *d_seeds,
                       cudaStream_t stream);
/* smem_bytes: dynamic shared memory per CTA, 0 = the staging area alone
 * (PB_PREF_BYTES_PER_THREAD per thread); more caps residency per SM
 * (pb_dev_label_balance_smem). */
int pb_dev_label(const pb_label_params_t *params, uint32_t grid, uint32_t cta_threads, uint32_t smem_bytes,
                 cudaStream_t stream);
int pb_dev_label_occupancy(uint32_t cta_threads, int *blocks_per_sm);
int pb_dev_label_balance_smem(uint32_t cta_threads, uint32_t per_sm, uint32_t *smem_bytes);
int pb_dev_label_single(uint32_t *d_out, int is_source, uint64_t node_index, const uint32_t *d_in,
                        int have_p0, int have_p1, cudaStream_t stream);
int pb_dev_compress_bench(uint32_t grid, uint32_t iters, uint32_t salt, uint32_t *d_sink,
                          int fma_adds, cudaStream_t stream);
int pb_dev_compress_latency(uint32_t iters, unsigned long long *d_cycles, uint32_t *d_sink,
                            cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif
