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
    uint32_t kernel;            /* 0 = automatic, 1 = basic lockstep kernel,
                                   3 = warp-specialised depth kernel (team_warps = hashing warps: 7 or 15);
                                   other values are refused */
    uint64_t scratch_cap_bytes; /* cap on the scratch pool (0 = free HBM less a margin) */
    uint32_t lane_efficiency;   /* batched launches: per-topology G reaches this lane efficiency,
                                   in percent; POSE_B200_PACK_CHAIN packs units while their chain
                                   stays within the launch's longest; 0 = automatic */
    uint32_t flags;             /* POSE_B200_BATCH_* (batched launches); 0 otherwise */
    uint32_t cluster_ctas;      /* depth kernel: CTAs per chunk copy, a thread-block cluster that
                                   shares the copy's wide levels (1 = none, 2..16); 0 = automatic */
} pose_b200_sched_t;

#define POSE_B200_PACK_CHAIN 255u
/* flags: run every request of a batch in one launch.  Without it, a batch
 * whose deepest topologies are much deeper than the rest runs them as a
 * second, concurrent launch (see pose_b200_batch_create). */
#define POSE_B200_BATCH_ONE_LAUNCH 1u

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
    uint32_t kernel;            /* 1 = basic lockstep kernel, 3 = warp-specialised depth kernel,
                                   4 = multi-topology batch kernel */
    uint32_t cluster_ctas;      /* depth kernel: CTAs per chunk copy (1 = no cluster) */
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

/* Timed-trial autotuner for one call shape.  It has no counterpart in the
 * reference; it tunes pose_graph_hbm_topo_label (common/include/gpu_label.h:
 * 80-83).  It plans every (team size, units per team) of the basic kernel
 * and the depth kernel with the schedule model and runs up to `trials`
 * (0 = 4) of them as real labeling calls on the given buffer: first the
 * modelled best of each team size and the depth kernel, then the other
 * units-per-team choices of the fastest team size; candidates modelled at
 * more than twice the cheapest are not run.  It remembers the
 * fastest: later calls on this topology with the same number of
 * super-chunks and no explicit schedule use it.  The buffer ends up holding the labels,
 * exactly as after pose_graph_hbm_topo_label.  Returns 0, or -1 on error;
 * `chosen` (may be NULL) gets the winning schedule and `stats` (may be NULL)
 * its timed call.  Same threading rule as the labeling call. */
int pose_b200_topo_autotune(pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                            void *hbm_dev_ptr, size_t hbm_len, uint64_t region_block_offset,
                            uint32_t trials, pose_b200_sched_t *chosen, pose_b200_stats_t *stats);

/* Sustained compression rate of this GPU for the labeler's instruction mix:
 * every SM full of threads chaining register-resident compressions.  Returns
 * compressions per second (0 on error); *latency_cycles gets the dependent
 * latency of one compression in SM clocks (NULL to skip). */
double pose_b200_compress_rate(uint32_t iters, double *latency_cycles);

/* ── batched labeling ────────────────────────────────────────────────────
 *
 * Extends pose_graph_hbm_topo_label (common/include/gpu_label.h:80-83) to many
 * requests at once: each request is one session seed, one topology (one
 * chunk_blocks), one device buffer and one region_block_offset, with exactly
 * the semantics of a pose_graph_hbm_topo_label call on it; all requests run
 * in ONE persistent kernel launch (teams take same-topology batches from a
 * device queue, longest first), replayed from a captured CUDA graph.  All
 * topologies must belong to the current device.  Bytes are identical to
 * labelling each request alone. */
typedef struct {
    const pose_hbm_topo_t *topo;
    const uint8_t *session_seed;
    size_t seed_len;
    void *hbm_dev_ptr;
    size_t hbm_len;
    uint64_t region_block_offset;
} pose_b200_request_t;

typedef struct pose_b200_batch pose_b200_batch_t;

/* Plan, upload and capture; NULL on error.  The requests' seeds are copied;
 * their buffers must stay valid until the batch is destroyed.  sched may fix
 * team_warps (1, 2, 4 or 8) and lane_efficiency, and cap units_per_team (the
 * largest G), max_teams and scratch_cap_bytes; what it leaves at 0 is chosen
 * by the makespan estimate.  Deep part: the requests whose topology's chain
 * (passes of an 8-warp team over one chunk copy) is at least 3/4 of the
 * deepest, when the others are shallower, run as a second launch captured
 * beside the first unless flags has POSE_B200_BATCH_ONE_LAUNCH; sched then
 * applies to the rest.  When the deep requests share one topology built with
 * its block-0 table, that launch is the multi-unit depth kernel (1, 2 or 4
 * chunk copies per CTA, at most one CTA per SM; the topology then also keeps
 * a second set of pipelined records, 32 bytes per node, built on first use).
 * Otherwise it is the lockstep kernel with 8-warp teams, units packed up to
 * 4 a team so that they hold about half the SMs' team slots.  The
 * environment variable POSE_B200_DEEP_KERNEL=0 selects the lockstep kernel
 * in every case.  With the multi-unit depth kernel, the requests of the
 * deepest remaining topology, when its chain is at least a third of the
 * deepest, run as a third launch of it (three chunk copies per CTA, on the
 * SMs the second launch leaves, its CTAs looping over their batches);
 * POSE_B200_DEEP2=0 keeps them with the rest. */
pose_b200_batch_t *pose_b200_batch_create(const pose_b200_request_t *reqs, size_t n,
                                          const pose_b200_sched_t *sched);
/* The empirical autotuner: rank the schedules sched leaves open (team size
 * 1/2/4/8 and the packing rule) by the makespan estimate, capture the best
 * `trials` of them (0 = 3), time one replay of each, and return the fastest
 * batch, already captured; *chosen (may be NULL) gets its schedule, which
 * pose_b200_batch_create reproduces, and *stats its timed replay.  Every
 * replay writes the same bytes.  NULL on error. */
pose_b200_batch_t *pose_b200_batch_autotune(const pose_b200_request_t *reqs, size_t n,
                                            const pose_b200_sched_t *sched, uint32_t trials,
                                            pose_b200_sched_t *chosen, pose_b200_stats_t *stats);
/* Replay the captured launch (synchronous).  0 on success, -1 on error. */
int pose_b200_batch_run(pose_b200_batch_t *batch, pose_b200_stats_t *stats);
/* Zero the batch's scratch and seeds, free it. */
void pose_b200_batch_destroy(pose_b200_batch_t *batch);
/* create + run + destroy. */
int pose_b200_label_batch(const pose_b200_request_t *reqs, size_t n, const pose_b200_sched_t *sched,
                          pose_b200_stats_t *stats);

/* ── streaming to a host sink ────────────────────────────────────────────
 *
 * Sink of labelled bytes, the shape of the reference's pose_label_sink_fn
 * (common/include/graph.h:244-245): called once per window with the pinned
 * host buffer holding it, its length and its absolute byte offset in the
 * target; returns 0 on success, non-zero to abort.  It is called from a
 * worker thread, one window at a time, in order. */
typedef int (*pose_b200_sink_fn)(void *ctx, const uint8_t *buf, size_t len, uint64_t off);

/* Label floor(region_bytes / (chunk_blocks*32)) super-chunks starting at
 * block offset region_block_offset (chunk index as in
 * pose_graph_hbm_topo_label) and deliver them to `sink` window by window
 * (window_bytes rounded down to whole super-chunks, at least one): window
 * k+1 is labelled on the GPU while window k is copied to pinned host memory
 * and sunk, which the reference's disk worker does one after the other
 * (tools/disk-wipe-bench/disk_wipe_bench.cu:646-697).  `off` of window k is
 * byte_offset + k*window.  Synchronous; 0 on success, -1 on error (including
 * a failing sink). */
int pose_b200_label_stream(const pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                           uint64_t region_bytes, uint64_t region_block_offset, uint64_t byte_offset,
                           size_t window_bytes, pose_b200_sink_fn sink, void *sink_ctx,
                           const pose_b200_sched_t *sched, pose_b200_stats_t *stats);

/* ── continuous-batching server ──────────────────────────────────────────
 *
 * A labeling service for many concurrent requests.  Session seeds are kept in
 * device memory; requests (the arguments of pose_graph_hbm_topo_label, with a
 * session instead of a seed) can be submitted from any thread at any time.  A
 * dispatcher thread admits pending requests whenever a slot is free and the
 * scratch arena (the HBM budget given at creation) has room, so work that
 * arrives while other work runs starts as memory frees up and overlaps it on
 * the device:
 *   - requests of deep topologies (chunk_blocks 2^17 and up) run on the
 *     multi-unit depth kernel, the pending ones of one topology together,
 *     three chunk copies per CTA, each CTA holding its SM alone, on
 *     high-priority streams; one that does not fit the free SMs waits;
 *   - the others run in waves: one persistent multi-topology launch per
 *     wave on its own stream, a request completing as soon as its chunk
 *     copies are in;
 *   - a request that waits for SMs or scratch never holds back the others,
 *     and the dispatcher never waits for the GPU.
 * Launches run on streams of their own; a launch starts only where no
 * running launch shares its host-to-device work queue, so
 * CUDA_DEVICE_MAX_CONNECTIONS (8 by default; 32 gives every slot its own)
 * bounds how many run at once.  Tuning variables, read at creation:
 * POSE_B200_SERVER_DEEP_LEVELS (levels from which a topology is deep),
 * POSE_B200_SERVER_DEEP_UNITS (copies per depth CTA; 0 = the fewest that fit
 * an idle GPU), POSE_B200_SERVER_DEEP_EXCL and POSE_B200_SERVER_DEEP_WAIT
 * (0: share SMs; 0: join a wave instead of waiting), POSE_B200_SERVER_DEEP=0
 * (every request in waves), POSE_B200_SERVER_DEEP_SMS (SMs the depth kernel
 * may hold).  Each result is byte-identical to labelling the request alone.
 * All topologies and buffers must be on the device that was current at
 * creation. */
typedef struct pose_b200_server pose_b200_server_t;

/* scratch_bytes: HBM arena for all waves (0 = half the free memory);
 * max_waves: concurrent waves (0 = 5 when CUDA_DEVICE_MAX_CONNECTIONS is 16
 * or more, else 3; at most 16).  NULL on error. */
pose_b200_server_t *pose_b200_server_create(uint64_t scratch_bytes, uint32_t max_waves);
/* Register a session seed (<= 1016 bytes); returns its id, or -1. */
int pose_b200_server_session(pose_b200_server_t *server, const uint8_t *seed, size_t seed_len);
/* Build ahead of the first request what requests of this topology need (the
 * depth kernel's 512-slot records, for a deep topology; kept with the
 * topology).  Optional: the first submit of a topology does it otherwise, in
 * the submitting thread.  0 on success, -1 on a bad argument. */
int pose_b200_server_prepare(pose_b200_server_t *server, const pose_hbm_topo_t *topo);
/* Queue one request; returns its ticket, or -1. */
int64_t pose_b200_server_submit(pose_b200_server_t *server, const pose_hbm_topo_t *topo, int session,
                                void *hbm_dev_ptr, size_t hbm_len, uint64_t region_block_offset);
/* Block until the request finished: 0 on success, -1 on failure; queue_ms
 * (submit to launch) and total_ms (submit to completion) may be NULL. */
int pose_b200_server_wait(pose_b200_server_t *server, int64_t ticket, double *queue_ms, double *total_ms);
/* 1 done, 0 pending or running, -1 failed or unknown. */
int pose_b200_server_query(pose_b200_server_t *server, int64_t ticket);
void pose_b200_server_stats(pose_b200_server_t *server, uint64_t *submitted, uint64_t *waves,
                            uint64_t *scratch_bytes);
/* Finish all submitted work, zero the arena and the session seeds, free. */
void pose_b200_server_destroy(pose_b200_server_t *server);

/* ── verifier: challenge recompute on the GPU ────────────────────────────── */

/* pose_graph_challenge (common/include/graph.h:99-102, common/src/graph.c:
 * 1019-1042) on the GPU: the label of output rank challenge_idx of the graph
 * of m = the topology's chunk_blocks outputs, labelled with `seed` as its
 * graph seed.  As in the reference, that seed is a chunk seed (for a region,
 * pose_chunk_seed(session seed, chunk index)) and only its first 32 bytes are
 * used.  The reference labels the whole graph on the CPU; here the chunk is
 * labelled on the device (both standalone copies run side by side, so the
 * latency is that of one copy) and 32 bytes come back.  0 on success; -1 when
 * challenge_idx >= m, seed is NULL or shorter than 32 bytes, or on a CUDA
 * error. */
int pose_b200_challenge(const pose_hbm_topo_t *topo, const uint8_t *seed, size_t seed_len,
                        uint64_t challenge_idx, uint8_t out[32]);

/* Many challenges of one session at once.  blocks[k] is an absolute block
 * index of a labelled region (the unit of region_block_offset): output rank
 * blocks[k] % cb of chunk blocks[k] / cb, whose chunk seed is
 * pose_chunk_seed(session_seed, blocks[k] / cb) (common/src/graph.c:
 * 1646-1649).  Each distinct chunk is recomputed once; the chunks run as
 * batched launches of at most 4 GiB of labels each, and out[32k..32k+31]
 * receives the label of blocks[k].  sched as for pose_b200_batch_create;
 * session seeds of at most 1016 bytes.
 * 0 on success, -1 on error. */
int pose_b200_challenge_blocks(const pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                               const uint64_t *blocks, size_t n, uint8_t *out,
                               const pose_b200_sched_t *sched, pose_b200_stats_t *stats);

/* Reads len bytes at byte offset off of the labelled target into buf, like
 * the pread of the reference's verify step; returns 0 on success. */
typedef int (*pose_b200_read_fn)(void *ctx, uint8_t *buf, size_t len, uint64_t off);

/* The sampled verify of disk-wipe-bench (verify_disk,
 * tools/disk-wipe-bench/disk_wipe_bench.cu:300-366) with the recompute on the
 * GPU.  The target holds n_super = wipe_len / (cb*32) super-chunks labelled
 * from region block 0 (super-chunk J at byte J*cb*32, chunk index J).
 * `samples` of them (clamped to [1, n_super]; J_k = k*(n_super-1)/(samples-1),
 * first and last included) are read through `read`, recomputed on the GPU in
 * batched launches while the reads run, and compared on the device (session
 * seeds of at most 1016 bytes).
 * *checked and *mismatched count super-chunks (either may be NULL);
 * first_bad, when not NULL, has `samples` entries and receives each sample's
 * first mismatching block within its super-chunk, or UINT64_MAX when it
 * matched.  The first three mismatches are also printed to stderr, as the
 * reference does.  0 when setup and I/O succeeded (mismatches are results,
 * not errors); -1 when nothing was labelled, a read failed, or on a CUDA
 * error. */
int pose_b200_verify_sampled(const pose_hbm_topo_t *topo, const uint8_t *session_seed, size_t seed_len,
                             uint64_t wipe_len, uint64_t samples, pose_b200_read_fn read, void *read_ctx,
                             uint64_t *checked, uint64_t *mismatched, uint64_t *first_bad,
                             const pose_b200_sched_t *sched, pose_b200_stats_t *stats);

/* Labeling that allocates no device memory during the call.
 *
 * No counterpart in the reference: it is an addition of this library.  Same
 * arguments, bytes and return convention as pose_graph_hbm_topo_label, for
 * callers that must not call cudaMalloc while they label — e.g. a wipe worker
 * that reserved the device's free memory for its label window before
 * starting (a late allocation could fail half-way through a disk), or a host
 * whose own allocator already holds the device's memory and forbids new
 * device allocations.  The topology, seed and output buffer are still the
 * caller's.
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
 * and the scratch, the seed table and the session seed copy are zeroed before
 * the call returns (when it fails too), but
 * calls whose device work overlaps (from several host threads, or on several
 * topologies of one device at once) race on them and must be serialised by
 * the caller. */
int pose_b200_topo_label_noalloc(const pose_hbm_topo_t *topo, const uint8_t *session_seed,
                                 size_t seed_len, void *hbm_dev_ptr, size_t hbm_len,
                                 uint64_t region_block_offset);

/* Workspace audit (no reference counterpart).  *nonzero_bytes = the nonzero
 * bytes left in the device memory that labeling calls on this topology use
 * besides the caller's buffer: the scratch labels, the chunk-seed table and
 * the session seed copy, plus, on the topology's device, the arrays of
 * pose_b200_topo_label_noalloc.  Every labeling call and every autotuner
 * trial zeroes them before it returns, whether it succeeded or not, so
 * between calls this is 0: no label, chunk seed or session key of a past
 * call stays on the device.  Synchronous; must not overlap a labeling call
 * on the same topology.  Returns 0 on success, -1 on error. */
int pose_b200_topo_residue(const pose_hbm_topo_t *topo, uint64_t *nonzero_bytes);

/* The counting of the workspace audit on any device buffer of the current
 * device: *nonzero_bytes = the nonzero bytes of dev_ptr[0, bytes).  dev_ptr
 * must be 16-byte aligned.  Synchronous.  Returns 0 on success, -1 on
 * error. */
int pose_b200_count_nonzero(const void *dev_ptr, size_t bytes, uint64_t *nonzero_bytes);

/* Last error message of the calling thread ("" when none). */
const char *pose_b200_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* POSE_B200_H */
