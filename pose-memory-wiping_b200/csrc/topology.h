/* topology.h — seed-independent labeling schedule of one chunk (C11, internal).
 *
 * A chunk of m = chunk_blocks outputs is two identical standalone copies of
 * the pose-db-drg-v1 DAG G_{n+1} (common/src/graph.c:1044-1100): the left
 * copy holds node ids [0, S), the right copy the same topology at ids
 * [S, 2S).  The schedule is therefore built for ONE copy and run twice (a
 * "unit" is one copy of one chunk); only the node-index input of the hash and
 * the output ranks differ between the copies.
 */
#ifndef PB_TOPOLOGY_H
#define PB_TOPOLOGY_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Packed node record, one per node, in dependency-level order:
 *   x = node id within the copy (bits 0..27) | predecessor count << 28
 *       | output flag << 30
 *   y = scratch slot of predecessor 0 (0 when absent)
 *   z = scratch slot of predecessor 1 (0 when absent)
 *   w = scratch slot this node's label is written to */
#define PB_REC_ID_MASK 0x0FFFFFFFu
#define PB_REC_NP_SHIFT 28
#define PB_REC_OUT_BIT (1u << 30)
#define PB_NO_RANK 0xFFFFFFFFu
#define PB_MAX_CHUNK_BLOCKS (1u << 20)

/* Pipelined records (8 words per node, level order), built for a shared-
 * memory label pool of `csm` slots per copy:
 *   [0] x as above
 *   [1] predecessor 0 reference, [2] predecessor 1 reference:
 *       PB_REF_PREV = the predecessor was born at the previous level (it is
 *       complete only after that level's barrier); PB_REF_SMEM = it lives in
 *       the shared-memory pool; low 30 bits = its slot in that pool.  A
 *       reference without PREV points at the global pool and may be fetched
 *       one level early.
 *   [3] global slot this node is copied to, PB_NO_SLOT if none (read by no
 *       node two or more levels later, and by its next level through shared
 *       memory)
 *   [4] shared-memory slot this node is copied to, PB_NO_SLOT if none
 *   [5] local output rank, PB_NO_RANK if not an output
 *   [6], [7] zero
 * A node's shared-memory copy lives for its own level and the next; nodes
 * whose level has more next-level-read labels than the pool holds fall back
 * to the global pool. */
#define PB_REF_PREV (1u << 31)
#define PB_REF_SMEM (1u << 30)
#define PB_REF_SLOT_MASK 0x3FFFFFFFu
#define PB_NO_SLOT 0xFFFFFFFFu

typedef struct pb_topo_host {
    uint32_t cb;        /* chunk_blocks (m) */
    int n;              /* graph parameter n */
    uint32_t half_w;    /* 2^n outputs taken from the left copy */
    uint32_t retained;  /* m - 2^n outputs taken from the right copy */
    uint32_t S;         /* nodes per copy */
    uint32_t L;         /* dependency levels per copy */
    uint32_t pool;      /* recycled 32-byte label slots per copy */
    uint32_t max_width; /* widest level */
    uint32_t *lstart;   /* [L + 1] offsets of each level in recs */
    uint32_t *recs;     /* [4 * S] packed records (x, y, z, w) */
    uint32_t *orank;    /* [S] local output rank per record, PB_NO_RANK otherwise */
    uint8_t desc[32];   /* graph descriptor digest */
    /* pipelined layout (present when built with csm > 0) */
    uint32_t csm;       /* shared-memory slots per copy */
    uint32_t gpool2;    /* global slots per copy */
    uint32_t *recs2;    /* [8 * S] pipelined records */
} pb_topo_host_t;

/* Build the schedule for chunk_blocks in [1, 2^20].  Returns 0, or -1 on a bad
 * argument or allocation failure (t is then left zeroed). */
int pb_topo_host_build(uint32_t chunk_blocks, pb_topo_host_t *t);
/* As pb_topo_host_build, plus the pipelined records for a shared-memory pool
 * of csm slots per copy (csm = 0: none). */
int pb_topo_host_build_ex(uint32_t chunk_blocks, uint32_t csm, pb_topo_host_t *t);
void pb_topo_host_free(pb_topo_host_t *t);

/* Nodes per copy and in a whole chunk (the reference's scaffold count). */
uint64_t pb_copy_node_count(uint32_t chunk_blocks);
uint64_t pb_chunk_node_count(uint32_t chunk_blocks);

/* Inspection for tests: the copy's edges in id order (np, p0, p1; preds 0
 * when absent; lower id first) and out_ids[r] = id of local output rank r
 * (2^n entries).  Arrays hold pb_copy_node_count entries.  Returns S or 0. */
uint64_t pb_topo_copy_edges(uint32_t chunk_blocks, uint8_t *np, uint32_t *p0,
                            uint32_t *p1, uint32_t *out_ids);

#ifdef __cplusplus
}
#endif
#endif
