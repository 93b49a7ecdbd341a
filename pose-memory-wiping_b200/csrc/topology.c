/*
 * topology.c — seed-independent labeling schedule of one chunk (C11).
 *
 * Emits one standalone copy of the pose-db-drg-v1 DAG with the node numbering
 * of the reference's edge-mode emitters (common/src/graph.c:156-520,
 * pose_graph_edges at graph.c:1044-1100):
 *   standalone(0)     = one source node;
 *   standalone(l)     = standalone(l-1) -> connector(l-1) over its base
 *                       outputs -> connected(l-1) over the connector outputs;
 *                       base outputs = standalone part | connected part;
 *   connected(0)      = one 1-pred node;
 *   connected(l)      = connected(l-1) over the first half of the inputs ->
 *                       merged(l-1)(primary = those outputs, ingress = second
 *                       half of the inputs) -> connected(l-1) over its output;
 *   connector(d)      = a 1-pred layer then d butterfly layers pairing i with
 *                       i ^ 2^(d-1-k);
 *   merged(d)         = the whole ingress butterfly (1-pred layer over the
 *                       ingress inputs + d butterfly layers), then the center
 *                       butterfly: layer 0 pairs primary[i] with the last
 *                       ingress layer, then d butterfly layers.
 * Ids are assigned in emission order, every predecessor id is smaller than
 * its reader's, and 2-pred nodes list the lower id first (graph.c:128-144).
 * The right copy of a chunk is the same topology shifted by S ids.
 *
 * From the edges it derives the GPU schedule: dependency levels
 * (level = 1 + max(level(pred)), as label_gpu_common.cu:126-162 does),
 * a stable level-sorted node order, and a recycled scratch-slot map with
 * level-granular lifetimes (a node occupies its slot from its own level up to
 * the level of its last reader; nodes of one level never share a slot, so a
 * level can be labelled in parallel).  Slots are reused last-freed-first for
 * cache locality.  The packed records are what the device kernels read.
 */
#include "topology.h"
#include "b3_host.h"

#include <stdlib.h>
#include <string.h>

static uint64_t cnt_bfly(int d) { return (uint64_t)(d + 1) << d; }
static uint64_t cnt_conn(int l) { return l == 0 ? 1 : 2 * cnt_conn(l - 1) + 2 * cnt_bfly(l - 1); }
static uint64_t cnt_stand(int l) { return l == 0 ? 1 : cnt_stand(l - 1) + cnt_bfly(l - 1) + cnt_conn(l - 1); }

uint64_t pb_copy_node_count(uint32_t cb)
{
    if (cb == 0 || cb > PB_MAX_CHUNK_BLOCKS) return 0;
    return cnt_stand(pb_parameter_n(cb) + 1);
}

uint64_t pb_chunk_node_count(uint32_t cb) { return 2 * pb_copy_node_count(cb); }

/* ── emitter ─────────────────────────────────────────────────────────────── */

typedef struct {
    uint32_t next;
    uint8_t *np;
    uint32_t *p0, *p1, *lvl;
    uint32_t *ws;     /* bump workspace for id arrays */
    size_t ws_top, ws_cap;
    int overflow;
} gen_t;

static uint32_t *ws_take(gen_t *g, size_t n)
{
    if (g->ws_top + n > g->ws_cap) { g->overflow = 1; g->ws_top = 0; }
    uint32_t *p = g->ws + g->ws_top;
    g->ws_top += n;
    return p;
}

static inline uint32_t mk(gen_t *g, int np, uint32_t a, uint32_t b)
{
    uint32_t id = g->next++;
    if (np == 2 && a > b) { uint32_t t = a; a = b; b = t; }
    uint32_t lv = 0;
    if (np >= 1) lv = g->lvl[a] + 1;
    if (np == 2 && g->lvl[b] + 1 > lv) lv = g->lvl[b] + 1;
    g->np[id] = (uint8_t)np;
    g->p0[id] = np >= 1 ? a : 0;
    g->p1[id] = np == 2 ? b : 0;
    g->lvl[id] = lv;
    return id;
}

/* d butterfly layers over cur (width 2^d), ping-ponging with tmp; returns the
 * buffer holding the last layer. */
static uint32_t *bfly_layers(gen_t *g, int d, uint32_t *cur, uint32_t *tmp)
{
    uint32_t w = 1u << d;
    for (int k = 0; k < d; k++) {
        uint32_t bit = 1u << (d - 1 - k);
        for (uint32_t i = 0; i < w; i++) tmp[i] = mk(g, 2, cur[i], cur[i ^ bit]);
        uint32_t *t = cur; cur = tmp; tmp = t;
    }
    return cur;
}

static void gen_connector(gen_t *g, int d, const uint32_t *in, uint32_t *out)
{
    uint32_t w = 1u << d;
    size_t mark = g->ws_top;
    uint32_t *a = ws_take(g, w), *b = ws_take(g, w);
    for (uint32_t i = 0; i < w; i++) a[i] = mk(g, 1, in[i], 0);
    uint32_t *last = bfly_layers(g, d, a, b);
    memcpy(out, last, sizeof(uint32_t) * w);
    g->ws_top = mark;
}

static void gen_merged(gen_t *g, int d, const uint32_t *prim, const uint32_t *ingr, uint32_t *out)
{
    uint32_t w = 1u << d;
    size_t mark = g->ws_top;
    uint32_t *a = ws_take(g, w), *b = ws_take(g, w);
    for (uint32_t i = 0; i < w; i++) a[i] = mk(g, 1, ingr[i], 0);
    uint32_t *ing = bfly_layers(g, d, a, b);
    uint32_t *ctr = ing == a ? b : a;
    for (uint32_t i = 0; i < w; i++) ctr[i] = mk(g, 2, prim[i], ing[i]);
    uint32_t *last = bfly_layers(g, d, ctr, ing);
    memcpy(out, last, sizeof(uint32_t) * w);
    g->ws_top = mark;
}

static void gen_connected(gen_t *g, int l, const uint32_t *in, uint32_t *out)
{
    if (l == 0) { out[0] = mk(g, 1, in[0], 0); return; }
    uint32_t h = 1u << (l - 1);
    size_t mark = g->ws_top;
    uint32_t *x = ws_take(g, h);
    gen_connected(g, l - 1, in, out);
    gen_merged(g, l - 1, out, in + h, x);
    gen_connected(g, l - 1, x, out + h);
    g->ws_top = mark;
}

static void gen_standalone(gen_t *g, int l, uint32_t *out)
{
    if (l == 0) { out[0] = mk(g, 0, 0, 0); return; }
    uint32_t h = 1u << (l - 1);
    size_t mark = g->ws_top;
    uint32_t *x = ws_take(g, h);
    gen_standalone(g, l - 1, out);
    gen_connector(g, l - 1, out, x);
    gen_connected(g, l - 1, x, out + h);
    g->ws_top = mark;
}

/* Emit one copy: fills np/p0/p1/lvl (S entries) and base[2^(n+1)]. */
static int emit_copy(uint32_t cb, uint8_t *np, uint32_t *p0, uint32_t *p1, uint32_t *lvl,
                     uint32_t *base)
{
    int level = pb_parameter_n(cb) + 1;
    gen_t g;
    memset(&g, 0, sizeof(g));
    g.np = np; g.p0 = p0; g.p1 = p1; g.lvl = lvl;
    g.ws_cap = ((size_t)8 << level) + 64;
    g.ws = (uint32_t *)malloc(g.ws_cap * sizeof(uint32_t));
    if (!g.ws) return -1;
    gen_standalone(&g, level, base);
    free(g.ws);
    if (g.overflow || g.next != pb_copy_node_count(cb)) return -1;
    return 0;
}

uint64_t pb_topo_copy_edges(uint32_t cb, uint8_t *np, uint32_t *p0, uint32_t *p1,
                            uint32_t *out_ids)
{
    uint64_t S = pb_copy_node_count(cb);
    if (S == 0) return 0;
    int n = pb_parameter_n(cb);
    uint32_t *lvl = (uint32_t *)malloc(S * sizeof(uint32_t));
    uint32_t *base = (uint32_t *)malloc(((size_t)2 << n) * sizeof(uint32_t));
    int rc = (lvl && base) ? emit_copy(cb, np, p0, p1, lvl, base) : -1;
    if (rc == 0) memcpy(out_ids, base + ((size_t)1 << n), ((size_t)1 << n) * sizeof(uint32_t));
    free(lvl);
    free(base);
    return rc == 0 ? S : 0;
}

/* ── schedule ────────────────────────────────────────────────────────────── */

void pb_topo_host_free(pb_topo_host_t *t)
{
    if (!t) return;
    free(t->lstart);
    free(t->recs);
    free(t->orank);
    free(t->recs2);
    memset(t, 0, sizeof(*t));
}

/* Pipelined records: every node read at its next level gets a shared-memory
 * copy (while the pool has room); a global slot is kept only for nodes read
 * two or more levels later or left without a shared-memory copy.  Both pools
 * are assigned greedily level by level, allocation before release, so two
 * labels that are live in the same level never share a slot. */
static int build_pipelined(uint32_t S, uint32_t L, const uint8_t *np, const uint32_t *p0,
                           const uint32_t *p1, const uint32_t *lvl, const uint32_t *dies,
                           const uint32_t *order, const uint32_t *lstart, const uint32_t *cntd,
                           const uint32_t *dorder, const uint32_t *rank_of, uint32_t csm,
                           pb_topo_host_t *t)
{
    uint8_t *d1 = (uint8_t *)calloc(S, 1);
    uint32_t *ss = (uint32_t *)malloc((size_t)S * 4), *gs = (uint32_t *)malloc((size_t)S * 4);
    uint32_t *gstack = (uint32_t *)malloc((size_t)S * 4);
    uint32_t *sstack = (uint32_t *)malloc(((size_t)csm + 1) * 4);
    uint32_t *recs = (uint32_t *)malloc((size_t)S * 32);
    int rc = -1;
    if (!d1 || !ss || !gs || !gstack || !sstack || !recs) goto out;
    for (uint32_t id = 0; id < S; id++) {
        if (np[id] >= 1 && lvl[p0[id]] + 1 == lvl[id]) d1[p0[id]] = 1;
        if (np[id] >= 2 && lvl[p1[id]] + 1 == lvl[id]) d1[p1[id]] = 1;
    }
    uint32_t gtop = 0, gfresh = 0, stop = 0, sfresh = 0;
    for (uint32_t l = 0; l < L; l++) {
        for (uint32_t p = lstart[l]; p < lstart[l + 1]; p++) {
            uint32_t id = order[p];
            ss[id] = PB_NO_SLOT;
            if (d1[id]) {
                if (stop) ss[id] = sstack[--stop];
                else if (sfresh < csm) ss[id] = sfresh++;
            }
        }
        for (uint32_t p = lstart[l]; p < lstart[l + 1]; p++) {
            uint32_t id = order[p];
            int need_g = dies[id] >= lvl[id] + 2 || (d1[id] && ss[id] == PB_NO_SLOT);
            gs[id] = need_g ? (gtop ? gstack[--gtop] : gfresh++) : PB_NO_SLOT;
        }
        for (uint32_t k = cntd[l]; k < cntd[l + 1]; k++) {
            uint32_t id = dorder[k];
            if (gs[id] != PB_NO_SLOT) gstack[gtop++] = gs[id];
        }
        if (l > 0)
            for (uint32_t p = lstart[l - 1]; p < lstart[l]; p++)
                if (ss[order[p]] != PB_NO_SLOT) sstack[stop++] = ss[order[p]];
    }
    for (uint32_t p = 0; p < S; p++) {
        uint32_t id = order[p], k = np[id], *r = recs + (size_t)8 * p;
        uint32_t ref[2] = {0, 0};
        for (uint32_t e = 0; e < k; e++) {
            uint32_t q = e == 0 ? p0[id] : p1[id];
            if (lvl[q] + 1 == lvl[id])
                ref[e] = PB_REF_PREV | (ss[q] != PB_NO_SLOT ? (PB_REF_SMEM | ss[q]) : gs[q]);
            else
                ref[e] = gs[q];
        }
        r[0] = id | (k << PB_REC_NP_SHIFT) | (rank_of[id] != PB_NO_RANK ? PB_REC_OUT_BIT : 0);
        r[1] = ref[0];
        r[2] = ref[1];
        r[3] = gs[id];
        r[4] = ss[id];
        r[5] = rank_of[id];
        r[6] = 0;
        r[7] = 0;
    }
    t->recs2 = recs;
    recs = NULL;
    t->csm = sfresh;
    t->gpool2 = gfresh;
    rc = 0;
out:
    free(d1); free(ss); free(gs); free(gstack); free(sstack); free(recs);
    return rc;
}

int pb_topo_host_build(uint32_t cb, pb_topo_host_t *t) { return pb_topo_host_build_ex(cb, 0, t); }

int pb_topo_host_build_ex(uint32_t cb, uint32_t csm, pb_topo_host_t *t)
{
    memset(t, 0, sizeof(*t));
    uint64_t S64 = pb_copy_node_count(cb);
    if (S64 == 0 || S64 > PB_REC_ID_MASK) return -1;
    const uint32_t S = (uint32_t)S64;
    const int n = pb_parameter_n(cb);
    const uint32_t half_w = 1u << n;

    uint8_t *np = (uint8_t *)malloc(S);
    uint32_t *p0 = (uint32_t *)malloc((size_t)S * 4), *p1 = (uint32_t *)malloc((size_t)S * 4);
    uint32_t *lvl = (uint32_t *)malloc((size_t)S * 4);
    uint32_t *base = (uint32_t *)malloc(((size_t)2 << n) * 4);
    uint32_t *order = NULL, *dies = NULL, *dorder = NULL, *slot = NULL, *stack = NULL;
    uint32_t *cntl = NULL, *cntd = NULL;
    int rc = -1;
    if (!np || !p0 || !p1 || !lvl || !base) goto out;
    if (emit_copy(cb, np, p0, p1, lvl, base) != 0) goto out;

    uint32_t L = 0;
    for (uint32_t id = 0; id < S; id++) if (lvl[id] + 1 > L) L = lvl[id] + 1;

    /* stable counting sort of ids by birth level */
    t->lstart = (uint32_t *)calloc((size_t)L + 1, 4);
    order = (uint32_t *)malloc((size_t)S * 4);
    cntl = (uint32_t *)malloc((size_t)L * 4);
    if (!t->lstart || !order || !cntl) goto out;
    for (uint32_t id = 0; id < S; id++) t->lstart[lvl[id] + 1]++;
    uint32_t maxw = 0;
    for (uint32_t l = 0; l < L; l++) {
        if (t->lstart[l + 1] > maxw) maxw = t->lstart[l + 1];
        t->lstart[l + 1] += t->lstart[l];
    }
    memcpy(cntl, t->lstart, (size_t)L * 4);
    for (uint32_t id = 0; id < S; id++) order[cntl[lvl[id]]++] = id;

    /* death level = level of the last reader (own level for a sink) */
    dies = (uint32_t *)malloc((size_t)S * 4);
    if (!dies) goto out;
    memcpy(dies, lvl, (size_t)S * 4);
    for (uint32_t id = 0; id < S; id++) {
        if (np[id] >= 1 && dies[p0[id]] < lvl[id]) dies[p0[id]] = lvl[id];
        if (np[id] >= 2 && dies[p1[id]] < lvl[id]) dies[p1[id]] = lvl[id];
    }
    cntd = (uint32_t *)calloc((size_t)L + 1, 4);
    dorder = (uint32_t *)malloc((size_t)S * 4);
    if (!cntd || !dorder) goto out;
    for (uint32_t id = 0; id < S; id++) cntd[dies[id] + 1]++;
    for (uint32_t l = 0; l < L; l++) cntd[l + 1] += cntd[l];
    memcpy(cntl, cntd, (size_t)L * 4);
    for (uint32_t id = 0; id < S; id++) dorder[cntl[dies[id]]++] = id;

    /* level-granular slot assignment: a level's nodes take slots before the
     * level's dying nodes release theirs */
    slot = (uint32_t *)malloc((size_t)S * 4);
    stack = (uint32_t *)malloc((size_t)S * 4);
    if (!slot || !stack) goto out;
    uint32_t top = 0, fresh = 0;
    for (uint32_t l = 0; l < L; l++) {
        for (uint32_t p = t->lstart[l]; p < t->lstart[l + 1]; p++)
            slot[order[p]] = top ? stack[--top] : fresh++;
        for (uint32_t k = cntd[l]; k < cntd[l + 1]; k++)
            stack[top++] = slot[dorder[k]];
    }
    free(stack); stack = NULL;

    /* id -> local output rank (kept in `stack`'s place) */
    stack = (uint32_t *)malloc((size_t)S * 4);
    if (!stack) goto out;
    for (uint32_t id = 0; id < S; id++) stack[id] = PB_NO_RANK;
    for (uint32_t r = 0; r < half_w; r++) stack[base[half_w + r]] = r;
    if (csm && build_pipelined(S, L, np, p0, p1, lvl, dies, order, t->lstart, cntd, dorder, stack,
                               csm, t) != 0)
        goto out;
    free(dies); dies = NULL;
    free(dorder); dorder = NULL;

    /* records; lvl is reused as the id -> local output rank map */
    memcpy(lvl, stack, (size_t)S * 4);
    t->recs = (uint32_t *)malloc((size_t)S * 16);
    t->orank = (uint32_t *)malloc((size_t)S * 4);
    if (!t->recs || !t->orank) goto out;
    for (uint32_t p = 0; p < S; p++) {
        uint32_t id = order[p];
        uint32_t k = np[id];
        uint32_t *r = t->recs + (size_t)4 * p;
        r[0] = id | (k << PB_REC_NP_SHIFT) | (lvl[id] != PB_NO_RANK ? PB_REC_OUT_BIT : 0);
        r[1] = k >= 1 ? slot[p0[id]] : 0;
        r[2] = k >= 2 ? slot[p1[id]] : 0;
        r[3] = slot[id];
        t->orank[p] = lvl[id];
    }

    t->cb = cb;
    t->n = n;
    t->half_w = half_w;
    t->retained = cb - half_w;
    t->S = S;
    t->L = L;
    t->pool = fresh;
    t->max_width = maxw;
    pb_graph_descriptor(t->desc, cb, (uint64_t)n);
    rc = 0;

out:
    free(np); free(p0); free(p1); free(lvl); free(base);
    free(order); free(dies); free(dorder); free(slot); free(stack);
    free(cntl); free(cntd);
    if (rc != 0) pb_topo_host_free(t);
    return rc;
}
