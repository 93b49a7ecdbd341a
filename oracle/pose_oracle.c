/*
 * pose_oracle.c — TEST INFRASTRUCTURE ONLY: the CPU oracle.
 *
 * A plain, scalar C restatement of the reference's labeling algorithm, used
 * only by tests/, __graft_entry__.smoke() and the bench's CPU-baseline leg to
 * check the product.  It is never linked into the product library.  It is
 * pinned against the official BLAKE3 vectors the reference tests hold
 * (common/test/test_hash.c:47-67) and against golden vectors produced by the
 * reference itself compiled from source (tests/golden/gen_golden.py).
 *
 * What it restates (reference file:line):
 *   - BLAKE3 compression, chunk chaining and the binary tree (the vendored
 *     BLAKE3 1.8.5, common/vendor/blake3/blake3_portable.c:8-98, blake3.c);
 *     derive_key (blake3.c:411-413 via blake3_hasher_init_derive_key).
 *   - label keys derive_key("pose-db/label/src" | "pose-db/label/int")
 *     (common/src/hash.c:46-67).
 *   - the 192-byte node message and its keyed hash
 *     (common/src/hash.c:80-144: block 0 = node index big-endian, block 1 =
 *     pred0 | pred1, block 2 = seed | descriptor; flags KEYED_HASH with
 *     CHUNK_START on block 0 and CHUNK_END|ROOT on block 2).
 *   - graph descriptor and chunk seed (common/src/hash.c:198-233).
 *   - pose-db-drg-v1 topology: counts (common/src/graph.c:33-54), the
 *     edge-mode emitters emit_connector / emit_merged_center_ingress /
 *     emit_standalone / emit_connected (graph.c:156-520) and
 *     pose_graph_edges (graph.c:1044-1100): two standalone copies, ids in
 *     emission order, 2-pred nodes list the lower id first, outputs = second
 *     half of the left copy's base outputs then the first `retained` of the
 *     right copy's.
 *   - labeling a chunk: every node in id order (do_label, graph.c:575-645),
 *     outputs gathered in rank order; super-chunk j of a region uses chunk
 *     index (rbo + j*cb)/cb (graph.c:1646-1649).
 *
 * The labeler keeps only live labels (a node's label is dropped after its
 * last reader), which changes memory use, never bytes.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ── BLAKE3 (from the public specification) ─────────────────────────────── */

enum {
    F_CHUNK_START = 1, F_CHUNK_END = 2, F_PARENT = 4, F_ROOT = 8,
    F_KEYED_HASH = 16, F_DERIVE_CONTEXT = 32, F_DERIVE_MATERIAL = 64,
};

static const uint32_t B3_IV[8] = {
    0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
    0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u,
};
static const int B3_PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};

static uint32_t ror(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

static void g(uint32_t *v, int a, int b, int c, int d, uint32_t x, uint32_t y)
{
    v[a] = v[a] + v[b] + x; v[d] = ror(v[d] ^ v[a], 16);
    v[c] = v[c] + v[d];     v[b] = ror(v[b] ^ v[c], 12);
    v[a] = v[a] + v[b] + y; v[d] = ror(v[d] ^ v[a], 8);
    v[c] = v[c] + v[d];     v[b] = ror(v[b] ^ v[c], 7);
}

/* Full compression: out[16] = final state with the feed-forward applied. */
static void b3_compress(const uint32_t cv[8], const uint32_t block[16],
                        uint64_t counter, uint32_t block_len, uint32_t flags,
                        uint32_t out[16])
{
    uint32_t v[16], m[16], t[16];
    for (int i = 0; i < 8; i++) v[i] = cv[i];
    for (int i = 0; i < 4; i++) v[8 + i] = B3_IV[i];
    v[12] = (uint32_t)counter; v[13] = (uint32_t)(counter >> 32);
    v[14] = block_len; v[15] = flags;
    memcpy(m, block, sizeof(m));
    for (int r = 0; r < 7; r++) {
        g(v, 0, 4, 8, 12, m[0], m[1]);   g(v, 1, 5, 9, 13, m[2], m[3]);
        g(v, 2, 6, 10, 14, m[4], m[5]);  g(v, 3, 7, 11, 15, m[6], m[7]);
        g(v, 0, 5, 10, 15, m[8], m[9]);  g(v, 1, 6, 11, 12, m[10], m[11]);
        g(v, 2, 7, 8, 13, m[12], m[13]); g(v, 3, 4, 9, 14, m[14], m[15]);
        for (int i = 0; i < 16; i++) t[i] = m[B3_PERM[i]];
        memcpy(m, t, sizeof(m));
    }
    for (int i = 0; i < 8; i++) { out[i] = v[i] ^ v[i + 8]; out[i + 8] = v[i + 8] ^ cv[i]; }
}

static uint32_t ld32(const uint8_t *p)
{
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static void st32(uint8_t *p, uint32_t w)
{
    p[0] = (uint8_t)w; p[1] = (uint8_t)(w >> 8); p[2] = (uint8_t)(w >> 16); p[3] = (uint8_t)(w >> 24);
}

/* One chunk (<= 1024 bytes) -> its chaining value; when root, the root output
 * words instead. */
static void b3_chunk(const uint32_t key[8], uint32_t base_flags, const uint8_t *in,
                     size_t len, uint64_t chunk_counter, int is_root, uint32_t out[8])
{
    uint32_t cv[8], blk[16], st[16];
    memcpy(cv, key, 32);
    size_t nblocks = len == 0 ? 1 : (len + 63) / 64;
    for (size_t b = 0; b < nblocks; b++) {
        uint8_t buf[64] = {0};
        size_t off = b * 64, bl = len - off < 64 ? len - off : 64;
        if (len == 0) bl = 0;
        memcpy(buf, in + off, bl);
        for (int i = 0; i < 16; i++) blk[i] = ld32(buf + 4 * i);
        uint32_t fl = base_flags;
        if (b == 0) fl |= F_CHUNK_START;
        if (b == nblocks - 1) { fl |= F_CHUNK_END; if (is_root) fl |= F_ROOT; }
        b3_compress(cv, blk, chunk_counter, (uint32_t)bl, fl, st);
        memcpy(cv, st, 32);
    }
    memcpy(out, cv, 32);
}

/* Subtree over whole chunks starting at chunk_counter: the left subtree holds
 * the largest power-of-two number of chunks that leaves at least one chunk on
 * the right. */
static void b3_subtree(const uint32_t key[8], uint32_t base_flags, const uint8_t *in,
                       size_t len, uint64_t chunk_counter, int is_root, uint32_t out[8])
{
    if (len <= 1024) { b3_chunk(key, base_flags, in, len, chunk_counter, is_root, out); return; }
    size_t nchunks = (len + 1023) / 1024, left = 1;
    while (left * 2 < nchunks) left *= 2;
    uint32_t l[8], r[8], blk[16], st[16];
    b3_subtree(key, base_flags, in, left * 1024, chunk_counter, 0, l);
    b3_subtree(key, base_flags, in + left * 1024, len - left * 1024, chunk_counter + left, 0, r);
    memcpy(blk, l, 32); memcpy(blk + 8, r, 32);
    b3_compress(key, blk, 0, 64, base_flags | F_PARENT | (is_root ? F_ROOT : 0), st);
    memcpy(out, st, 32);
}

static void b3_hash(const uint32_t key[8], uint32_t base_flags, const uint8_t *in,
                    size_t len, uint8_t out[32])
{
    uint32_t w[8];
    b3_subtree(key, base_flags, in, len, 0, 1, w);
    for (int i = 0; i < 8; i++) st32(out + 4 * i, w[i]);
}

static void b3_context_key(const char *context, uint32_t key[8])
{
    uint8_t k[32];
    b3_hash(B3_IV, F_DERIVE_CONTEXT, (const uint8_t *)context, strlen(context), k);
    for (int i = 0; i < 8; i++) key[i] = ld32(k + 4 * i);
}

/* Exported for the tests: plain BLAKE3 hash (official-vector check). */
void oracle_blake3(const uint8_t *in, size_t len, uint8_t out[32])
{
    b3_hash(B3_IV, 0, in, len, out);
}

void oracle_derive_key(const char *context, const uint8_t *material, size_t len, uint8_t out[32])
{
    uint32_t key[8];
    b3_context_key(context, key);
    b3_hash(key, F_DERIVE_MATERIAL, material, len, out);
}

/* ── PoSE node hash, keys, descriptor, chunk seed ───────────────────────── */

void oracle_label_keys(uint32_t ksrc[8], uint32_t kint[8])
{
    b3_context_key("pose-db/label/src", ksrc);
    b3_context_key("pose-db/label/int", kint);
}

static uint32_t g_ksrc[8], g_kint[8];
static int g_keys;

void oracle_label_node(uint8_t out[32], int is_source, uint64_t node_index,
                       const uint8_t *pred0, const uint8_t *pred1,
                       const uint8_t seed[32], const uint8_t desc[32])
{
    if (!g_keys) { oracle_label_keys(g_ksrc, g_kint); g_keys = 1; }
    uint8_t msg[192];
    memset(msg, 0, sizeof(msg));
    for (int i = 0; i < 8; i++) msg[i] = (uint8_t)(node_index >> (56 - 8 * i));
    if (!is_source && pred0) memcpy(msg + 64, pred0, 32);
    if (!is_source && pred1) memcpy(msg + 96, pred1, 32);
    memcpy(msg + 128, seed, 32);
    memcpy(msg + 160, desc, 32);
    b3_hash(is_source ? g_ksrc : g_kint, F_KEYED_HASH, msg, sizeof(msg), out);
}

static void be64(uint8_t *p, uint64_t v)
{
    for (int i = 0; i < 8; i++) p[i] = (uint8_t)(v >> (56 - 8 * i));
}

void oracle_descriptor(uint8_t out[32], uint64_t m, uint64_t n)
{
    uint8_t buf[24];
    be64(buf, m); be64(buf + 8, n); be64(buf + 16, 256);
    oracle_derive_key("pose-db/descriptor", buf, sizeof(buf), out);
}

void oracle_chunk_seed(uint8_t out[32], const uint8_t *seed, size_t seed_len, uint64_t chunk_index)
{
    uint8_t *buf = (uint8_t *)malloc(seed_len + 8);
    if (!buf) { memset(out, 0, 32); return; }
    memcpy(buf, seed, seed_len);
    be64(buf + seed_len, chunk_index);
    oracle_derive_key("pose-db/chunk-seed", buf, seed_len + 8, out);
    free(buf);
}

/* ── pose-db-drg-v1 topology (edge mode) ─────────────────────────────────── */

int oracle_parameter_n(uint64_t m)
{
    if (m <= 1) return 0;
    int bits = 0;
    for (uint64_t v = m - 1; v; v >>= 1) bits++;
    return bits - 1;
}

static uint64_t cnt_butterfly(int d) { return (uint64_t)(d + 1) << d; }
static uint64_t cnt_connected(int l) { return l == 0 ? 1 : 2 * cnt_connected(l - 1) + 2 * cnt_butterfly(l - 1); }
static uint64_t cnt_standalone(int l)
{
    return l == 0 ? 1 : cnt_standalone(l - 1) + cnt_butterfly(l - 1) + cnt_connected(l - 1);
}

uint64_t oracle_node_count(uint64_t m)
{
    return 2 * cnt_standalone(oracle_parameter_n(m) + 1);
}

typedef struct {
    uint64_t next;
    uint8_t *np;
    uint32_t *p0, *p1;
} em_t;

static uint32_t node1(em_t *e, uint32_t a)
{
    uint32_t id = (uint32_t)e->next++;
    e->np[id] = 1; e->p0[id] = a; e->p1[id] = 0;
    return id;
}
static uint32_t node2(em_t *e, uint32_t a, uint32_t b)
{
    uint32_t id = (uint32_t)e->next++;
    e->np[id] = 2; e->p0[id] = a < b ? a : b; e->p1[id] = a < b ? b : a;
    return id;
}

/* Butterfly connector (graph.c:156-264 edge path): a one-pred layer, then dim
 * two-pred layers pairing i with i ^ 2^(dim-1-k). */
static void em_connector(em_t *e, int dim, const uint32_t *in, uint32_t *out)
{
    int w = 1 << dim;
    uint32_t *a = (uint32_t *)malloc(sizeof(uint32_t) * w), *b = (uint32_t *)malloc(sizeof(uint32_t) * w);
    for (int i = 0; i < w; i++) a[i] = node1(e, in[i]);
    for (int k = 0; k < dim; k++) {
        int bit = 1 << (dim - 1 - k);
        for (int i = 0; i < w; i++) b[i] = node2(e, a[i], a[i ^ bit]);
        uint32_t *t = a; a = b; b = t;
    }
    memcpy(out, a, sizeof(uint32_t) * w);
    free(a); free(b);
}

/* Merged center ingress (graph.c:466-520 edge path): the whole ingress
 * butterfly over ingress_inputs, then the center butterfly whose layer 0
 * pairs primary[i] with the last ingress layer. */
static void em_merged(em_t *e, int dim, const uint32_t *prim, const uint32_t *ingr, uint32_t *out)
{
    int w = 1 << dim;
    uint32_t *a = (uint32_t *)malloc(sizeof(uint32_t) * w), *b = (uint32_t *)malloc(sizeof(uint32_t) * w);
    for (int i = 0; i < w; i++) a[i] = node1(e, ingr[i]);
    for (int k = 1; k <= dim; k++) {
        int bit = 1 << (dim - k);
        for (int i = 0; i < w; i++) b[i] = node2(e, a[i], a[i ^ bit]);
        uint32_t *t = a; a = b; b = t;
    }
    for (int i = 0; i < w; i++) b[i] = node2(e, prim[i], a[i]);
    { uint32_t *t = a; a = b; b = t; }
    for (int k = 1; k <= dim; k++) {
        int bit = 1 << (dim - k);
        for (int i = 0; i < w; i++) b[i] = node2(e, a[i], a[i ^ bit]);
        uint32_t *t = a; a = b; b = t;
    }
    memcpy(out, a, sizeof(uint32_t) * w);
    free(a); free(b);
}

static void em_connected(em_t *e, int level, const uint32_t *in, uint32_t *out)
{
    if (level == 0) { out[0] = node1(e, in[0]); return; }
    int h = 1 << (level - 1);
    uint32_t *l = (uint32_t *)malloc(sizeof(uint32_t) * h), *c = (uint32_t *)malloc(sizeof(uint32_t) * h);
    em_connected(e, level - 1, in, l);
    em_merged(e, level - 1, l, in + h, c);
    em_connected(e, level - 1, c, out + h);
    memcpy(out, l, sizeof(uint32_t) * h);
    free(l); free(c);
}

static void em_standalone(em_t *e, int level, uint32_t *out)
{
    if (level == 0) {
        uint32_t id = (uint32_t)e->next++;
        e->np[id] = 0; e->p0[id] = 0; e->p1[id] = 0;
        out[0] = id;
        return;
    }
    int h = 1 << (level - 1);
    uint32_t *c = (uint32_t *)malloc(sizeof(uint32_t) * h);
    em_standalone(e, level - 1, out);
    em_connector(e, level - 1, out, c);
    em_connected(e, level - 1, c, out + h);
    free(c);
}

/* pose_graph_edges restated: fills np/p0/p1/rank for the whole chunk of m
 * outputs.  Arrays must hold oracle_node_count(m) entries.  Returns the
 * count, or 0 when m is out of range (0 or > 2^20). */
uint64_t oracle_edges(uint64_t m, uint8_t *np, uint32_t *p0, uint32_t *p1, int32_t *rank)
{
    if (m == 0 || m > (1u << 20)) return 0;
    int n = oracle_parameter_n(m), level = n + 1;
    uint64_t half_w = (uint64_t)1 << n, retained = m - half_w;
    uint64_t width = (uint64_t)1 << level;
    uint32_t *lb = (uint32_t *)malloc(sizeof(uint32_t) * width), *rb = (uint32_t *)malloc(sizeof(uint32_t) * width);
    em_t e = {0, np, p0, p1};
    em_standalone(&e, level, lb);
    em_standalone(&e, level, rb);
    for (uint64_t i = 0; i < e.next; i++) rank[i] = -1;
    for (uint64_t i = 0; i < half_w; i++) rank[lb[half_w + i]] = (int32_t)i;
    for (uint64_t i = 0; i < retained; i++) rank[rb[half_w + i]] = (int32_t)(half_w + i);
    free(lb); free(rb);
    return e.next;
}

/* ── chunk labeling ─────────────────────────────────────────────────────── */

/* Label one chunk of m outputs with chunk seed cseed; out = m * 32 bytes in
 * rank order.  Optionally (all != NULL) also every scaffold label in id
 * order.  Returns 0 on success, -1 on error. */
int oracle_label_chunk(const uint8_t cseed[32], uint64_t m, uint8_t *out, uint8_t *all)
{
    uint64_t count = oracle_node_count(m);
    if (m == 0 || m > (1u << 20)) return -1;
    uint8_t *np = (uint8_t *)malloc(count);
    uint32_t *p0 = (uint32_t *)malloc(4 * count), *p1 = (uint32_t *)malloc(4 * count);
    int32_t *rank = (int32_t *)malloc(4 * count);
    uint32_t *last = (uint32_t *)malloc(4 * count), *slot = (uint32_t *)malloc(4 * count);
    uint32_t *freel = (uint32_t *)malloc(4 * count);
    if (!np || !p0 || !p1 || !rank || !last || !slot || !freel) {
        free(np); free(p0); free(p1); free(rank); free(last); free(slot); free(freel);
        return -1;
    }
    oracle_edges(m, np, p0, p1, rank);
    uint8_t desc[32];
    oracle_descriptor(desc, m, (uint64_t)oracle_parameter_n(m));
    /* last reader of every node (readers come in increasing id order) */
    for (uint64_t id = 0; id < count; id++) last[id] = (uint32_t)id;
    for (uint64_t id = 0; id < count; id++) {
        if (np[id] >= 1) last[p0[id]] = (uint32_t)id;
        if (np[id] >= 2) last[p1[id]] = (uint32_t)id;
    }
    size_t cap = 1024;
    uint8_t *lab = (uint8_t *)malloc(cap * 32);
    uint64_t nfree = 0, used = 0;
    int rc = 0;
    for (uint64_t id = 0; id < count && rc == 0; id++) {
        uint32_t s;
        if (nfree) s = freel[--nfree];
        else {
            if (used == cap) {
                cap *= 2;
                uint8_t *nl = (uint8_t *)realloc(lab, cap * 32);
                if (!nl) { rc = -1; break; }
                lab = nl;
            }
            s = (uint32_t)used++;
        }
        slot[id] = s;
        const uint8_t *a = np[id] >= 1 ? lab + (size_t)slot[p0[id]] * 32 : NULL;
        const uint8_t *b = np[id] >= 2 ? lab + (size_t)slot[p1[id]] * 32 : NULL;
        uint8_t tmp[32];
        oracle_label_node(tmp, np[id] == 0, id, a, b, cseed, desc);
        memcpy(lab + (size_t)s * 32, tmp, 32);
        if (all) memcpy(all + id * 32, tmp, 32);
        if (rank[id] >= 0) memcpy(out + (size_t)rank[id] * 32, tmp, 32);
        if (np[id] >= 1 && last[p0[id]] == id) freel[nfree++] = slot[p0[id]];
        if (np[id] >= 2 && last[p1[id]] == id) freel[nfree++] = slot[p1[id]];
        if (last[id] == id) freel[nfree++] = s;
    }
    free(lab);
    free(np); free(p0); free(p1); free(rank); free(last); free(slot); free(freel);
    return rc;
}

/* Label num_super super-chunks of a region at block offset rbo (region layout
 * of pose_graph_label_region_pooled_inplace / the GPU labeler: super-chunk j
 * at j*cb*32 holds rank r at +32r). */
int oracle_label_region(const uint8_t *seed, size_t seed_len, uint32_t cb,
                        uint8_t *out, uint64_t num_super, uint64_t rbo)
{
    for (uint64_t j = 0; j < num_super; j++) {
        uint8_t cs[32];
        oracle_chunk_seed(cs, seed, seed_len, (rbo + j * (uint64_t)cb) / cb);
        if (oracle_label_chunk(cs, cb, out + j * (uint64_t)cb * 32, NULL) != 0) return -1;
    }
    return 0;
}
