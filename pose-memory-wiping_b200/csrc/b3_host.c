/*
 * b3_host.c — host-side BLAKE3 (C11) for the labeler's seed-independent
 * constants and per-chunk seeds.
 *
 * Written from the BLAKE3 specification (compression function, chunk
 * chaining, and the streaming chaining-value stack that merges subtrees by the
 * trailing zeros of the chunk count).  The PoSE-specific inputs follow the
 * reference:
 *   - label keys: derive_key context keys of "pose-db/label/src" and
 *     "pose-db/label/int" (common/src/hash.c:46-67);
 *   - descriptor: derive_key("pose-db/descriptor",
 *     be64(m) | be64(n) | be64(256)) (common/src/hash.c:198-216);
 *   - chunk seed: derive_key("pose-db/chunk-seed",
 *     session_seed | be64(chunk_index)) (common/src/hash.c:218-233).
 */
#include "b3_host.h"

#include <stdlib.h>
#include <string.h>

static const uint32_t kIV[8] = {
    0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
    0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u,
};

/* Message word order of each of the 7 rounds: row r is the BLAKE3 message
 * permutation applied r times. */
static const uint8_t kSchedule[7][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15},
    {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8},
    {3, 4, 10, 12, 13, 2, 7, 14, 6, 5, 9, 0, 11, 15, 8, 1},
    {10, 7, 12, 9, 14, 3, 13, 15, 4, 0, 11, 2, 5, 8, 1, 6},
    {12, 13, 9, 11, 15, 10, 14, 8, 7, 2, 5, 3, 0, 1, 6, 4},
    {9, 14, 11, 5, 8, 12, 15, 1, 13, 3, 0, 10, 2, 6, 4, 7},
    {11, 15, 5, 0, 1, 9, 8, 6, 14, 10, 2, 12, 3, 4, 7, 13},
};

static inline uint32_t rotr(uint32_t x, unsigned n) { return (x >> n) | (x << (32 - n)); }

#define QR(a, b, c, d, x, y)                                  \
    do {                                                      \
        s[a] += s[b] + (x); s[d] = rotr(s[d] ^ s[a], 16);     \
        s[c] += s[d];       s[b] = rotr(s[b] ^ s[c], 12);     \
        s[a] += s[b] + (y); s[d] = rotr(s[d] ^ s[a], 8);      \
        s[c] += s[d];       s[b] = rotr(s[b] ^ s[c], 7);      \
    } while (0)

/* Compression returning the 8-word chaining value (first half of the output). */
static void compress_cv(uint32_t cv[8], const uint32_t m[16], uint64_t ctr,
                        uint32_t len, uint32_t flags)
{
    uint32_t s[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                      kIV[0], kIV[1], kIV[2], kIV[3],
                      (uint32_t)ctr, (uint32_t)(ctr >> 32), len, flags};
    for (int r = 0; r < 7; r++) {
        const uint8_t *o = kSchedule[r];
        QR(0, 4, 8, 12, m[o[0]], m[o[1]]);
        QR(1, 5, 9, 13, m[o[2]], m[o[3]]);
        QR(2, 6, 10, 14, m[o[4]], m[o[5]]);
        QR(3, 7, 11, 15, m[o[6]], m[o[7]]);
        QR(0, 5, 10, 15, m[o[8]], m[o[9]]);
        QR(1, 6, 11, 12, m[o[10]], m[o[11]]);
        QR(2, 7, 8, 13, m[o[12]], m[o[13]]);
        QR(3, 4, 9, 14, m[o[14]], m[o[15]]);
    }
    for (int i = 0; i < 8; i++) cv[i] = s[i] ^ s[i + 8];
}

static void words_le(uint32_t *w, const uint8_t *p, size_t nbytes)
{
    uint8_t blk[64];
    memset(blk, 0, sizeof(blk));
    memcpy(blk, p, nbytes);
    for (int i = 0; i < 16; i++)
        w[i] = (uint32_t)blk[4 * i] | ((uint32_t)blk[4 * i + 1] << 8) |
               ((uint32_t)blk[4 * i + 2] << 16) | ((uint32_t)blk[4 * i + 3] << 24);
}

/* Chaining value of one chunk (len <= 1024; len 0 only for an empty root). */
static void chunk_cv(const uint32_t key[8], uint32_t flags, const uint8_t *in, size_t len,
                     uint64_t counter, int root, uint32_t out[8])
{
    memcpy(out, key, 32);
    size_t off = 0;
    do {
        size_t take = len - off > 64 ? 64 : len - off;
        uint32_t m[16];
        words_le(m, in + off, take);
        uint32_t f = flags | (off == 0 ? PB_B3_CHUNK_START : 0);
        int last = off + take >= len;
        if (last) f |= PB_B3_CHUNK_END | (root ? PB_B3_ROOT : 0);
        compress_cv(out, m, counter, (uint32_t)take, f);
        off += take;
    } while (off < len);
}

static void parent_cv(const uint32_t key[8], uint32_t flags, const uint32_t l[8],
                      const uint32_t r[8], int root, uint32_t out[8])
{
    uint32_t m[16];
    memcpy(m, l, 32);
    memcpy(m + 8, r, 32);
    memcpy(out, key, 32);
    compress_cv(out, m, 0, 64, flags | PB_B3_PARENT | (root ? PB_B3_ROOT : 0));
}

void pb_b3_hash(const uint32_t key[8], uint32_t flags, const uint8_t *in, size_t len,
                uint8_t out[32])
{
    uint32_t cv[8];
    size_t nchunks = len == 0 ? 1 : (len + 1023) / 1024;
    if (nchunks == 1) {
        chunk_cv(key, flags, in, len, 0, 1, cv);
    } else {
        uint32_t stack[64][8];
        int depth = 0;
        for (size_t i = 0; i + 1 < nchunks; i++) {
            uint32_t c[8];
            chunk_cv(key, flags, in + i * 1024, 1024, i, 0, c);
            /* merge completed subtrees: as many as the trailing zeros of the
             * number of chunks absorbed so far */
            for (uint64_t t = (uint64_t)i + 1; (t & 1) == 0; t >>= 1) {
                uint32_t p[8];
                parent_cv(key, flags, stack[--depth], c, 0, p);
                memcpy(c, p, 32);
            }
            memcpy(stack[depth++], c, 32);
        }
        size_t last = nchunks - 1;
        chunk_cv(key, flags, in + last * 1024, len - last * 1024, last, 0, cv);
        while (depth > 0) {
            uint32_t p[8];
            depth--;
            parent_cv(key, flags, stack[depth], cv, depth == 0, p);
            memcpy(cv, p, 32);
        }
    }
    for (int i = 0; i < 8; i++) {
        out[4 * i] = (uint8_t)cv[i];
        out[4 * i + 1] = (uint8_t)(cv[i] >> 8);
        out[4 * i + 2] = (uint8_t)(cv[i] >> 16);
        out[4 * i + 3] = (uint8_t)(cv[i] >> 24);
    }
}

void pb_context_key(const char *ctx, uint32_t key[8])
{
    uint8_t k[32];
    pb_b3_hash(kIV, PB_B3_DERIVE_KEY_CONTEXT, (const uint8_t *)ctx, strlen(ctx), k);
    for (int i = 0; i < 8; i++)
        key[i] = (uint32_t)k[4 * i] | ((uint32_t)k[4 * i + 1] << 8) |
                 ((uint32_t)k[4 * i + 2] << 16) | ((uint32_t)k[4 * i + 3] << 24);
}

void pb_label_keys(uint32_t key_src[8], uint32_t key_int[8])
{
    pb_context_key("pose-db/label/src", key_src);
    pb_context_key("pose-db/label/int", key_int);
}

static void put_be64(uint8_t *p, uint64_t v)
{
    for (int i = 0; i < 8; i++) p[i] = (uint8_t)(v >> (56 - 8 * i));
}

void pb_graph_descriptor(uint8_t out[32], uint64_t m, uint64_t n)
{
    uint32_t key[8];
    uint8_t buf[24];
    put_be64(buf, m);
    put_be64(buf + 8, n);
    put_be64(buf + 16, 256);
    pb_context_key("pose-db/descriptor", key);
    pb_b3_hash(key, PB_B3_DERIVE_KEY_MATERIAL, buf, sizeof(buf), out);
}

void pb_chunk_seed(uint8_t out[32], const uint8_t *session_seed, size_t seed_len,
                   uint64_t chunk_index)
{
    uint32_t key[8];
    pb_context_key("pose-db/chunk-seed", key);
    uint8_t small[256];
    uint8_t *buf = seed_len + 8 <= sizeof(small) ? small : (uint8_t *)malloc(seed_len + 8);
    if (!buf) { memset(out, 0, 32); return; }
    if (seed_len) memcpy(buf, session_seed, seed_len);
    put_be64(buf + seed_len, chunk_index);
    pb_b3_hash(key, PB_B3_DERIVE_KEY_MATERIAL, buf, seed_len + 8, out);
    if (buf != small) free(buf);
}

int pb_parameter_n(uint64_t m)
{
    if (m <= 1) return 0;
    int bits = 64 - __builtin_clzll(m - 1);
    return bits - 1;
}
