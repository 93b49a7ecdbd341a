/* b3_host.h — host-side BLAKE3 for the seed-independent constants and the
 * per-chunk seeds the labeler feeds to the device (C11, internal). */
#ifndef PB_B3_HOST_H
#define PB_B3_HOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* BLAKE3 block flags (BLAKE3 specification, section 2.1). */
enum {
    PB_B3_CHUNK_START = 1u << 0,
    PB_B3_CHUNK_END = 1u << 1,
    PB_B3_PARENT = 1u << 2,
    PB_B3_ROOT = 1u << 3,
    PB_B3_KEYED_HASH = 1u << 4,
    PB_B3_DERIVE_KEY_CONTEXT = 1u << 5,
    PB_B3_DERIVE_KEY_MATERIAL = 1u << 6,
};

/* The two keyed-hash keys of the node labels, 8 little-endian words each:
 * derive_key context keys of "pose-db/label/src" (source nodes) and
 * "pose-db/label/int" (all other nodes). */
void pb_label_keys(uint32_t key_src[8], uint32_t key_int[8]);

/* derive_key("pose-db/descriptor", be64(m) | be64(n) | be64(256)). */
void pb_graph_descriptor(uint8_t out[32], uint64_t m, uint64_t n);

/* derive_key("pose-db/chunk-seed", session_seed | be64(chunk_index)). */
void pb_chunk_seed(uint8_t out[32], const uint8_t *session_seed, size_t seed_len,
                   uint64_t chunk_index);

/* Generic one-shot BLAKE3 over any input length with a key (8 words) and
 * base flags; writes the first 32 output bytes. */
void pb_b3_hash(const uint32_t key[8], uint32_t flags, const uint8_t *in, size_t len,
                uint8_t out[32]);

/* derive_key context key of a context string (8 little-endian words). */
void pb_context_key(const char *context, uint32_t key[8]);

/* pose-db-drg-v1 graph parameter n = max(0, bit_length(m-1) - 1). */
int pb_parameter_n(uint64_t m);

#ifdef __cplusplus
}
#endif
#endif
