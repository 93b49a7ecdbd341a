/*
 * b3_device.cuh — register-resident BLAKE3 compression for sm_100a.
 *
 * Written from the BLAKE3 specification.  The 16-word state stays in
 * registers for the whole compression; the message schedule is resolved at
 * compile time (round r reads message word sched(r, i), the BLAKE3 message
 * permutation applied r times), so permuting costs no instructions.  The G
 * function maps to the minimal integer form: a three-input add (IADD3) for
 * a + b + m, a two-input add for c + d, a LOP3 xor before each rotation,
 * byte permutes (PRMT) for the rotations by 16 and 8 and funnel shifts (SHF)
 * for 12 and 7.
 */
#ifndef PB_B3_DEVICE_CUH
#define PB_B3_DEVICE_CUH

#include <cstdint>

namespace pb {

/* BLAKE3 flags used by the node hash. */
constexpr uint32_t kFlagChunkStart = 1u << 0;
constexpr uint32_t kFlagChunkEnd = 1u << 1;
constexpr uint32_t kFlagRoot = 1u << 3;
constexpr uint32_t kFlagKeyed = 1u << 4;
constexpr uint32_t kFlagDeriveMaterial = 1u << 6;

/* Node message blocks: block 0 (node index) starts the chunk, block 2
 * (seed | descriptor) ends it and is the root (common/src/hash.c:136-140). */
constexpr uint32_t kFlagsBlock0 = kFlagKeyed | kFlagChunkStart;
constexpr uint32_t kFlagsBlock1 = kFlagKeyed;
constexpr uint32_t kFlagsBlock2 = kFlagKeyed | kFlagChunkEnd | kFlagRoot;

constexpr uint32_t kIV0 = 0x6A09E667u, kIV1 = 0xBB67AE85u, kIV2 = 0x3C6EF372u,
                   kIV3 = 0xA54FF53Au, kIV4 = 0x510E527Fu, kIV5 = 0x9B05688Cu,
                   kIV6 = 0x1F83D9ABu, kIV7 = 0x5BE0CD19u;

__host__ __device__ constexpr int perm16(int i)
{
    /* BLAKE3 message permutation */
    return i == 0 ? 2 : i == 1 ? 6 : i == 2 ? 3 : i == 3 ? 10 : i == 4 ? 7 : i == 5 ? 0
         : i == 6 ? 4 : i == 7 ? 13 : i == 8 ? 1 : i == 9 ? 11 : i == 10 ? 12
         : i == 11 ? 5 : i == 12 ? 9 : i == 13 ? 14 : i == 14 ? 15 : 8;
}

__host__ __device__ constexpr int sched(int r, int i)
{
    return r == 0 ? i : sched(r - 1, perm16(i));
}

__device__ __forceinline__ uint32_t rotr16(uint32_t x) { return __byte_perm(x, 0, 0x1032); }
__device__ __forceinline__ uint32_t rotr8(uint32_t x) { return __byte_perm(x, 0, 0x0321); }
__device__ __forceinline__ uint32_t rotr12(uint32_t x) { return __funnelshift_r(x, x, 12); }
__device__ __forceinline__ uint32_t rotr7(uint32_t x) { return __funnelshift_r(x, x, 7); }

__device__ __forceinline__ void g_mix(uint32_t &a, uint32_t &b, uint32_t &c, uint32_t &d,
                                      uint32_t x, uint32_t y)
{
    a = a + b + x;
    d = rotr16(d ^ a);
    c = c + d;
    b = rotr12(b ^ c);
    a = a + b + y;
    d = rotr8(d ^ a);
    c = c + d;
    b = rotr7(b ^ c);
}

/* The same G with its additions issued as integer multiply-adds by a
 * run-time 1 (`one`, opaque to the compiler): they then execute on the FMA
 * pipe instead of the integer ALU pipe, which otherwise carries all twelve
 * operations of G (adds, xors, funnel shifts and byte permutes) and bounds
 * throughput when every SM is full.  a + b + m becomes two multiply-adds
 * (b*1 + m, then a*1 + that), so the dependent chain is longer: use it where
 * throughput, not latency, is the limit. */
__device__ __forceinline__ uint32_t madd(uint32_t a, uint32_t one, uint32_t b)
{
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(one), "r"(b));
    return r;
}

__device__ __forceinline__ void g_mix_fma(uint32_t &a, uint32_t &b, uint32_t &c, uint32_t &d,
                                          uint32_t x, uint32_t y, uint32_t one)
{
    a = madd(a, one, madd(b, one, x));
    d = rotr16(d ^ a);
    c = madd(c, one, d);
    b = rotr12(b ^ c);
    a = madd(a, one, madd(b, one, y));
    d = rotr8(d ^ a);
    c = madd(c, one, d);
    b = rotr7(b ^ c);
}

template <int R>
__device__ __forceinline__ void round_fma(uint32_t (&v)[16], const uint32_t (&m)[16], uint32_t one)
{
    g_mix_fma(v[0], v[4], v[8], v[12], m[sched(R, 0)], m[sched(R, 1)], one);
    g_mix_fma(v[1], v[5], v[9], v[13], m[sched(R, 2)], m[sched(R, 3)], one);
    g_mix_fma(v[2], v[6], v[10], v[14], m[sched(R, 4)], m[sched(R, 5)], one);
    g_mix_fma(v[3], v[7], v[11], v[15], m[sched(R, 6)], m[sched(R, 7)], one);
    g_mix_fma(v[0], v[5], v[10], v[15], m[sched(R, 8)], m[sched(R, 9)], one);
    g_mix_fma(v[1], v[6], v[11], v[12], m[sched(R, 10)], m[sched(R, 11)], one);
    g_mix_fma(v[2], v[7], v[8], v[13], m[sched(R, 12)], m[sched(R, 13)], one);
    g_mix_fma(v[3], v[4], v[9], v[14], m[sched(R, 14)], m[sched(R, 15)], one);
}

template <int R>
__device__ __forceinline__ void round_fn(uint32_t (&v)[16], const uint32_t (&m)[16])
{
    g_mix(v[0], v[4], v[8], v[12], m[sched(R, 0)], m[sched(R, 1)]);
    g_mix(v[1], v[5], v[9], v[13], m[sched(R, 2)], m[sched(R, 3)]);
    g_mix(v[2], v[6], v[10], v[14], m[sched(R, 4)], m[sched(R, 5)]);
    g_mix(v[3], v[7], v[11], v[15], m[sched(R, 6)], m[sched(R, 7)]);
    g_mix(v[0], v[5], v[10], v[15], m[sched(R, 8)], m[sched(R, 9)]);
    g_mix(v[1], v[6], v[11], v[12], m[sched(R, 10)], m[sched(R, 11)]);
    g_mix(v[2], v[7], v[8], v[13], m[sched(R, 12)], m[sched(R, 13)]);
    g_mix(v[3], v[4], v[9], v[14], m[sched(R, 14)], m[sched(R, 15)]);
}

/* One compression with counter 0: cv <- first 8 output words (the chaining
 * value; for a ROOT block these are the first 32 output bytes). */
__device__ __forceinline__ void compress(uint32_t (&cv)[8], const uint32_t (&m)[16],
                                         uint32_t block_len, uint32_t flags)
{
    uint32_t v[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                      kIV0,  kIV1,  kIV2,  kIV3,  0u,    0u,    block_len, flags};
    round_fn<0>(v, m);
    round_fn<1>(v, m);
    round_fn<2>(v, m);
    round_fn<3>(v, m);
    round_fn<4>(v, m);
    round_fn<5>(v, m);
    round_fn<6>(v, m);
#pragma unroll
    for (int i = 0; i < 8; i++) cv[i] = v[i] ^ v[i + 8];
}

/* compress() with the FMA-pipe additions of g_mix_fma (same result). */
__device__ __forceinline__ void compress_fma(uint32_t (&cv)[8], const uint32_t (&m)[16],
                                             uint32_t block_len, uint32_t flags, uint32_t one)
{
    uint32_t v[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                      kIV0,  kIV1,  kIV2,  kIV3,  0u,    0u,    block_len, flags};
    round_fma<0>(v, m, one);
    round_fma<1>(v, m, one);
    round_fma<2>(v, m, one);
    round_fma<3>(v, m, one);
    round_fma<4>(v, m, one);
    round_fma<5>(v, m, one);
    round_fma<6>(v, m, one);
#pragma unroll
    for (int i = 0; i < 8; i++) cv[i] = v[i] ^ v[i + 8];
}

/* Block 0 of a node message: node index big-endian in bytes 0..7, the rest
 * zero.  As little-endian words: w0 = bswap(index >> 32), w1 = bswap(index). */
__device__ __forceinline__ void block0_words(uint32_t (&m)[16], uint64_t node_index)
{
    m[0] = __byte_perm((uint32_t)(node_index >> 32), 0, 0x0123);
    m[1] = __byte_perm((uint32_t)node_index, 0, 0x0123);
#pragma unroll
    for (int i = 2; i < 16; i++) m[i] = 0;
}

} /* namespace pb */

#endif
