/*
 * label_kernels.cu — sm_100a labeling kernels and their C-ABI launchers.
 *
 * Replaces the reference's per-strategy kernels (common/src/cuda/
 * label_gpu_{level,block,thread,warp}.cu) and its device hash
 * (common/src/cuda/blake3_node.cuh:195-230) with one persistent kernel:
 *
 *   - A "unit" is one standalone copy of one chunk (left copy: node ids
 *     [0, S); right copy: ids [S, 2S)).  Both copies share the topology
 *     records, so a team runs G units of the same topology in lockstep and a
 *     level of width w becomes G*w independent node hashes.  That packs the
 *     many narrow levels of the depth-robust DAG into full warps.
 *   - A team is T warps (T = 1: __syncwarp between levels; T > 1: a named
 *     barrier per team).  Teams pull batches of G units from a device work
 *     counter until the launch's units are exhausted (no waiting on other
 *     teams, so no spin-waits exist anywhere).
 *   - Scratch is the recycled slot pool of the topology, one per unit,
 *     interleaved by unit: label (slot s, unit u) lives at
 *     team_base + (s*G + u)*32, so the G lanes that hash the same node read
 *     and write G adjacent labels (coalesced 128-bit accesses).
 *   - Block 0 of a node message depends only on (key type, node index): it
 *     is either hashed in registers while the parent loads are in flight, or
 *     read from a per-topology chaining-value table built once per
 *     chunk_blocks (k_cv0_table).  Output bytes are identical either way.
 *   - An output node's label is also stored to the persisted super-chunk at
 *     its challenge rank the moment it is computed
 *     (label_gpu_warp.cu:110-117 does the same).
 */
#include "b3_device.cuh"
#include "kernels.h"

#include <cuda_runtime.h>
#include <stdint.h>

namespace pb {

__constant__ uint32_t c_key_src[8];
__constant__ uint32_t c_key_int[8];
__constant__ uint32_t c_key_chunk_seed[8];

__device__ __forceinline__ void team_sync(uint32_t team_warps, uint32_t bar_id, uint32_t nthreads)
{
    if (team_warps == 1) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
    }
}

__device__ __forceinline__ void key_words(uint32_t (&cv)[8], bool source)
{
#pragma unroll
    for (int i = 0; i < 8; i++) cv[i] = source ? c_key_src[i] : c_key_int[i];
}

/* ── per-topology block-0 chaining values ─────────────────────────────────── */

/* cv0[(copy*S + pos)*2 + {0,1}] = chaining value after block 0 of the node at
 * level-order position pos in copy `copy` (node index id + copy*S). */
__global__ void __launch_bounds__(256) k_cv0_table(const uint4 *__restrict__ recs, uint32_t S,
                                                    uint32_t copies, uint4 *__restrict__ cv0)
{
    uint64_t total = (uint64_t)S * copies;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total;
         k += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t copy = (uint32_t)(k / S), pos = (uint32_t)(k % S);
        uint32_t x = recs[pos].x;
        uint32_t id = (x & PB_REC_ID_MASK) + copy * S;
        uint32_t np = (x >> PB_REC_NP_SHIFT) & 3u;
        uint32_t cv[8], m[16];
        key_words(cv, np == 0);
        block0_words(m, id);
        compress(cv, m, 64, kFlagsBlock0);
        cv0[2 * k] = make_uint4(cv[0], cv[1], cv[2], cv[3]);
        cv0[2 * k + 1] = make_uint4(cv[4], cv[5], cv[6], cv[7]);
    }
}

/* ── chunk seeds on the device ───────────────────────────────────────────── */

/* seeds[8*j..] = derive_key("pose-db/chunk-seed",
 *   session_seed | be64((rbo + j*cb) / cb))  (common/src/hash.c:218-233,
 * chunk index as common/src/graph.c:1646-1649).  One thread per chunk; the
 * material (seed_len + 8 <= 1024 bytes) is one BLAKE3 chunk. */
__global__ void __launch_bounds__(128) k_chunk_seeds(const uint8_t *__restrict__ session_seed,
                                                      uint32_t seed_len, uint64_t rbo, uint32_t cb,
                                                      uint32_t nchunks, uint64_t first_super,
                                                      uint32_t *__restrict__ seeds)
{
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nchunks) return;
    uint64_t idx = (rbo + (first_super + j) * (uint64_t)cb) / cb;
    uint32_t len = seed_len + 8;
    uint32_t nblocks = (len + 63) / 64;
    uint32_t cv[8];
#pragma unroll
    for (int i = 0; i < 8; i++) cv[i] = c_key_chunk_seed[i];
    for (uint32_t b = 0; b < nblocks; b++) {
        uint32_t m[16];
#pragma unroll
        for (int i = 0; i < 16; i++) {
            uint32_t w = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                uint32_t off = b * 64 + 4 * i + k;
                uint32_t byte = 0;
                if (off < seed_len) byte = session_seed[off];
                else if (off < len) byte = (uint32_t)(idx >> (8 * (7 - (off - seed_len)))) & 0xFFu;
                w |= byte << (8 * k);
            }
            m[i] = w;
        }
        uint32_t blen = (b + 1 == nblocks) ? len - b * 64 : 64;
        uint32_t flags = kFlagDeriveMaterial | (b == 0 ? kFlagChunkStart : 0u) |
                         (b + 1 == nblocks ? (kFlagChunkEnd | kFlagRoot) : 0u);
        compress(cv, m, blen, flags);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) seeds[8 * (size_t)j + i] = cv[i];
}

/* ── the labeling kernel ─────────────────────────────────────────────────── */

template <bool FMA>
__global__ void __launch_bounds__(PB_CTA_THREADS) k_label(const __grid_constant__ pb_label_params_t p)
{
    const uint32_t T = p.team_warps;
    const uint32_t TT = T * 32;
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t team = warp / T;
    const uint32_t tt = threadIdx.x - team * TT;
    const uint32_t teams_per_cta = blockDim.x / TT;
    const uint64_t gteam = (uint64_t)blockIdx.x * teams_per_cta + team;
    const uint32_t bar_id = 1 + team;
    const uint32_t glog = p.g_log2;
    const uint32_t G = 1u << glog;
    const uint32_t u = tt & (G - 1);
    const uint32_t q = tt >> glog;
    const uint32_t stride = TT >> glog;
    uint4 *tscr = reinterpret_cast<uint4 *>(p.scratch + gteam * p.team_scratch_bytes);
    const pb_topo_view_t &tp = p.topo;
    __shared__ uint32_t s_batch[PB_CTA_THREADS / 32];

    for (;;) {
        uint32_t batch;
        if (T == 1) {
            uint32_t b = 0;
            if ((threadIdx.x & 31) == 0) b = atomicAdd(p.queue, 1u);
            batch = __shfl_sync(0xFFFFFFFFu, b, 0);
        } else {
            if (tt == 0) s_batch[team] = atomicAdd(p.queue, 1u);
            team_sync(T, bar_id, TT);
            batch = s_batch[team];
            team_sync(T, bar_id, TT);
        }
        if (batch >= p.nbatches) break;

        const uint32_t unit = (batch << glog) + u;
        const bool valid = unit < p.nunits;
        const uint32_t chunk = unit >> p.copies_log2;
        const uint32_t copy = unit & ((1u << p.copies_log2) - 1u);
        const uint32_t id_off = copy ? tp.S : 0u;
        const uint32_t rank_base = copy ? tp.half_w : 0u;
        const uint32_t rank_lim = copy ? tp.retained : tp.half_w;
        uint8_t *out = p.persist + (uint64_t)(p.first_super + chunk) * p.super_bytes;
        const uint4 *cv0 = tp.cv0 ? tp.cv0 + (uint64_t)copy * tp.S * 2 : nullptr;
        uint32_t seed[8];
#pragma unroll
        for (int i = 0; i < 8; i++) seed[i] = valid ? p.seeds[8 * (size_t)chunk + i] : 0u;

        for (uint32_t l = 0; l < tp.L; l++) {
            const uint32_t s0 = __ldg(tp.lstart + l);
            const uint32_t w = __ldg(tp.lstart + l + 1) - s0;
            if (valid) {
                for (uint32_t j = q; j < w; j += stride) {
                    const uint32_t pos = s0 + j;
                    const uint4 rec = __ldg(tp.recs + pos);
                    const uint32_t np = (rec.x >> PB_REC_NP_SHIFT) & 3u;
                    uint32_t m[16];
                    if (np >= 1) {
                        const uint4 *s = tscr + (((size_t)rec.y << glog) + u) * 2;
                        uint4 a = s[0], b = s[1];
                        m[0] = a.x; m[1] = a.y; m[2] = a.z; m[3] = a.w;
                        m[4] = b.x; m[5] = b.y; m[6] = b.z; m[7] = b.w;
                    } else {
#pragma unroll
                        for (int i = 0; i < 8; i++) m[i] = 0;
                    }
                    if (np >= 2) {
                        const uint4 *s = tscr + (((size_t)rec.z << glog) + u) * 2;
                        uint4 a = s[0], b = s[1];
                        m[8] = a.x; m[9] = a.y; m[10] = a.z; m[11] = a.w;
                        m[12] = b.x; m[13] = b.y; m[14] = b.z; m[15] = b.w;
                    } else {
#pragma unroll
                        for (int i = 8; i < 16; i++) m[i] = 0;
                    }
                    uint32_t cv[8];
                    if (cv0) {
                        const uint4 c0 = __ldg(cv0 + 2 * (size_t)pos);
                        const uint4 c1 = __ldg(cv0 + 2 * (size_t)pos + 1);
                        cv[0] = c0.x; cv[1] = c0.y; cv[2] = c0.z; cv[3] = c0.w;
                        cv[4] = c1.x; cv[5] = c1.y; cv[6] = c1.z; cv[7] = c1.w;
                    } else {
                        uint32_t m0[16];
                        key_words(cv, np == 0);
                        block0_words(m0, (rec.x & PB_REC_ID_MASK) + id_off);
                        if (FMA) compress_fma(cv, m0, 64, kFlagsBlock0, p.one);
                        else compress(cv, m0, 64, kFlagsBlock0);
                    }
                    uint32_t m2[16];
#pragma unroll
                    for (int i = 0; i < 8; i++) { m2[i] = seed[i]; m2[8 + i] = tp.desc[i]; }
                    if (FMA) {
                        compress_fma(cv, m, 64, kFlagsBlock1, p.one);
                        compress_fma(cv, m2, 64, kFlagsBlock2, p.one);
                    } else {
                        compress(cv, m, 64, kFlagsBlock1);
                        compress(cv, m2, 64, kFlagsBlock2);
                    }
                    const uint4 o0 = make_uint4(cv[0], cv[1], cv[2], cv[3]);
                    const uint4 o1 = make_uint4(cv[4], cv[5], cv[6], cv[7]);
                    uint4 *d = tscr + (((size_t)rec.w << glog) + u) * 2;
                    d[0] = o0;
                    d[1] = o1;
                    if (rec.x & PB_REC_OUT_BIT) {
                        const uint32_t r = __ldg(tp.orank + pos);
                        if (r < rank_lim) {
                            uint4 *o = reinterpret_cast<uint4 *>(out + (size_t)(rank_base + r) * 32);
                            o[0] = o0;
                            o[1] = o1;
                        }
                    }
                }
            }
            team_sync(T, bar_id, TT);
        }
    }
}

/* ── known-answer single node ────────────────────────────────────────────── */

/* in = pred0[8] | pred1[8] | seed[8] | descriptor[8] | key_src[8] | key_int[8]
 * (little-endian words); the caller's keys are used, as the reference KAT
 * helper does (common/src/cuda/blake3_node.cu:18-29). */
__global__ void k_label_single(uint32_t *out, int is_source, uint64_t node_index,
                               const uint32_t *in, int have_p0, int have_p1)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t cv[8], m[16];
#pragma unroll
    for (int i = 0; i < 8; i++) cv[i] = is_source ? in[32 + i] : in[40 + i];
    block0_words(m, node_index);
    compress(cv, m, 64, kFlagsBlock0);
#pragma unroll
    for (int i = 0; i < 8; i++) {
        m[i] = (!is_source && have_p0) ? in[i] : 0u;
        m[8 + i] = (!is_source && have_p1) ? in[8 + i] : 0u;
    }
    compress(cv, m, 64, kFlagsBlock1);
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = in[16 + i];
    compress(cv, m, 64, kFlagsBlock2);
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = cv[i];
}

/* ── compression-rate microbenchmark (the INT32 roofline denominator) ───── */

/* Each thread chains `iters` node-style compressions (block 1 then block 2
 * message shapes) entirely in registers; xor-folds the result to `sink` so the
 * work cannot be elided.  Counting compressions / time with every SM full
 * gives the sustained compression rate of this GPU for the exact instruction
 * mix the labeler issues. */
template <bool FMA>
__global__ void __launch_bounds__(256) k_compress_bench(uint32_t iters, uint32_t salt,
                                                        uint32_t *sink, uint32_t one)
{
    uint32_t cv[8], m[16];
#pragma unroll
    for (int i = 0; i < 8; i++) cv[i] = threadIdx.x * 0x9E3779B9u + i + salt;
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = blockIdx.x * 0x85EBCA6Bu + i * 0x27D4EB2Fu;
    for (uint32_t k = 0; k < iters; k++) {
        if (FMA) compress_fma(cv, m, 64, kFlagsBlock1, one);
        else compress(cv, m, 64, kFlagsBlock1);
#pragma unroll
        for (int i = 0; i < 8; i++) m[i] ^= cv[i];
    }
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) x ^= cv[i];
    if (x == 0x12345678u) sink[blockIdx.x] = x; /* practically never stored */
}

/* Dependent-latency probe: one thread chains `iters` compressions and reports
 * the elapsed SM clocks. */
__global__ void k_compress_latency(uint32_t iters, unsigned long long *cycles, uint32_t *sink)
{
    uint32_t cv[8], m[16];
#pragma unroll
    for (int i = 0; i < 8; i++) cv[i] = threadIdx.x + i;
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = i * 0x27D4EB2Fu;
    unsigned long long t0 = clock64();
    for (uint32_t k = 0; k < iters; k++) compress(cv, m, 64, kFlagsBlock1);
    unsigned long long t1 = clock64();
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) x ^= cv[i];
    sink[0] = x;
    cycles[0] = t1 - t0;
}

} /* namespace pb */

/* ── C-ABI launchers (called from the C11 host code) ─────────────────────── */

extern "C" int pb_dev_set_keys(const uint32_t ksrc[8], const uint32_t kint[8],
                               const uint32_t kseed[8])
{
    if (cudaMemcpyToSymbol(pb::c_key_src, ksrc, 32) != cudaSuccess) return -1;
    if (cudaMemcpyToSymbol(pb::c_key_int, kint, 32) != cudaSuccess) return -1;
    if (cudaMemcpyToSymbol(pb::c_key_chunk_seed, kseed, 32) != cudaSuccess) return -1;
    return 0;
}

extern "C" int pb_dev_cv0_table(const void *recs, uint32_t S, uint32_t copies, void *cv0,
                                cudaStream_t stream)
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint64_t total = (uint64_t)S * copies;
    uint64_t blocks = (total + 255) / 256;
    uint64_t cap = (uint64_t)(sms > 0 ? sms : 148) * 8;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    pb::k_cv0_table<<<(unsigned)blocks, 256, 0, stream>>>((const uint4 *)recs, S, copies,
                                                          (uint4 *)cv0);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_chunk_seeds(const uint8_t *d_session_seed, uint32_t seed_len, uint64_t rbo,
                                  uint32_t cb, uint32_t nchunks, uint64_t first_super,
                                  uint32_t *d_seeds, cudaStream_t stream)
{
    if (nchunks == 0) return 0;
    pb::k_chunk_seeds<<<(nchunks + 127) / 128, 128, 0, stream>>>(d_session_seed, seed_len, rbo, cb,
                                                                  nchunks, first_super, d_seeds);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_label(const pb_label_params_t *params, uint32_t grid, uint32_t cta_threads,
                            cudaStream_t stream)
{
    if (params->fma_adds) pb::k_label<true><<<grid, cta_threads, 0, stream>>>(*params);
    else pb::k_label<false><<<grid, cta_threads, 0, stream>>>(*params);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_label_occupancy(uint32_t cta_threads, int *blocks_per_sm)
{
    int a = 0, b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, pb::k_label<false>, (int)cta_threads, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, pb::k_label<true>, (int)cta_threads, 0) != cudaSuccess)
        return -1;
    *blocks_per_sm = a < b ? a : b;
    return 0;
}

extern "C" int pb_dev_label_single(uint32_t *d_out, int is_source, uint64_t node_index,
                                   const uint32_t *d_in, int have_p0, int have_p1,
                                   cudaStream_t stream)
{
    pb::k_label_single<<<1, 32, 0, stream>>>(d_out, is_source, node_index, d_in, have_p0, have_p1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_compress_bench(uint32_t grid, uint32_t iters, uint32_t salt, uint32_t *d_sink,
                                     int fma_adds, cudaStream_t stream)
{
    if (fma_adds) pb::k_compress_bench<true><<<grid, 256, 0, stream>>>(iters, salt, d_sink, 1u);
    else pb::k_compress_bench<false><<<grid, 256, 0, stream>>>(iters, salt, d_sink, 1u);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_compress_latency(uint32_t iters, unsigned long long *d_cycles, uint32_t *d_sink,
                                       cudaStream_t stream)
{
    pb::k_compress_latency<<<1, 1, 0, stream>>>(iters, d_cycles, d_sink);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
