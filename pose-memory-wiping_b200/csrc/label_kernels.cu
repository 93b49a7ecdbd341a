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

/* Team barrier.  CTA_TEAM: the team is the whole CTA, so barrier 0 serves
 * (a kernel that names only barrier 0 reserves one barrier per CTA, not all
 * sixteen, and its CTAs are not held back by the SM's barrier count);
 * otherwise the named barrier bar_id over the team's nthreads threads. */
template <bool CTA_TEAM>
__device__ __forceinline__ void team_sync(uint32_t team_warps, uint32_t bar_id, uint32_t nthreads)
{
    if (team_warps == 1) {
        __syncwarp();
    } else if (CTA_TEAM) {
        __syncthreads();
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

/* What one thread needs to run its unit through the levels. */
struct UnitCtx {
    uint4 *tscr;       /* team scratch, label (slot, u) at (slot*G + u)*2 */
    uint32_t glog, u, q, stride;
    bool valid;
    uint32_t id_off, rank_base, rank_lim;
    uint8_t *out;      /* persisted super-chunk of this unit's chunk */
    const uint4 *cv0;  /* this copy's block-0 table, or null */
    uint32_t seed[8];
};

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc)
{
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

/* Copy the record and block-0 chaining value of node `pos` into this
 * thread's staging buffer b (dynamic shared memory, PB_PREF_BYTES_PER_THREAD
 * a thread: [buffer][record, cv lo, cv hi][thread]). */
__device__ __forceinline__ void stage_node(const pb_topo_view_t &tp, const UnitCtx &c, uint32_t pos, uint32_t b)
{
    extern __shared__ uint4 s_stage[];
    const uint32_t nt = blockDim.x;
    uint4 *slot = s_stage + (size_t)b * 3 * nt + threadIdx.x;
    cp_async16(slot, tp.recs + pos);
    if (c.cv0) {
        cp_async16(slot + nt, c.cv0 + 2 * (size_t)pos);
        cp_async16(slot + 2 * nt, c.cv0 + 2 * (size_t)pos + 1);
    }
}

__device__ __forceinline__ uint4 staged(uint32_t b, uint32_t k)
{
    extern __shared__ uint4 s_stage[];
    return s_stage[((size_t)b * 3 + k) * blockDim.x + threadIdx.x];
}

/* All levels of one batch: thread (q, u) hashes nodes q, q+stride, ... of
 * every level for unit u; the team syncs between levels.
 *
 * The seed-independent inputs of a thread's first node of a level (its
 * record and block-0 chaining value) are copied into shared memory one level
 * ahead (cp.async, double-buffered per thread), and the level bounds are read
 * two levels ahead, so that a level's dependent chain is only the
 * predecessor loads, the two compressions and the barrier.  Each thread
 * reads back only its own staging slots, after waiting for its own copies. */
template <bool FMA, bool CTA_TEAM>
__device__ __forceinline__ void label_levels(const pb_topo_view_t &tp, const UnitCtx &c, uint32_t T,
                                             uint32_t bar_id, uint32_t TT, uint32_t one)
{
    const uint32_t L = tp.L;
    uint32_t s0 = __ldg(tp.lstart);
    uint32_t s1 = __ldg(tp.lstart + 1);
    uint32_t s2 = L >= 2 ? __ldg(tp.lstart + 2) : s1;
    if (c.valid && c.q < s1 - s0) stage_node(tp, c, s0 + c.q, 0);
    cp_async_commit();
    for (uint32_t l = 0; l < L; l++) {
        const uint32_t w = s1 - s0;
        const uint32_t cur = l & 1u;
        const uint32_t s3 = l + 3 <= L ? __ldg(tp.lstart + l + 3) : s2;
        cp_async_wait_all(); /* this level's staged node has landed */
        if (c.valid && l + 1 < L && c.q < s2 - s1) stage_node(tp, c, s1 + c.q, cur ^ 1u);
        cp_async_commit();
        if (c.valid) {
            for (uint32_t j = c.q; j < w; j += c.stride) {
                const uint32_t pos = s0 + j;
                const bool first = j == c.q;
                const uint4 rec = first ? staged(cur, 0) : __ldg(tp.recs + pos);
                const uint32_t np = (rec.x >> PB_REC_NP_SHIFT) & 3u;
                uint32_t m[16];
                if (np >= 1) {
                    const uint4 *s = c.tscr + (((size_t)rec.y << c.glog) + c.u) * 2;
                    uint4 a = s[0], b = s[1];
                    m[0] = a.x; m[1] = a.y; m[2] = a.z; m[3] = a.w;
                    m[4] = b.x; m[5] = b.y; m[6] = b.z; m[7] = b.w;
                } else {
#pragma unroll
                    for (int i = 0; i < 8; i++) m[i] = 0;
                }
                if (np >= 2) {
                    const uint4 *s = c.tscr + (((size_t)rec.z << c.glog) + c.u) * 2;
                    uint4 a = s[0], b = s[1];
                    m[8] = a.x; m[9] = a.y; m[10] = a.z; m[11] = a.w;
                    m[12] = b.x; m[13] = b.y; m[14] = b.z; m[15] = b.w;
                } else {
#pragma unroll
                    for (int i = 8; i < 16; i++) m[i] = 0;
                }
                uint32_t cv[8];
                if (c.cv0) {
                    const uint4 c0 = first ? staged(cur, 1) : __ldg(c.cv0 + 2 * (size_t)pos);
                    const uint4 c1 = first ? staged(cur, 2) : __ldg(c.cv0 + 2 * (size_t)pos + 1);
                    cv[0] = c0.x; cv[1] = c0.y; cv[2] = c0.z; cv[3] = c0.w;
                    cv[4] = c1.x; cv[5] = c1.y; cv[6] = c1.z; cv[7] = c1.w;
                } else {
                    uint32_t m0[16];
                    key_words(cv, np == 0);
                    block0_words(m0, (rec.x & PB_REC_ID_MASK) + c.id_off);
                    if (FMA) compress_fma(cv, m0, 64, kFlagsBlock0, one);
                    else compress(cv, m0, 64, kFlagsBlock0);
                }
                uint32_t m2[16];
#pragma unroll
                for (int i = 0; i < 8; i++) { m2[i] = c.seed[i]; m2[8 + i] = tp.desc[i]; }
                if (FMA) {
                    compress_fma(cv, m, 64, kFlagsBlock1, one);
                    compress_fma(cv, m2, 64, kFlagsBlock2, one);
                } else {
                    compress(cv, m, 64, kFlagsBlock1);
                    compress(cv, m2, 64, kFlagsBlock2);
                }
                const uint4 o0 = make_uint4(cv[0], cv[1], cv[2], cv[3]);
                const uint4 o1 = make_uint4(cv[4], cv[5], cv[6], cv[7]);
                uint4 *d = c.tscr + (((size_t)rec.w << c.glog) + c.u) * 2;
                d[0] = o0;
                d[1] = o1;
                if (rec.x & PB_REC_OUT_BIT) {
                    const uint32_t r = __ldg(tp.orank + pos);
                    if (r < c.rank_lim) {
                        uint4 *o = reinterpret_cast<uint4 *>(c.out + (size_t)(c.rank_base + r) * 32);
                        o[0] = o0;
                        o[1] = o1;
                    }
                }
            }
        }
        team_sync<CTA_TEAM>(T, bar_id, TT);
        s0 = s1;
        s1 = s2;
        s2 = s3;
    }
}

/* Team-wide batch index from the work counter. */
template <bool CTA_TEAM>
__device__ __forceinline__ uint32_t grab_batch(unsigned int *queue, uint32_t T, uint32_t team, uint32_t tt,
                                               uint32_t bar_id, uint32_t TT, uint32_t *s_batch)
{
    if (T == 1) {
        uint32_t b = 0;
        if ((threadIdx.x & 31) == 0) b = atomicAdd(queue, 1u);
        return __shfl_sync(0xFFFFFFFFu, b, 0);
    }
    if (tt == 0) s_batch[team] = atomicAdd(queue, 1u);
    team_sync<CTA_TEAM>(T, bar_id, TT);
    const uint32_t b = s_batch[team];
    team_sync<CTA_TEAM>(T, bar_id, TT);
    return b;
}

/* The lockstep kernel for one topology: one team of T warps per CTA
 * (blockDim.x == 32 T), so any number of teams can be resident per SM. */
template <bool FMA>
__global__ void __launch_bounds__(PB_CTA_THREADS) k_label(const __grid_constant__ pb_label_params_t p)
{
    const uint32_t T = p.team_warps;
    const uint32_t TT = T * 32;
    const uint32_t team = 0;
    const uint32_t tt = threadIdx.x;
    const uint64_t gteam = blockIdx.x;
    const uint32_t bar_id = 0;
    const pb_topo_view_t &tp = p.topo;
    __shared__ uint32_t s_batch[1];
    UnitCtx c;
    c.glog = p.g_log2;
    c.u = tt & ((1u << c.glog) - 1);
    c.q = tt >> c.glog;
    c.stride = TT >> c.glog;
    c.tscr = reinterpret_cast<uint4 *>(p.scratch + gteam * p.team_scratch_bytes);

    for (;;) {
        const uint32_t batch = grab_batch<true>(p.queue, T, team, tt, bar_id, TT, s_batch);
        if (batch >= p.nbatches) break;
        const uint32_t unit = (batch << c.glog) + c.u;
        c.valid = unit < p.nunits;
        const uint32_t chunk = unit >> p.copies_log2;
        const uint32_t copy = unit & ((1u << p.copies_log2) - 1u);
        c.id_off = copy ? tp.S : 0u;
        c.rank_base = copy ? tp.half_w : 0u;
        c.rank_lim = copy ? tp.retained : tp.half_w;
        c.out = p.persist + (uint64_t)(p.first_super + chunk) * p.super_bytes;
        c.cv0 = tp.cv0 ? tp.cv0 + (uint64_t)copy * tp.S * 2 : nullptr;
#pragma unroll
        for (int i = 0; i < 8; i++) c.seed[i] = c.valid ? p.seeds[8 * (size_t)chunk + i] : 0u;
        label_levels<FMA, true>(tp, c, T, bar_id, TT, p.one);
    }
}

/* Many topologies in one launch: teams take batches (same topology, up to
 * G = 2^glog units) from a queue sorted longest first, and copy the batch's
 * topology view into shared memory.  One team of T warps per CTA
 * (blockDim.x == 32 T), ending its levels with the CTA barrier. */
template <bool FMA>
__global__ void __launch_bounds__(PB_MULTI_CTA_THREADS, 3) k_label_multi(const __grid_constant__ pb_multi_params_t p)
{
    const uint32_t T = p.team_warps;
    const uint32_t TT = T * 32;
    const uint32_t team = 0;
    const uint32_t tt = threadIdx.x;
    const uint64_t gteam = blockIdx.x;
    const uint32_t bar_id = 0;
    __shared__ uint32_t s_batch[1];
    __shared__ pb_topo_view_t s_topo[1];
    UnitCtx c;
    c.tscr = reinterpret_cast<uint4 *>(p.scratch + gteam * p.team_scratch_bytes);

    for (;;) {
        const uint32_t batch = grab_batch<true>(p.queue, T, team, tt, bar_id, TT, s_batch);
        if (batch >= p.nbatches) break;
        const pb_mbatch_t bd = p.batches[batch];
        if (tt < sizeof(pb_topo_view_t) / 4)
            reinterpret_cast<uint32_t *>(&s_topo[team])[tt] =
                reinterpret_cast<const uint32_t *>(p.topos + bd.topo)[tt];
        team_sync<true>(T, bar_id, TT);
        const pb_topo_view_t &tp = s_topo[team];
        c.glog = bd.glog;
        c.u = tt & ((1u << c.glog) - 1);
        c.q = tt >> c.glog;
        c.stride = TT >> c.glog;
        c.valid = c.u < bd.count;
        const pb_munit_t un = p.units[bd.first_unit + (c.valid ? c.u : 0)];
        const uint32_t copy = un.copy;
        c.id_off = copy ? tp.S : 0u;
        c.rank_base = copy ? tp.half_w : 0u;
        c.rank_lim = copy ? tp.retained : tp.half_w;
        c.out = reinterpret_cast<uint8_t *>(un.out);
        c.cv0 = tp.cv0 ? tp.cv0 + (uint64_t)copy * tp.S * 2 : nullptr;
#pragma unroll
        for (int i = 0; i < 8; i++) c.seed[i] = c.valid ? p.seeds[8 * (size_t)un.seed + i] : 0u;
        label_levels<FMA, true>(tp, c, T, bar_id, TT, p.one);
        /* label_levels ended with a team barrier, so every persisted label of
         * the batch is ordered before this fence */
        if (p.req_done != nullptr && tt < bd.count) {
            __threadfence_system();
            atomicAdd_system(p.req_done + p.unit_req[bd.first_unit + tt], 1u);
        }
        team_sync<true>(T, bar_id, TT); /* s_topo[team] is rewritten by the next batch */
    }
}

/* Chunk seeds of arbitrary (session, chunk index) jobs: job j derives
 * seeds[8j..] = derive_key("pose-db/chunk-seed", blob[off..off+len) |
 * be64(index)) (common/src/hash.c:218-233). */
__global__ void __launch_bounds__(128) k_seed_jobs(const pb_seedjob_t *__restrict__ jobs, uint32_t njobs,
                                                    const uint8_t *__restrict__ blob, uint32_t *__restrict__ seeds)
{
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    const pb_seedjob_t jb = jobs[j];
    const uint8_t *session_seed = blob + jb.seed_off;
    const uint32_t seed_len = jb.seed_len;
    const uint64_t idx = jb.chunk_index;
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
    cudaGetLastError(); /* report only this launch */
    pb::k_cv0_table<<<(unsigned)blocks, 256, 0, stream>>>((const uint4 *)recs, S, copies,
                                                          (uint4 *)cv0);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_chunk_seeds(const uint8_t *d_session_seed, uint32_t seed_len, uint64_t rbo,
                                  uint32_t cb, uint32_t nchunks, uint64_t first_super,
                                  uint32_t *d_seeds, cudaStream_t stream)
{
    if (nchunks == 0) return 0;
    cudaGetLastError(); /* report only this launch */
    pb::k_chunk_seeds<<<(nchunks + 127) / 128, 128, 0, stream>>>(d_session_seed, seed_len, rbo, cb,
                                                                  nchunks, first_super, d_seeds);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* k_label's 512-thread CTAs stage 48 KiB, which with the static shared
 * memory is above the default per-CTA limit: opt in (idempotent). */
static void allow_stage_smem()
{
    const int bytes = (int)(PB_PREF_BYTES_PER_THREAD * PB_CTA_THREADS);
    cudaFuncSetAttribute(pb::k_label<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(pb::k_label<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

extern "C" int pb_dev_label(const pb_label_params_t *params, uint32_t grid, uint32_t cta_threads,
                            uint32_t smem_bytes, cudaStream_t stream)
{
    if (cta_threads != 32u * params->team_warps || cta_threads > PB_CTA_THREADS) return -1; /* one team per CTA */
    cudaGetLastError(); /* report only this launch */
    uint32_t smem = PB_PREF_BYTES_PER_THREAD * cta_threads;
    if (smem_bytes > smem) {
        if (cudaFuncSetAttribute(pb::k_label<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes) !=
                cudaSuccess ||
            cudaFuncSetAttribute(pb::k_label<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes) !=
                cudaSuccess)
            return -1;
        smem = smem_bytes;
    } else if (smem > 48 * 1024 - 1024) {
        allow_stage_smem();
    }
    cudaGetLastError();
    if (params->fma_adds) pb::k_label<true><<<grid, cta_threads, smem, stream>>>(*params);
    else pb::k_label<false><<<grid, cta_threads, smem, stream>>>(*params);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_label_multi(const pb_multi_params_t *params, uint32_t grid, uint32_t cta_threads,
                                  cudaStream_t stream)
{
    if (cta_threads != 32u * params->team_warps || cta_threads > PB_MULTI_CTA_THREADS) return -1; /* one team per CTA */
    cudaGetLastError(); /* report only this launch */
    const uint32_t smem = PB_PREF_BYTES_PER_THREAD * cta_threads;
    if (params->fma_adds) pb::k_label_multi<true><<<grid, cta_threads, smem, stream>>>(*params);
    else pb::k_label_multi<false><<<grid, cta_threads, smem, stream>>>(*params);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_label_multi_occupancy(uint32_t cta_threads, int *blocks_per_sm)
{
    int a = 0, b = 0;
    const size_t smem = PB_PREF_BYTES_PER_THREAD * cta_threads;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, pb::k_label_multi<false>, (int)cta_threads, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, pb::k_label_multi<true>, (int)cta_threads, smem) != cudaSuccess)
        return -1;
    *blocks_per_sm = a < b ? a : b;
    return 0;
}

extern "C" int pb_dev_seed_jobs(const void *jobs, uint32_t njobs, const uint8_t *blob, uint32_t *seeds,
                                cudaStream_t stream)
{
    if (njobs == 0) return 0;
    cudaGetLastError(); /* report only this launch */
    pb::k_seed_jobs<<<(njobs + 127) / 128, 128, 0, stream>>>((const pb_seedjob_t *)jobs, njobs, blob, seeds);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* Dynamic shared memory per CTA of k_label with cta_threads threads that
 * lets at most `per_sm` such CTAs reside on one SM (the staging area is the
 * least it gets): *smem_bytes = 0 when the staging area alone already holds
 * residency to per_sm or below.  A launch of per_sm x SMs CTAs then puts
 * exactly per_sm teams on every SM, so the waves of a persistent launch end
 * together on every SM. */
extern "C" int pb_dev_label_balance_smem(uint32_t cta_threads, uint32_t per_sm, uint32_t *smem_bytes)
{
    int dev = 0, cap = 0, resv = 0, optin = 0, occ = 0;
    *smem_bytes = 0;
    if (per_sm == 0 || cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return -1;
    const uint32_t base = PB_PREF_BYTES_PER_THREAD * cta_threads;
    if (pb_dev_label_occupancy(cta_threads, &occ) != 0) return -1;
    if ((uint32_t)occ <= per_sm) return 0;
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, pb::k_label<true>) != cudaSuccess) return -1;
    /* largest multiple of 1 KiB with per_sm CTAs fitting the SM's shared memory */
    int64_t each = (int64_t)cap / per_sm - resv - (int64_t)fa.sharedSizeBytes;
    each -= each % 1024;
    if (each > optin - (int64_t)fa.sharedSizeBytes) each = optin - (int64_t)fa.sharedSizeBytes;
    if (each < (int64_t)base) return 0;
    for (; each >= (int64_t)base; each -= 1024) {
        int a = 0, b = 0;
        if (cudaFuncSetAttribute(pb::k_label<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)each) !=
                cudaSuccess ||
            cudaFuncSetAttribute(pb::k_label<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)each) !=
                cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, pb::k_label<false>, (int)cta_threads, each) !=
                cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, pb::k_label<true>, (int)cta_threads, each) !=
                cudaSuccess)
            return -1;
        const int m = a > b ? a : b;
        if ((uint32_t)m == per_sm) {
            *smem_bytes = (uint32_t)each;
            return 0;
        }
        if ((uint32_t)m > per_sm) break;
    }
    return 0;
}

extern "C" int pb_dev_label_occupancy(uint32_t cta_threads, int *blocks_per_sm)
{
    int a = 0, b = 0;
    const size_t smem = PB_PREF_BYTES_PER_THREAD * cta_threads;
    allow_stage_smem();
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, pb::k_label<false>, (int)cta_threads, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, pb::k_label<true>, (int)cta_threads, smem) != cudaSuccess)
        return -1;
    *blocks_per_sm = a < b ? a : b;
    return 0;
}

extern "C" int pb_dev_label_single(uint32_t *d_out, int is_source, uint64_t node_index,
                                   const uint32_t *d_in, int have_p0, int have_p1,
                                   cudaStream_t stream)
{
    cudaGetLastError(); /* report only this launch */
    pb::k_label_single<<<1, 32, 0, stream>>>(d_out, is_source, node_index, d_in, have_p0, have_p1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_compress_bench(uint32_t grid, uint32_t iters, uint32_t salt, uint32_t *d_sink,
                                     int fma_adds, cudaStream_t stream)
{
    cudaGetLastError(); /* report only this launch */
    if (fma_adds) pb::k_compress_bench<true><<<grid, 256, 0, stream>>>(iters, salt, d_sink, 1u);
    else pb::k_compress_bench<false><<<grid, 256, 0, stream>>>(iters, salt, d_sink, 1u);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_compress_latency(uint32_t iters, unsigned long long *d_cycles, uint32_t *d_sink,
                                       cudaStream_t stream)
{
    cudaGetLastError(); /* report only this launch */
    pb::k_compress_latency<<<1, 1, 0, stream>>>(iters, d_cycles, d_sink);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
