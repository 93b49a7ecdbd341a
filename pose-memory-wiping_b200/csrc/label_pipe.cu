/*
 * label_pipe.cu — the software-pipelined labeling kernel (sm_100a).
 *
 * Same work, same bytes as k_label (label_kernels.cu): teams of T warps run
 * G chunk copies of one topology in lockstep, level by level, pulling batches
 * from a device work counter.  What changes is where a label waits between
 * the level that writes it and the level that reads it, and when it is
 * fetched (records from topology.c's pipelined layout, PB_REF_* bits):
 *
 *   - a label read by the next level also goes to a shared-memory pool
 *     (slot * G + u), so the next level reads it without a round trip to L2;
 *   - a label read two or more levels later goes to the global pool; its
 *     readers fetch it ONE LEVEL EARLY with cp.async into a per-thread
 *     staging buffer in shared memory, together with the reader's block-0
 *     chaining value, while the current level is being hashed;
 *   - records are loaded two levels ahead into registers.
 *
 * So on the critical path of a level there is a barrier, a shared-memory
 * read, and the two dependent compressions of block 1 and block 2; the
 * memory latency of everything else overlaps the previous level's hashing.
 * The pipeline covers each thread's first item of a level; further items of
 * a wide level load what they need when they run (other warps cover that).
 *
 * cp.async waits are per thread (each thread reads only its own staging
 * slots), the level barrier orders the shared pool, and no thread ever waits
 * on another team: there are no spin-waits.
 */
#include "b3_device.cuh"
#include "kernels.h"

#include <cuda_runtime.h>
#include <stdint.h>

namespace pb {
namespace {

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc)
{
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ void team_sync(uint32_t T, uint32_t bar_id, uint32_t nthreads)
{
    if (T == 1) __syncwarp();
    else asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
}

/* staging slots of one thread: [stage][k] at stg[(stage*6 + k) * nthreads + tid]
 * (k: 0,1 = block-0 chaining value; 2,3 = predecessor 0; 4,5 = predecessor 1) */
struct Stage {
    uint4 *base;
    uint32_t nthr, tid;
    __device__ __forceinline__ uint4 *at(uint32_t stage, uint32_t k) const
    {
        return base + (size_t)(stage * 6 + k) * nthr + tid;
    }
};

__device__ __forceinline__ void put8(uint32_t *w, uint4 a, uint4 b)
{
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
}

struct Unit {
    uint32_t u, glog, copy, rank_base, rank_lim;
    uint32_t seed[8];
    uint8_t *out;
    const uint4 *cv0;   /* this copy's block-0 table */
    uint4 *gscr;        /* team's global pool (slot*G + u)*2 */
    uint4 *spool;       /* team's shared pool (slot*G + u)*2 */
};

/* Hash one node whose chaining value and predecessor words are in cv/m and
 * store the label wherever its record says. */
__device__ __forceinline__ void finish_node(const pb_pipe_params_t &p, const Unit &un, uint4 r0, uint4 r1,
                                            uint32_t (&cv)[8], const uint32_t (&m)[16])
{
    compress(cv, m, 64, kFlagsBlock1);
    uint32_t m2[16];
#pragma unroll
    for (int i = 0; i < 8; i++) { m2[i] = un.seed[i]; m2[8 + i] = p.topo.desc[i]; }
    compress(cv, m2, 64, kFlagsBlock2);
    const uint4 o0 = make_uint4(cv[0], cv[1], cv[2], cv[3]);
    const uint4 o1 = make_uint4(cv[4], cv[5], cv[6], cv[7]);
    if (r1.x != PB_NO_SLOT) {
        uint4 *d = un.spool + (((size_t)r1.x << un.glog) + un.u) * 2;
        d[0] = o0;
        d[1] = o1;
    }
    if (r0.w != PB_NO_SLOT) {
        uint4 *d = un.gscr + (((size_t)r0.w << un.glog) + un.u) * 2;
        d[0] = o0;
        d[1] = o1;
    }
    if ((r0.x & PB_REC_OUT_BIT) && r1.y < un.rank_lim) {
        uint4 *o = reinterpret_cast<uint4 *>(un.out + (size_t)(un.rank_base + r1.y) * 32);
        o[0] = o0;
        o[1] = o1;
    }
}

/* Read predecessor e of a record from wherever it lives (no staging). */
__device__ __forceinline__ void load_pred(const Unit &un, uint32_t ref, uint32_t *w)
{
    const uint32_t slot = ref & PB_REF_SLOT_MASK;
    const uint4 *s = ((ref & PB_REF_PREV) && (ref & PB_REF_SMEM)) ? un.spool : un.gscr;
    s += (((size_t)slot << un.glog) + un.u) * 2;
    put8(w, s[0], s[1]);
}

__device__ __forceinline__ void load_item_direct(const pb_pipe_params_t &p, const Unit &un, uint32_t pos)
{
    const uint4 *rp = p.topo.recs2 + 2 * (size_t)pos;
    const uint4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
    const uint32_t np = (r0.x >> PB_REC_NP_SHIFT) & 3u;
    uint32_t m[16], cv[8];
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = 0;
    if (np >= 1) load_pred(un, r0.y, m);
    if (np >= 2) load_pred(un, r0.z, m + 8);
    put8(cv, __ldg(un.cv0 + 2 * (size_t)pos), __ldg(un.cv0 + 2 * (size_t)pos + 1));
    finish_node(p, un, r0, r1, cv, m);
}

} /* namespace */

__global__ void __launch_bounds__(PB_CTA_THREADS) k_label_pipe(const __grid_constant__ pb_pipe_params_t p)
{
    extern __shared__ uint4 smem[];
    const uint32_t T = p.team_warps, TT = T * 32;
    const uint32_t team = (threadIdx.x >> 5) / T;
    const uint32_t tt = threadIdx.x - team * TT;
    const uint32_t teams_per_cta = blockDim.x / TT;
    const uint64_t gteam = (uint64_t)blockIdx.x * teams_per_cta + team;
    const uint32_t bar_id = 1 + team;
    const uint32_t glog = p.g_log2, G = 1u << glog;
    const uint32_t q = tt >> glog, stride = TT >> glog;
    const pb_topo_view2_t &tp = p.topo;
    const uint32_t L = tp.L;
    __shared__ uint32_t s_batch[PB_CTA_THREADS / 32];

    Unit un;
    un.u = tt & (G - 1);
    un.glog = glog;
    un.gscr = reinterpret_cast<uint4 *>(p.scratch + gteam * p.team_scratch_bytes);
    un.spool = smem + (size_t)team * tp.csm * G * 2;
    Stage stg;
    stg.base = smem + (size_t)teams_per_cta * tp.csm * G * 2;
    stg.nthr = blockDim.x;
    stg.tid = threadIdx.x;

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

        const uint32_t unit = (batch << glog) + un.u;
        const bool valid = unit < p.nunits;
        const uint32_t chunk = unit >> p.copies_log2;
        un.copy = unit & ((1u << p.copies_log2) - 1u);
        un.rank_base = un.copy ? tp.half_w : 0u;
        un.rank_lim = un.copy ? tp.retained : tp.half_w;
        un.out = p.persist + (uint64_t)(p.first_super + chunk) * p.super_bytes;
        un.cv0 = tp.cv0 + (uint64_t)un.copy * tp.S * 2;
#pragma unroll
        for (int i = 0; i < 8; i++) un.seed[i] = valid ? p.seeds[8 * (size_t)chunk + i] : 0u;

        /* level starts l, l+1, l+2, l+3 (clamped to S past the end) */
        uint32_t ls0 = __ldg(tp.lstart), ls1 = __ldg(tp.lstart + 1);
        uint32_t ls2 = L >= 2 ? __ldg(tp.lstart + 2) : ls1;
        uint32_t ls3 = L >= 3 ? __ldg(tp.lstart + 3) : ls2;
        /* records of this thread's first item at levels l (c), l+1 (n), l+2 (f) */
        uint4 c0 = make_uint4(0, 0, 0, 0), c1 = c0, n0 = c0, n1 = c0, f0 = c0, f1 = c0;
        bool c_ok = valid && q < ls1 - ls0, n_ok = valid && q < ls2 - ls1;
        if (c_ok) { c0 = __ldg(tp.recs2 + 2 * (size_t)(ls0 + q)); c1 = __ldg(tp.recs2 + 2 * (size_t)(ls0 + q) + 1); }
        if (n_ok) { n0 = __ldg(tp.recs2 + 2 * (size_t)(ls1 + q)); n1 = __ldg(tp.recs2 + 2 * (size_t)(ls1 + q) + 1); }
        /* stage 0: level 0's chaining value (level 0 has no predecessors) */
        if (c_ok) {
            cp_async16(stg.at(0, 0), un.cv0 + 2 * (size_t)(ls0 + q));
            cp_async16(stg.at(0, 1), un.cv0 + 2 * (size_t)(ls0 + q) + 1);
        }
        cp_async_commit();

        for (uint32_t l = 0; l < L; l++) {
            const uint32_t w = ls1 - ls0;
            const uint32_t st_next = (l + 1) & 1, st_cur = l & 1;
            /* (1) fetch the next level's first item: chaining value and the
             * predecessors born two or more levels back (complete since the
             * barrier that ended level l-1) */
            if (n_ok) {
                const uint32_t pos = ls1 + q;
                cp_async16(stg.at(st_next, 0), un.cv0 + 2 * (size_t)pos);
                cp_async16(stg.at(st_next, 1), un.cv0 + 2 * (size_t)pos + 1);
                const uint32_t np = (n0.x >> PB_REC_NP_SHIFT) & 3u;
                if (np >= 1 && !(n0.y & PB_REF_PREV)) {
                    const uint4 *s = un.gscr + (((size_t)(n0.y & PB_REF_SLOT_MASK) << glog) + un.u) * 2;
                    cp_async16(stg.at(st_next, 2), s);
                    cp_async16(stg.at(st_next, 3), s + 1);
                }
                if (np >= 2 && !(n0.z & PB_REF_PREV)) {
                    const uint4 *s = un.gscr + (((size_t)(n0.z & PB_REF_SLOT_MASK) << glog) + un.u) * 2;
                    cp_async16(stg.at(st_next, 4), s);
                    cp_async16(stg.at(st_next, 5), s + 1);
                }
            }
            cp_async_commit();
            /* (2) records two levels ahead */
            const uint32_t ls4 = (l + 4 <= L) ? __ldg(tp.lstart + l + 4) : ls3;
            const bool f_ok = valid && l + 2 < L && q < ls3 - ls2;
            if (f_ok) { f0 = __ldg(tp.recs2 + 2 * (size_t)(ls2 + q)); f1 = __ldg(tp.recs2 + 2 * (size_t)(ls2 + q) + 1); }
            /* (3) this level's staged data is complete once only the newest
             * group may still be in flight */
            cp_async_wait_1();
            /* (4) the first item */
            if (c_ok) {
                const uint32_t np = (c0.x >> PB_REC_NP_SHIFT) & 3u;
                uint32_t m[16], cv[8];
                put8(cv, *stg.at(st_cur, 0), *stg.at(st_cur, 1));
#pragma unroll
                for (int i = 0; i < 16; i++) m[i] = 0;
                if (np >= 1) {
                    if (c0.y & PB_REF_PREV) load_pred(un, c0.y, m);
                    else put8(m, *stg.at(st_cur, 2), *stg.at(st_cur, 3));
                }
                if (np >= 2) {
                    if (c0.z & PB_REF_PREV) load_pred(un, c0.z, m + 8);
                    else put8(m + 8, *stg.at(st_cur, 4), *stg.at(st_cur, 5));
                }
                finish_node(p, un, c0, c1, cv, m);
            }
            /* (5) further items of a wide level */
            if (valid)
                for (uint32_t j = q + stride; j < w; j += stride) load_item_direct(p, un, ls0 + j);
            team_sync(T, bar_id, TT);
            /* (6) advance the pipeline */
            c0 = n0; c1 = n1; c_ok = n_ok;
            n0 = f0; n1 = f1; n_ok = f_ok;
            ls0 = ls1; ls1 = ls2; ls2 = ls3; ls3 = ls4;
        }
        /* drain the (empty) trailing group before the staging is reused */
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        team_sync(T, bar_id, TT);
    }
}

} /* namespace pb */

extern "C" int pb_dev_label_pipe(const pb_pipe_params_t *params, uint32_t grid, uint32_t cta_threads,
                                 uint32_t smem_bytes, cudaStream_t stream)
{
    if (cudaFuncSetAttribute(pb::k_label_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes) != cudaSuccess)
        return -1;
    cudaGetLastError(); /* report only this launch */
    pb::k_label_pipe<<<grid, cta_threads, smem_bytes, stream>>>(*params);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_label_pipe_occupancy(uint32_t cta_threads, uint32_t smem_bytes, int *blocks_per_sm)
{
    if (cudaFuncSetAttribute(pb::k_label_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes) != cudaSuccess)
        return -1;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pb::k_label_pipe, (int)cta_threads,
                                                         smem_bytes) == cudaSuccess
               ? 0
               : -1;
}
