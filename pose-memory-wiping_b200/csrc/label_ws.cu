/*
 * label_ws.cu — warp-specialised labeling kernel for the depth-bound regime
 * (few chunks in flight; sm_100a).
 *
 * When a launch has about one chunk copy per SM, its time is the number of
 * dependency levels times the time of one level, and a level's floor is two
 * dependent compressions (block 1 needs the predecessors, block 2 needs
 * block 1).  Everything else a level does — finding its width, loading node
 * records, block-0 chaining values and predecessors born earlier, computing
 * addresses — is taken off that path by a producer warp that works one and
 * two levels ahead, using the pipelined records of topology.c (PB_REF_*):
 *
 *   CTA = NC hashing warps + 1 producer warp, one chunk copy per CTA.
 *   During level l the producer
 *     - copies the records of level l+2 into a three-stage ring (cp.async),
 *       and writes that level's start and width into the ring header;
 *     - from the records of level l+1 (copied during level l-1), copies the
 *       block-0 chaining value and every predecessor born at level l-1 or
 *       earlier (complete since the barrier that ended level l-1) into a
 *       two-stage data area (cp.async), then waits for its copies.
 *   During level l the hashing threads read their record and data from shared
 *   memory, read predecessors born at level l-1 from the shared-memory label
 *   pool (or global memory when that level overflowed the pool), hash, and
 *   store.  One barrier of the whole CTA ends the level.
 *
 * Items beyond the first NC*32 of a wide level are hashed with direct loads.
 * No thread waits on anything but its own cp.async groups and the CTA
 * barrier: there are no spin-waits.
 *
 * k_label_wsg is the same design for up to four chunk copies of one topology
 * per CTA (the deep part of a batch): records are staged once for all units,
 * and each unit has its own shared-memory pool, built for 512 slots.
 */
#include "b3_device.cuh"
#include "kernels.h"

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cg = cooperative_groups;

namespace pb {
namespace {

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc)
{
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ void put8(uint32_t *w, uint4 a, uint4 b)
{
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
}

/* Shared-memory layout (uint4 units):
 *   pool  [csm][2]                    next-level labels
 *   rec   [3][slots][2]               records, ring of three levels
 *   dat   [2][slots][6]               cv0 (2), predecessor 0 (2), predecessor 1 (2)
 *   hdr   [3]                         (level start, width) of each ring stage */
struct Smem {
    uint4 *pool, *rec, *dat, *hdr;
    uint32_t slots;
    __device__ __forceinline__ uint4 *r(uint32_t st, uint32_t j) const { return rec + ((size_t)st * slots + j) * 2; }
    __device__ __forceinline__ uint4 *d(uint32_t st, uint32_t j) const { return dat + ((size_t)st * slots + j) * 6; }
};

struct Unit {
    uint32_t copy, rank_base, rank_lim;
    uint32_t seed[8];
    uint8_t *out;
    const uint4 *cv0;
    uint4 *gscr; /* this unit's global pool, slot * 2 */
};

__device__ __forceinline__ void store_label(const Unit &un, const Smem &sm, uint4 r0, uint4 r1,
                                            const uint32_t (&cv)[8])
{
    const uint4 o0 = make_uint4(cv[0], cv[1], cv[2], cv[3]);
    const uint4 o1 = make_uint4(cv[4], cv[5], cv[6], cv[7]);
    if (r1.x != PB_NO_SLOT) {
        uint4 *d = sm.pool + (size_t)r1.x * 2;
        d[0] = o0;
        d[1] = o1;
    }
    if (r0.w != PB_NO_SLOT) {
        uint4 *d = un.gscr + (size_t)r0.w * 2;
        d[0] = o0;
        d[1] = o1;
    }
    if ((r0.x & PB_REC_OUT_BIT) && r1.y < un.rank_lim) {
        uint4 *o = reinterpret_cast<uint4 *>(un.out + (size_t)(un.rank_base + r1.y) * 32);
        o[0] = o0;
        o[1] = o1;
    }
}

template <class P>
__device__ __forceinline__ void hash_node(const P &p, const Unit &un, uint32_t (&cv)[8], const uint32_t (&m)[16])
{
    compress(cv, m, 64, kFlagsBlock1);
    uint32_t m2[16];
#pragma unroll
    for (int i = 0; i < 8; i++) { m2[i] = un.seed[i]; m2[8 + i] = p.topo.desc[i]; }
    compress(cv, m2, 64, kFlagsBlock2);
}

/* A predecessor born at the previous level: shared pool, or global pool when
 * its level overflowed the shared pool. */
__device__ __forceinline__ void load_prev(const Unit &un, const Smem &sm, uint32_t ref, uint32_t *w)
{
    const uint4 *s = (ref & PB_REF_SMEM) ? sm.pool : un.gscr;
    s += (size_t)(ref & PB_REF_SLOT_MASK) * 2;
    put8(w, s[0], s[1]);
}

/* An item with everything loaded on the spot (wide levels). */
template <class P>
__device__ __forceinline__ void direct_item(const P &p, const Unit &un, const Smem &sm, uint32_t pos)
{
    const uint4 *rp = p.topo.recs2 + 2 * (size_t)pos;
    const uint4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
    const uint32_t np = (r0.x >> PB_REC_NP_SHIFT) & 3u;
    uint32_t m[16], cv[8];
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = 0;
    if (np >= 1) {
        if (r0.y & PB_REF_PREV) load_prev(un, sm, r0.y, m);
        else { const uint4 *s = un.gscr + (size_t)(r0.y & PB_REF_SLOT_MASK) * 2; put8(m, s[0], s[1]); }
    }
    if (np >= 2) {
        if (r0.z & PB_REF_PREV) load_prev(un, sm, r0.z, m + 8);
        else { const uint4 *s = un.gscr + (size_t)(r0.z & PB_REF_SLOT_MASK) * 2; put8(m + 8, s[0], s[1]); }
    }
    put8(cv, __ldg(un.cv0 + 2 * (size_t)pos), __ldg(un.cv0 + 2 * (size_t)pos + 1));
    hash_node(p, un, cv, m);
    store_label(un, sm, r0, r1, cv);
}

/* Producer: records of `lv` (when < L) into ring stage lv % 3, and its header. */
template <class P, class S>
__device__ __forceinline__ void stage_records(const P &p, const S &sm, uint32_t lv, uint32_t lane)
{
    const pb_topo_view2_t &tp = p.topo;
    if (lv >= tp.L) return;
    const uint32_t st = lv % 3;
    const uint32_t ls = __ldg(tp.lstart + lv), w = __ldg(tp.lstart + lv + 1) - ls;
    const uint32_t n = w < sm.slots ? w : sm.slots;
    for (uint32_t j = lane; j < n; j += 32) {
        const uint4 *src = tp.recs2 + 2 * (size_t)(ls + j);
        cp_async16(sm.r(st, j), src);
        cp_async16(sm.r(st, j) + 1, src + 1);
    }
    if (lane == 0) sm.hdr[st] = make_uint4(ls, w, 0, 0);
}

/* Producer: block-0 values and older predecessors of level `lv` into data
 * stage lv & 1, from its records (ring stage lv % 3, already complete). */
__device__ __forceinline__ void stage_data(const pb_pipe_params_t &p, const Smem &sm, const Unit &un, uint32_t lv,
                                           uint32_t ls, uint32_t w, uint32_t lane)
{
    if (lv >= p.topo.L) return;
    const uint32_t n = w < sm.slots ? w : sm.slots;
    const uint32_t rs = lv % 3, ds = lv & 1;
    for (uint32_t j = lane; j < n; j += 32) {
        const uint4 r0 = *sm.r(rs, j);
        uint4 *d = sm.d(ds, j);
        const uint4 *c = un.cv0 + 2 * (size_t)(ls + j);
        cp_async16(d, c);
        cp_async16(d + 1, c + 1);
        const uint32_t np = (r0.x >> PB_REC_NP_SHIFT) & 3u;
        if (np >= 1 && !(r0.y & PB_REF_PREV)) {
            const uint4 *s = un.gscr + (size_t)(r0.y & PB_REF_SLOT_MASK) * 2;
            cp_async16(d + 2, s);
            cp_async16(d + 3, s + 1);
        }
        if (np >= 2 && !(r0.z & PB_REF_PREV)) {
            const uint4 *s = un.gscr + (size_t)(r0.z & PB_REF_SLOT_MASK) * 2;
            cp_async16(d + 4, s);
            cp_async16(d + 5, s + 1);
        }
    }
}

} /* namespace */

__global__ void __launch_bounds__(PB_CTA_THREADS, 1) k_label_ws(const __grid_constant__ pb_pipe_params_t p)
{
    extern __shared__ uint4 smem[];
    __shared__ uint32_t s_batch;
    const pb_topo_view2_t &tp = p.topo;
    const uint32_t NC = p.team_warps;           /* hashing warps */
    const uint32_t nthr = NC * 32;              /* hashing threads */
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = warp == NC;
    const uint32_t c = threadIdx.x;             /* hashing thread index when !producer */
    Smem sm;
    sm.slots = nthr;
    sm.pool = smem;
    sm.rec = sm.pool + (size_t)tp.csm * 2;
    sm.dat = sm.rec + (size_t)3 * nthr * 2;
    sm.hdr = sm.dat + (size_t)2 * nthr * 6;
    Unit un;
    un.gscr = reinterpret_cast<uint4 *>(p.scratch + (uint64_t)blockIdx.x * p.team_scratch_bytes);

    for (;;) {
        if (threadIdx.x == 0) s_batch = atomicAdd(p.queue, 1u);
        __syncthreads();
        const uint32_t unit = s_batch;
        __syncthreads();
        if (unit >= p.nunits) break;
        const uint32_t chunk = unit >> p.copies_log2;
        un.copy = unit & ((1u << p.copies_log2) - 1u);
        un.rank_base = un.copy ? tp.half_w : 0u;
        un.rank_lim = un.copy ? tp.retained : tp.half_w;
        un.out = p.persist + (uint64_t)(p.first_super + chunk) * p.super_bytes;
        un.cv0 = tp.cv0 + (uint64_t)un.copy * tp.S * 2;
#pragma unroll
        for (int i = 0; i < 8; i++) un.seed[i] = p.seeds[8 * (size_t)chunk + i];

        /* prologue: records of levels 0 and 1, then level 0's data */
        if (producer) {
            stage_records(p, sm, 0, lane);
            stage_records(p, sm, 1, lane);
            cp_async_commit();
            cp_async_wait_all();
            __syncwarp();
            const uint32_t ls0 = __ldg(tp.lstart), w0 = __ldg(tp.lstart + 1) - ls0;
            stage_data(p, sm, un, 0, ls0, w0, lane);
            cp_async_commit();
            cp_async_wait_all();
        }
        __syncthreads();

        for (uint32_t l = 0; l < tp.L; l++) {
            if (producer) {
                /* level l+2's records; level l+1's block-0 values and older
                 * predecessors (their records arrived during level l-1) */
                stage_records(p, sm, l + 2, lane);
                if (l + 1 < tp.L) {
                    const uint4 h = sm.hdr[(l + 1) % 3];
                    stage_data(p, sm, un, l + 1, h.x, h.y, lane);
                }
                cp_async_commit();
                cp_async_wait_all();
            } else {
                const uint4 h = sm.hdr[l % 3];
                const uint32_t ls = h.x, w = h.y;
                if (c < w && c < nthr) {
                    const uint4 r0 = *sm.r(l % 3, c), r1 = *(sm.r(l % 3, c) + 1);
                    const uint4 *d = sm.d(l & 1, c);
                    const uint32_t np = (r0.x >> PB_REC_NP_SHIFT) & 3u;
                    uint32_t m[16], cv[8];
#pragma unroll
                    for (int i = 0; i < 16; i++) m[i] = 0;
                    if (np >= 1) {
                        if (r0.y & PB_REF_PREV) load_prev(un, sm, r0.y, m);
                        else put8(m, d[2], d[3]);
                    }
                    if (np >= 2) {
                        if (r0.z & PB_REF_PREV) load_prev(un, sm, r0.z, m + 8);
                        else put8(m + 8, d[4], d[5]);
                    }
                    put8(cv, d[0], d[1]);
                    hash_node(p, un, cv, m);
                    store_label(un, sm, r0, r1, cv);
                }
                for (uint32_t j = c + nthr; j < w; j += nthr) direct_item(p, un, sm, ls + j);
            }
            __syncthreads();
        }
    }
}

/* k_label_ws with a thread-block cluster of C CTAs per chunk copy, for
 * launches with fewer copies than SMs.  CTA rank 0 runs the copy exactly as
 * k_label_ws does (producer warp, shared-memory pool, a CTA barrier per
 * level).  A level wider than split_width is shared: rank 0 hashes its
 * staged nodes and as many of the rest as bring it to ceil(w / C) nodes; the
 * other ranks hash the remainder, striding over it, with direct loads, and
 * read and write rank 0's shared-memory pool through distributed shared
 * memory.  Every boundary between levels l - 1 and l where l - 1 or l is
 * split is a cluster barrier instead of rank 0's CTA barrier; the other
 * ranks walk only the split levels (split_levels, nsplit of them, ascending)
 * and meet rank 0 at exactly those barriers, so every CTA of the cluster
 * passes the same barrier sequence.  One copy per cluster: the grid is
 * nunits * C CTAs, and copy k's global pool is at scratch + k *
 * team_scratch_bytes.  No spin-waits: only CTA and cluster barriers. */
__global__ void __launch_bounds__(PB_CTA_THREADS, 1) k_label_wsc(const __grid_constant__ pb_pipe_params_t p)
{
    extern __shared__ uint4 smem[];
    cg::cluster_group cl = cg::this_cluster();
    const pb_topo_view2_t &tp = p.topo;
    const uint32_t C = p.cluster;
    const uint32_t rank = cl.block_rank();
    const uint32_t unit = blockIdx.x / C;
    const uint32_t NC = p.team_warps;
    const uint32_t nthr = NC * 32;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = warp == NC;
    const uint32_t c = threadIdx.x;
    const uint32_t sw = p.split_width;
    Smem sm;
    sm.slots = nthr;
    sm.pool = smem;
    sm.rec = sm.pool + (size_t)tp.csm * 2;
    sm.dat = sm.rec + (size_t)3 * nthr * 2;
    sm.hdr = sm.dat + (size_t)2 * nthr * 6;
    Unit un;
    un.gscr = reinterpret_cast<uint4 *>(p.scratch + (uint64_t)unit * p.team_scratch_bytes);
    const uint32_t chunk = unit >> p.copies_log2;
    un.copy = unit & ((1u << p.copies_log2) - 1u);
    un.rank_base = un.copy ? tp.half_w : 0u;
    un.rank_lim = un.copy ? tp.retained : tp.half_w;
    un.out = p.persist + (uint64_t)(p.first_super + chunk) * p.super_bytes;
    un.cv0 = tp.cv0 + (uint64_t)un.copy * tp.S * 2;
#pragma unroll
    for (int i = 0; i < 8; i++) un.seed[i] = p.seeds[8 * (size_t)chunk + i];

    if (rank != 0) {
        /* rank 0's pool, through distributed shared memory */
        Smem rs;
        rs.slots = 0;
        rs.pool = cl.map_shared_rank(smem, 0);
        rs.rec = rs.dat = rs.hdr = nullptr;
        for (uint32_t k = 0; k < p.nsplit; k++) {
            const uint32_t l = __ldg(p.split_levels + k);
            if (k == 0 || __ldg(p.split_levels + k - 1) + 1 != l) cl.sync(); /* boundary l */
            const uint32_t ls = __ldg(tp.lstart + l), w = __ldg(tp.lstart + l + 1) - ls;
            const uint32_t per = (w + C - 1) / C, a = per > nthr ? per - nthr : 0;
            if (!producer)
                for (uint32_t j = nthr + a + (rank - 1) * nthr + c; j < w; j += (C - 1) * nthr)
                    direct_item(p, un, rs, ls + j);
            cl.sync(); /* boundary l + 1 */
        }
        return;
    }

    /* rank 0: prologue as k_label_ws */
    if (producer) {
        stage_records(p, sm, 0, lane);
        stage_records(p, sm, 1, lane);
        cp_async_commit();
        cp_async_wait_all();
        __syncwarp();
        const uint32_t ls0 = __ldg(tp.lstart), w0 = __ldg(tp.lstart + 1) - ls0;
        stage_data(p, sm, un, 0, ls0, w0, lane);
        cp_async_commit();
        cp_async_wait_all();
    }
    __syncthreads();
    if (tp.L > 0 && __ldg(tp.lstart + 1) - __ldg(tp.lstart) > sw) cl.sync(); /* boundary 0 */

    for (uint32_t l = 0; l < tp.L; l++) {
        const uint4 h = sm.hdr[l % 3];
        const uint32_t ls = h.x, w = h.y;
        /* the next level's width (its header arrived during level l - 1) */
        const uint32_t wn = l + 1 < tp.L ? sm.hdr[(l + 1) % 3].y : 0u;
        if (producer) {
            stage_records(p, sm, l + 2, lane);
            if (l + 1 < tp.L) stage_data(p, sm, un, l + 1, sm.hdr[(l + 1) % 3].x, wn, lane);
            cp_async_commit();
            cp_async_wait_all();
        } else {
            if (c < w && c < nthr) {
                const uint4 r0 = *sm.r(l % 3, c), r1 = *(sm.r(l % 3, c) + 1);
                const uint4 *d = sm.d(l & 1, c);
                const uint32_t np = (r0.x >> PB_REC_NP_SHIFT) & 3u;
                uint32_t m[16], cv[8];
#pragma unroll
                for (int i = 0; i < 16; i++) m[i] = 0;
                if (np >= 1) {
                    if (r0.y & PB_REF_PREV) load_prev(un, sm, r0.y, m);
                    else put8(m, d[2], d[3]);
                }
                if (np >= 2) {
                    if (r0.z & PB_REF_PREV) load_prev(un, sm, r0.z, m + 8);
                    else put8(m + 8, d[4], d[5]);
                }
                put8(cv, d[0], d[1]);
                hash_node(p, un, cv, m);
                store_label(un, sm, r0, r1, cv);
            }
            uint32_t lim = w;
            if (w > sw) { /* split: rank 0 stops at ceil(w / C) nodes */
                const uint32_t per = (w + C - 1) / C, a = per > nthr ? per - nthr : 0;
                lim = nthr + a < w ? nthr + a : w;
            }
            for (uint32_t j = c + nthr; j < lim; j += nthr) direct_item(p, un, sm, ls + j);
        }
        if (w > sw || wn > sw) cl.sync(); /* boundary l + 1 */
        else __syncthreads();
    }
}

namespace {

/* Shared-memory layout of the multi-unit kernel (uint4 units):
 *   pool  [G][csm][2]   next-level labels, one pool per unit
 *   rec   [3][slots][2] records of up to `slots` nodes per level (shared by the units)
 *   dat   [2][items][6] cv0 (2), predecessor 0 (2), predecessor 1 (2) per item
 *   hdr   [3]           (level start, width) of each ring stage
 * slots = hashing threads / G, items = slots * G; item i is node i / G of
 * the batch's unit i % G. */
struct SmemG {
    uint4 *pool, *rec, *dat, *hdr;
    uint32_t slots, items;
    __device__ __forceinline__ uint4 *r(uint32_t st, uint32_t j) const { return rec + ((size_t)st * slots + j) * 2; }
    __device__ __forceinline__ uint4 *d(uint32_t st, uint32_t i) const { return dat + ((size_t)st * items + i) * 6; }
};

/* Producer: block-0 values and older predecessors of level `lv` into data
 * stage lv & 1, for every item of the level's staged nodes whose unit is in
 * the batch (cnt units; s_copy = their copies).  The lanes stride over the
 * level's items, so a narrow level of G units is one pass; item i is node
 * i / G (a multiply-high by ginv = ceil(2^32 / G), exact for these counts)
 * of unit i % G. */
__device__ __forceinline__ void stage_data_g(const pb_wsg_params_t &p, const SmemG &sm, const uint32_t *s_copy,
                                             uint32_t cnt, uint32_t lv, uint32_t ls, uint32_t w, uint32_t lane,
                                             uint32_t ginv)
{
    if (lv >= p.topo.L) return;
    const uint32_t G = p.units_per_cta;
    const uint32_t ns = w < sm.slots ? w : sm.slots;
    const uint32_t rs = lv % 3, ds = lv & 1;
    for (uint32_t i = lane; i < ns * G; i += 32) {
        const uint32_t j = G == 1 ? i : __umulhi(i, ginv), u = i - j * G;
        if (u >= cnt) continue;
        const uint4 r0 = *sm.r(rs, j);
        uint4 *d = sm.d(ds, i);
        const uint4 *c = p.topo.cv0 + ((size_t)s_copy[u] * p.topo.S + ls + j) * 2;
        cp_async16(d, c);
        cp_async16(d + 1, c + 1);
        const uint4 *gs =
            reinterpret_cast<const uint4 *>(p.scratch + ((uint64_t)blockIdx.x * G + u) * p.unit_scratch_bytes);
        const uint32_t np = (r0.x >> PB_REC_NP_SHIFT) & 3u;
        if (np >= 1 && !(r0.y & PB_REF_PREV)) {
            const uint4 *s = gs + (size_t)(r0.y & PB_REF_SLOT_MASK) * 2;
            cp_async16(d + 2, s);
            cp_async16(d + 3, s + 1);
        }
        if (np >= 2 && !(r0.z & PB_REF_PREV)) {
            const uint4 *s = gs + (size_t)(r0.z & PB_REF_SLOT_MASK) * 2;
            cp_async16(d + 4, s);
            cp_async16(d + 5, s + 1);
        }
    }
}

} /* namespace */

/* k_label_ws with G (1 to 4) units of one topology per CTA.  The producer
 * warp stages each level's records once for all units and the block-0
 * values and older predecessors of every (node, unit) item; hashing thread
 * c < slots * G works item c (node c / G of unit c % G) and, on levels wider
 * than the staged slots, that unit's further nodes with direct loads.  One
 * CTA barrier ends a level, as in k_label_ws; there are no spin-waits. */
__global__ void __launch_bounds__(PB_CTA_THREADS, 1) k_label_wsg(const __grid_constant__ pb_wsg_params_t p)
{
    extern __shared__ uint4 smem[];
    __shared__ uint32_t s_batch, s_cnt;
    __shared__ uint32_t s_copy[4];
    const pb_topo_view2_t &tp = p.topo;
    const uint32_t NC = p.team_warps;
    const uint32_t nthr = NC * 32;
    const uint32_t G = p.units_per_cta;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = warp == NC;
    const uint32_t c = threadIdx.x;
    const uint32_t u = c % G, j0 = c / G;
    const uint32_t ginv = G > 1 ? (uint32_t)((0x100000000ull + G - 1) / G) : 0u;
    SmemG sg;
    sg.slots = nthr / G;
    sg.items = sg.slots * G;
    sg.pool = smem;
    sg.rec = sg.pool + (size_t)G * tp.csm * 2;
    sg.dat = sg.rec + (size_t)3 * sg.slots * 2;
    sg.hdr = sg.dat + (size_t)2 * nthr * 6;
    Smem su; /* this thread's unit pool, for load_prev / store_label / direct_item */
    su.pool = sg.pool + (size_t)u * tp.csm * 2;
    su.rec = su.dat = su.hdr = nullptr;
    su.slots = 0;
    Unit un;
    un.gscr = reinterpret_cast<uint4 *>(p.scratch + ((uint64_t)blockIdx.x * G + u) * p.unit_scratch_bytes);

    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t b = atomicAdd(p.queue, 1u);
            s_batch = b;
            s_cnt = 0;
            if (b < p.nbatches) {
                const uint32_t left = p.nunits - b * G;
                s_cnt = left < G ? left : G;
                for (uint32_t k = 0; k < s_cnt; k++) s_copy[k] = p.units[b * G + k].copy;
            }
        }
        __syncthreads();
        const uint32_t batch = s_batch, cnt = s_cnt;
        __syncthreads();
        if (batch >= p.nbatches) break;
        const bool act = !producer && u < cnt && c < sg.items;
        if (act) {
            const pb_munit_t mu = p.units[batch * G + u];
            un.copy = mu.copy;
            un.rank_base = mu.copy ? tp.half_w : 0u;
            un.rank_lim = mu.copy ? tp.retained : tp.half_w;
            un.out = reinterpret_cast<uint8_t *>(mu.out);
            un.cv0 = tp.cv0 + (uint64_t)mu.copy * tp.S * 2;
#pragma unroll
            for (int i = 0; i < 8; i++) un.seed[i] = p.seeds[8 * (size_t)mu.seed + i];
        }

        /* prologue: records of levels 0 and 1, then level 0's data */
        if (producer) {
            stage_records(p, sg, 0, lane);
            stage_records(p, sg, 1, lane);
            cp_async_commit();
            cp_async_wait_all();
            __syncwarp();
            const uint32_t ls0 = __ldg(tp.lstart), w0 = __ldg(tp.lstart + 1) - ls0;
            stage_data_g(p, sg, s_copy, cnt, 0, ls0, w0, lane, ginv);
            cp_async_commit();
            cp_async_wait_all();
        }
        __syncthreads();

        for (uint32_t l = 0; l < tp.L; l++) {
            if (producer) {
                stage_records(p, sg, l + 2, lane);
                if (l + 1 < tp.L) {
                    const uint4 h = sg.hdr[(l + 1) % 3];
                    stage_data_g(p, sg, s_copy, cnt, l + 1, h.x, h.y, lane, ginv);
                }
                cp_async_commit();
                cp_async_wait_all();
            } else if (act) {
                const uint4 h = sg.hdr[l % 3];
                const uint32_t ls = h.x, w = h.y;
                const uint32_t ns = w < sg.slots ? w : sg.slots;
                if (j0 < ns) {
                    const uint4 r0 = *sg.r(l % 3, j0), r1 = *(sg.r(l % 3, j0) + 1);
                    const uint4 *d = sg.d(l & 1, c);
                    const uint32_t np = (r0.x >> PB_REC_NP_SHIFT) & 3u;
                    uint32_t m[16], cv[8];
#pragma unroll
                    for (int i = 0; i < 16; i++) m[i] = 0;
                    if (np >= 1) {
                        if (r0.y & PB_REF_PREV) load_prev(un, su, r0.y, m);
                        else put8(m, d[2], d[3]);
                    }
                    if (np >= 2) {
                        if (r0.z & PB_REF_PREV) load_prev(un, su, r0.z, m + 8);
                        else put8(m + 8, d[4], d[5]);
                    }
                    put8(cv, d[0], d[1]);
                    hash_node(p, un, cv, m);
                    store_label(un, su, r0, r1, cv);
                }
                for (uint32_t j = j0 + sg.slots; j < w; j += sg.slots) direct_item(p, un, su, ls + j);
            }
            __syncthreads();
        }
    }
}

} /* namespace pb */

extern "C" int pb_dev_label_ws(const pb_pipe_params_t *params, uint32_t grid, uint32_t cta_threads,
                               uint32_t smem_bytes, cudaStream_t stream)
{
    if (cudaFuncSetAttribute(pb::k_label_ws, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes) !=
        cudaSuccess)
        return -1;
    cudaGetLastError(); /* report only this launch */
    pb::k_label_ws<<<grid, cta_threads, smem_bytes, stream>>>(*params);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_label_wsc(const pb_pipe_params_t *params, uint32_t smem_bytes, cudaStream_t stream)
{
    const uint32_t C = params->cluster;
    if (C < 2 || C > 16 || (params->team_warps != 7 && params->team_warps != 15) || params->nunits == 0)
        return -1;
    if (cudaFuncSetAttribute(pb::k_label_wsc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes) !=
            cudaSuccess ||
        (C > 8 && cudaFuncSetAttribute(pb::k_label_wsc, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                      cudaSuccess))
        return -1;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(params->nunits * C);
    cfg.blockDim = dim3(32 * (params->team_warps + 1));
    cfg.dynamicSmemBytes = smem_bytes;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaGetLastError(); /* report only this launch */
    if (cudaLaunchKernelEx(&cfg, pb::k_label_wsc, *params) != cudaSuccess) return -1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* How many clusters of C CTAs (team_warps hashing warps + 1, smem_bytes of
 * dynamic shared memory each) the device holds at once. */
extern "C" int pb_dev_label_wsc_max_clusters(uint32_t C, uint32_t team_warps, uint32_t smem_bytes, int *clusters)
{
    *clusters = 0;
    if (C < 2 || C > 16) return -1;
    if (cudaFuncSetAttribute(pb::k_label_wsc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes) !=
            cudaSuccess ||
        (C > 8 && cudaFuncSetAttribute(pb::k_label_wsc, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                      cudaSuccess))
        return -1;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(C * 148);
    cfg.blockDim = dim3(32 * (team_warps + 1));
    cfg.dynamicSmemBytes = smem_bytes;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(clusters, pb::k_label_wsc, &cfg) == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_label_ws_occupancy(uint32_t cta_threads, uint32_t smem_bytes, int *blocks_per_sm)
{
    if (cudaFuncSetAttribute(pb::k_label_ws, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes) !=
        cudaSuccess)
        return -1;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pb::k_label_ws, (int)cta_threads,
                                                         smem_bytes) == cudaSuccess
               ? 0
               : -1;
}

extern "C" uint32_t pb_wsg_smem_bytes(uint32_t csm, uint32_t units_per_cta, uint32_t team_warps)
{
    const uint32_t nthr = 32u * team_warps, slots = nthr / units_per_cta;
    return (2u * units_per_cta * csm + 3u * 2u * slots + 2u * 6u * nthr + 3u) * 16u;
}

extern "C" int pb_dev_label_wsg(const pb_wsg_params_t *params, uint32_t grid, uint32_t cta_threads,
                                uint32_t smem_bytes, cudaStream_t stream)
{
    if (params->units_per_cta < 1 || params->units_per_cta > 4 ||
        (params->team_warps != 7 && params->team_warps != 15) || cta_threads != 32u * (params->team_warps + 1) ||
        smem_bytes < pb_wsg_smem_bytes(params->topo.csm, params->units_per_cta, params->team_warps))
        return -1;
    cudaGetLastError(); /* report only this launch */
    pb::k_label_wsg<<<grid, cta_threads, smem_bytes, stream>>>(*params);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* Allow k_label_wsg the largest dynamic shared memory a CTA can have (the
 * device's opt-in limit less the kernel's static shared memory) and report
 * it; call before capturing a launch (the attribute is per function, not per
 * launch). */
extern "C" int pb_dev_label_wsg_prepare(uint32_t *max_smem_bytes)
{
    int dev = 0, optin = 0;
    cudaFuncAttributes fa;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, pb::k_label_wsg) != cudaSuccess)
        return -1;
    const int lim = optin - (int)fa.sharedSizeBytes;
    if (lim <= 0 || cudaFuncSetAttribute(pb::k_label_wsg, cudaFuncAttributeMaxDynamicSharedMemorySize, lim) !=
                        cudaSuccess)
        return -1;
    if (max_smem_bytes) *max_smem_bytes = (uint32_t)lim;
    return 0;
}
