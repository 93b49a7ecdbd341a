/*
 * label_noalloc.cu — labeling with no device allocation in the call.
 *
 * pose_b200_topo_label_noalloc produces the same bytes as
 * pose_graph_hbm_topo_label, but its scratch pool, chunk-seed table, session
 * seed copy and work counter live in file-scope static device arrays instead
 * of memory the call allocates.  It exists for callers that must not call
 * cudaMalloc while they label: a wipe worker that reserved the device's free
 * memory for its label window up front (an allocation there could fail
 * half-way through a disk, or land in memory another tenant is about to
 * claim), or a host whose own memory pool already holds the device's memory.
 * The topology (an input built
 * earlier by pose_graph_hbm_topo_build), the session seed and the output
 * buffer still come from the caller.
 *
 * Limits: PB_NOALLOC_SCRATCH_BYTES of scratch (enough for two concurrent
 * chunk copies at chunk_blocks = 2^20 and 16 at 2^17; the schedule adapts to
 * it, so any chunk_blocks the library accepts fits), session seeds of at most
 * PB_NOALLOC_MAX_SEED bytes, and PB_NOALLOC_MAX_CHUNKS super-chunks per
 * kernel launch (larger buffers are labelled in several launches).  Every
 * GPU that loads this library holds these arrays until the process exits.
 */
#include "kernels.h"
#include "pose_b200.h"
#include "topo_internal.h"

#include <cuda_runtime.h>
#include <pthread.h>
#include <string.h>

#define PB_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define PB_NOALLOC_MAX_CHUNKS 8192u
#define PB_NOALLOC_MAX_SEED 1016u
#define PB_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) uint8_t g_na_scratch[PB_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) uint32_t g_na_seeds[PB_NOALLOC_MAX_CHUNKS * 8];
static __device__ __align__(256) uint8_t g_na_session[PB_NOALLOC_MAX_SEED];
static __device__ __align__(256) unsigned int g_na_queue[64];

/* Device addresses of the arrays above, looked up once per device.  In host
 * code the array names are host-side stand-ins, not device addresses; only
 * these looked-up pointers may be handed to kernels and copies. */
typedef struct {
    int ready;
    uint8_t *scratch;
    uint32_t *seeds;
    uint8_t *session;
    unsigned int *queue;
} na_addrs_t;

static na_addrs_t g_na_addrs[PB_NOALLOC_MAX_DEVICES];
static pthread_mutex_t g_na_lock = PTHREAD_MUTEX_INITIALIZER;

/* With `device` current: resolve the arrays' device addresses (first call on
 * a device only). */
static int na_setup(int device, na_addrs_t *out)
{
    if (device < 0 || device >= PB_NOALLOC_MAX_DEVICES) return -1;
    pthread_mutex_lock(&g_na_lock);
    na_addrs_t *a = &g_na_addrs[device];
    int rc = 0;
    if (!a->ready) {
        if (cudaGetSymbolAddress((void **)&a->scratch, g_na_scratch) != cudaSuccess ||
            cudaGetSymbolAddress((void **)&a->seeds, g_na_seeds) != cudaSuccess ||
            cudaGetSymbolAddress((void **)&a->session, g_na_session) != cudaSuccess ||
            cudaGetSymbolAddress((void **)&a->queue, g_na_queue) != cudaSuccess) {
            rc = -1;
        } else {
            a->ready = 1;
        }
    }
    if (rc == 0) *out = *a;
    pthread_mutex_unlock(&g_na_lock);
    return rc;
}

/* Same bytes as pose_graph_hbm_topo_label; see include/pose_b200.h. */
extern "C" int pose_b200_topo_label_noalloc(const pose_hbm_topo_t *topo, const uint8_t *session_seed,
                                            size_t seed_len, void *hbm_dev_ptr, size_t hbm_len,
                                            uint64_t region_block_offset)
{
    pb_topo_internal_t ti;
    if (pb_topo_internal(topo, &ti) != 0) {
        pb_set_err("pose_b200_topo_label_noalloc: NULL topology");
        return -1;
    }
    const uint64_t num_super = hbm_len / ti.super_bytes;
    if (num_super == 0) return 0; /* smaller than one super-chunk: nothing to label */
    if (!hbm_dev_ptr || (!session_seed && seed_len)) {
        pb_set_err("pose_b200_topo_label_noalloc: NULL buffer or seed");
        return -1;
    }
    if (seed_len > PB_NOALLOC_MAX_SEED) {
        pb_set_err("pose_b200_topo_label_noalloc: session seed of %zu bytes exceeds the %u-byte maximum "
                   "of the no-allocation entry point",
                   seed_len, PB_NOALLOC_MAX_SEED);
        return -1;
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != ti.device && cudaSetDevice(ti.device) != cudaSuccess) {
        pb_set_err("pose_b200_topo_label_noalloc: cannot select the topology's device");
        return -1;
    }
    int rc = -1;
    na_addrs_t na;
    pb_plan_out_t plan;
    const uint64_t per_launch = num_super < PB_NOALLOC_MAX_CHUNKS ? num_super : PB_NOALLOC_MAX_CHUNKS;
    cudaStream_t s = ti.stream;
    if (na_setup(ti.device, &na) != 0) {
        pb_set_err("pose_b200_topo_label_noalloc: cudaGetSymbolAddress failed: %s",
                   cudaGetErrorString(cudaGetLastError()));
        goto out;
    }
    if (pb_plan_for_budget(topo, per_launch * ti.copies, PB_NOALLOC_SCRATCH_BYTES, &plan) != 0) {
        pb_set_err("pose_b200_topo_label_noalloc: chunk_blocks %u needs %llu bytes of scratch per chunk copy, "
                   "more than the %llu bytes the no-allocation entry point holds",
                   ti.cb, (unsigned long long)ti.view.pool * 32ull, PB_NOALLOC_SCRATCH_BYTES);
        goto out;
    }
    if (seed_len && cudaMemcpyAsync(na.session, session_seed, seed_len, cudaMemcpyHostToDevice, s) != cudaSuccess)
        goto cuda_fail;
    for (uint64_t first = 0; first < num_super; first += per_launch) {
        uint64_t n = num_super - first < per_launch ? num_super - first : per_launch;
        if (pb_dev_chunk_seeds(na.session, (uint32_t)seed_len, region_block_offset, ti.cb, (uint32_t)n, first,
                               na.seeds, s) != 0)
            goto cuda_fail;
        /* the work counter must start at zero for every launch */
        if (cudaMemsetAsync(na.queue, 0, sizeof(unsigned int), s) != cudaSuccess) goto cuda_fail;
        pb_label_params_t p;
        memset(&p, 0, sizeof(p));
        p.topo = ti.view;
        p.seeds = na.seeds;
        p.persist = (uint8_t *)hbm_dev_ptr;
        p.super_bytes = ti.super_bytes;
        p.first_super = first;
        p.scratch = na.scratch;
        p.team_scratch_bytes = plan.team_scratch;
        p.nunits = (uint32_t)(n * ti.copies);
        p.copies_log2 = ti.copies == 2 ? 1 : 0;
        p.g_log2 = (uint32_t)__builtin_ctz(plan.G);
        p.team_warps = plan.T;
        p.nbatches = (uint32_t)((p.nunits + plan.G - 1) / plan.G);
        p.queue = na.queue;
        p.one = 1;
        if (pb_dev_label(&p, plan.grid, plan.cta, 0, s) != 0) goto cuda_fail;
    }
    /* labels and seeds never outlive the call: clear the shared scratch, the
     * seed table and the session seed copy */
    if (cudaMemsetAsync(na.scratch, 0, plan.scratch_bytes, s) != cudaSuccess) goto cuda_fail;
    if (cudaMemsetAsync(na.seeds, 0, per_launch * 32, s) != cudaSuccess) goto cuda_fail;
    if (seed_len && cudaMemsetAsync(na.session, 0, seed_len, s) != cudaSuccess) goto cuda_fail;
    if (cudaStreamSynchronize(s) != cudaSuccess) goto cuda_fail;
    rc = 0;
    goto out;
cuda_fail:
    pb_set_err("pose_b200_topo_label_noalloc: CUDA error: %s", cudaGetErrorString(cudaGetLastError()));
    /* a call that stopped part way clears all three arrays, best effort */
    cudaMemsetAsync(na.scratch, 0, PB_NOALLOC_SCRATCH_BYTES, s);
    cudaMemsetAsync(na.seeds, 0, sizeof(g_na_seeds), s);
    cudaMemsetAsync(na.session, 0, PB_NOALLOC_MAX_SEED, s);
    cudaStreamSynchronize(s);
    cudaGetLastError();
out:
    if (prev >= 0 && prev != ti.device) cudaSetDevice(prev);
    return rc;
}

/* Count the nonzero bytes of this device's no-allocation workspace (scratch,
 * seed table, session seed) into *d_count on stream s; nothing to count (0)
 * when the entry point never ran on the device.  The device is current. */
extern "C" int pb_noalloc_residue(int device, unsigned long long *d_count, uint32_t grid, cudaStream_t s)
{
    if (device < 0 || device >= PB_NOALLOC_MAX_DEVICES) return -1;
    pthread_mutex_lock(&g_na_lock);
    const na_addrs_t a = g_na_addrs[device];
    pthread_mutex_unlock(&g_na_lock);
    if (!a.ready) return 0;
    if (pb_dev_count_nonzero(a.scratch, PB_NOALLOC_SCRATCH_BYTES, d_count, grid, s) != 0 ||
        pb_dev_count_nonzero(a.seeds, sizeof(g_na_seeds), d_count, grid, s) != 0 ||
        pb_dev_count_nonzero(a.session, PB_NOALLOC_MAX_SEED, d_count, grid, s) != 0)
        return -1;
    return 0;
}
