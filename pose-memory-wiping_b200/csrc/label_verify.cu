/*
 * label_verify.cu — device helpers of the GPU verifier (label_verify.c) and
 * of the workspace audit (pose_b200_topo_residue).
 *
 * All are plain HBM streams: the compare reads two labelled super-chunk
 * images 32 bytes per thread-iteration with 128-bit loads, the gather moves
 * one 32-byte label per challenge, and the count reads a buffer 16 bytes per
 * thread-iteration.  None is on the labeling path.
 */
#include "kernels.h"

#include <cuda_runtime.h>

namespace pb {

__global__ void __launch_bounds__(256) k_compare_blocks(const uint4 *__restrict__ a, const uint4 *__restrict__ b,
                                                        uint64_t nblocks, uint64_t per_group,
                                                        unsigned long long *__restrict__ first_bad)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nblocks; i += stride) {
        const uint4 x0 = a[2 * i], x1 = a[2 * i + 1];
        const uint4 y0 = b[2 * i], y1 = b[2 * i + 1];
        const uint32_t d = (x0.x ^ y0.x) | (x0.y ^ y0.y) | (x0.z ^ y0.z) | (x0.w ^ y0.w) |
                           (x1.x ^ y1.x) | (x1.y ^ y1.y) | (x1.z ^ y1.z) | (x1.w ^ y1.w);
        if (d) atomicMin(&first_bad[i / per_group], (unsigned long long)(i % per_group));
    }
}

__global__ void __launch_bounds__(128) k_gather_labels(const uint4 *__restrict__ work,
                                                       const uint64_t *__restrict__ src, uint32_t n,
                                                       uint4 *__restrict__ out)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint64_t s = src[k];
    out[2 * k] = work[2 * s];
    out[2 * k + 1] = work[2 * s + 1];
}

__device__ __forceinline__ uint32_t nonzero_bytes_of(uint32_t w)
{
    return (uint32_t)((w & 0xFFu) != 0) + (uint32_t)((w & 0xFF00u) != 0) + (uint32_t)((w & 0xFF0000u) != 0) +
           (uint32_t)((w & 0xFF000000u) != 0);
}

/* *count += nonzero bytes of buf[0, bytes); buf is 16-byte aligned. */
__global__ void __launch_bounds__(256) k_count_nonzero(const uint8_t *__restrict__ buf, uint64_t bytes,
                                                       unsigned long long *__restrict__ count)
{
    const uint4 *v = (const uint4 *)buf;
    const uint64_t words = bytes / 16;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t n = 0;
    for (uint64_t i = tid; i < words; i += stride) {
        const uint4 x = v[i];
        n += nonzero_bytes_of(x.x) + nonzero_bytes_of(x.y) + nonzero_bytes_of(x.z) + nonzero_bytes_of(x.w);
    }
    if (tid == 0)
        for (uint64_t j = words * 16; j < bytes; j++) n += buf[j] != 0;
    n = __reduce_add_sync(0xFFFFFFFFu, n);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(count, (unsigned long long)n);
}

}  // namespace pb

extern "C" int pb_dev_compare_blocks(const void *a, const void *b, uint64_t nblocks, uint64_t blocks_per_group,
                                     unsigned long long *first_bad, uint32_t grid, cudaStream_t stream)
{
    if (nblocks == 0) return 0;
    if (blocks_per_group == 0 || grid == 0) return -1;
    cudaGetLastError();
    pb::k_compare_blocks<<<grid, 256, 0, stream>>>((const uint4 *)a, (const uint4 *)b, nblocks, blocks_per_group,
                                                   first_bad);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_gather_labels(const void *work, const uint64_t *src, uint32_t n, void *out,
                                    cudaStream_t stream)
{
    if (n == 0) return 0;
    cudaGetLastError();
    pb::k_gather_labels<<<(n + 127) / 128, 128, 0, stream>>>((const uint4 *)work, src, n, (uint4 *)out);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_dev_count_nonzero(const void *buf, uint64_t bytes, unsigned long long *d_count, uint32_t grid,
                                    cudaStream_t stream)
{
    if (bytes == 0) return 0;
    if (!buf || !d_count || grid == 0 || ((uintptr_t)buf & 15u)) return -1;
    const uint64_t words = bytes / 16;
    const uint64_t need = (words + 255) / 256;
    const uint32_t g = need == 0 ? 1u : need < grid ? (uint32_t)need : grid;
    cudaGetLastError();
    pb::k_count_nonzero<<<g, 256, 0, stream>>>((const uint8_t *)buf, bytes, d_count);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
