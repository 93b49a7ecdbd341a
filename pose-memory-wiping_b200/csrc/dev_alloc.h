/* dev_alloc.h — the library's one device-allocation call (internal).
 *
 * Every device allocation of the library goes through pb_dev_malloc, which is
 * cudaMalloc plus a host-side fault injector for tests: with
 * POSE_B200_FAIL_ALLOC=n in the environment, the next n allocation attempts
 * after the variable was set (or changed) fail with cudaErrorMemoryAllocation
 * without touching the device.  The failure is made on the host, so no GPU
 * fault is involved. */
#ifndef PB_DEV_ALLOC_H
#define PB_DEV_ALLOC_H

#include <stddef.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

cudaError_t pb_dev_malloc(void **ptr, size_t bytes);

#ifdef __cplusplus
}
#endif
#endif
