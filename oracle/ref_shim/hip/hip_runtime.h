/* Host-only stand-in for <hip/hip_runtime.h>.
 *
 * Test infrastructure: lets the reference's HOST headers (macros.h, format.h,
 * coo2block.h, utils.h under cb-spmv-dcu/src/) compile with g++ so the oracle
 * can be pinned against the reference's own CB builder and CPU SpMV.  Nothing
 * here touches a GPU; the device-side helpers of utils.h are never called.
 */
#pragma once
#include <climits> /* the real HIP header brings INT_MAX in transitively */
#include <cstddef>
#include <cstring>

typedef int hipError_t;
static const hipError_t hipSuccess = 0;

typedef enum hipMemcpyKind {
    hipMemcpyHostToHost = 0,
    hipMemcpyHostToDevice = 1,
    hipMemcpyDeviceToHost = 2,
    hipMemcpyDeviceToDevice = 3
} hipMemcpyKind;

typedef struct hipDeviceProp_t {
    char name[256];
    int major, minor;
    size_t totalGlobalMem, totalConstMem, sharedMemPerBlock;
    size_t maxSharedMemoryPerMultiProcessor;
    int maxGridSize[3], maxThreadsDim[3];
    int multiProcessorCount, regsPerBlock, maxThreadsPerBlock;
    int maxThreadsPerMultiProcessor, warpSize;
} hipDeviceProp_t;

static inline const char *hipGetErrorString(hipError_t) { return "host stub"; }
static inline hipError_t hipDeviceReset() { return hipSuccess; }
static inline hipError_t hipSetDevice(int) { return hipSuccess; }
static inline hipError_t hipGetDeviceProperties(hipDeviceProp_t *p, int) {
    std::memset(p, 0, sizeof(*p));
    return hipSuccess;
}
static inline hipError_t hipMemcpy(void *dst, const void *src, size_t bytes,
                                   hipMemcpyKind) {
    std::memcpy(dst, src, bytes);
    return hipSuccess;
}
