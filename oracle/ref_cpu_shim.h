/*
 * Test infrastructure only (part of the oracle).
 *
 * Force-included (g++ -include) when the reference's own sources are compiled
 * as plain C++ for the CPU oracle in oracle/_ref/.  The reference's CPU FMM
 * path still calls cudaHostAlloc / cudaHostGetDevicePointer for its mapped
 * pinned buffers (fmm_calc.cu:119-123, fmm_calc.cu:360-364) even when
 * use_gpu == 0, which needs a CUDA driver.  These stand-ins map that memory to
 * ordinary host memory so the unmodified CPU paths run on any host.  Nothing
 * here is part of the product library.
 */
#ifndef MMS_ORACLE_REF_CPU_SHIM_H
#define MMS_ORACLE_REF_CPU_SHIM_H

#include <stdlib.h>
#include <string.h>
#include <math.h> /* nvcc's host pass pulls these in implicitly; g++ does not */

typedef int cudaError_t;
#define cudaSuccess 0
#define cudaHostAllocMapped 2u

static inline cudaError_t cudaHostAlloc(void **p, size_t n, unsigned int flags)
{
    (void)flags;
    *p = calloc(1, n);
    return *p ? cudaSuccess : 2;
}

static inline cudaError_t cudaHostGetDevicePointer(void **d, void *h, unsigned int flags)
{
    (void)flags;
    *d = h;
    return cudaSuccess;
}

/* defined by the harness (the reference defines it in potential_calc.cu, which
 * is CUDA-only and not compiled into the CPU oracle) */
void checkCUDAError(const char *msg);

#endif
