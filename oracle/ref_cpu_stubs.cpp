/*
 * Test infrastructure only (part of the oracle).
 *
 * CPU-only stand-ins for the reference's CUDA-side symbols, linked with the
 * reference's own CPU sources in oracle/_ref/.  The oracle only ever runs the
 * reference with use_gpu == 0, so these are never reached on a correct call;
 * they exist so the reference's CPU objects link without its CUDA translation
 * unit (potential_calc.cu, fmm_kernel.cu).
 */
#include <cstdio>
#include <cstdlib>

#include "mydefs.hpp"
#include "Vector3.hpp"
#include "helper_functions.hpp"

void checkCUDAError(const char *msg) { (void)msg; }

int calc_potential_exact_gpu(const fptype *, const int, const int, const int,
                             const fptype, const fptype, const fptype, fptype *)
{
    fprintf(stderr, "oracle: the reference's GPU direct path is not part of the CPU oracle\n");
    return EXIT_FAILURE;
}

int fmm_gpu(const Box *const, const Cmpx *const, fptype *, const unsigned int, const int,
            const int, const int, const int, const fptype, const fptype, const fptype,
            const int, const int, const int)
{
    fprintf(stderr, "oracle: the reference's GPU FMM path is not part of the CPU oracle\n");
    return EXIT_FAILURE;
}
