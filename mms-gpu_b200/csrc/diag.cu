// Diagnostics: an FP32 FMA throughput microbenchmark.  Its result is the
// denominator of the roofline fraction for the FP32-pipe-bound kernels (the
// direct sum and the FMM near field), which the HBM-copy and bf16-GEMM peaks
// do not cover.
#include "mms_internal.cuh"

namespace {

constexpr int FMA_CHAINS = 8;
constexpr int FMA_ITERS = 4096;

__global__ void __launch_bounds__(256) k_fma_peak(float *out, float a, float b)
{
    float v[FMA_CHAINS];
#pragma unroll
    for (int c = 0; c < FMA_CHAINS; c++) v[c] = threadIdx.x * 1e-7f + c;
    for (int it = 0; it < FMA_ITERS; it++) {
#pragma unroll
        for (int c = 0; c < FMA_CHAINS; c++) v[c] = fmaf(v[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < FMA_CHAINS; c++) s += v[c];
    if (s == 12345.678f) out[0] = s;  // keeps the chains alive
}

}  // namespace

extern "C" int mms_diag_fma_tflops(int reps, double *tflops)
{
    if (!tflops || reps < 1) {
        mms_set_error("mms_diag_fma_tflops: bad argument");
        return MMS_ERR_ARG;
    }
    int dev = 0, sms = 0;
    MMS_CUDA_TRY(cudaGetDevice(&dev));
    MMS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    float *out = nullptr;
    MMS_CUDA_TRY(cudaMalloc(&out, sizeof(float)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8;
    k_fma_peak<<<blocks, 256>>>(out, 0.999999f, 1e-7f);  // warm-up
    cudaEventRecord(e0);
    for (int r = 0; r < reps; r++) k_fma_peak<<<blocks, 256>>>(out, 0.999999f, 1e-7f);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) {
        mms_set_error("mms_diag_fma_tflops: %s", cudaGetErrorString(e));
        return MMS_ERR_CUDA;
    }
    const double flops = 2.0 * FMA_CHAINS * (double)FMA_ITERS * 256.0 * blocks * reps;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return MMS_OK;
}
