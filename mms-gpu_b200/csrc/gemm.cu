// BF16 tensor-core GEMM entry points on the tcgen05 core (umma.cuh):
// C = A B^T or C += A B^T with A (M x K) and B (N x K) K-major.
#include "mms_internal.cuh"
#include "umma.cuh"

namespace {

__device__ int g_umma_err;

template <int BN>
__global__ void __launch_bounds__(128) k_gemm_bf16(const __nv_bfloat16 *__restrict__ A, int lda,
                                                   const __nv_bfloat16 *__restrict__ B, int ldb, float *__restrict__ C,
                                                   int ldc, int M, int N, int K, int beta)
{
    extern __shared__ uint8_t raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
    umma::Smem<BN> &s = *reinterpret_cast<umma::Smem<BN> *>(base);
    umma::gemm_tile<BN>(A, lda, B, ldb, C, ldc, M, N, K, blockIdx.x * umma::BM, blockIdx.y * BN, beta, &g_umma_err,
                        s);
}

template <int BN>
size_t gemm_smem() { return sizeof(umma::Smem<BN>) + 1024; }

template <int BN>
int gemm_launch(const void *A, int lda, const void *B, int ldb, float *C, int ldc, int M, int N, int K, int beta,
                cudaStream_t st)
{
    static bool attr = false;  // per process; the attribute is set on the current device
    if (!attr) {
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)gemm_smem<BN>()));
        attr = true;
    }
    dim3 grid(div_up(M, umma::BM), div_up(N, BN));
    k_gemm_bf16<BN><<<grid, 128, gemm_smem<BN>(), st>>>((const __nv_bfloat16 *)A, lda, (const __nv_bfloat16 *)B,
                                                         ldb, C, ldc, M, N, K, beta);
    MMS_CUDA_TRY(cudaGetLastError());
    return MMS_OK;
}

}  // namespace

int umma_gemm_bf16(const void *A, int lda, const void *B, int ldb, float *C, int ldc, int M, int N, int K, int beta,
                   int bn, cudaStream_t st)
{
    if (M < 1 || N < 1 || K < 0 || (K % 8) || (lda % 8) || (ldb % 8) || lda < K || ldb < K || ldc < N) {
        mms_set_error("gemm: K, lda, ldb must be multiples of 8 with lda, ldb >= K, ldc >= N");
        return MMS_ERR_ARG;
    }
    switch (bn) {
    case 64: return gemm_launch<64>(A, lda, B, ldb, C, ldc, M, N, K, beta, st);
    case 128: return gemm_launch<128>(A, lda, B, ldb, C, ldc, M, N, K, beta, st);
    default:
        mms_set_error("gemm: tile N must be 64 or 128");
        return MMS_ERR_ARG;
    }
}

int umma_check_error()
{
    int e = 0;
    MMS_CUDA_TRY(cudaMemcpyFromSymbol(&e, g_umma_err, sizeof(int)));
    if (e) {
        const int z = 0;
        cudaMemcpyToSymbol(g_umma_err, &z, sizeof(int));
        mms_set_error("tensor-core GEMM: an mbarrier wait timed out");
        return MMS_ERR_CUDA;
    }
    return MMS_OK;
}

extern "C" int mms_diag_gemm_bf16(const void *A, int lda, const void *B, int ldb, float *C, int ldc, int M, int N,
                                  int K, int beta, int bn, void *stream)
{
    if (!A || !B || !C) {
        mms_set_error("mms_diag_gemm_bf16: NULL argument");
        return MMS_ERR_ARG;
    }
    MMS_TRY(umma_gemm_bf16(A, lda, B, ldb, C, ldc, M, N, K, beta, bn, (cudaStream_t)stream));
    MMS_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return umma_check_error();
}
