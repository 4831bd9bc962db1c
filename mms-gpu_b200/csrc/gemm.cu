// BF16 tensor-core GEMM entry points on the tcgen05 core (umma.cuh):
// C = A B^T or C += A B^T with A (M x K) and B (N x K) K-major.
#include <algorithm>

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

// split-K: CTA (m tile, n tile, split s) multiplies the K range
// [s kchunk, (s + 1) kchunk) into its own partial C (Cp + s M N, beta 0)
template <int BN>
__global__ void __launch_bounds__(128) k_gemm_bf16_splitk(const __nv_bfloat16 *__restrict__ A, int lda,
                                                          const __nv_bfloat16 *__restrict__ B, int ldb,
                                                          float *__restrict__ Cp, int M, int N, int K, int kchunk)
{
    extern __shared__ uint8_t raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
    umma::Smem<BN> &s = *reinterpret_cast<umma::Smem<BN> *>(base);
    const int k0 = blockIdx.z * kchunk;
    const int kn = min(kchunk, K - k0);
    umma::gemm_tile<BN>(A + k0, lda, B + k0, ldb, Cp + (size_t)blockIdx.z * M * N, N, M, N, kn, blockIdx.x * umma::BM,
                        blockIdx.y * BN, 0, &g_umma_err, s);
}

// C = sum of the splits' partials, in split order
__global__ void k_splitk_reduce(const float *__restrict__ Cp, int splits, long long MN, float *__restrict__ C)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MN) return;
    float v = Cp[i];
    for (int s = 1; s < splits; s++) v += Cp[(long long)s * MN + i];
    C[i] = v;
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

int umma_gemm_bf16_splitk_plan(int M, int N, int K, int bn, int *splits, int *kchunk)
{
    const int tiles = (int)(div_up(M, umma::BM) * div_up(N, bn));
    int sp = std::max(1, std::min(148 / std::max(tiles, 1), (K + 63) / 64));
    int kc = ((K + sp - 1) / sp + 63) / 64 * 64;
    sp = (K + kc - 1) / kc;
    *splits = sp;
    *kchunk = kc;
    return MMS_OK;
}

int umma_gemm_bf16_splitk(const void *A, int lda, const void *B, int ldb, float *C, float *Cpart, int M, int N,
                          int K, int bn, int splits, int kchunk, cudaStream_t st)
{
    if (M < 1 || N < 1 || K < 8 || (K % 8) || (lda % 8) || (ldb % 8) || lda < K || ldb < K || kchunk % 64 ||
        (long long)splits * kchunk < K || (long long)(splits - 1) * kchunk >= K) {
        mms_set_error("gemm split-K: bad shape");
        return MMS_ERR_ARG;
    }
    // the two tile widths have the same function type: one set-up flag each
    static bool attr64 = false, attr128 = false;
    auto launch = [&](auto kern, size_t smem, bool &attr) -> int {
        if (!attr) {
            MMS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr = true;
        }
        dim3 grid(div_up(M, umma::BM), div_up(N, bn), splits);
        kern<<<grid, 128, smem, st>>>((const __nv_bfloat16 *)A, lda, (const __nv_bfloat16 *)B, ldb, Cpart, M, N, K,
                                      kchunk);
        MMS_CUDA_TRY(cudaGetLastError());
        return MMS_OK;
    };
    if (bn == 64)
        MMS_TRY(launch(k_gemm_bf16_splitk<64>, gemm_smem<64>(), attr64));
    else if (bn == 128)
        MMS_TRY(launch(k_gemm_bf16_splitk<128>, gemm_smem<128>(), attr128));
    else {
        mms_set_error("gemm split-K: tile N must be 64 or 128");
        return MMS_ERR_ARG;
    }
    const long long MN = (long long)M * N;
    k_splitk_reduce<<<div_up(MN, 256), 256, 0, st>>>(Cpart, splits, MN, C);
    MMS_CUDA_TRY(cudaGetLastError());
    return MMS_OK;
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
