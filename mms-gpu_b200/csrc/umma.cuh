// tcgen05 (5th-generation tensor core) GEMM core for sm_100a.
//
//   C[M x N] (+)= A[M x K] * B[N x K]^T      A, B: BF16, row-major (K-major)
//                                            C: FP32, row-major, leading dim ldc
//
// One CTA computes a 128 x BN tile with a single-CTA MMA (cta_group::1,
// M = 128): operands are staged in shared memory in the canonical K-major
// 128-byte-swizzled layout (8-row x 128-byte atoms, 16-byte chunks XOR-ed with
// the row), the accumulator lives in tensor memory (BN columns allocated per
// CTA), one elected thread issues the MMAs, and a commit to an mbarrier tells
// the CTA when a stage's shared memory may be refilled.  Two stages: the
// cp.async loads of K-tile k+1 run while the tensor core works on tile k.
// Every mbarrier wait is bounded; a timeout sets an error word and the CTA
// still releases its tensor memory.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace umma {

constexpr int BM = 128;          // MMA M (rows of the accumulator = TMEM lanes)
constexpr int BK = 64;           // K per stage: 64 BF16 = one 128-byte swizzle row
constexpr int STAGES = 2;
constexpr long long WAIT_CYCLES = 2000000000LL;  // ~1 s at the B200's SM clock

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major, SWIZZLE_128B, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);   // start address (16-byte units)
    d |= (uint64_t)1u << 16;                  // leading byte offset (unused for swizzled K-major): 1
    d |= (uint64_t)(1024u >> 4) << 32;        // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1u << 46;                  // descriptor version (sm_100)
    d |= (uint64_t)2u << 61;                  // layout: 128-byte swizzle
    return d;
}

// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_bf16(int n)
{
    return (1u << 4)                       // D format F32
           | (1u << 7)                     // A format BF16
           | (1u << 10)                    // B format BF16
           | ((uint32_t)(n >> 3) << 17)    // N / 8
           | ((uint32_t)(BM >> 4) << 24);  // M / 16
}

// byte offset of 16-byte chunk c (0..7) of row r inside a swizzled tile
__device__ __forceinline__ uint32_t sw128_off(int r, int c) { return (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4)); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid)
{
    const int n = valid ? 16 : 0;  // zero-fill when out of range
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(1) : "memory");
}

// bounded wait for the completion of the phase with the given parity:
// non-blocking test_wait with a short back-off, giving up after ~2e9 cycles
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const long long t0 = clock64();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > WAIT_CYCLES) return false;
        __nanosleep(32);
    }
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 lanes x 16 consecutive FP32 columns of the accumulator
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float v[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// shared memory of one CTA: S x (A tile 16 KB + B tile BN x 128 B), 1024-aligned
template <int BN, int S = STAGES>
struct Smem {
    alignas(1024) uint8_t a[S][BM * 128];
    alignas(1024) uint8_t b[S][BN * 128];
    uint64_t done[S];        // MMA of this stage finished (stage may be refilled)
    uint32_t tmem;           // allocated tensor-memory address
    int err;
};

__device__ __forceinline__ void cp_async_wait_pending(int pending)
{
    // wait until at most `pending` committed groups are still in flight
    if (pending >= 6)
        asm volatile("cp.async.wait_group 6;\n" ::: "memory");
    else if (pending == 5)
        asm volatile("cp.async.wait_group 5;\n" ::: "memory");
    else if (pending == 4)
        asm volatile("cp.async.wait_group 4;\n" ::: "memory");
    else if (pending == 3)
        asm volatile("cp.async.wait_group 3;\n" ::: "memory");
    else if (pending == 2)
        asm volatile("cp.async.wait_group 2;\n" ::: "memory");
    else if (pending == 1)
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    else
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// One 128 x BN tile of C.  A is M x K (lda), B is N x K (ldb), both BF16 with
// K contiguous; rows beyond M / N and columns beyond K read as zero.
// beta != 0: C += A B^T, else C = A B^T.  err: set to 1 on a barrier timeout.
// rowmap (may be NULL): row r of the tile result goes to C row rowmap[r].
// S pipeline stages (S - 1 tiles of cp.async loads in flight ahead of the
// tensor core); NT = 128 or 256 threads (256: two warps per TMEM lane quarter,
// splitting the loads and the epilogue's columns).
template <int BN, int S = STAGES, int NT = 128>
__device__ void gemm_tile(const __nv_bfloat16 *__restrict__ A, int lda, const __nv_bfloat16 *__restrict__ B, int ldb,
                          float *__restrict__ C, int ldc, int M, int N, int K, int m0, int n0, int beta,
                          int *__restrict__ err, Smem<BN, S> &s, const int *__restrict__ rowmap = nullptr)
{
    static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "BN must be a power of two in [32, 256]");
    static_assert(S >= 2 && S <= 8, "2..8 stages");
    static_assert(NT == 128 || NT == 256, "128 or 256 threads");
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s.tmem)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < S; i++) mbar_init(&s.done[i]);
        s.err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = s.tmem;
    const uint32_t idesc = idesc_bf16(BN);
    const int nk = (K + BK - 1) / BK;

    auto load_stage = [&](int st, int kt) {
        const int k0 = kt * BK;
        const uint32_t sa = smem_u32(s.a[st]), sb = smem_u32(s.b[st]);
        for (int i = tid; i < BM * 8; i += NT) {
            const int r = i >> 3, c = i & 7;
            const int gr = m0 + r, gk = k0 + c * 8;
            const bool ok = gr < M && gk < K;  // K is a multiple of 8 (16-byte rows)
            cp_async16(sa + sw128_off(r, c), ok ? (const void *)(A + (long long)gr * lda + gk) : (const void *)A, ok);
        }
        for (int i = tid; i < BN * 8; i += NT) {
            const int r = i >> 3, c = i & 7;
            const int gr = n0 + r, gk = k0 + c * 8;
            const bool ok = gr < N && gk < K;
            cp_async16(sb + sw128_off(r, c), ok ? (const void *)(B + (long long)gr * ldb + gk) : (const void *)B, ok);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    bool ok = true;
    int issued = 0;
    for (; issued < S - 1 && issued < nk; issued++) load_stage(issued % S, issued);
    for (int kt = 0; kt < nk && ok; kt++) {
        const int st = kt % S;
        cp_async_wait_pending(issued - kt - 1);  // tile kt has landed
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t sa = smem_u32(s.a[st]), sb = smem_u32(s.b[st]);
#pragma unroll
            for (int kk = 0; kk < BK / 16; kk++)
                mma_bf16(tmem, desc_sw128(sa + kk * 32), desc_sw128(sb + kk * 32), idesc, (kt > 0 || kk > 0) ? 1u : 0u);
            mma_commit(&s.done[st]);
        }
        __syncwarp();
        if (issued < nk) {
            // the stage to refill was read by the MMAs of tile kt - 1
            if (kt >= 1) ok = mbar_wait(&s.done[(kt - 1) % S], (uint32_t)(((kt - 1) / S) & 1));
            if (ok) {
                load_stage(issued % S, issued);
                issued++;
            }
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");  // no copy may still be in flight at exit
    // the last commit covers every earlier MMA of this thread
    if (ok && nk > 0) ok = mbar_wait(&s.done[(nk - 1) % S], (uint32_t)(((nk - 1) / S) & 1));
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    // epilogue: warp w reads accumulator rows 32 (w % 4) .. +31 (its TMEM lane
    // quarter); with 256 threads warps 4..7 take the upper half of the columns
    const int quarter = warp & 3;
    const int cbeg = (NT == 256) ? (warp >> 2) * (BN / 2) : 0;
    const int cend = (NT == 256) ? cbeg + BN / 2 : BN;
    if (!ok) {
        if (lane == 0) atomicExch(err, 1);
    } else if (nk > 0) {
        const int row = m0 + quarter * 32 + lane;
        for (int c0 = cbeg; c0 < cend; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0, v);
            if (row < M) {
                const long long crow_i = rowmap ? (long long)rowmap[row] : (long long)row;
                float *crow = C + crow_i * ldc + n0 + c0;
#pragma unroll
                for (int i = 0; i < 16; i++)
                    if (n0 + c0 + i < N) crow[i] = beta ? crow[i] + v[i] : v[i];
            }
        }
    } else if (!beta) {
        const int row = m0 + quarter * 32 + lane;
        if (row < M) {
            const long long crow_i = rowmap ? (long long)rowmap[row] : (long long)row;
            for (int c = cbeg; c < cend && n0 + c < N; c++) C[crow_i * ldc + n0 + c] = 0.f;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(BN) : "memory");
}

}  // namespace umma
