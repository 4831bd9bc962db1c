// Local stencils of the field evaluation and the fused field + LLG + RK4 stage.
//
// Two families:
//  * FP32 AoS operators behind the reference-facing API (divergence_3d,
//    gradient_3d, add_exchange_field, Hfield: vector_functions.cpp:8-103,
//    ode_functions.cpp:21-70).  They keep the reference's operation order and
//    use explicitly rounded intrinsics (no FMA contraction), so for the same
//    FP32 input they return the reference's bits.
//  * The resident-state path: FP64 SoA state planes (M, stage buffers, the RK4
//    slope sum), FP32 rho/phi.  One kernel per RK4 stage fuses
//    H = (1/4pi) grad(phi) + exchange(M_stage) + H_ext(t_stage), the LLG
//    right-hand side (ode_functions.cpp:11-18) and the RK4 stage combination
//    (ode_functions.cpp:96-145), so every state array is read once and written
//    once per stage.
#include <cuda_bf16.h>

#include "mms_internal.cuh"

#include <math.h>

#include "stencil_dev.cuh"

namespace {

using namespace mmsdev;

constexpr int TPB = 256;

// ---- FP32 AoS, reference operation order ---------------------------------

// vector_functions.cpp:8-28
__global__ void k_div_aos(const float *__restrict__ M, float *__restrict__ rho, GridK g, float dx, float dy, float dz)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    int x, y, z;
    cell_xyz(i, g, x, y, z);
    const long long sx = 1, sy = g.X, sz = (long long)g.X * g.Y;
    float x2 = (x != g.X - 1) ? M[3 * (i + sx) + 0] : 0.f;
    float x0 = (x != 0) ? M[3 * (i - sx) + 0] : 0.f;
    float y2 = (y != g.Y - 1) ? M[3 * (i + sy) + 1] : 0.f;
    float y0 = (y != 0) ? M[3 * (i - sy) + 1] : 0.f;
    float z2 = (z != g.Z - 1) ? M[3 * (i + sz) + 2] : 0.f;
    float z0 = (z != 0) ? M[3 * (i - sz) + 2] : 0.f;
    float s = __fadd_rn(__fadd_rn(__fdiv_rn(__fsub_rn(x2, x0), dx), __fdiv_rn(__fsub_rn(y2, y0), dy)),
                        __fdiv_rn(__fsub_rn(z2, z0), dz));
    rho[i] = s * 0.5f;  // (s / 2.0) in double then to float: exact halving
}

// vector_functions.cpp:31-54; c is the reference's fptype constant_multiple
__device__ __forceinline__ void grad_aos_cell(const float *__restrict__ S, long long i, int x, int y, int z,
                                              const GridK &g, float dx2, float dy2, float dz2, float c, float H[3])
{
    const long long sy = g.X, sz = (long long)g.X * g.Y;
    float x2 = (x != g.X - 1) ? S[i + 1] : 0.f;
    float x0 = (x != 0) ? S[i - 1] : 0.f;
    float y2 = (y != g.Y - 1) ? S[i + sy] : 0.f;
    float y0 = (y != 0) ? S[i - sy] : 0.f;
    float z2 = (z != g.Z - 1) ? S[i + sz] : 0.f;
    float z0 = (z != 0) ? S[i - sz] : 0.f;
    H[0] = __fmul_rn(__fdiv_rn(__fsub_rn(x2, x0), dx2), c);
    H[1] = __fmul_rn(__fdiv_rn(__fsub_rn(y2, y0), dy2), c);
    H[2] = __fmul_rn(__fdiv_rn(__fsub_rn(z2, z0), dz2), c);
}

// vector_functions.cpp:57-103: H += cm * lap(M), M = 0 outside
__device__ __forceinline__ void exch_aos_cell(const float *__restrict__ M, long long i, int x, int y, int z,
                                              const GridK &g, float ddx, float ddy, float ddz, float cm, float H[3])
{
    const long long sy = g.X, sz = (long long)g.X * g.Y;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float m0 = M[3 * i + c];
        float xp = (x != g.X - 1) ? M[3 * (i + 1) + c] : 0.f;
        float xm = (x != 0) ? M[3 * (i - 1) + c] : 0.f;
        float yp = (y != g.Y - 1) ? M[3 * (i + sy) + c] : 0.f;
        float ym = (y != 0) ? M[3 * (i - sy) + c] : 0.f;
        float zp = (z != g.Z - 1) ? M[3 * (i + sz) + c] : 0.f;
        float zm = (z != 0) ? M[3 * (i - sz) + c] : 0.f;
        float m2 = __fmul_rn(2.f, m0);
        float lx = __fdiv_rn(__fsub_rn(__fadd_rn(xp, xm), m2), ddx);
        float ly = __fdiv_rn(__fsub_rn(__fadd_rn(yp, ym), m2), ddy);
        float lz = __fdiv_rn(__fsub_rn(__fadd_rn(zp, zm), m2), ddz);
        float L = __fadd_rn(__fadd_rn(lx, ly), lz);
        H[c] = __fadd_rn(H[c], __fmul_rn(cm, L));
    }
}

struct AosConsts {
    float dx2, dy2, dz2;   // 2*dx etc. (fptype)
    float ddx, ddy, ddz;   // dx*dx etc. (fptype)
    float cgrad;           // (fptype)(1/(4 pi)) or caller's constant
    float cm;              // (fptype)(2 A / (mu Ms Ms)) in fptype arithmetic
    float hx, hy, hz;      // H_ext as the reference's Vector3
    int demag, exchange, external;
};

__global__ void k_grad_aos(const float *__restrict__ S, float *__restrict__ H, GridK g, AosConsts k)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    int x, y, z;
    cell_xyz(i, g, x, y, z);
    float h[3];
    grad_aos_cell(S, i, x, y, z, g, k.dx2, k.dy2, k.dz2, k.cgrad, h);
    H[3 * i + 0] = h[0];
    H[3 * i + 1] = h[1];
    H[3 * i + 2] = h[2];
}

__global__ void k_exch_aos(const float *__restrict__ M, float *__restrict__ H, GridK g, AosConsts k)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    int x, y, z;
    cell_xyz(i, g, x, y, z);
    float h[3] = {H[3 * i + 0], H[3 * i + 1], H[3 * i + 2]};
    exch_aos_cell(M, i, x, y, z, g, k.ddx, k.ddy, k.ddz, k.cm, h);
    H[3 * i + 0] = h[0];
    H[3 * i + 1] = h[1];
    H[3 * i + 2] = h[2];
}

// ode_functions.cpp:33-67 after the potential: zero, grad, exchange, external
__global__ void k_hfield_aos(const float *__restrict__ M, const float *__restrict__ phi, float *__restrict__ H,
                             GridK g, AosConsts k)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    int x, y, z;
    cell_xyz(i, g, x, y, z);
    float h[3] = {0.f, 0.f, 0.f};
    if (k.demag) grad_aos_cell(phi, i, x, y, z, g, k.dx2, k.dy2, k.dz2, k.cgrad, h);
    if (k.exchange) exch_aos_cell(M, i, x, y, z, g, k.ddx, k.ddy, k.ddz, k.cm, h);
    if (k.external) {
        h[0] = __fadd_rn(h[0], k.hx);
        h[1] = __fadd_rn(h[1], k.hy);
        h[2] = __fadd_rn(h[2], k.hz);
    }
    H[3 * i + 0] = h[0];
    H[3 * i + 1] = h[1];
    H[3 * i + 2] = h[2];
}

// ---- FP64 SoA resident state ----------------------------------------------

// rho = div M; with rhi != NULL also the BF16 hi / lo split of rho in the
// box-major layout of the tensor-core near field ([Z][nby][nbx][8][8], leaf
// side 8; the padding cells beyond the grid stay zero from the plan)
__global__ void k_div_soa(const double *__restrict__ M, float *__restrict__ rho, GridK g, DivScale h,
                          __nv_bfloat16 *__restrict__ rhi, __nv_bfloat16 *__restrict__ rlo, int nbx, int nby)
{
    pdl_begin();
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    int x, y, z;
    cell_xyz(i, g, x, y, z);
    const float v = div_soa_cell(M, i, x, y, z, g, h);
    rho[i] = v;
    if (rhi) {
        const long long j = ntc_index(x, y, z, nbx, nby);
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        rhi[j] = h;
        rlo[j] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

// One RK4 stage (ode_functions.cpp:96-145):
//   stage 0: K  = k1;       Mnext = M + dt/2 k1   (Mst == M)
//   stage 1: K += 2 k2;     Mnext = M + dt/2 k2
//   stage 2: K += 2 k3;     Mnext = M + dt   k3
//   stage 3: K += k4;       M = renorm(M + dt/6 K) (Mnext unused, written in place)
// Empty cells keep M = 0 in every buffer.
__device__ __forceinline__ void rk4_stage_cell(long long i, const float *__restrict__ phi,
                                               const double *__restrict__ Mst, double *__restrict__ M,
                                               double *__restrict__ K, double *__restrict__ Mnext,
                                               const uint8_t *__restrict__ mat, const double *__restrict__ tstate,
                                               const double *__restrict__ htab, double *__restrict__ stats,
                                               const GridK &g, const PhysK &p, int stage)
{
    const long long N = g.N;
    const double t = tstate[TIME_T], dt = tstate[TIME_DT];
    if (!mat[i]) {
        if (stage < 3) {
            Mnext[i] = 0.0;
            Mnext[i + N] = 0.0;
            Mnext[i + 2 * N] = 0.0;
        } else {
            M[i] = 0.0;
            M[i + N] = 0.0;
            M[i + 2 * N] = 0.0;
        }
        return;
    }
    int x, y, z;
    cell_xyz(i, g, x, y, z);
    double ts;
    if (p.ref_stage_time)
        ts = (stage == 0) ? tstate[TIME_TK1] : t;
    else
        ts = t + ((stage == 0) ? 0.0 : (stage == 3 ? dt : 0.5 * dt));
    double he[3];
    hext_at(p, htab, ts, he);
    double h[3];
    field_soa(phi, Mst, i, x, y, z, g, p, he, h);
    const double ms[3] = {Mst[i], Mst[i + N], Mst[i + 2 * N]};
    double k[3];
    llg(ms, h, p, k);
    const double m[3] = {M[i], M[i + N], M[i + 2 * N]};
    if (stage == 0) {
        K[i] = k[0];
        K[i + N] = k[1];
        K[i + 2 * N] = k[2];
    } else {
        const double w = (stage == 3) ? 1.0 : 2.0;
        K[i] += w * k[0];
        K[i + N] += w * k[1];
        K[i + 2 * N] += w * k[2];
    }
    if (stage < 3) {
        const double a = (stage == 2) ? dt : 0.5 * dt;
        Mnext[i] = m[0] + a * k[0];
        Mnext[i + N] = m[1] + a * k[1];
        Mnext[i + 2 * N] = m[2] + a * k[2];
    } else {
        double n0 = m[0] + dt * K[i] * (1 / 6.0);
        double n1 = m[1] + dt * K[i + N] * (1 / 6.0);
        double n2 = m[2] + dt * K[i + 2 * N] * (1 / 6.0);
        const double s = p.Ms / sqrt(n0 * n0 + n1 * n1 + n2 * n2);
        n0 *= s;
        n1 *= s;
        n2 *= s;
        if (!(isfinite(n0) && isfinite(n1) && isfinite(n2))) stats[7] = 1.0;  // benign race: any writer sets 1
        M[i] = n0;
        M[i + N] = n1;
        M[i + 2 * N] = n2;
    }
}


// The stage kernel: thread per cell.  At the last stage (advance != 0) the
// last CTA to finish also advances the time of the state, so that no launch
// of its own follows the step: every CTA has read t and dt before it arrives
// on the counter, and the counter is reset for the next step.
__global__ void __launch_bounds__(TPB) k_rk4_stage(const float *__restrict__ phi, const double *__restrict__ Mst,
                                                   double *__restrict__ M, double *__restrict__ K,
                                                   double *__restrict__ Mnext, const uint8_t *__restrict__ mat,
                                                   double *__restrict__ tstate, const double *__restrict__ htab,
                                                   double *__restrict__ stats, GridK g, PhysK p, int stage,
                                                   int advance)
{
    pdl_begin();
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < g.N) rk4_stage_cell(i, phi, Mst, M, K, Mnext, mat, tstate, htab, stats, g, p, stage);
    if (!advance) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned *ctr = reinterpret_cast<unsigned *>(tstate + TIME_CTR);
        if (atomicAdd(ctr, 1u) == gridDim.x - 1) {
            // t_k1: the time at which the next step's k1 field is taken (the
            // reference evaluates the post-step field at the OLD t,
            // ode_functions.cpp:267)
            tstate[TIME_TK1] = tstate[TIME_T];
            tstate[TIME_T] += tstate[TIME_DT];
            *ctr = 0u;
        }
    }
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// per-block partial sums over material cells of the state M with H(M) built
// from the current phi:  M.H, max|MxH|, sum M, sum |M|, count  (fixed order)
__global__ void __launch_bounds__(TPB) k_stats_part(const float *__restrict__ phi, const double *__restrict__ M,
                                                    const uint8_t *__restrict__ mat, const double *__restrict__ tstate,
                                                    const double *__restrict__ htab, double *__restrict__ part,
                                                    GridK g, PhysK p)
{
    __shared__ double sh[TPB / 32][7];
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    if (i < g.N && mat[i]) {
        int x, y, z;
        cell_xyz(i, g, x, y, z);
        const double t = p.ref_stage_time ? tstate[TIME_TK1] : tstate[TIME_T];
        double he[3], h[3];
        hext_at(p, htab, t, he);
        field_soa(phi, M, i, x, y, z, g, p, he, h);
        const double m[3] = {M[i], M[i + g.N], M[i + 2 * g.N]};
        v[0] = m[0] * h[0] + m[1] * h[1] + m[2] * h[2];
        const double cx = m[1] * h[2] - m[2] * h[1];
        const double cy = m[2] * h[0] - m[0] * h[2];
        const double cz = m[0] * h[1] - m[1] * h[0];
        v[1] = sqrt(cx * cx + cy * cy + cz * cz);
        v[2] = m[0];
        v[3] = m[1];
        v[4] = m[2];
        v[5] = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        v[6] = 1.0;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 7; k++) {
        double r = (k == 1) ? warp_max(v[k]) : warp_sum(v[k]);
        if (lane == 0) sh[w][k] = r;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        const int k = threadIdx.x;
        double r = sh[0][k];
        for (int j = 1; j < TPB / 32; j++) r = (k == 1) ? fmax(r, sh[j][k]) : r + sh[j][k];
        part[(long long)blockIdx.x * 8 + k] = r;
    }
}

__global__ void k_stats_final(const double *__restrict__ part, int nblocks, double *__restrict__ stats)
{
    // one warp, fixed order: lane j sums blocks j, j+32, ...; then a fixed tree
    const int lane = threadIdx.x;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int b = lane; b < nblocks; b += 32)
        for (int k = 0; k < 7; k++) v[k] = (k == 1) ? fmax(v[k], part[(long long)b * 8 + k]) : v[k] + part[(long long)b * 8 + k];
    for (int k = 0; k < 7; k++) {
        double r = (k == 1) ? warp_max(v[k]) : warp_sum(v[k]);
        if (lane == 0) stats[k] = r;
    }
}

AosConsts aos_consts(const mms_ctx *ctx, double cgrad, double t)
{
    AosConsts k;
    const float dx = (float)ctx->g.dx, dy = (float)ctx->g.dy, dz = (float)ctx->g.dz;
    k.dx2 = 2 * dx;
    k.dy2 = 2 * dy;
    k.dz2 = 2 * dz;
    k.ddx = dx * dx;
    k.ddy = dy * dy;
    k.ddz = dz * dz;
    k.cgrad = (float)cgrad;
    const float A = (float)ctx->p.Aexch, mu = (float)ctx->p.mu0, Ms = (float)ctx->p.Ms;
    k.cm = 2 * A / (mu * Ms * Ms);  // vector_functions.cpp:64 in fptype
    k.demag = ctx->p.demag;
    k.exchange = ctx->p.exchange;
    k.external = ctx->p.external;
    k.hx = k.hy = k.hz = 0.f;
    if (ctx->p.external) {
        if (ctx->p.n_hext == 0) {
            // ode_functions.cpp:61 evaluated exactly as the reference does
            const float inv_mu = 1 / mu;
            const double ramp = (t < 1e-9) ? (-0.3 / 1e-9 * t + 0.3) : 0;
            k.hx = (float)(inv_mu * ramp);
        } else {
            const std::vector<double> &tt = ctx->hext_t, &bb = ctx->hext_b;
            const int n = (int)tt.size();
            double B[3];
            if (t <= tt[0]) {
                for (int c = 0; c < 3; c++) B[c] = bb[c];
            } else if (t >= tt[n - 1]) {
                for (int c = 0; c < 3; c++) B[c] = bb[3 * (n - 1) + c];
            } else {
                int j = 0;
                while (j + 1 < n && tt[j + 1] < t) j++;
                const double w = (t - tt[j]) / (tt[j + 1] - tt[j]);
                for (int c = 0; c < 3; c++) B[c] = (1 - w) * bb[3 * j + c] + w * bb[3 * (j + 1) + c];
            }
            k.hx = (float)(B[0] / ctx->p.mu0);
            k.hy = (float)(B[1] / ctx->p.mu0);
            k.hz = (float)(B[2] / ctx->p.mu0);
        }
    }
    return k;
}

}  // namespace

PhysK mms_ctx::pk() const
{
    PhysK k;
    k.Ms = p.Ms;
    k.alpha = p.alpha;
    k.gamma = p.gamma;
    k.mu0 = p.mu0;
    k.cexch = 2 * p.Aexch / (p.mu0 * p.Ms * p.Ms);
    k.cdemag = 1.0 / (4.0 * M_PI);
    k.demag = p.demag;
    k.exchange = p.exchange;
    k.external = p.external;
    k.n_hext = p.external ? (int)hext_t.size() : 0;
    k.ref_stage_time = p.ref_stage_time;
    physk_derive(k, g.dx, g.dy, g.dz);
    return k;
}

int launch_divergence_aos(mms_ctx *ctx, const float *M, float *rho)
{
    fmm_split_written(ctx, nullptr);  // rho changes without its BF16 split
    k_div_aos<<<div_up(ctx->N, TPB), TPB, 0, ctx->stream>>>(M, rho, ctx->gk(), (float)ctx->g.dx, (float)ctx->g.dy,
                                                           (float)ctx->g.dz);
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

int launch_divergence_soa(mms_ctx *ctx, const double *M, float *rho)
{
    void *hi = nullptr, *lo = nullptr;
    int nbx = 0, nby = 0;
    const int split = fmm_split_target(ctx, &hi, &lo, &nbx, &nby);
    MMS_CUDA_TRY(launch_k(k_div_soa, dim3(div_up(ctx->N, TPB)), dim3(TPB), 0, ctx->stream, M, rho, ctx->gk(),
                          div_scale(ctx->g.dx, ctx->g.dy, ctx->g.dz), (__nv_bfloat16 *)(split ? hi : nullptr),
                          (__nv_bfloat16 *)(split ? lo : nullptr), nbx, nby));
    MMS_LAUNCH_CHECK(ctx);
    fmm_split_written(ctx, split ? rho : nullptr);
    return MMS_OK;
}

int launch_gradient_aos(mms_ctx *ctx, const float *phi, double c, float *H)
{
    k_grad_aos<<<div_up(ctx->N, TPB), TPB, 0, ctx->stream>>>(phi, H, ctx->gk(), aos_consts(ctx, c, 0.0));
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

int launch_exchange_aos(mms_ctx *ctx, const float *M, float *H)
{
    k_exch_aos<<<div_up(ctx->N, TPB), TPB, 0, ctx->stream>>>(M, H, ctx->gk(), aos_consts(ctx, 0.0, 0.0));
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

int launch_hfield_aos(mms_ctx *ctx, const float *M, const float *phi, double t, float *H)
{
    k_hfield_aos<<<div_up(ctx->N, TPB), TPB, 0, ctx->stream>>>(M, phi, H, ctx->gk(),
                                                              aos_consts(ctx, 1 / (4.0 * M_PI), t));
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

int launch_rk4_stage(mms_ctx *ctx, int stage, const double *Mst, double *Mnext)
{
    MMS_CUDA_TRY(launch_k(k_rk4_stage, dim3(div_up(ctx->N, TPB)), dim3(TPB), 0, ctx->stream,
                          (const float *)ctx->phi, Mst, ctx->M, ctx->K, Mnext, (const uint8_t *)ctx->mat,
                          ctx->tstate, (const double *)ctx->hext, ctx->stats, ctx->gk(), ctx->pk(), stage,
                          stage == 3 ? 1 : 0));
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

int launch_stats(mms_ctx *ctx)
{
    const unsigned nb = div_up(ctx->N, TPB);
    k_stats_part<<<nb, TPB, 0, ctx->stream>>>(ctx->phi, ctx->M, ctx->mat, ctx->tstate, ctx->hext, ctx->stat_part,
                                              ctx->gk(), ctx->pk());
    MMS_LAUNCH_CHECK(ctx);
    k_stats_final<<<1, 32, 0, ctx->stream>>>(ctx->stat_part, (int)nb, ctx->stats);
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}
