// Exact O(N^2) demag potential: phi_i = sum_{j != i} rho_j dV / |r_i - r_j|
// (the reference's calc_potential_exact, fmm_calc.cu:412-461, and its GPU
// kernel potential_calc.cu:18-116).
//
// B200 design.  On a regular grid 1/|r_i - r_j| depends only on the integer
// offset, so the sum is a 3-D aperiodic convolution.  A table
// G[|dz|][|dy|][|dx|] = dV/|r| is built once per context in FP64 and rounded to
// FP32 (more accurate than a per-pair rsqrt, and it takes the MUFU pipe out of
// the inner loop), with G[0][0][0] = 0 so the self term drops out.  The pair
// loop then is one FP32 FMA per (target, source) pair:
//
//   * one warp owns a 256-cell segment of one target row (y_t, z_t); each lane
//     holds TX = 8 consecutive targets in registers;
//   * source rows sharing the same |y_t - y_s|, |z_t - z_s| share one G row, so
//     they are pre-summed (up to 4 rows) into one shared-memory row: a "group";
//   * per group the lane walks the source row 8 cells at a time with a
//     16-entry sliding window of the mirrored G row in registers: 64 FMAs per
//     two conflict-free LDS.128 (lanes 4-7 of every quarter-warp load the two
//     halves in swapped order, so the 8 lanes of a phase hit 8 distinct
//     16-byte bank groups) and two broadcast LDS.128 of the source row;
//   * the groups of a target row are split over the CTA's warps (split-K);
//     each warp keeps a Kahan-compensated FP32 sum per target across its
//     groups (the long reduction), each group's row product (one FP32 FMA chain
//     per target) being a plain FP32 partial; the warps' partials are combined in FP64 in a fixed
//     order, so results are bitwise reproducible run to run.
#include "mms_internal.cuh"

#include <math.h>

#include <mutex>

namespace {

constexpr int TX = 8;            // targets per lane
constexpr int SEG = 32 * TX;     // targets per warp segment
constexpr int DWARPS = 4;        // warps per CTA splitting the groups of a row
constexpr int MAX_X = 2048;      // row length limit of the shared-memory staging

__global__ void k_build_gtab(float *__restrict__ gtab, GridK g)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    const int ax = (int)(i % g.X);
    const int ay = (int)((i / g.X) % g.Y);
    const int az = (int)(i / ((long long)g.X * g.Y));
    const double rx = ax * g.dx, ry = ay * g.dy, rz = az * g.dz;
    const double r2 = rx * rx + ry * ry + rz * rz;
    gtab[i] = (r2 == 0.0) ? 0.f : (float)(g.dx * g.dy * g.dz / sqrt(r2));
}

struct DirectShape {
    int Xr;      // row length rounded up to 8
    int C;       // centre of the mirrored G row: gm[C + d] = G[|d|]
    int GM;      // mirrored row length (floats), multiple of 4
};

__host__ __device__ inline DirectShape direct_shape(int X)
{
    DirectShape s;
    s.Xr = (X + 7) & ~7;
    s.C = s.Xr + 3;
    s.GM = 2 * s.Xr + 8;
    return s;
}

__global__ void __launch_bounds__(DWARPS * 32) k_direct(const float *__restrict__ rho, const float *__restrict__ gtab,
                                                         float *__restrict__ phi, GridK g)
{
    extern __shared__ __align__(16) float smem[];
    const DirectShape sh = direct_shape(g.X);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *qs = smem + warp * (sh.Xr + sh.GM);   // pre-summed source row
    float *gm = qs + sh.Xr;                      // mirrored G row
    float *red = smem + DWARPS * (sh.Xr + sh.GM);  // [DWARPS][SEG][2] combine area

    const int row = blockIdx.x;                  // target row = zt*Y + yt
    const int yt = row % g.Y, zt = row / g.Y;
    const int seg0 = blockIdx.y * SEG;
    const int x0 = seg0 + lane * TX;             // this lane's first target
    const bool active = x0 < g.X;

    const int nY = max(yt, g.Y - 1 - yt) + 1;    // |dy| = 0 .. nY-1 has a source row
    const int nZ = max(zt, g.Z - 1 - zt) + 1;
    const int ngroups = nY * nZ;
    const long long plane = (long long)g.X * g.Y;

    float s[TX], c[TX];
#pragma unroll
    for (int i = 0; i < TX; i++) s[i] = c[i] = 0.f;

    const bool swap = (lane & 4) != 0;
    for (int grp = warp; grp < ngroups; grp += DWARPS) {
        const int ady = grp / nZ, adz = grp % nZ;
        // source rows of this group: {y_t -/+ |dy|} x {z_t -/+ |dz|}, inside the grid
        const int ya = yt - ady, yb = yt + ady, za = zt - adz, zb = zt + adz;
        const bool hya = ya >= 0, hyb = ady != 0 && yb < g.Y;
        const bool hza = za >= 0, hzb = adz != 0 && zb < g.Z;
        const float *raa = rho + (long long)za * plane + (long long)ya * g.X;
        const float *rab = rho + (long long)za * plane + (long long)yb * g.X;
        const float *rba = rho + (long long)zb * plane + (long long)ya * g.X;
        const float *rbb = rho + (long long)zb * plane + (long long)yb * g.X;
        __syncwarp();
        bool nzl = false;
        for (int k = lane; k < sh.Xr; k += 32) {
            float q = 0.f;
            if (k < g.X) {
                if (hza && hya) q += raa[k];
                if (hza && hyb) q += rab[k];
                if (hzb && hya) q += rba[k];
                if (hzb && hyb) q += rbb[k];
            }
            qs[k] = q;
            nzl |= q != 0.f;
        }
        // a group whose source rows carry no charge adds nothing: skip it
        // (e.g. the empty padding layers of an in-plane magnetised film)
        if (!__any_sync(0xffffffffu, nzl)) continue;
        const float *grow = gtab + ((long long)adz * g.Y + ady) * g.X;
        for (int k = lane; k < sh.GM; k += 32) {
            const int d = abs(k - sh.C);
            gm[k] = (d < g.X) ? grow[d] : 0.f;
        }
        __syncwarp();
        if (active) {
            float acc[TX];
#pragma unroll
            for (int i = 0; i < TX; i++) acc[i] = 0.f;
            // window: win[k] = gm[base + k], base = C - 7 + x0 - xb
            int base = sh.C - 7 + x0;
            float wb[8];  // upper half gm[base+8 .. base+15]
            {
                const float4 u = *reinterpret_cast<const float4 *>(&gm[base + 8]);
                const float4 v = *reinterpret_cast<const float4 *>(&gm[base + 12]);
                wb[0] = u.x; wb[1] = u.y; wb[2] = u.z; wb[3] = u.w;
                wb[4] = v.x; wb[5] = v.y; wb[6] = v.z; wb[7] = v.w;
            }
#pragma unroll 2
            for (int xb = 0; xb < sh.Xr; xb += 8) {
                float wa[8];
                {
                    const float4 f0 = *reinterpret_cast<const float4 *>(&gm[base + (swap ? 4 : 0)]);
                    const float4 f1 = *reinterpret_cast<const float4 *>(&gm[base + (swap ? 0 : 4)]);
                    const float4 lo = swap ? f1 : f0, hi = swap ? f0 : f1;
                    wa[0] = lo.x; wa[1] = lo.y; wa[2] = lo.z; wa[3] = lo.w;
                    wa[4] = hi.x; wa[5] = hi.y; wa[6] = hi.z; wa[7] = hi.w;
                }
                const float4 q0 = *reinterpret_cast<const float4 *>(&qs[xb]);
                const float4 q1 = *reinterpret_cast<const float4 *>(&qs[xb + 4]);
                const float q[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
                for (int j = 0; j < 8; j++)
#pragma unroll
                    for (int i = 0; i < TX; i++) {
                        const int k = 7 + i - j;  // 0..14
                        const float w = (k < 8) ? wa[k] : wb[k - 8];
                        acc[i] = fmaf(q[j], w, acc[i]);
                    }
#pragma unroll
                for (int k = 0; k < 8; k++) wb[k] = wa[k];
                base -= 8;
            }
#pragma unroll
            for (int i = 0; i < TX; i++) {  // Kahan across groups
                const float y = acc[i] - c[i];
                const float t = s[i] + y;
                c[i] = (t - s[i]) - y;
                s[i] = t;
            }
        }
    }
    // combine the DWARPS split-K partials in a fixed order
    __syncthreads();
#pragma unroll
    for (int i = 0; i < TX; i++) {
        red[((warp * SEG) + lane * TX + i) * 2 + 0] = s[i];
        red[((warp * SEG) + lane * TX + i) * 2 + 1] = c[i];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < SEG; t += blockDim.x) {
        const int x = seg0 + t;
        if (x >= g.X) continue;
        double tot = 0.0;
        for (int w = 0; w < DWARPS; w++)
            tot += (double)red[(w * SEG + t) * 2 + 0] - (double)red[(w * SEG + t) * 2 + 1];
        phi[(long long)zt * plane + (long long)yt * g.X + x] = (float)tot;
    }
}

size_t direct_smem_bytes(int X)
{
    const DirectShape sh = direct_shape(X);
    return (size_t)DWARPS * (sh.Xr + sh.GM) * sizeof(float) + (size_t)DWARPS * SEG * 2 * sizeof(float);
}

}  // namespace

int direct_build_table(mms_ctx *ctx)
{
    if (ctx->g.xdim > MAX_X) {
        mms_set_error("direct sum: xdim %d exceeds the supported %d", ctx->g.xdim, MAX_X);
        return MMS_ERR_ARG;
    }
    if (!ctx->gtab) MMS_TRY(ctx_alloc(ctx, &ctx->gtab, (size_t)ctx->N));
    k_build_gtab<<<div_up(ctx->N, 256), 256, 0, ctx->stream>>>(ctx->gtab, ctx->gk());
    MMS_LAUNCH_CHECK(ctx);
    // The attribute is per kernel, shared by every context and by the
    // allocation-free entry point: always raise it to the widest supported
    // row, so that no caller ever lowers it below another caller's need.
    if (direct_smem_bytes(ctx->g.xdim) > 48 * 1024)
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_direct, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)direct_smem_bytes(MAX_X)));
    return MMS_OK;
}

int launch_potential_direct(mms_ctx *ctx, const float *rho, float *phi)
{
    MmsRange nvtx_("mms/direct_potential");
    if (!ctx->gtab) MMS_TRY(direct_build_table(ctx));
    dim3 grid((unsigned)(ctx->g.ydim * ctx->g.zdim), div_up(ctx->g.xdim, SEG));
    k_direct<<<grid, DWARPS * 32, direct_smem_bytes(ctx->g.xdim), ctx->stream>>>(rho, ctx->gtab, phi, ctx->gk());
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the exact potential.
//
// For callers that cannot call cudaMalloc: a host that has handed the device
// memory to its own pool allocator, code that runs while a CUDA graph is being
// captured (where allocation is not permitted), or a latency-critical loop that
// must not take the driver's allocation lock.  The direct sum's only scratch
// is its table G[|dz|][|dy|][|dx|] = dV/|r|; here it lives in a fixed array in
// the library's own device memory (module global), so a call needs nothing but
// the caller's input and output buffers.
//
// Limit: X*Y*Z <= MMS_NOALLOC_MAX_CELLS (1,048,576 cells, a 4 MiB table that
// every GPU which loads the library holds until the process exits) and
// xdim <= 2048.
constexpr long long MMS_NOALLOC_MAX_CELLS = 1LL << 20;
static __device__ __align__(256) float g_noalloc_gtab[MMS_NOALLOC_MAX_CELLS];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
float *g_noalloc_ptr[NOALLOC_MAX_DEVICES];   // device address of g_noalloc_gtab, per device
std::once_flag g_noalloc_once[NOALLOC_MAX_DEVICES];
cudaError_t g_noalloc_setup_err[NOALLOC_MAX_DEVICES];
}  // namespace

extern "C" int mms_potential_direct_noalloc(const float *rho, float *phi, int xdim, int ydim, int zdim, double dx,
                                            double dy, double dz, void *stream)
{
    if (!rho || !phi || xdim < 1 || ydim < 1 || zdim < 1 || !(dx > 0 && dy > 0 && dz > 0)) {
        mms_set_error("mms_potential_direct_noalloc: bad argument");
        return MMS_ERR_ARG;
    }
    const long long N = (long long)xdim * ydim * zdim;
    if (N > MMS_NOALLOC_MAX_CELLS || xdim > MAX_X) {
        mms_set_error("mms_potential_direct_noalloc: %d x %d x %d exceeds the fixed table of %lld cells "
                      "(or xdim > %d)", xdim, ydim, zdim, MMS_NOALLOC_MAX_CELLS, MAX_X);
        return MMS_ERR_ARG;
    }
    int dev = 0;
    MMS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        mms_set_error("mms_potential_direct_noalloc: device %d out of range", dev);
        return MMS_ERR_ARG;
    }
    // An error left pending by the caller's earlier work is not this call's:
    // report it as such instead of blaming the launches below.
    {
        const cudaError_t pend = cudaPeekAtLastError();
        if (pend != cudaSuccess) {
            mms_set_error("mms_potential_direct_noalloc: a CUDA error was pending before the call: %s",
                          cudaGetErrorString(pend));
            return MMS_ERR_CUDA;
        }
    }
    // one-time set-up on this device (the first call, with the device
    // current): the table's device address.  Host threads racing on the
    // first call run it once.
    std::call_once(g_noalloc_once[dev], [dev]() {
        float *p = nullptr;
        g_noalloc_setup_err[dev] = cudaGetSymbolAddress((void **)&p, g_noalloc_gtab);
        if (g_noalloc_setup_err[dev] == cudaSuccess) g_noalloc_ptr[dev] = p;
    });
    if (g_noalloc_setup_err[dev] != cudaSuccess || !g_noalloc_ptr[dev]) {
        mms_set_error("mms_potential_direct_noalloc: cudaGetSymbolAddress: %s",
                      cudaGetErrorString(g_noalloc_setup_err[dev]));
        return MMS_ERR_CUDA;
    }
    // The kernel's shared-memory limit is a per-kernel attribute that a
    // context may also set; set it on every call (host-side, allocates
    // nothing) so that it always covers this call's row length.
    const size_t smem = direct_smem_bytes(xdim);
    if (smem > 48 * 1024)
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_direct, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)direct_smem_bytes(MAX_X)));
    float *gtab = g_noalloc_ptr[dev];
    GridK g;
    g.X = xdim;
    g.Y = ydim;
    g.Z = zdim;
    g.N = N;
    g.dx = dx;
    g.dy = dy;
    g.dz = dz;
    cudaStream_t st = (cudaStream_t)stream;
    // every table entry the sum reads is rewritten here: nothing has to start at zero
    k_build_gtab<<<div_up(N, 256), 256, 0, st>>>(gtab, g);
    MMS_CUDA_TRY(cudaGetLastError());
    dim3 grid((unsigned)(ydim * zdim), div_up(xdim, SEG));
    k_direct<<<grid, DWARPS * 32, smem, st>>>(rho, gtab, phi, g);
    MMS_CUDA_TRY(cudaGetLastError());
    return MMS_OK;
}
