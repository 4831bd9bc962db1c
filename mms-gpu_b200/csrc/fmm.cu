// Spherical-harmonic FMM for the demag potential on a thin film grid.
//
// Replaces the reference's fmm_calc / fmm_bfs tree code (fmm_calc.cu:20-408)
// and its per-box GPU M2P kernel (fmm_kernel.cu:21-155) with a full FMM on the
// same quadtree over (x, y):
//   P2M   leaf multipoles from the cell charges          (k_p2m)
//   M2M   upward pass, level L-1 .. 2                    (k_m2m)
//   M2L   interaction lists of every level >= 2         (k_m2l, one launch)
//   L2L   downward pass, level 3 .. L                    (k_l2l)
//   L2P + P2P  leaf locals at the cells plus the exact near field over the
//         3x3 leaf neighbourhood, all layers             (k_l2p_p2p)
// The interaction list of a box is the reference's: children of the parent's
// neighbours that are not neighbours (Box.cu:171-195), here an implicit set of
// 27 offsets per parity class.  Each box holds all zdim layers; expansion
// centres sit in the middle layer.  The tree is implicit (box index = row-major
// position at its level) and covers any X x Y grid, padded to 2^L leaves.
//
// All translation operators are level independent (lengths in box widths) and
// built once on the host in FP64 (fmm_ops.cpp), stored in FP32.  Expansions
// are FP32 real vectors of the (re, im) pairs for m >= 0, even n + m first;
// M2M, M2L and L2L act on the two parity blocks separately.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "fmm_ops.hpp"
#include "mms_internal.cuh"

namespace {

constexpr int KW = 16;        // k values per warp in k_m2l (4 x float4)
constexpr int M2L_WARPS = 4;  // up to 64 k per parity block

struct FmmDev {
    int P, s, L, nb, NR, NE, C, Z;
    int X, Y;
    float inv_w;              // 1 / leaf width (m): L2P scale
};

}  // namespace

struct FmmPlan {
    FmmDev d{};
    int KPb[2] = {0, 0};      // padded k extent per parity block in k_m2l
    std::vector<long long> lev_off;  // first box of each level in Mall / Lall
    long long nbox_total = 0;
    int n_m2l_items = 0;
    // device
    float *Wt = nullptr;      // [C][NR]  P2M weights (dV folded in)
    float *Vt = nullptr;      // [NR][C]  L2P weights (1/w folded in)
    float *Tm2m = nullptr;    // [4][NR(j)][NR(k)]
    float *Tl2l = nullptr;    // [4][NR(j)][NR(k)]
    float *Tm2l = nullptr;    // [49][2][NBmax(j)][KP(k)] parity blocks, k padded
    float *Gn = nullptr;      // [Z][2s][2s] near-field dV/|r|
    float *Mall = nullptr;    // [boxes of all levels][NR]
    float *Lall = nullptr;
    int4 *m2l_items = nullptr;  // {level, parity, first target, 0}
    long long *lev_dev = nullptr;  // device copy of lev_off
    size_t bytes = 0;
    // algorithmic work per evaluation (for the roofline)
    double flops = 0, bytes_min = 0;
    long long p2p_pairs = 0, m2l_pairs = 0;
};

namespace {

// ---- P2M: leaf multipoles.  CTA per leaf box, thread per coefficient.
__global__ void k_p2m(const float *__restrict__ rho, const float *__restrict__ Wt, float *__restrict__ Mleaf,
                      FmmDev f)
{
    extern __shared__ float q[];  // C charges of the box (z, y, x order)
    const int box = blockIdx.x;
    const int bx = box % f.nb, by = box / f.nb;
    const int s = f.s;
    for (int c = threadIdx.x; c < f.C; c += blockDim.x) {
        const int x = bx * s + c % s, y = by * s + (c / s) % s, z = c / (s * s);
        q[c] = (x < f.X && y < f.Y) ? rho[((long long)z * f.Y + y) * f.X + x] : 0.f;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < f.NR; k += blockDim.x) {
        float acc = 0.f;
        for (int c = 0; c < f.C; c++) acc = fmaf(Wt[(long long)c * f.NR + k], q[c], acc);
        Mleaf[(long long)box * f.NR + k] = acc;
    }
}

// ---- M2M: parent level l from children at l+1.  CTA per parent, thread per k.
__global__ void k_m2m(float *__restrict__ Mall, const float *__restrict__ Tm2m, long long off_p, long long off_c,
                      int np, FmmDev f)
{
    const int box = blockIdx.x;
    const int bx = box % np, by = box / np, nc = 2 * np;
    const int k = threadIdx.x;
    if (k >= f.NR) return;
    const int j0 = (k < f.NE) ? 0 : f.NE, j1 = (k < f.NE) ? f.NE : f.NR;
    float acc = 0.f;
    for (int c = 0; c < 4; c++) {
        const int cx = 2 * bx + (c & 1), cy = 2 * by + (c >> 1);
        const float *Mc = Mall + (off_c + (long long)cy * nc + cx) * f.NR;
        const float *T = Tm2m + (long long)c * f.NR * f.NR;
        for (int j = j0; j < j1; j++) acc = fmaf(T[(long long)j * f.NR + k], Mc[j], acc);
    }
    Mall[(off_p + box) * f.NR + k] = acc;
}

// ---- M2L: all levels >= 2 in one launch.
// CTA = 32 targets of one (level, parity class) x one parity block of k;
// lane <-> target, warp <-> 16 consecutive k.  The 27 offsets of the class are
// walked in order; each offset's operator block is staged in shared memory and
// read as warp-uniform float4 broadcasts, each lane streams its own source
// multipole from global (L1).  Results overwrite Lall (the downward pass adds
// the parents' contributions afterwards).
__global__ void __launch_bounds__(32 * M2L_WARPS) k_m2l(const float *__restrict__ Mall, float *__restrict__ Lall,
                                                        const float *__restrict__ Tm2l, const int4 *__restrict__ items,
                                                        const long long *__restrict__ lev_off, FmmDev f, int KP0,
                                                        int KP1, int NBmax)
{
    extern __shared__ __align__(16) float Ts[];  // [NBmax][KP]
    const int4 it = items[blockIdx.x];
    const int lev = it.x, px = it.y & 1, py = it.y >> 1;
    const int blk = blockIdx.y;
    const int KP = blk ? KP1 : KP0;
    const int NB = blk ? (f.NR - f.NE) : f.NE;
    const int boff = blk ? f.NE : 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = 1 << lev, nh = n >> 1;
    const int ti = it.z + lane;
    const bool tvalid = ti < nh * nh;
    const int tx = 2 * (ti % nh) + px, ty = 2 * (ti / nh) + py;
    const long long off = lev_off[lev];
    const int k0 = warp * KW;
    const bool wactive = k0 < NB;

    float acc[KW];
#pragma unroll
    for (int i = 0; i < KW; i++) acc[i] = 0.f;

    for (int oy = py - 3; oy <= py + 2; oy++)
        for (int ox = px - 3; ox <= px + 2; ox++) {
            if (max(abs(ox), abs(oy)) < 2) continue;
            const int o = (oy + 3) * 7 + (ox + 3);
            const float *Tg = Tm2l + ((long long)o * 2 + blk) * NBmax * max(KP0, KP1);
            __syncthreads();
            for (int i = threadIdx.x * 4; i < NB * KP; i += blockDim.x * 4)
                *reinterpret_cast<float4 *>(&Ts[i]) = *reinterpret_cast<const float4 *>(&Tg[i]);
            __syncthreads();
            const int sx = tx - ox, sy = ty - oy;
            if (!(wactive && tvalid && sx >= 0 && sy >= 0 && sx < n && sy < n)) continue;
            const float *Ms = Mall + (off + (long long)sy * n + sx) * f.NR + boff;
            for (int j = 0; j < NB; j++) {
                const float m = __ldg(&Ms[j]);
                const float4 *tr = reinterpret_cast<const float4 *>(&Ts[j * KP + k0]);
#pragma unroll
                for (int v = 0; v < KW / 4; v++) {
                    const float4 t = tr[v];
                    acc[4 * v + 0] = fmaf(t.x, m, acc[4 * v + 0]);
                    acc[4 * v + 1] = fmaf(t.y, m, acc[4 * v + 1]);
                    acc[4 * v + 2] = fmaf(t.z, m, acc[4 * v + 2]);
                    acc[4 * v + 3] = fmaf(t.w, m, acc[4 * v + 3]);
                }
            }
        }
    if (!(wactive && tvalid)) return;
    float *Lt = Lall + (off + (long long)ty * n + tx) * f.NR + boff;
#pragma unroll
    for (int i = 0; i < KW; i++)
        if (k0 + i < NB) Lt[k0 + i] = acc[i];
}

// ---- L2L: child level l += shifted parent locals.  CTA per child, thread per k.
__global__ void k_l2l(float *__restrict__ Lall, const float *__restrict__ Tl2l, long long off_p, long long off_c,
                      int nc, FmmDev f)
{
    const int box = blockIdx.x;
    const int cx = box % nc, cy = box / nc;
    const int k = threadIdx.x;
    if (k >= f.NR) return;
    const int c = (cx & 1) | ((cy & 1) << 1);
    const int np = nc >> 1;
    const float *Lp = Lall + (off_p + (long long)(cy >> 1) * np + (cx >> 1)) * f.NR;
    const float *T = Tl2l + (long long)c * f.NR * f.NR;
    const int j0 = (k < f.NE) ? 0 : f.NE, j1 = (k < f.NE) ? f.NE : f.NR;
    float acc = 0.f;
    for (int j = j0; j < j1; j++) acc = fmaf(T[(long long)j * f.NR + k], Lp[j], acc);
    Lall[(off_c + box) * f.NR + k] += acc;
}

// ---- L2P + P2P: CTA per leaf box, thread per target cell.
__global__ void k_l2p_p2p(const float *__restrict__ rho, const float *__restrict__ Lleaf,
                          const float *__restrict__ Vt, const float *__restrict__ Gn, float *__restrict__ phi,
                          FmmDev f, int far)
{
    extern __shared__ float sm[];
    const int s = f.s, S3 = 3 * s, Z = f.Z;
    float *qn = sm;                         // [Z][3s][3s] neighbourhood charges
    float *g = qn + Z * S3 * S3;            // [Z][2s][2s]
    float *Lb = g + Z * 4 * s * s;          // [NR]
    const int box = blockIdx.x;
    const int bx = box % f.nb, by = box / f.nb;
    const int x0 = bx * s - s, y0 = by * s - s;
    for (int i = threadIdx.x; i < Z * S3 * S3; i += blockDim.x) {
        const int xx = x0 + i % S3, yy = y0 + (i / S3) % S3, zz = i / (S3 * S3);
        qn[i] = (xx >= 0 && yy >= 0 && xx < f.X && yy < f.Y) ? rho[((long long)zz * f.Y + yy) * f.X + xx] : 0.f;
    }
    for (int i = threadIdx.x; i < Z * 4 * s * s; i += blockDim.x) g[i] = Gn[i];
    if (far)
        for (int i = threadIdx.x; i < f.NR; i += blockDim.x) Lb[i] = Lleaf[(long long)box * f.NR + i];
    __syncthreads();
    const int c = threadIdx.x;
    if (c >= f.C) return;
    const int lx = c % s, ly = (c / s) % s, lz = c / (s * s);
    const int x = bx * s + lx, y = by * s + ly;
    if (x >= f.X || y >= f.Y) return;
    float farv = 0.f;
    if (far)
        for (int k = 0; k < f.NR; k++) farv = fmaf(Vt[(long long)k * f.C + c], Lb[k], farv);
    // near field: sources at (sx, sy) in [0, 3s) of the neighbourhood
    const int tx = lx + s, ty = ly + s;
    float near = 0.f;
    for (int sz = 0; sz < Z; sz++) {
        const int dz = abs(sz - lz);
        for (int sy = 0; sy < S3; sy++) {
            const int dy = abs(sy - ty);
            if (dy >= 2 * s) continue;
            const float *grow = g + (dz * 2 * s + dy) * 2 * s;
            const float *qrow = qn + (sz * S3 + sy) * S3;
            for (int sx = 0; sx < S3; sx++) {
                const int dx = abs(sx - tx);
                if (dx < 2 * s) near = fmaf(qrow[sx], grow[dx], near);
            }
        }
    }
    phi[((long long)lz * f.Y + y) * f.X + x] = farv * f.inv_w + near;
}

__global__ void k_build_gn(float *__restrict__ Gn, int Z, int s, double dx, double dy, double dz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n2 = 2 * s;
    if (i >= Z * n2 * n2) return;
    const int ax = i % n2, ay = (i / n2) % n2, az = i / (n2 * n2);
    const double rx = ax * dx, ry = ay * dy, rz = az * dz;
    const double r2 = rx * rx + ry * ry + rz * rz;
    Gn[i] = (r2 == 0.0) ? 0.f : (float)(dx * dy * dz / sqrt(r2));
}

template <class T>
int upload(mms_ctx *ctx, FmmPlan *pl, T **dst, const std::vector<T> &v)
{
    const size_t bytes = std::max<size_t>(v.size() * sizeof(T), 16);
    if (cudaMalloc((void **)dst, bytes) != cudaSuccess) {
        *dst = nullptr;
        mms_set_error("FMM plan: cudaMalloc(%zu) failed", bytes);
        return MMS_ERR_NOMEM;
    }
    pl->bytes += bytes;
    if (!v.empty()) MMS_CUDA_TRY(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice,
                                                 ctx->stream));
    return MMS_OK;
}

}  // namespace

int fmm_default_leaf(int P, int X, int Y);

int fmm_plan_create(mms_ctx *ctx)
{
    const int P = ctx->s.fmm_order;
    if (P < 1 || P > 12) {
        mms_set_error("FMM order P must be 1..12 (got %d)", P);
        return MMS_ERR_ARG;
    }
    int s = ctx->s.fmm_leaf;
    if (s == 0) s = fmm_default_leaf(P, ctx->g.xdim, ctx->g.ydim);
    if (s < 1 || s > 16) {
        mms_set_error("FMM leaf side must be 1..16 cells (got %d)", s);
        return MMS_ERR_ARG;
    }
    const int Z = ctx->g.zdim;
    if ((long long)s * s * Z > 1024) {
        mms_set_error("FMM leaf of %d x %d x %d cells exceeds 1024 cells", s, s, Z);
        return MMS_ERR_ARG;
    }
    FmmPlan *pl = new FmmPlan();
    ctx->fmm = pl;
    FmmDev &f = pl->d;
    f.P = P;
    f.s = s;
    f.Z = Z;
    f.X = ctx->g.xdim;
    f.Y = ctx->g.ydim;
    f.C = s * s * Z;
    const int nleaf = std::max(1, (std::max(f.X, f.Y) + s - 1) / s);
    f.L = 0;
    while ((1 << f.L) < nleaf) f.L++;
    f.nb = 1 << f.L;
    fmmops::Layout lay(P);
    f.NR = lay.NR;
    f.NE = lay.NE;
    const double w = s * ctx->g.dx;  // leaf width (x), the length unit of the leaf level
    f.inv_w = (float)(1.0 / w);
    const double ay = ctx->g.dy / ctx->g.dx, az = ctx->g.dz / ctx->g.dx;
    const double dV = ctx->g.dx * ctx->g.dy * ctx->g.dz;

    // P2M / L2P weights over the leaf cells
    std::vector<double> rx(f.C), ry(f.C), rz(f.C), W, V;
    const double zc = (Z - 1) / 2.0;
    for (int c = 0; c < f.C; c++) {
        const int lx = c % s, ly = (c / s) % s, lz = c / (s * s);
        rx[c] = (lx - (s - 1) / 2.0) / s;
        ry[c] = (ly - (s - 1) / 2.0) / s * ay;
        rz[c] = (lz - zc) / s * az;
    }
    fmmops::p2m_l2p(lay, rx, ry, rz, W, V);
    std::vector<float> Wt((size_t)f.C * f.NR), Vt((size_t)f.NR * f.C);
    for (int k = 0; k < f.NR; k++)
        for (int c = 0; c < f.C; c++) {
            Wt[(size_t)c * f.NR + k] = (float)(W[(size_t)k * f.C + c] * dV);
            Vt[(size_t)k * f.C + c] = (float)V[(size_t)c * f.NR + k];
        }
    // M2M / L2L, transposed to [j][k]
    const int NR = f.NR;
    std::vector<float> Tm2m((size_t)4 * NR * NR), Tl2l((size_t)4 * NR * NR);
    for (int c = 0; c < 4; c++) {
        const double dxv = ((c & 1) - 0.5) / 2, dyv = ((c >> 1) - 0.5) / 2 * ay;
        const std::vector<double> a = fmmops::m2m(lay, dxv, dyv, 0.0);
        const std::vector<double> b = fmmops::l2l(lay, -dxv, -dyv, 0.0);
        for (int k = 0; k < NR; k++)
            for (int j = 0; j < NR; j++) {
                Tm2m[((size_t)c * NR + j) * NR + k] = (float)a[(size_t)k * NR + j];
                Tl2l[((size_t)c * NR + j) * NR + k] = (float)b[(size_t)k * NR + j];
            }
    }
    // M2L parity blocks, [o][blk][j][k padded]
    const int NB0 = f.NE, NB1 = NR - f.NE, NBmax = std::max(NB0, NB1);
    pl->KPb[0] = ((NB0 + KW - 1) / KW) * KW;
    pl->KPb[1] = ((NB1 + KW - 1) / KW) * KW;
    const int KPmax = std::max(pl->KPb[0], pl->KPb[1]);
    if (KPmax > KW * M2L_WARPS) {
        delete pl;
        ctx->fmm = nullptr;
        mms_set_error("FMM order %d too high for the M2L kernel (block of %d > %d)", P, NBmax, KW * M2L_WARPS);
        return MMS_ERR_ARG;
    }
    std::vector<float> Tm2l((size_t)49 * 2 * NBmax * KPmax, 0.f);
    double max_offblock = 0.0;
    for (int oy = -3; oy <= 3; oy++)
        for (int ox = -3; ox <= 3; ox++) {
            if (std::max(abs(ox), abs(oy)) < 2) continue;
            const int o = (oy + 3) * 7 + (ox + 3);
            const std::vector<double> T = fmmops::m2l(lay, -ox, -oy * ay, 0.0);  // source - target
            for (int blk = 0; blk < 2; blk++) {
                const int b0 = blk ? f.NE : 0, NB = blk ? NB1 : NB0, KP = pl->KPb[blk];
                float *dst = &Tm2l[((size_t)o * 2 + blk) * NBmax * KPmax];
                for (int j = 0; j < NB; j++)
                    for (int k = 0; k < NB; k++) dst[(size_t)j * KP + k] = (float)T[(size_t)(b0 + k) * NR + (b0 + j)];
            }
            for (int k = 0; k < NR; k++)
                for (int j = 0; j < NR; j++)
                    if ((k < f.NE) != (j < f.NE)) max_offblock = std::max(max_offblock, fabs(T[(size_t)k * NR + j]));
        }
    if (max_offblock > 1e-9) {
        delete pl;
        ctx->fmm = nullptr;
        mms_set_error("FMM operator parity blocks are not decoupled (%g)", max_offblock);
        return MMS_ERR_ARG;
    }
    // levels, work items
    pl->lev_off.assign(f.L + 2, 0);
    long long tot = 0;
    for (int l = 0; l <= f.L; l++) {
        pl->lev_off[l] = tot;
        tot += (long long)(1 << l) * (1 << l);
    }
    pl->lev_off[f.L + 1] = tot;
    pl->nbox_total = tot;
    std::vector<int4> items;
    for (int l = 2; l <= f.L; l++) {
        const int nh = (1 << l) / 2;
        for (int par = 0; par < 4; par++)
            for (int t0 = 0; t0 < nh * nh; t0 += 32) items.push_back(make_int4(l, par, t0, 0));
    }
    pl->n_m2l_items = (int)items.size();

    int st = MMS_OK;
    if (!st) st = upload(ctx, pl, &pl->Wt, Wt);
    if (!st) st = upload(ctx, pl, &pl->Vt, Vt);
    if (!st) st = upload(ctx, pl, &pl->Tm2m, Tm2m);
    if (!st) st = upload(ctx, pl, &pl->Tl2l, Tl2l);
    if (!st) st = upload(ctx, pl, &pl->Tm2l, Tm2l);
    if (!st) st = upload(ctx, pl, &pl->m2l_items, items);
    long long *lev_dev = nullptr;
    if (!st) st = upload(ctx, pl, &lev_dev, pl->lev_off);
    if (st) {
        if (lev_dev) cudaFree(lev_dev);
        fmm_plan_destroy(ctx);
        return st;
    }
    {
        const size_t ncoef = (size_t)tot * NR;
        if (cudaMalloc((void **)&pl->Mall, ncoef * sizeof(float)) != cudaSuccess ||
            cudaMalloc((void **)&pl->Lall, ncoef * sizeof(float)) != cudaSuccess ||
            cudaMalloc((void **)&pl->Gn, (size_t)Z * 4 * s * s * sizeof(float)) != cudaSuccess) {
            cudaFree(lev_dev);
            fmm_plan_destroy(ctx);
            mms_set_error("FMM plan: device allocation failed");
            return MMS_ERR_NOMEM;
        }
        pl->bytes += 2 * ncoef * sizeof(float) + (size_t)Z * 4 * s * s * sizeof(float);
        MMS_CUDA_TRY(cudaMemsetAsync(pl->Mall, 0, ncoef * sizeof(float), ctx->stream));
        MMS_CUDA_TRY(cudaMemsetAsync(pl->Lall, 0, ncoef * sizeof(float), ctx->stream));
    }
    k_build_gn<<<div_up((long long)Z * 4 * s * s, 128), 128, 0, ctx->stream>>>(pl->Gn, Z, s, ctx->g.dx, ctx->g.dy,
                                                                            ctx->g.dz);
    MMS_LAUNCH_CHECK(ctx);
    pl->lev_dev = lev_dev;
    const size_t m2l_smem = (size_t)NBmax * KPmax * sizeof(float);
    if (m2l_smem > 48 * 1024)
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_m2l, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m2l_smem));

    // algorithmic work of one evaluation (FMA = 2 flops)
    const long long nleafb = (long long)f.nb * f.nb;
    double fl = 0;
    fl += 2.0 * nleafb * f.C * NR;  // P2M
    fl += 2.0 * nleafb * f.C * NR;  // L2P
    long long m2l_pairs = 0;
    for (int l = 2; l <= f.L; l++) {
        const int n = 1 << l;
        for (int by = 0; by < n; by++)
            for (int bx = 0; bx < n; bx++)
                for (int oy = (by & 1) - 3; oy <= (by & 1) + 2; oy++)
                    for (int ox = (bx & 1) - 3; ox <= (bx & 1) + 2; ox++)
                        if (std::max(abs(ox), abs(oy)) >= 2 && bx - ox >= 0 && bx - ox < n && by - oy >= 0 &&
                            by - oy < n)
                            m2l_pairs++;
    }
    const double blk2 = (double)NB0 * NB0 + (double)NB1 * NB1;
    fl += 2.0 * m2l_pairs * blk2;
    for (int l = 2; l < f.L; l++) fl += 2.0 * 4.0 * (double)(1 << l) * (1 << l) * blk2;           // M2M
    for (int l = 3; l <= f.L; l++) fl += 2.0 * (double)(1 << l) * (1 << l) * blk2;               // L2L
    // P2P: each target cell against every cell of its 3x3 leaf neighbourhood inside the grid
    long long pairs = 0;
    for (int by = 0; by < f.nb; by++)
        for (int bx = 0; bx < f.nb; bx++) {
            const int tx = std::max(0, std::min(f.X, (bx + 1) * s) - bx * s);
            const int ty = std::max(0, std::min(f.Y, (by + 1) * s) - by * s);
            if (!tx || !ty) continue;
            const int sx = std::max(0, std::min(f.X, (bx + 2) * s) - std::max(0, (bx - 1) * s));
            const int sy = std::max(0, std::min(f.Y, (by + 2) * s) - std::max(0, (by - 1) * s));
            pairs += (long long)tx * ty * Z * sx * sy * Z;
        }
    fl += 2.0 * pairs;
    pl->flops = fl;
    pl->p2p_pairs = pairs;
    pl->m2l_pairs = m2l_pairs;
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return MMS_OK;
}

void fmm_plan_destroy(mms_ctx *ctx)
{
    FmmPlan *pl = ctx->fmm;
    if (!pl) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    void *b[] = {pl->Wt, pl->Vt, pl->Tm2m, pl->Tl2l, pl->Tm2l, pl->Gn, pl->Mall, pl->Lall, pl->m2l_items,
                 pl->lev_dev};
    for (void *p : b)
        if (p) cudaFree(p);
    delete pl;
    ctx->fmm = nullptr;
}

size_t fmm_plan_bytes(const mms_ctx *ctx) { return ctx->fmm ? ctx->fmm->bytes : 0; }

int launch_potential_fmm(mms_ctx *ctx, const float *rho, float *phi)
{
    FmmPlan *pl = ctx->fmm;
    if (!pl) {
        mms_set_error("FMM plan missing");
        return MMS_ERR_ARG;
    }
    const FmmDev &f = pl->d;
    const int far = f.L >= 2;
    if (far) {
        const long long leaf_off = pl->lev_off[f.L];
        k_p2m<<<f.nb * f.nb, 128, f.C * sizeof(float), ctx->stream>>>(rho, pl->Wt, pl->Mall + leaf_off * f.NR, f);
        MMS_LAUNCH_CHECK(ctx);
        for (int l = f.L - 1; l >= 2; l--) {
            const int np = 1 << l;
            k_m2m<<<np * np, ((f.NR + 31) / 32) * 32, 0, ctx->stream>>>(pl->Mall, pl->Tm2m, pl->lev_off[l],
                                                                       pl->lev_off[l + 1], np, f);
            MMS_LAUNCH_CHECK(ctx);
        }
        const int NBmax = std::max(f.NE, f.NR - f.NE);
        const int KPmax = std::max(pl->KPb[0], pl->KPb[1]);
        dim3 grid(pl->n_m2l_items, 2);
        k_m2l<<<grid, 32 * M2L_WARPS, (size_t)NBmax * KPmax * sizeof(float), ctx->stream>>>(
            pl->Mall, pl->Lall, pl->Tm2l, pl->m2l_items, pl->lev_dev, f, pl->KPb[0], pl->KPb[1], NBmax);
        MMS_LAUNCH_CHECK(ctx);
        for (int l = 3; l <= f.L; l++) {
            const int nc = 1 << l;
            k_l2l<<<nc * nc, ((f.NR + 31) / 32) * 32, 0, ctx->stream>>>(pl->Lall, pl->Tl2l, pl->lev_off[l - 1],
                                                                       pl->lev_off[l], nc, f);
            MMS_LAUNCH_CHECK(ctx);
        }
    }
    const size_t smem = ((size_t)f.Z * 9 * f.s * f.s + (size_t)f.Z * 4 * f.s * f.s + f.NR) * sizeof(float);
    const int threads = ((f.C + 31) / 32) * 32;
    k_l2p_p2p<<<f.nb * f.nb, threads, smem, ctx->stream>>>(rho, pl->Lall + pl->lev_off[f.L] * f.NR, pl->Vt, pl->Gn,
                                                          phi, f, far);
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

int fmm_default_leaf(int P, int X, int Y)
{
    // near field vs far field balance: higher orders favour bigger leaves
    (void)X;
    (void)Y;
    return P <= 4 ? 4 : 8;
}

extern "C" int mms_fmm_info(const mms_ctx *ctx, int *levels, int *leaf, int *order, double *flops,
                            long long *p2p_pairs, long long *m2l_pairs)
{
    if (!ctx || !ctx->fmm) {
        mms_set_error("context has no FMM plan");
        return MMS_ERR_ARG;
    }
    const FmmPlan *pl = ctx->fmm;
    if (levels) *levels = pl->d.L;
    if (leaf) *leaf = pl->d.s;
    if (order) *order = pl->d.P;
    if (flops) *flops = pl->flops;
    if (p2p_pairs) *p2p_pairs = pl->p2p_pairs;
    if (m2l_pairs) *m2l_pairs = pl->m2l_pairs;
    return MMS_OK;
}
