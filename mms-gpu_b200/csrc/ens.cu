// Batched ensemble: many independent simulations of uneven grid size advance
// together, one kernel launch per stage for the whole ensemble.
//
// Layout: the instances' cells are concatenated (instance order, each in the
// reference's z*Y*X + y*X + x order); the FP64 state is SoA planes over all
// cells; an offset table gives each instance's first cell and dims, and a tile
// table cuts every instance into <= 256-cell tiles that never cross an
// instance, so the per-cell kernels (divergence, field + LLG + RK4 stage) are
// one launch over all tiles.  The exact potential is one launch over
// (instance, block of target rows) items: several short target rows share a
// warp, each lane keeps 8 consecutive targets in registers and slides a window
// over a mirrored table G[|dz|][|dy|][.] = dV/|r| kept in shared memory, with
// the source row broadcast from shared memory (one FMA per pair); FP32 sums
// over groups of KG source rows are combined with Kahan compensation.
//
// Per-step physics is the single-grid path's (stencil_dev.cuh); each instance
// has its own constant external field.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "mms_internal.cuh"
#include "stencil_dev.cuh"

namespace {

using namespace mmsdev;

constexpr int ETPB = 256;       // cells per tile / threads per block in the cell kernels
constexpr int EW_MAX = 16;      // warps per CTA in the batched direct kernel (runtime, autotuned)
constexpr int ETX = 8;          // targets per lane
constexpr int QROWS_MAX = 32;   // source rows staged per batch (runtime, autotuned)
constexpr int KG = 4;           // source rows summed in FP32 between compensated (Kahan) adds

struct EnsInst {
    int X, Y, Z;
    int pad;
    long long off;              // first cell
    double hx, hy, hz;          // external field (A/m)
};

struct EnsTile {
    int inst;
    int start;                  // first cell within the instance
    int count;
    int pad;
};

struct EnsDirectItem {
    int inst;
    int row0;                   // first target row (z*Y + y) of the CTA
    int rpw;                    // target rows per warp
    int lpr;                    // lanes per target row (Xr / 8)
};

struct TableShape {
    int Xm, Ym, Z;              // table extents (max over instances, Xm multiple of 8)
    int C;                      // centre of a mirrored row
    int pitch;                  // floats per mirrored row
};

__global__ void k_ens_table(float *__restrict__ gm, TableShape t, double dx, double dy, double dz)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long n = (long long)t.Z * t.Ym * t.pitch;
    if (i >= n) return;
    const int k = (int)(i % t.pitch);
    const int ady = (int)((i / t.pitch) % t.Ym), adz = (int)(i / ((long long)t.pitch * t.Ym));
    const int d = abs(k - t.C);
    float v = 0.f;
    if (d < t.Xm) {
        const double rx = d * dx, ry = ady * dy, rz = adz * dz;
        const double r2 = rx * rx + ry * ry + rz * rz;
        v = (r2 == 0.0) ? 0.f : (float)(dx * dy * dz / sqrt(r2));
    }
    gm[i] = v;
}

__device__ __forceinline__ GridK inst_grid(const EnsInst &in, long long Ntot, double dx, double dy, double dz)
{
    GridK g;
    g.X = in.X;
    g.Y = in.Y;
    g.Z = in.Z;
    g.N = Ntot;  // plane stride of the SoA state
    g.dx = dx;
    g.dy = dy;
    g.dz = dz;
    return g;
}

// Persistent cell kernels: an occupancy-sized grid walks the tile table
// (tile = blockIdx.x, blockIdx.x + gridDim.x, ...).
__global__ void __launch_bounds__(ETPB) k_ens_div(const double *__restrict__ M, float *__restrict__ rho,
                                                  const EnsInst *__restrict__ inst, const EnsTile *__restrict__ tiles,
                                                  int ntiles, long long Ntot, double dx, double dy, double dz,
                                                  DivScale h)
{
  for (int tix = blockIdx.x; tix < ntiles; tix += gridDim.x) {
    const EnsTile tl = tiles[tix];
    if ((int)threadIdx.x >= tl.count) continue;
    const EnsInst in = inst[tl.inst];
    const long long i = tl.start + threadIdx.x;
    const long long plane = (long long)in.X * in.Y;
    const int x = (int)(i % in.X), y = (int)((i / in.X) % in.Y), z = (int)(i / plane);
    // the single-grid expression on the instance's planes
    rho[in.off + i] = div_soa_cell(M + in.off, i, x, y, z, inst_grid(in, Ntot, dx, dy, dz), h);
  }
}

// one RK4 stage for every instance (see k_rk4_stage in stencil.cu)
__global__ void __launch_bounds__(ETPB) k_ens_stage(const float *__restrict__ phi, const double *__restrict__ Mst,
                                                    double *__restrict__ M, double *__restrict__ K,
                                                    double *__restrict__ Mnext, const uint8_t *__restrict__ mat,
                                                    const double *__restrict__ tstate, const EnsInst *__restrict__ inst,
                                                    const EnsTile *__restrict__ tiles, double *__restrict__ flag,
                                                    int ntiles, long long Ntot, double dx, double dy, double dz,
                                                    PhysK p, int stage)
{
  for (int tix = blockIdx.x; tix < ntiles; tix += gridDim.x) {
    const EnsTile tl = tiles[tix];
    if ((int)threadIdx.x >= tl.count) continue;
    const EnsInst in = inst[tl.inst];
    const long long i = tl.start + threadIdx.x;   // within the instance
    const long long gi = in.off + i;              // global cell
    const long long N = Ntot;
    if (!mat[gi]) {
        double *dst = (stage < 3) ? Mnext : M;
        dst[gi] = 0.0;
        dst[gi + N] = 0.0;
        dst[gi + 2 * N] = 0.0;
        continue;
    }
    const double dt = tstate[TIME_DT];
    const GridK g = inst_grid(in, Ntot, dx, dy, dz);
    int x, y, z;
    const long long plane = (long long)in.X * in.Y;
    x = (int)(i % in.X);
    y = (int)((i / in.X) % in.Y);
    z = (int)(i / plane);
    const double he[3] = {p.external ? in.hx : 0.0, p.external ? in.hy : 0.0, p.external ? in.hz : 0.0};
    double h[3];
    field_soa(phi + in.off, Mst + in.off, i, x, y, z, g, p, he, h);
    const double ms[3] = {Mst[gi], Mst[gi + N], Mst[gi + 2 * N]};
    double k[3];
    llg(ms, h, p, k);
    const double m[3] = {M[gi], M[gi + N], M[gi + 2 * N]};
    if (stage == 0) {
        K[gi] = k[0];
        K[gi + N] = k[1];
        K[gi + 2 * N] = k[2];
    } else {
        const double w = (stage == 3) ? 1.0 : 2.0;
        K[gi] += w * k[0];
        K[gi + N] += w * k[1];
        K[gi + 2 * N] += w * k[2];
    }
    if (stage < 3) {
        const double a = (stage == 2) ? dt : 0.5 * dt;
        Mnext[gi] = m[0] + a * k[0];
        Mnext[gi + N] = m[1] + a * k[1];
        Mnext[gi + 2 * N] = m[2] + a * k[2];
    } else {
        double n0 = m[0] + dt * K[gi] * (1 / 6.0);
        double n1 = m[1] + dt * K[gi + N] * (1 / 6.0);
        double n2 = m[2] + dt * K[gi + 2 * N] * (1 / 6.0);
        const double s = p.Ms / sqrt(n0 * n0 + n1 * n1 + n2 * n2);
        n0 *= s;
        n1 *= s;
        n2 *= s;
        if (!(isfinite(n0) && isfinite(n1) && isfinite(n2))) flag[0] = 1.0;
        M[gi] = n0;
        M[gi + N] = n1;
        M[gi + 2 * N] = n2;
    }
  }
}

__global__ void k_ens_advance(double *tstate)
{
    tstate[TIME_TK1] = tstate[TIME_T];
    tstate[TIME_T] += tstate[TIME_DT];
}

__global__ void k_ens_set_dt(double *tstate, double dt) { tstate[TIME_DT] = dt; }

// batched exact potential (see the file comment).  Persistent: an
// occupancy-sized grid; each CTA stages the mirrored table once, then takes
// work items (instance, block of target rows) from a shared counter in the
// order of the item table (costliest first).  blockDim.x / 32 warps per CTA
// and `qrows` staged source rows per batch are the autotuned shape the items
// were built for.
__global__ void __launch_bounds__(EW_MAX * 32) k_ens_direct(const float *__restrict__ rho,
                                                            const float *__restrict__ gtab, float *__restrict__ phi,
                                                            const EnsInst *__restrict__ inst,
                                                            const EnsDirectItem *__restrict__ items, int nitems,
                                                            unsigned *__restrict__ next, TableShape t, int qrows)
{
    extern __shared__ __align__(16) float se[];
    const int tsz = t.Z * t.Ym * t.pitch;
    float *gm = se;                       // mirrored table
    float *qs = se + tsz;                 // [qrows][Xm] staged source rows
    for (int i = threadIdx.x * 4; i < tsz; i += blockDim.x * 4)
        *reinterpret_cast<float4 *>(&gm[i]) = __ldg(reinterpret_cast<const float4 *>(&gtab[i]));
    __shared__ int nz[QROWS_MAX];  // staged source row holds a non-zero charge
    __shared__ int s_item;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (;;) {
        __syncthreads();  // the previous item is done with the staged rows
        if (threadIdx.x == 0) s_item = (int)atomicAdd(next, 1u);
        __syncthreads();
        const int itx = s_item;
        if (itx >= nitems) break;
        const EnsDirectItem it = items[itx];
        const EnsInst in = inst[it.inst];
        const int r = lane / it.lpr, l = lane % it.lpr;
        const int nrows = in.Y * in.Z;
        const int trow = it.row0 + warp * it.rpw + r;
        const bool active = r < it.rpw && trow < nrows && l * ETX < in.X;
        const int yt = active ? trow % in.Y : 0, zt = active ? trow / in.Y : 0;
        const int x0 = l * ETX;
        const int Xr = (in.X + 7) & ~7;
        float s[ETX], c[ETX];
#pragma unroll
        for (int i = 0; i < ETX; i++) s[i] = c[i] = 0.f;
        for (int sr0 = 0; sr0 < nrows; sr0 += qrows) {
            __syncthreads();
            if (threadIdx.x < qrows) nz[threadIdx.x] = 0;
            __syncthreads();
            const int nq = min(qrows, nrows - sr0);
            for (int i = threadIdx.x; i < qrows * t.Xm; i += blockDim.x) {
                const int qr = i / t.Xm, xs = i % t.Xm;
                const float v = (qr < nq && xs < in.X) ? rho[in.off + (long long)(sr0 + qr) * in.X + xs] : 0.f;
                qs[i] = v;
                if (v != 0.f) nz[qr] = 1;  // benign race: every writer stores 1
            }
            __syncthreads();
            if (!active) continue;
            float acc[ETX];
#pragma unroll
            for (int i = 0; i < ETX; i++) acc[i] = 0.f;
            for (int qr = 0; qr < nq; qr++) {
                if (nz[qr]) {  // an all-zero source row adds nothing
                    const int srow = sr0 + qr;
                    const int ys = srow % in.Y, zs = srow / in.Y;
                    const float *grow = gm + (abs(zt - zs) * t.Ym + abs(yt - ys)) * t.pitch;
                    const float *q = qs + qr * t.Xm;
                    // window: win[k] = grow[base + k], base = C - 7 + x0 - xb
                    // C = Xm + 3 with Xm a multiple of 8: base is a multiple of 4, so
                    // the window is read as two 16-byte vectors (a row's lanes are 32 B
                    // apart: at most 2-way bank conflicts instead of 8-way scalar ones)
                    int base = t.C - 7 + x0;
                    float wb[8];
                    {
                        const float4 u0 = *reinterpret_cast<const float4 *>(grow + base + 8);
                        const float4 u1 = *reinterpret_cast<const float4 *>(grow + base + 12);
                        wb[0] = u0.x; wb[1] = u0.y; wb[2] = u0.z; wb[3] = u0.w;
                        wb[4] = u1.x; wb[5] = u1.y; wb[6] = u1.z; wb[7] = u1.w;
                    }
                    for (int xb = 0; xb < Xr; xb += 8) {
                        float wa[8];
                        {
                            const float4 u0 = *reinterpret_cast<const float4 *>(grow + base);
                            const float4 u1 = *reinterpret_cast<const float4 *>(grow + base + 4);
                            wa[0] = u0.x; wa[1] = u0.y; wa[2] = u0.z; wa[3] = u0.w;
                            wa[4] = u1.x; wa[5] = u1.y; wa[6] = u1.z; wa[7] = u1.w;
                        }
                        const float4 q0 = *reinterpret_cast<const float4 *>(&q[xb]);
                        const float4 q1 = *reinterpret_cast<const float4 *>(&q[xb + 4]);
                        const float qv[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
                        for (int j = 0; j < 8; j++)
#pragma unroll
                            for (int i = 0; i < ETX; i++) {
                                const int k = 7 + i - j;
                                acc[i] = fmaf(qv[j], (k < 8) ? wa[k] : wb[k - 8], acc[i]);
                            }
#pragma unroll
                        for (int k = 0; k < 8; k++) wb[k] = wa[k];
                        base -= 8;
                    }
                }
                if ((qr + 1) % KG == 0 || qr + 1 == nq) {
#pragma unroll
                    for (int i = 0; i < ETX; i++) {  // Kahan across groups of KG source rows
                        const float y = acc[i] - c[i];
                        const float tt = s[i] + y;
                        c[i] = (tt - s[i]) - y;
                        s[i] = tt;
                        acc[i] = 0.f;
                    }
                }
            }
        }
        if (active) {
            float *out = phi + in.off + (long long)trow * in.X;
#pragma unroll
            for (int i = 0; i < ETX; i++)
                if (x0 + i < in.X) out[x0 + i] = s[i] - c[i];
        }
    }
}

__global__ void k_aos_to_soa_ens(const double *__restrict__ in, const uint8_t *__restrict__ mat,
                                 double *__restrict__ out, long long N)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const bool m = mat[i] != 0;
    out[i] = m ? in[3 * i + 0] : 0.0;
    out[i + N] = m ? in[3 * i + 1] : 0.0;
    out[i + 2 * N] = m ? in[3 * i + 2] : 0.0;
}

__global__ void k_soa_to_aos_ens(const double *__restrict__ in, double *__restrict__ out, long long N)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= N) return;
    out[3 * i + 0] = in[i];
    out[3 * i + 1] = in[i + N];
    out[3 * i + 2] = in[i + 2 * N];
}

}  // namespace

struct mms_ens {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int n = 0;
    double dx = 0, dy = 0, dz = 0;
    mms_params p{};
    long long Ntot = 0;
    int ntiles = 0, nitems = 0;
    TableShape ts{};
    size_t direct_smem = 0;
    int ew = 8, qrows = 16;           // direct-kernel shape (mms_ens_autotune)
    int grid_direct = 0, grid_cells = 0;
    unsigned *next = nullptr;         // work counter of the persistent direct kernel
    std::vector<EnsInst> hin;         // host copy of the offset table
    int64_t launches = 0;
    size_t dev_bytes = 0;
    EnsInst *inst = nullptr;
    EnsTile *tiles = nullptr;
    EnsDirectItem *items = nullptr;
    float *gtab = nullptr, *rho = nullptr, *phi = nullptr;
    uint8_t *mat = nullptr;
    double *M = nullptr, *A = nullptr, *B = nullptr, *K = nullptr, *tstate = nullptr, *flag = nullptr;
    double *h_scratch = nullptr;
    bool ready = false, phi_valid = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_kernels = 0;
    PhysK pk() const
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
        k.n_hext = 0;
        k.ref_stage_time = 0;
        physk_derive(k, dx, dy, dz);
        return k;
    }
};

namespace {

#define ENS_LAUNCH_CHECK(e)                                                                          \
    do {                                                                                             \
        (e)->launches++;                                                                             \
        cudaError_t e_ = cudaGetLastError();                                                         \
        if (e_ != cudaSuccess) {                                                                     \
            mms_set_error("%s:%d ensemble kernel launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            return MMS_ERR_CUDA;                                                                     \
        }                                                                                            \
    } while (0)

template <class T>
int ens_alloc(mms_ens *e, T **p, size_t count)
{
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    if (cudaMalloc((void **)p, bytes) != cudaSuccess) {
        *p = nullptr;
        mms_set_error("ensemble: cudaMalloc(%zu) failed", bytes);
        return MMS_ERR_NOMEM;
    }
    e->dev_bytes += bytes;
    return MMS_OK;
}

// direct-kernel work items for `ew` warps per CTA: (instance, first target
// row), rpw rows per warp; sorted by decreasing cost (rows x row length x
// source cells) so that the dynamic schedule ends with the cheapest items
std::vector<EnsDirectItem> build_items(const std::vector<EnsInst> &hin, int ew)
{
    std::vector<std::pair<double, EnsDirectItem>> v;
    for (int i = 0; i < (int)hin.size(); i++) {
        const EnsInst &a = hin[i];
        const int Xr = (a.X + 7) & ~7;
        const int lpr = Xr / ETX;                       // lanes per target row (<= 32)
        const int rpw = std::max(1, 32 / lpr);          // target rows per warp
        const int nrows = a.Y * a.Z;
        for (int r0 = 0; r0 < nrows; r0 += rpw * ew) {
            EnsDirectItem d;
            d.inst = i;
            d.row0 = r0;
            d.rpw = rpw;
            d.lpr = lpr;
            const double cost = (double)std::min(rpw * ew, nrows - r0) * Xr * ((double)a.X * a.Y * a.Z);
            v.push_back({cost, d});
        }
    }
    std::stable_sort(v.begin(), v.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
    std::vector<EnsDirectItem> out;
    for (auto &p : v) out.push_back(p.second);
    return out;
}

size_t direct_smem_for(const TableShape &ts, int qrows)
{
    return ((size_t)ts.Z * ts.Ym * ts.pitch + (size_t)qrows * ts.Xm) * sizeof(float);
}

// uploads the item table of shape (ew, qrows) and sizes the persistent grids
int ens_set_shape(mms_ens *e, int ew, int qrows)
{
    const std::vector<EnsDirectItem> items = build_items(e->hin, ew);
    if ((int)items.size() > e->nitems) {
        cudaFree(e->items);
        e->items = nullptr;
        if (cudaMalloc((void **)&e->items, items.size() * sizeof(EnsDirectItem)) != cudaSuccess) {
            mms_set_error("ensemble: cudaMalloc of the item table failed");
            return MMS_ERR_NOMEM;
        }
    }
    e->nitems = (int)items.size();
    MMS_CUDA_TRY(cudaMemcpyAsync(e->items, items.data(), items.size() * sizeof(EnsDirectItem), cudaMemcpyHostToDevice,
                                 e->stream));
    e->ew = ew;
    e->qrows = qrows;
    e->direct_smem = direct_smem_for(e->ts, qrows);
    {
        // the limit is per kernel and shared by every ensemble: only ever raise it
        cudaFuncAttributes fa{};
        MMS_CUDA_TRY(cudaFuncGetAttributes(&fa, k_ens_direct));
        if ((size_t)fa.maxDynamicSharedSizeBytes < e->direct_smem)
            MMS_CUDA_TRY(cudaFuncSetAttribute(k_ens_direct, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)e->direct_smem));
    }
    int dev = 0, sms = 0, per = 0, perc = 0;
    MMS_CUDA_TRY(cudaGetDevice(&dev));
    MMS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MMS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_ens_direct, ew * 32, e->direct_smem));
    MMS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perc, k_ens_stage, ETPB, 0));
    e->grid_direct = std::max(1, std::min(e->nitems, std::max(per, 1) * sms));
    e->grid_cells = std::max(1, std::min(e->ntiles, std::max(perc, 1) * sms));
    if (e->exec) {  // a captured step holds the old launch shape
        cudaGraphExecDestroy(e->exec);
        e->exec = nullptr;
    }
    if (e->graph) {
        cudaGraphDestroy(e->graph);
        e->graph = nullptr;
    }
    return MMS_OK;
}

int ens_direct(mms_ens *e)
{
    MMS_CUDA_TRY(cudaMemsetAsync(e->next, 0, sizeof(unsigned), e->stream));
    k_ens_direct<<<e->grid_direct, e->ew * 32, e->direct_smem, e->stream>>>(e->rho, e->gtab, e->phi, e->inst,
                                                                           e->items, e->nitems, e->next, e->ts,
                                                                           e->qrows);
    ENS_LAUNCH_CHECK(e);
    return MMS_OK;
}

int ens_potential(mms_ens *e, const double *Mst)
{
    if (!e->p.demag) return MMS_OK;
    k_ens_div<<<e->grid_cells, ETPB, 0, e->stream>>>(Mst, e->rho, e->inst, e->tiles, e->ntiles, e->Ntot, e->dx, e->dy,
                                                     e->dz, div_scale(e->dx, e->dy, e->dz));
    ENS_LAUNCH_CHECK(e);
    return ens_direct(e);
}

int ens_stage(mms_ens *e, int stage, const double *Mst, double *Mnext)
{
    k_ens_stage<<<e->grid_cells, ETPB, 0, e->stream>>>(e->phi, Mst, e->M, e->K, Mnext, e->mat, e->tstate, e->inst,
                                                       e->tiles, e->flag, e->ntiles, e->Ntot, e->dx, e->dy, e->dz,
                                                       e->pk(), stage);
    ENS_LAUNCH_CHECK(e);
    return MMS_OK;
}

int ens_step(mms_ens *e)
{
    MMS_TRY(ens_stage(e, 0, e->M, e->A));
    MMS_TRY(ens_potential(e, e->A));
    MMS_TRY(ens_stage(e, 1, e->A, e->B));
    MMS_TRY(ens_potential(e, e->B));
    MMS_TRY(ens_stage(e, 2, e->B, e->A));
    MMS_TRY(ens_potential(e, e->A));
    MMS_TRY(ens_stage(e, 3, e->A, nullptr));
    MMS_TRY(ens_potential(e, e->M));
    k_ens_advance<<<1, 1, 0, e->stream>>>(e->tstate);
    ENS_LAUNCH_CHECK(e);
    return MMS_OK;
}

}  // namespace

extern "C" {

int mms_ens_create(const mms_ens_instance *inst, int n, double dx, double dy, double dz, const mms_params *params,
                   void *stream, mms_ens **out)
{
    if (!out || !inst || n < 1 || !params || !(dx > 0 && dy > 0 && dz > 0)) {
        mms_set_error("mms_ens_create: bad argument");
        return MMS_ERR_ARG;
    }
    *out = nullptr;
    TableShape ts{};
    long long Ntot = 0;
    std::vector<EnsInst> hin(n);
    std::vector<EnsTile> htiles;
    for (int i = 0; i < n; i++) {
        const mms_ens_instance &a = inst[i];
        if (a.xdim < 1 || a.ydim < 1 || a.zdim < 1 || a.xdim > 256) {
            mms_set_error("mms_ens_create: instance %d has dims %d x %d x %d (1 <= xdim <= 256)", i, a.xdim, a.ydim,
                          a.zdim);
            return MMS_ERR_ARG;
        }
        hin[i].X = a.xdim;
        hin[i].Y = a.ydim;
        hin[i].Z = a.zdim;
        hin[i].pad = 0;
        hin[i].off = Ntot;
        hin[i].hx = a.bext[0] / params->mu0;
        hin[i].hy = a.bext[1] / params->mu0;
        hin[i].hz = a.bext[2] / params->mu0;
        const long long Ni = (long long)a.xdim * a.ydim * a.zdim;
        for (long long s0 = 0; s0 < Ni; s0 += ETPB) {
            EnsTile t;
            t.inst = i;
            t.start = (int)s0;
            t.count = (int)std::min<long long>(ETPB, Ni - s0);
            t.pad = 0;
            htiles.push_back(t);
        }
        const int Xr = (a.xdim + 7) & ~7;
        Ntot += Ni;
        ts.Xm = std::max(ts.Xm, Xr);
        ts.Ym = std::max(ts.Ym, a.ydim);
        ts.Z = std::max(ts.Z, a.zdim);
    }
    ts.C = ts.Xm + 3;
    ts.pitch = 2 * ts.Xm + 8;
    const size_t smem = direct_smem_for(ts, QROWS_MAX);
    if (smem > 200 * 1024) {
        mms_set_error("mms_ens_create: the shared kernel table (%zu B) exceeds 200 KiB; largest instance too big",
                      smem);
        return MMS_ERR_ARG;
    }
    mms_ens *e = new (std::nothrow) mms_ens();
    if (!e) {
        mms_set_error("host allocation failed");
        return MMS_ERR_NOMEM;
    }
    int st = MMS_OK;
    do {
        cudaGetDevice(&e->device);
        e->n = n;
        e->dx = dx;
        e->dy = dy;
        e->dz = dz;
        e->p = *params;
        e->p.hext_t = e->p.hext_b = nullptr;
        e->p.n_hext = 0;
        e->Ntot = Ntot;
        e->ts = ts;
        e->ntiles = (int)htiles.size();
        e->nitems = 0;
        e->hin = hin;
        if (stream) {
            e->stream = (cudaStream_t)stream;
        } else {
            if (cudaStreamCreate(&e->stream) != cudaSuccess) {
                mms_set_error("cudaStreamCreate failed");
                st = MMS_ERR_CUDA;
                break;
            }
            e->own_stream = true;
        }
        const size_t N = (size_t)Ntot;
        if ((st = ens_alloc(e, &e->inst, (size_t)n))) break;
        if ((st = ens_alloc(e, &e->tiles, htiles.size()))) break;
        if ((st = ens_alloc(e, &e->next, 1))) break;
        if ((st = ens_alloc(e, &e->gtab, (size_t)ts.Z * ts.Ym * ts.pitch))) break;
        if ((st = ens_alloc(e, &e->rho, N))) break;
        if ((st = ens_alloc(e, &e->phi, N))) break;
        if ((st = ens_alloc(e, &e->mat, N))) break;
        if ((st = ens_alloc(e, &e->M, 3 * N))) break;
        if ((st = ens_alloc(e, &e->A, 3 * N))) break;
        if ((st = ens_alloc(e, &e->B, 3 * N))) break;
        if ((st = ens_alloc(e, &e->K, 3 * N))) break;
        if ((st = ens_alloc(e, &e->tstate, TIME_SLOTS))) break;
        if ((st = ens_alloc(e, &e->flag, 1))) break;
        if (cudaMallocHost((void **)&e->h_scratch, 8 * sizeof(double)) != cudaSuccess) {
            st = MMS_ERR_NOMEM;
            mms_set_error("cudaMallocHost failed");
            break;
        }
        if (cudaMemcpyAsync(e->inst, hin.data(), n * sizeof(EnsInst), cudaMemcpyHostToDevice, e->stream) ||
            cudaMemcpyAsync(e->tiles, htiles.data(), htiles.size() * sizeof(EnsTile), cudaMemcpyHostToDevice,
                            e->stream) ||
            cudaMemsetAsync(e->tstate, 0, TIME_SLOTS * sizeof(double), e->stream) ||
            cudaMemsetAsync(e->flag, 0, sizeof(double), e->stream)) {
            mms_set_error("ensemble set-up copies failed");
            st = MMS_ERR_CUDA;
            break;
        }
        const long long tn = (long long)ts.Z * ts.Ym * ts.pitch;
        k_ens_table<<<div_up(tn, 256), 256, 0, e->stream>>>(e->gtab, ts, dx, dy, dz);
        if ((st = ens_set_shape(e, 8, 16))) break;
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(e->stream) != cudaSuccess) {
            mms_set_error("ensemble set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
            st = MMS_ERR_CUDA;
            break;
        }
    } while (0);
    if (st != MMS_OK) {
        char keep[512];
        strncpy(keep, mms_last_error(), sizeof keep - 1);
        keep[sizeof keep - 1] = 0;
        mms_ens_destroy(e);
        mms_set_error("%s", keep);
        return st;
    }
    *out = e;
    return MMS_OK;
}

int mms_ens_destroy(mms_ens *e)
{
    if (!e) return MMS_OK;
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    void *b[] = {e->inst, e->tiles, e->items, e->gtab, e->rho, e->phi, e->mat, e->M, e->A, e->B, e->K, e->tstate,
                 e->flag, e->next};
    for (void *p : b)
        if (p) cudaFree(p);
    if (e->h_scratch) cudaFreeHost(e->h_scratch);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return MMS_OK;
}

long long mms_ens_cells(const mms_ens *e) { return e ? e->Ntot : 0; }

int64_t mms_ens_kernel_launches(const mms_ens *e) { return e ? e->launches : 0; }

int mms_ens_state_set(mms_ens *e, const uint8_t *material, const double *M)
{
    if (!e || !material || !M) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    const size_t N = (size_t)e->Ntot;
    MMS_CUDA_TRY(cudaMemcpyAsync(e->mat, material, N, cudaMemcpyHostToDevice, e->stream));
    MMS_CUDA_TRY(cudaMemcpyAsync(e->K, M, 3 * N * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    k_aos_to_soa_ens<<<div_up(e->Ntot, 256), 256, 0, e->stream>>>(e->K, e->mat, e->M, e->Ntot);
    ENS_LAUNCH_CHECK(e);
    MMS_CUDA_TRY(cudaMemsetAsync(e->tstate, 0, TIME_SLOTS * sizeof(double), e->stream));
    MMS_CUDA_TRY(cudaMemsetAsync(e->flag, 0, sizeof(double), e->stream));
    MMS_CUDA_TRY(cudaStreamSynchronize(e->stream));
    e->ready = true;
    e->phi_valid = false;
    return MMS_OK;
}

int mms_ens_state_get(mms_ens *e, double *M, double *t)
{
    if (!e || !e->ready) {
        mms_set_error("ensemble state not set");
        return MMS_ERR_NOT_READY;
    }
    const size_t N = (size_t)e->Ntot;
    if (M) {
        k_soa_to_aos_ens<<<div_up(e->Ntot, 256), 256, 0, e->stream>>>(e->M, e->K, e->Ntot);
        ENS_LAUNCH_CHECK(e);
        MMS_CUDA_TRY(cudaMemcpyAsync(M, e->K, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    }
    MMS_CUDA_TRY(cudaMemcpyAsync(e->h_scratch, e->tstate, TIME_SLOTS * sizeof(double), cudaMemcpyDeviceToHost,
                                 e->stream));
    MMS_CUDA_TRY(cudaMemcpyAsync(e->h_scratch + TIME_SLOTS, e->flag, sizeof(double), cudaMemcpyDeviceToHost,
                                 e->stream));
    MMS_CUDA_TRY(cudaStreamSynchronize(e->stream));
    if (t) *t = e->h_scratch[TIME_T];
    if (e->h_scratch[TIME_SLOTS] != 0.0) {
        mms_set_error("non-finite magnetisation in the ensemble");
        return MMS_ERR_NUMERIC;
    }
    return MMS_OK;
}

int mms_ens_run_fixed(mms_ens *e, double dt, int nsteps, int use_graph)
{
    if (!e || !e->ready) {
        mms_set_error("ensemble state not set");
        return MMS_ERR_NOT_READY;
    }
    if (!(dt > 0) || nsteps < 0) {
        mms_set_error("dt must be positive and nsteps >= 0");
        return MMS_ERR_ARG;
    }
    k_ens_set_dt<<<1, 1, 0, e->stream>>>(e->tstate, dt);
    ENS_LAUNCH_CHECK(e);
    if (!e->phi_valid) {
        MMS_TRY(ens_potential(e, e->M));
        e->phi_valid = true;
    }
    if (!use_graph) {
        for (int s = 0; s < nsteps; s++) MMS_TRY(ens_step(e));
        return MMS_OK;
    }
    if (!e->exec) {
        const int64_t before = e->launches;
        MMS_CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        const int st = ens_step(e);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (st != MMS_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (ce != cudaSuccess) {
            mms_set_error("ensemble graph capture: %s", cudaGetErrorString(ce));
            return MMS_ERR_CUDA;
        }
        e->graph = g;
        MMS_CUDA_TRY(cudaGraphInstantiate(&e->exec, g, 0));
        e->graph_kernels = (int)(e->launches - before);
        e->launches = before;
    }
    for (int s = 0; s < nsteps; s++) {
        MMS_CUDA_TRY(cudaGraphLaunch(e->exec, e->stream));
        e->launches += e->graph_kernels;
    }
    return MMS_OK;
}

int mms_ens_autotune(mms_ens *e, int reps, int *ew, int *qrows, double *best_ms)
{
    if (!e || !e->ready || reps < 1) {
        mms_set_error("mms_ens_autotune: ensemble state not set or reps < 1");
        return MMS_ERR_NOT_READY;
    }
    // the charges of the current state
    k_ens_div<<<e->grid_cells, ETPB, 0, e->stream>>>(e->M, e->rho, e->inst, e->tiles, e->ntiles, e->Ntot, e->dx, e->dy,
                                                     e->dz, div_scale(e->dx, e->dy, e->dz));
    ENS_LAUNCH_CHECK(e);
    cudaEvent_t e0, e1;
    MMS_CUDA_TRY(cudaEventCreate(&e0));
    MMS_CUDA_TRY(cudaEventCreate(&e1));
    const int ews[] = {4, 8, 16}, qs[] = {8, 16, 32};
    double best = 1e30;
    int bew = e->ew, bq = e->qrows, st = MMS_OK;
    for (int a : ews)
        for (int q : qs) {
            if (st != MMS_OK) break;
            if ((st = ens_set_shape(e, a, q))) break;
            if ((st = ens_direct(e))) break;  // warm
            cudaEventRecord(e0, e->stream);
            for (int r = 0; r < reps && st == MMS_OK; r++) st = ens_direct(e);
            cudaEventRecord(e1, e->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                mms_set_error("mms_ens_autotune: %s", cudaGetErrorString(cudaGetLastError()));
                st = MMS_ERR_CUDA;
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms / reps < best) {
                best = ms / reps;
                bew = a;
                bq = q;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MMS_TRY(st);
    MMS_TRY(ens_set_shape(e, bew, bq));
    e->phi_valid = false;
    MMS_CUDA_TRY(cudaStreamSynchronize(e->stream));
    if (ew) *ew = bew;
    if (qrows) *qrows = bq;
    if (best_ms) *best_ms = best;
    return MMS_OK;
}

int mms_ens_sync(mms_ens *e)
{
    if (!e) {
        mms_set_error("NULL ensemble");
        return MMS_ERR_ARG;
    }
    MMS_CUDA_TRY(cudaStreamSynchronize(e->stream));
    return MMS_OK;
}

}  // extern "C"
