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
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include "farnet.cuh"
#include "fmm_ops.hpp"
#include "mms_internal.cuh"
#include "stencil_dev.cuh"
#include "umma.cuh"

namespace {

constexpr int KW = 16;        // k values per warp in k_m2l (4 x float4)
constexpr int M2L_WARPS = 4;  // up to 64 k per parity block

struct FmmDev {
    int P, s, L, nb, NR, NE, C, Z;
    int X, Y;
    float inv_w;              // 1 / leaf width (m): L2P scale
};

// The divergence an upward-pass kernel forms from the FP64 state as it stages
// the charges (the state path of a field evaluation, no separate divergence
// launch): the state, its grid, and where rho and, when hi != nullptr, its
// BF16 hi / lo split for the tensor-core near field go.
struct DivSrc {
    const double *M;
    float *rho;
    __nv_bfloat16 *hi, *lo;
    GridK g;
    mmsdev::DivScale h;
    int nbx, nby;
};

// rho at cell (x, y, z) inside the grid (div_soa_cell: the bits of the
// divergence kernel), and its stores
__device__ __forceinline__ float div_value(const DivSrc &dv, int x, int y, int z)
{
    const long long i = ((long long)z * dv.g.Y + y) * dv.g.X + x;
    return mmsdev::div_soa_cell(dv.M, i, x, y, z, dv.g, dv.h);
}

__device__ __forceinline__ void div_store(const DivSrc &dv, int x, int y, int z, float v)
{
    dv.rho[((long long)z * dv.g.Y + y) * dv.g.X + x] = v;
    if (dv.hi) {
        const long long j = mmsdev::ntc_index(x, y, z, dv.nbx, dv.nby);
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        dv.hi[j] = h;
        dv.lo[j] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

// one GEMM of the grouped tensor-core M2L (a parity class x a parity block)
struct TcGroup {
    const __nv_bfloat16 *A;
    const __nv_bfloat16 *B;
    float *C;
    const int *rowmap;
    int lda, ldb, ldc, M, N, K;
    int pad[2];
};


}  // namespace

struct FarSync;

struct FmmPlan {
    FmmDev d{};
    int KPb[2] = {0, 0};      // padded k extent per parity block in k_m2l
    std::vector<long long> lev_off;  // first box of each level in Mall / Lall
    long long nbox_total = 0;
    int n_m2l_items = 0;
    // device
    float *Wt = nullptr;      // [C][NR]  P2M weights (dV folded in)
    float *Vt = nullptr;      // [NR][C]  L2P weights (1/leaf width folded in)
    float *Tm2m = nullptr;    // [4][parity block][j][k]
    float *Tl2l = nullptr;    // [4][parity block][j][k]
    float *Tm2l = nullptr;    // [49][2][NBmax(j)][KP(k)] parity blocks, k padded
    float *Tm2lc = nullptr;   // [49][even NE x NE | odd NO x NO] compact, j-major (low orders)
    int m2l_resident = 0;     // 1: k_m2l_res (all operators in shared memory)
    int far_fused = 0;        // 1: P2M .. L2L in one cooperative launch (k_far)
    int far_grid = 0;
    size_t far_smem = 0;
    struct FarSync *far_sync = nullptr;
    int m2l_tc = 0;           // 1: tensor-core M2L (gather + grouped tcgen05 GEMM)
    // tensor-core M2L: per parity block b, A'_b rows = every box of levels >= 2
    // grouped by parity class, each row [S_hi | S_hi | S_lo] over the class's
    // 27 offsets; B'_{p,b} = [T_hi | T_lo | T_hi] operator rows
    int tcK[2] = {0, 0};      // 27 * NB padded to 8, per block
    int tcNBp[2] = {0, 0};
    int tc_rows = 0;
    __nv_bfloat16 *tcA[2] = {nullptr, nullptr};
    __nv_bfloat16 *tcB = nullptr;   // [4 parities][2 blocks] regions
    int *tc_rowmap = nullptr;       // row -> box index (all levels)
    int4 *tc_rowinfo = nullptr;     // row -> {level, parity, target in class}
    TcGroup *tc_groups = nullptr;   // [8] on the device
    std::vector<TcGroup> tc_group_host;
    int tc_maxm = 0;
    int tc_ksplit = 1;        // K split of the grouped GEMM: partial locals, summed by L2L / L2P
    float *Gn = nullptr;      // [Z][2s][2s] near-field dV/|r|
    float *Mall = nullptr;    // [boxes of all levels][NR]
    float *Lall = nullptr;    // final locals
    float *Lpart = nullptr;   // [NSPLIT][boxes][NR] M2L partial locals
    int4 *m2l_items = nullptr;  // {level, parity, first target, 0}: 32 targets (k_m2l_split)
    int4 *res_items = nullptr;  // the same with RES_TPI targets (k_m2l_res, k_far)
    int n_res_items = 0;
    long long *lev_dev = nullptr;  // device copy of lev_off
    float *near = nullptr;    // [N] near-field potential (P2P) before L2P adds the far field
    int p2p_tc = 0;           // 1: near field on the tensor cores (leaf side 8): k_p2p_tc
    __nv_bfloat16 *ntcT = nullptr;  // [3 dy][C][2 parts (hi, lo)][3 dx][C] near-field operators
    __nv_bfloat16 *ntcR = nullptr;  // [2][Z][nby][nbx][8][8] BF16 hi, lo of rho, box-major, zero-padded
    CUtensorMap ntc_map[3];   // TMA maps: rho hi, rho lo (4-D, box-major), operators (2-D)
    const float *split_of = nullptr;  // rho whose BF16 split ntcR holds (written by the divergence)
    float *near3 = nullptr;   // [3 dy][N] near-field partials of k_p2p_tc, summed by L2P
    cudaStream_t side = nullptr;   // P2P runs here, concurrently with P2M .. L2L
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    size_t bytes = 0;
    // learned far-field network (solver MMS_SOLVER_SURROGATE): tables per
    // level, bound by farnet_bind from a weight vector indexed by depth
    int fn_ready = 0;
    float *fnW = nullptr;     // [NR][C] encoder (transposed), dx^2 folded in
    float *fnV = nullptr;     // [NR][C] decoder
    float *fnM2L = nullptr;   // [levels 2..L][49][OSZ]
    float *fnM2M = nullptr;   // [parent levels 2..L-1][4][OSZ]
    float *fnL2L = nullptr;   // [parent levels 2..L-1][4][OSZ]
    float *fnM = nullptr;     // [boxes of all levels][NR] multipoles
    float *fnLp = nullptr;    // [boxes of all levels][NR] interaction-list locals
    unsigned *fnCtr = nullptr;  // [boxes] arrival counters of the upward pass (zero between launches)
    int fn_nr = 0, fn_ne = 0;   // width of the bound network
    // algorithmic work per evaluation (for the roofline)
    double flops = 0;
    double stage_flops[5] = {0, 0, 0, 0, 0};  // P2M, M2M, M2L, L2L, L2P+P2P
    long long p2p_pairs = 0, m2l_pairs = 0;
};

namespace {

// ---- generic L2P + P2P (any leaf side): CTA per leaf box, thread per target cell.
__global__ void k_l2p_p2p(const float *__restrict__ rho, const float *__restrict__ Lleaf,
                          const float *__restrict__ Vt, const float *__restrict__ Gn, float *__restrict__ phi,
                          FmmDev f, int far)
{
    pdl_begin();
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
    phi[((long long)lz * f.Y + y) * f.X + x] = farv + near;
}


// ===========================================================================
// Stage kernels.

constexpr int BB = 8;         // leaf boxes per CTA along x in the leaf kernels
constexpr int NSPLIT = 9;     // M2L offset groups (3 offsets each) -> partial locals

// one float into shared memory by an asynchronous copy; zero when !valid
// (src must still be a readable address)
__device__ __forceinline__ void cp_async4(float *dst, const float *src, bool valid)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(umma::smem_u32(dst)), "l"(src),
                 "r"(valid ? 4 : 0)
                 : "memory");
}

// Stage n floats (n a multiple of 4, both addresses 16-byte aligned) into
// shared memory with asynchronous copies, every chunk in flight at once, and
// wait for this thread's copies; a __syncthreads must follow before any
// other thread reads them.
__device__ __forceinline__ void stage_async(float *dst, const float *src, int n)
{
    for (int i = threadIdx.x * 4; i < n; i += blockDim.x * 4) umma::cp_async16(umma::smem_u32(dst + i), src + i, true);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// One P2M output: sum over the leaf's C cells of W[c][k] q[c], w = &W[0][k]
// (row pitch NR), qq = &q[0] (pitch QS).  Four interleaved partial sums
// (cells c = 0, 1, 2, 3 mod 4) joined as (s0 + s1) + (s2 + s3): four
// independent FMA chains a quarter as long as one running sum.
template <int QS>
__device__ __forceinline__ float p2m_dot(const float *w, int NR, const float *qq, int C)
{
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    const int C4 = C & ~3;
#pragma unroll 2
    for (int c = 0; c < C4; c += 4) {
        a0 = fmaf(w[0], qq[0], a0);
        a1 = fmaf(w[NR], qq[QS], a1);
        a2 = fmaf(w[2 * NR], qq[2 * QS], a2);
        a3 = fmaf(w[3 * NR], qq[3 * QS], a3);
        w += 4 * NR;
        qq += 4 * QS;
    }
    if (C4 < C) a0 = fmaf(w[0], qq[0], a0);
    if (C4 + 1 < C) a1 = fmaf(w[NR], qq[QS], a1);
    if (C4 + 2 < C) a2 = fmaf(w[2 * NR], qq[2 * QS], a2);
    return (a0 + a1) + (a2 + a3);
}

// P2M of one item = BB leaf boxes of one row: the boxes' charges are staged
// transposed in shared memory ([cell][box]); thread per (box, coefficient),
// each output by p2m_dot.  Wt: [C][NR] weights (shared or global memory).
// q: C * BB floats of shared memory.
__device__ __forceinline__ void p2m_item(const float *__restrict__ rho, const float *Wt, float *q,
                                         float *__restrict__ Mleaf, const FmmDev &f, int by, int bx0)
{
    const int s = f.s;
    for (int i = threadIdx.x; i < f.C * BB; i += blockDim.x) {
        const int b = i % BB, c = i / BB;
        const int x = (bx0 + b) * s + c % s, y = by * s + (c / s) % s, z = c / (s * s);
        q[i] = (x < f.X && y < f.Y) ? rho[((long long)z * f.Y + y) * f.X + x] : 0.f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < BB * f.NR; e += blockDim.x) {
        const int b = e / f.NR, k = e % f.NR;
        const float acc = p2m_dot<BB>(Wt + k, f.NR, q + b, f.C);
        if (bx0 + b < f.nb) Mleaf[((long long)by * f.nb + bx0 + b) * f.NR + k] = acc;
    }
    __syncthreads();
}

__device__ __forceinline__ void m2m_reduce(float *__restrict__ Mall, const float *Ts, const float *Mc, float *red,
                                           long long off_p, int box, const FmmDev &f, int t, int KT, bool valid,
                                           float *keep = nullptr);

// P2M: CTA = one item, PB leaf boxes of one row (up == 0) or of two rows
// (up != 0, NR <= 32), thread per (row, box, coefficient).  The charges are
// read a row of PB boxes at a time (one warp per cell row, consecutive
// lanes on consecutive cells) into [rows][C][PB] in shared memory while the
// weights W (when wsm) and, with up, the M2M operators stream in by cp.async.
// With up the CTA then forms the PB/2 parents (the M2M of level L-1), one
// 4 KT-thread group per parent, from the children it keeps in shared memory;
// (PB/2) 4 KT threads.  PB = 8, or 4 at leaf side >= 8 or NR > 32.  Per output
// the arithmetic of p2m_item / m2m_item.
// Shared memory: charges [rows][C][PB], W [C][NR] when wsm, then (up) the M2M
// operators and the per-parent M2M scratch.
// DIV: the charges are the divergence of the state dv.M, formed here and also
// stored to dv.rho (and its split) for the near field; rho is not read.
template <int PB, bool DIV>
__global__ void __launch_bounds__(512) k_p2m_row(const float *__restrict__ rho, const float *__restrict__ Wg,
                                                 float *__restrict__ Mall, long long off_leaf, FmmDev f, int wsm,
                                                 int up, const float *__restrict__ Tm2m, long long off_par, DivSrc dv)
{
    extern __shared__ __align__(16) float q[];
    const int rows = up ? 2 : 1;
    const int NE = f.NE, NO = f.NR - f.NE, s = f.s, CB = f.C * PB;
    const int tsz = 4 * (NE * NE + NO * NO);
    const int KT = ((f.NR + 31) / 32) * 32;
    const float *Wt = Wg;
    float *tail = q + rows * CB;
    // weights and operators: every chunk in flight before the charges load
    if (wsm) {
        for (int i = threadIdx.x * 4; i < f.C * f.NR; i += blockDim.x * 4)
            umma::cp_async16(umma::smem_u32(tail + i), Wg + i, true);
        Wt = tail;
        tail += f.C * f.NR;
    }
    float *Ts = tail, *scr = Ts + tsz;
    if (up)
        for (int i = threadIdx.x * 4; i < tsz; i += blockDim.x * 4)
            umma::cp_async16(umma::smem_u32(Ts + i), Tm2m + i, true);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    // weights and operators are constant and already in flight; the charges
    // are the predecessor's output
    pdl_begin();
    const int bx0 = blockIdx.x * PB, by0 = rows * blockIdx.y;
    if constexpr (DIV) {
        // element e = (row, xx) as below; each thread forms up to DR values
        // (all their state loads in flight) before it stores any
        constexpr int DR = 8;
        const int RW = PB * s, ntot = rows * f.Z * s * RW;
        for (int base = 0; base < ntot; base += DR * blockDim.x) {
            float v[DR];
#pragma unroll
            for (int k = 0; k < DR; k++) {
                const int e = base + threadIdx.x + k * blockDim.x, row = e / RW, xx = e - row * RW;
                const int yy = row % s, z = (row / s) % f.Z, r = row / (s * f.Z);
                const int x = bx0 * s + xx, y = (by0 + r) * s + yy;
                v[k] = (e < ntot && x < f.X && y < f.Y) ? div_value(dv, x, y, z) : 0.f;
            }
#pragma unroll
            for (int k = 0; k < DR; k++) {
                const int e = base + threadIdx.x + k * blockDim.x, row = e / RW, xx = e - row * RW;
                if (e >= ntot) break;
                const int yy = row % s, z = (row / s) % f.Z, r = row / (s * f.Z);
                const int x = bx0 * s + xx, y = (by0 + r) * s + yy;
                const int b = xx / s, cx = xx - b * s;
                q[r * CB + (z * s + yy) * s * PB + cx * PB + b] = v[k];
                if (x < f.X && y < f.Y) div_store(dv, x, y, z, v[k]);
            }
        }
    } else {
        const int RW = PB * s, nrow = rows * f.Z * s;
        const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        for (int row = threadIdx.x >> 5; row < nrow; row += nw) {
            const int yy = row % s, z = (row / s) % f.Z, r = row / (s * f.Z);
            const int y = (by0 + r) * s + yy;
            const float *src = rho + ((long long)z * f.Y + y) * f.X + (long long)bx0 * s;
            float *dst = q + r * CB + (z * s + yy) * s * PB;
            for (int xx = lane; xx < RW; xx += 32) {
                const int b = xx / s, cx = xx - b * s;
                dst[cx * PB + b] = (bx0 * s + xx < f.X && y < f.Y) ? src[xx] : 0.f;
            }
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    float *Mleaf = Mall + off_leaf * f.NR;
    // with up, the children's expansions also go to the parents' scratch
    const int np = f.nb >> 1;
    for (int e = threadIdx.x; e < rows * PB * f.NR; e += blockDim.x) {
        const int r = e / (PB * f.NR), rem = e % (PB * f.NR), b = rem / f.NR, k = rem % f.NR;
        const float acc = p2m_dot<PB>(Wt + k, f.NR, q + r * CB + b, f.C);
        if (bx0 + b < f.nb) Mleaf[((long long)(by0 + r) * f.nb + bx0 + b) * f.NR + k] = acc;
        if (up) scr[(b >> 1) * (4 * f.NR + 4 * KT) + ((b & 1) | (r << 1)) * f.NR + k] = acc;
    }
    if (!up) return;
    __syncthreads();
    const int grp = threadIdx.x / (4 * KT), t = threadIdx.x % (4 * KT);
    const int pc = (bx0 >> 1) + grp;
    float *Mc = scr + grp * (4 * f.NR + 4 * KT), *red = Mc + 4 * f.NR;
    m2m_reduce(Mall, Ts, Mc, red, off_par, blockIdx.y * np + pc, f, t, KT, grp < PB / 2 && pc < np);
}

// M2M: CTA per parent box, thread per (child c, output coefficient k).  The
// four child operators (parity blocks only, [c][blk][j][k]) and the children's
// expansions are staged in shared memory with one wave of bulk loads; the four
// child contributions are summed in a fixed order.
__device__ __forceinline__ int blk_base(int c, int NE, int NO, int blk)
{
    return c * (NE * NE + NO * NO) + (blk ? NE * NE : 0);
}

// one parent box of M2M with a group of 4 KT threads (t = thread in group):
// thread (child c, coefficient k); Ts = the 4 child operators in shared
// memory; Mc (4 NR: the children's expansions, child c = (cy & 1) 2 +
// (cx & 1)) and red (4 KT) are the group's shared scratch
__device__ __forceinline__ void m2m_reduce(float *__restrict__ Mall, const float *Ts, const float *Mc, float *red,
                                           long long off_p, int box, const FmmDev &f, int t, int KT, bool valid,
                                           float *keep)
{
    const int NE = f.NE, NO = f.NR - f.NE;
    const int c = t / KT, k = t % KT;
    float acc = 0.f;
    if (k < f.NR) {
        const int blk = k >= NE, NB = blk ? NO : NE, kk = blk ? k - NE : k, boff = blk ? NE : 0;
        const float *T = Ts + blk_base(c, NE, NO, blk);
        const float *m = Mc + c * f.NR + boff;
#pragma unroll 8
        for (int j = 0; j < NB; j++) acc = fmaf(T[j * NB + kk], m[j], acc);
    }
    red[c * KT + k] = acc;
    __syncthreads();
    if (valid && c == 0 && k < f.NR) {
        const float v = (red[k] + red[KT + k]) + (red[2 * KT + k] + red[3 * KT + k]);
        Mall[(off_p + box) * f.NR + k] = v;
        if (keep) keep[k] = v;  // (the caller's shared copy for the next level up)
    }
    __syncthreads();
}

// m2m_reduce with the children's expansions read from Mall first
__device__ __forceinline__ void m2m_item(float *__restrict__ Mall, const float *Ts, float *Mc, float *red,
                                         long long off_p, long long off_c, int np, int box, const FmmDev &f, int t,
                                         int KT, bool valid = true)
{
    const int bx = box % np, by = box / np, nc = 2 * np;
    for (int i = t; valid && i < 4 * f.NR; i += 4 * KT) {
        const int c = i / f.NR, j = i % f.NR;
        const int cx = 2 * bx + (c & 1), cy = 2 * by + (c >> 1);
        Mc[i] = Mall[(off_c + (long long)cy * nc + cx) * f.NR + j];
    }
    __syncthreads();
    m2m_reduce(Mall, Ts, Mc, red, off_p, box, f, t, KT, valid);
}

__global__ void k_m2m_c(float *__restrict__ Mall, const float *__restrict__ Tb, long long off_p, long long off_c,
                        int np, FmmDev f)
{
    pdl_begin();
    extern __shared__ __align__(16) float smb[];
    const int NE = f.NE, NO = f.NR - f.NE;
    const int tsz = 4 * (NE * NE + NO * NO);
    const int KT = blockDim.x / 4;            // threads per child
    float *Ts = smb;                          // [4][blocks]
    float *Mc = smb + tsz;                    // [4][NR]
    float *red = Mc + 4 * f.NR;               // [4][KT]
    stage_async(Ts, Tb, tsz);
    m2m_item(Mall, Ts, Mc, red, off_p, off_c, np, blockIdx.x, f, threadIdx.x, KT);
}

// M2L, all levels >= 2 in one launch.  CTA = 32 targets of one (level, parity
// class) x one parity block of k x one of NSPLIT groups of 3 of the class's 27
// offsets (blockIdx.z; each group writes its own partial locals, summed in a
// fixed order by the downward pass).  Lane <-> target, warp <-> 16
// consecutive k.  Per offset the operator block and the 32 source expansions
// are staged in shared memory (odd row pitch: conflict-free per-lane reads);
// the operator is read as warp-uniform float4 broadcasts, 16 FMAs per source
// coefficient per lane.
__global__ void __launch_bounds__(32 * M2L_WARPS) k_m2l_split(const float *__restrict__ Mall,
                                                              float *__restrict__ Lpart,
                                                              const float *__restrict__ Tm2l,
                                                              const int4 *__restrict__ items,
                                                              const long long *__restrict__ lev_off, FmmDev f,
                                                              int KP0, int KP1, int NBmax, long long part_stride)
{
    pdl_begin();
    extern __shared__ __align__(16) float sm2[];
    const int4 it = items[blockIdx.x];
    const int lev = it.x, px = it.y & 1, py = it.y >> 1;
    const int blk = blockIdx.y, grp = blockIdx.z;
    const int KP = blk ? KP1 : KP0;
    const int KPmax = max(KP0, KP1);
    const int NB = blk ? (f.NR - f.NE) : f.NE;
    const int NBp = NB | 1;
    const int boff = blk ? f.NE : 0;
    float *Ts = sm2;                     // [NB][KP]
    float *Ms = sm2 + NBmax * KPmax;     // [32][NBp]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = 1 << lev, nh = n >> 1;
    const long long off = lev_off[lev];
    const int k0 = warp * KW;
    const bool wactive = k0 < NB;
    const int ti = it.z + lane;
    const bool tvalid = ti < nh * nh;
    const int tx = 2 * (ti % nh) + px, ty = 2 * (ti / nh) + py;

    float acc[KW];
#pragma unroll
    for (int i = 0; i < KW; i++) acc[i] = 0.f;

    int idx = 0;
    for (int oy = py - 3; oy <= py + 2; oy++)
        for (int ox = px - 3; ox <= px + 2; ox++) {
            if (max(abs(ox), abs(oy)) < 2) continue;
            const int mine = (idx++ / (27 / NSPLIT)) == grp;
            if (!mine) continue;
            const int o = (oy + 3) * 7 + (ox + 3);
            const float *Tg = Tm2l + ((long long)o * 2 + blk) * NBmax * KPmax;
            __syncthreads();
            stage_async(Ts, Tg, NB * KP);
            for (int i = threadIdx.x; i < 32 * NB; i += blockDim.x) {
                const int t = i / NB, j = i % NB;
                const int tj = it.z + t;
                const int ux = 2 * (tj % nh) + px - ox, uy = 2 * (tj / nh) + py - oy;
                const bool ok = tj < nh * nh && ux >= 0 && uy >= 0 && ux < n && uy < n;
                Ms[t * NBp + j] = ok ? __ldg(&Mall[(off + (long long)uy * n + ux) * f.NR + boff + j]) : 0.f;
            }
            __syncthreads();
            if (!wactive) continue;
            const float *mrow = Ms + lane * NBp;
#pragma unroll 2
            for (int j = 0; j < NB; j++) {
                const float m = mrow[j];
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
    float *Lt = Lpart + grp * part_stride + (off + (long long)ty * n + tx) * f.NR + boff;
#pragma unroll
    for (int i = 0; i < KW; i++)
        if (k0 + i < NB) Lt[k0 + i] = acc[i];
}

// M2L for low orders, all levels >= 2 in one launch: every operator block of
// the 49 offset slots stays resident in shared memory (P <= 5).  CTA = 32
// targets of one (level, parity class) x 8 warps; warp w takes offsets
// w, w+8, w+16, w+24 of the class's 27; lane <-> target.  Each lane keeps its
// source expansion and both parity blocks of its partial local in registers
// and reads the operator rows as warp-uniform float2 broadcasts.  The 8 warps'
// partials are summed in a fixed order in shared memory; the result is the
// complete M2L local (one partial buffer).
constexpr int RES_WARPS = 8;
constexpr int RES_TPI = 16;  // targets per resident-M2L item

// one M2L item (32 targets of one level and parity class, all 27 offsets) on
// RES_WARPS warps; Ts = all 49 operator slots in shared memory; red =
// RES_WARPS * 32 * (NR + 1) floats of shared scratch (may alias Ts: it is
// written only after the last operator read)
// one M2L item (RES_TPI = 16 targets of one level and parity class, all 27
// offsets) on RES_WARPS warps; lane = (half, target): the 16 slots (warp,
// half) take the class's offsets s, s + 16 (class order), the two halves of a
// warp are added with one shuffle and the warps in a fixed order.  Ts = all
// 49 operator slots in shared memory; red = RES_WARPS * RES_TPI * (NR + 1)
// floats of shared scratch (may alias Ts: it is written only after the last
// operator read)
template <int NR_, int NE_, bool NC>
__device__ __forceinline__ void m2l_res_item(const float *__restrict__ Mall, float *__restrict__ Lout, const float *Ts,
                                             float *red, const int4 it, const long long *__restrict__ lev_off)
{
    constexpr int NO_ = NR_ - NE_;
    constexpr int OSZ = NE_ * NE_ + NO_ * NO_;
    constexpr int NSLOT = 2 * RES_WARPS;
    const int lev = it.x, px = it.y & 1, py = it.y >> 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int half = lane >> 4, tl = lane & 15, slot = 2 * warp + half;
    const int n = 1 << lev, nh = n >> 1;
    const long long off = lev_off[lev];
    const int ti = it.z + tl;
    const bool tvalid = ti < nh * nh;
    const int tx = 2 * (ti % nh) + px, ty = 2 * (ti / nh) + py;
    // this slot's offsets (s, s + 16) of the class's 27, in class order
    int ox_l[2], oy_l[2], no = 0;
    {
        int idx = 0;
        for (int oy = py - 3; oy <= py + 2; oy++)
            for (int ox = px - 3; ox <= px + 2; ox++) {
                if (max(abs(ox), abs(oy)) < 2) continue;
                if ((idx++ % NSLOT) == slot && no < 2) {
                    ox_l[no] = ox;
                    oy_l[no] = oy;
                    no++;
                }
            }
    }
    float acc[NR_];
#pragma unroll
    for (int k = 0; k < NR_; k++) acc[k] = 0.f;
    float m[NR_], mn[NR_];
    auto fetch = [&](int q, float *dst) {
        const int sx = tx - ox_l[q], sy = ty - oy_l[q];
        const bool ok = tvalid && sx >= 0 && sy >= 0 && sx < n && sy < n;
        const float2 *ms = reinterpret_cast<const float2 *>(Mall + (off + (long long)(ok ? sy : 0) * n + (ok ? sx : 0)) * NR_);
#pragma unroll
        for (int v = 0; v < NR_ / 2; v++) {
            const float2 u = ok ? (NC ? __ldg(&ms[v]) : ms[v]) : make_float2(0.f, 0.f);
            dst[2 * v] = u.x;
            dst[2 * v + 1] = u.y;
        }
    };
    if (no > 0) fetch(0, m);
    __syncthreads();
#pragma unroll 1
    for (int q = 0; q < 2; q++) {
        if (q >= no) break;
        if (q + 1 < no) fetch(q + 1, mn);
        const float *T = Ts + ((oy_l[q] + 3) * 7 + (ox_l[q] + 3)) * OSZ;
#pragma unroll
        for (int j = 0; j < NE_; j++) {
            const float2 *row = reinterpret_cast<const float2 *>(T + j * NE_);
#pragma unroll
            for (int v = 0; v < NE_ / 2; v++) {
                const float2 t = row[v];
                acc[2 * v] = fmaf(t.x, m[j], acc[2 * v]);
                acc[2 * v + 1] = fmaf(t.y, m[j], acc[2 * v + 1]);
            }
        }
        T += NE_ * NE_;
#pragma unroll
        for (int j = 0; j < NO_; j++) {
            const float2 *row = reinterpret_cast<const float2 *>(T + j * NO_);
#pragma unroll
            for (int v = 0; v < NO_ / 2; v++) {
                const float2 t = row[v];
                acc[NE_ + 2 * v] = fmaf(t.x, m[NE_ + j], acc[NE_ + 2 * v]);
                acc[NE_ + 2 * v + 1] = fmaf(t.y, m[NE_ + j], acc[NE_ + 2 * v + 1]);
            }
        }
#pragma unroll
        for (int k = 0; k < NR_; k++) m[k] = mn[k];
    }
    // the two halves of the warp hold the same targets: lower + upper
#pragma unroll
    for (int k = 0; k < NR_; k++) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], 16);
    __syncthreads();  // (when red aliases Ts) operators no longer needed
    if (half == 0) {
        float *rw = red + (warp * RES_TPI + tl) * (NR_ + 1);
#pragma unroll
        for (int k = 0; k < NR_; k++) rw[k] = acc[k];
    }
    __syncthreads();
    // fixed-order sum over the warps: thread t handles (target, k) pairs
    for (int e = threadIdx.x; e < RES_TPI * NR_; e += blockDim.x) {
        const int t = e / NR_, k = e % NR_;
        const int tj = it.z + t;
        if (tj >= nh * nh) continue;
        float v = 0.f;
#pragma unroll
        for (int w = 0; w < RES_WARPS; w++) v += red[(w * RES_TPI + t) * (NR_ + 1) + k];
        const int ux = 2 * (tj % nh) + px, uy = 2 * (tj / nh) + py;
        Lout[(off + (long long)uy * n + ux) * NR_ + k] = v;
    }
    __syncthreads();
}

// Registers: at most 112 for NR <= 30 (P <= 4, no spills), so that one CTA
// fits beside two k_p2p CTAs of 288 threads x 64 registers; the near field
// runs concurrently with the M2L and, at 117 registers, the M2L's CTAs waited
// for the near field's to finish.  256 threads per CTA.
// lstride: floats between the operator tables of consecutive levels (tables
// of level l at Tc + (l - 2) lstride); 0 when one table serves every level
// (the spherical-harmonic operators, lengths in box widths).
template <int NR_, int NE_>
__global__ void __maxnreg__(NR_ <= 30 ? 112 : 255) k_m2l_res(const float *__restrict__ Mall, float *__restrict__ Lout,
                                                            const float *__restrict__ Tc, const int4 *__restrict__ items,
                                                            const long long *__restrict__ lev_off, FmmDev f,
                                                            long long lstride)
{
    constexpr int NO_ = NR_ - NE_;
    constexpr int OSZ = NE_ * NE_ + NO_ * NO_;
    extern __shared__ __align__(16) float sr[];
    Tc += (long long)(items[blockIdx.x].x - 2) * lstride;
    // stage the operator table with asynchronous copies: every 16-byte chunk
    // in flight at once instead of one load-store round trip per chunk; the
    // table is constant, so it streams in while the predecessor finishes
    for (int i = threadIdx.x * 4; i < 49 * OSZ; i += blockDim.x * 4)
        umma::cp_async16(umma::smem_u32(&sr[i]), &Tc[i], true);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    pdl_begin();
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    (void)f;
    m2l_res_item<NR_, NE_, true>(Mall, Lout, sr, sr, items[blockIdx.x], lev_off);
}

// one parent box of the downward pass with a group of 4 KT threads: child
// locals = L2L of the parent's final local + the M2L partials; Ts = the 4
// operators in shared memory; Lp = NR floats of the group's shared scratch
__device__ __forceinline__ void l2l_item(float *__restrict__ Lfin, const float *__restrict__ Lpart, const float *Ts,
                                         float *Lp, long long off_p, long long off_c, int nc, int np, int pb,
                                         long long part_stride, int nsplit, const FmmDev &f, int t, int KT,
                                         bool valid = true)
{
    const int NE = f.NE, NO = f.NR - f.NE;
    for (int i = t; valid && i < f.NR; i += 4 * KT) Lp[i] = Lfin[(off_p + pb) * (long long)f.NR + i];
    __syncthreads();
    const int c = t / KT, k = t % KT;
    if (valid && k < f.NR) {
        const int blk = k >= NE, NB = blk ? NO : NE, kk = blk ? k - NE : k, boff = blk ? NE : 0;
        const float *T = Ts + blk_base(c, NE, NO, blk);
        const float *lp = Lp + boff;
        float acc = 0.f;
#pragma unroll 8
        for (int j = 0; j < NB; j++) acc = fmaf(T[j * NB + kk], lp[j], acc);
        const int cx = 2 * (pb % np) + (c & 1), cy = 2 * (pb / np) + (c >> 1);
        const long long b = off_c + (long long)cy * nc + cx;
        float v = acc;
        for (int g = 0; g < nsplit; g++) v += Lpart[g * part_stride + b * f.NR + k];
        Lfin[b * f.NR + k] = v;
    }
    __syncthreads();
}

// level 2 has no far-field parent: its locals are the partial sums alone
__device__ __forceinline__ void l2l_top_box(float *__restrict__ Lfin, const float *__restrict__ Lpart, long long b,
                                            long long part_stride, int nsplit, const FmmDev &f, int t, int nt)
{
    for (int k = t; k < f.NR; k += nt) {
        float v = 0.f;
        for (int g = 0; g < nsplit; g++) v += Lpart[g * part_stride + b * f.NR + k];
        Lfin[b * f.NR + k] = v;
    }
}

// The two top levels in one launch each way (NR <= 32).  CTA = one level-2
// box.  Upward: its four level-3 children (one 4 KT-thread group each, from
// their level-4 children, which are staged with the operators in one wave of
// asynchronous copies), then the box itself from those four, kept in shared
// memory.  Downward: the box's local from its M2L partials, then its four
// level-3 children.  The arithmetic of the per-level kernels, so the same bits.
__global__ void __launch_bounds__(512) k_top_m2m(float *__restrict__ Mall, const float *__restrict__ Tb,
                                                 long long off2, long long off3, long long off4, FmmDev f)
{
    extern __shared__ __align__(16) float smb[];
    const int NE = f.NE, NO = f.NR - f.NE;
    const int tsz = 4 * (NE * NE + NO * NO);
    const int KT = blockDim.x / 16;
    float *Ts = smb;
    const int grp = threadIdx.x / (4 * KT), t = threadIdx.x % (4 * KT);
    float *Mc = Ts + tsz + grp * (4 * f.NR + 4 * KT), *red = Mc + 4 * f.NR;
    float *G = Ts + tsz + 4 * (4 * f.NR + 4 * KT);  // [4][NR]: the level-3 children, child index = grp
    const int P = blockIdx.x;
    const int cx = 2 * (P % 4) + (grp & 1), cy = 2 * (P / 4) + (grp >> 1);
    // the operators are constant: they stream in while the predecessor finishes
    for (int i = threadIdx.x * 4; i < tsz; i += blockDim.x * 4) umma::cp_async16(umma::smem_u32(Ts + i), Tb + i, true);
    pdl_begin();
    for (int i = t; i < 4 * f.NR; i += 4 * KT) {  // the group's four level-4 children
        const int c = i / f.NR, j = i % f.NR;
        cp_async4(Mc + i, Mall + (off4 + (long long)(2 * cy + (c >> 1)) * 16 + 2 * cx + (c & 1)) * f.NR + j, true);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    m2m_reduce(Mall, Ts, Mc, red, off3, cy * 8 + cx, f, t, KT, true, G + grp * f.NR);
    m2m_reduce(Mall, Ts, G, red, off2, P, f, t, KT, grp == 0);
}

// ---- upward pass in one launch (leaf side 8, 3 layers) ----------------------
// The learned far field's encoder and upward pass (NR_ channels, NE_ of them
// even).  The FMM's own P2M + M2M launches stay separate: at P = 4 this one
// launch of 64 CTAs measured 10.9 us in the RK4 step against 10.6 us for
// k_p2m_row (128 CTAs) + k_top_m2m under programmatic launch.
constexpr int UP_THREADS = 384;
constexpr int UP_S = 8, UP_Z = 3, UP_C = UP_S * UP_S * UP_Z;  // leaf box: 8 x 8 cells x 3 layers
constexpr int UP_WP = UP_C + 4;  // weight row pitch in shared memory (floats): conflict-free 16-byte reads

// one output k of a block-diagonal map: sum_j T[blk][j][k] x[j], T one
// operator [even NE_ x NE_ | odd NO x NO] input-major, in the order of
// m2m_reduce's per-child sums
template <int NR_, int NE_>
__device__ __forceinline__ float blk_apply(const float *T, const float *x, int k)
{
    constexpr int NO_ = NR_ - NE_;
    if (k < NE_) {
        float acc = 0.f;
#pragma unroll
        for (int j = 0; j < NE_; j++) acc = fmaf(T[j * NE_ + k], x[j], acc);
        return acc;
    }
    const int kk = k - NE_;
    const float *To = T + NE_ * NE_;
    float acc = 0.f;
#pragma unroll
    for (int j = 0; j < NO_; j++) acc = fmaf(To[j * NO_ + kk], x[NE_ + j], acc);
    return acc;
}

// Leaf multipoles and the whole upward pass.  CTA = one box of level cb =
// max(2, L - 2), i.e. gs x gs leaf boxes (gs = 2^(L - cb) <= 4): their
// charges and the weights W ([NR][C], k-major) are staged in shared memory,
// the leaf multipoles (p2m_dot's four interleaved chains, so the same bits)
// and every level up to cb formed there and written out.  Levels above cb:
// the CTA that completes the fourth child of a box forms that box (an
// arrival counter per box in ctr, reset by that CTA for the next launch;
// writers fence their stores before they arrive, the last arriver fences
// before it reads the siblings through L2), and so on up to level 2.  No CTA
// waits for another.  M2M sums the four children as m2m_reduce does,
// (c0 + c1) + (c2 + c3).  tls: floats between the M2M tables of consecutive
// levels (0: one table for every level).
template <int NR_, int NE_>
__global__ void __launch_bounds__(UP_THREADS) k_up(const float *__restrict__ rho, const float *__restrict__ W,
                                                   const float *__restrict__ Tm2m, long long tls,
                                                   float *__restrict__ Mall, const long long *__restrict__ lev_off,
                                                   unsigned *__restrict__ ctr, FmmDev f, int cb)
{
    constexpr int OSZ = NE_ * NE_ + (NR_ - NE_) * (NR_ - NE_);
    extern __shared__ __align__(16) float usm[];
    const int gs = 1 << (f.L - cb), G = gs * gs, ncb = 1 << cb;
    const int cbx = blockIdx.x % ncb, cby = blockIdx.x / ncb;  // the CTA's box at level cb
    const int bx0 = cbx * gs, by0 = cby * gs;                  // its first leaf box
    const int ntab = tls ? f.L - 2 : 1;
    float *Ws = usm;                       // [NR][UP_WP]: weight rows, padded
    float *Ts = Ws + NR_ * UP_WP;          // M2M tables: [ntab][4][OSZ]
    float *q = Ts + ntab * 4 * OSZ;        // [G][C]
    float *mb = q + G * UP_C;              // multipoles of levels L .. cb, G NR + G/4 NR + ...
    __shared__ int s_last;
    for (int i = threadIdx.x; i < NR_ * UP_C / 4; i += blockDim.x) {
        const int k = i / (UP_C / 4), c4 = i % (UP_C / 4);
        umma::cp_async16(umma::smem_u32(Ws + k * UP_WP + 4 * c4), W + k * UP_C + 4 * c4, true);
    }
    for (int i = threadIdx.x * 4; i < ntab * 4 * OSZ; i += blockDim.x * 4)
        umma::cp_async16(umma::smem_u32(Ts + i), Tm2m + i, true);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    pdl_begin();  // the weights above are constant; the charges are the predecessor's output
    // charges, a region row at a time (consecutive threads on consecutive x);
    // every load of a thread is issued before the first store
    const int rw = gs * UP_S, ne = UP_Z * rw * rw;
    constexpr int QR = (UP_Z * 32 * 32 + UP_THREADS - 1) / UP_THREADS;
    float qv[QR];
#pragma unroll
    for (int r = 0; r < QR; r++) {
        const int e = threadIdx.x + r * blockDim.x;
        const int rx = e % rw, ry = (e / rw) % rw, lz = e / (rw * rw);
        const int x = bx0 * UP_S + rx, y = by0 * UP_S + ry;
        qv[r] = (e < ne && x < f.X && y < f.Y) ? __ldg(&rho[((long long)lz * f.Y + y) * f.X + x]) : 0.f;
    }
#pragma unroll
    for (int r = 0; r < QR; r++) {
        const int e = threadIdx.x + r * blockDim.x;
        if (e >= ne) break;
        const int rx = e % rw, ry = (e / rw) % rw, lz = e / (rw * rw);
        const int b = (ry / UP_S) * gs + rx / UP_S, c = lz * UP_S * UP_S + (ry % UP_S) * UP_S + rx % UP_S;
        q[b * UP_C + c] = qv[r];
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    // leaf multipoles: four interleaved chains per output (p2m_dot's order)
    const long long offL = lev_off[f.L];
    for (int o = threadIdx.x; o < G * NR_; o += blockDim.x) {
        const int b = o / NR_, k = o % NR_;
        const float4 *qb = reinterpret_cast<const float4 *>(q + b * UP_C);
        const float4 *wk = reinterpret_cast<const float4 *>(Ws + k * UP_WP);
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll 8
        for (int c4 = 0; c4 < UP_C / 4; c4++) {
            const float4 wv = wk[c4], qv4 = qb[c4];
            a0 = fmaf(wv.x, qv4.x, a0);
            a1 = fmaf(wv.y, qv4.y, a1);
            a2 = fmaf(wv.z, qv4.z, a2);
            a3 = fmaf(wv.w, qv4.w, a3);
        }
        const float v = (a0 + a1) + (a2 + a3);
        mb[o] = v;
        const int bx = bx0 + b % gs, by = by0 + b / gs;
        Mall[(offL + (long long)by * f.nb + bx) * NR_ + k] = v;
    }
    __syncthreads();
    // levels L-1 .. cb inside the CTA
    const float *child = mb;
    float *par = mb + G * NR_;
    int gc = gs;
    for (int l = f.L - 1; l >= cb; l--) {
        const int gp = gc / 2, n = 1 << l;
        const float *T = Ts + (tls ? (l - 2) : 0) * 4 * OSZ;
        const int px0 = bx0 >> (f.L - l), py0 = by0 >> (f.L - l);
        for (int o = threadIdx.x; o < gp * gp * NR_; o += blockDim.x) {
            const int p = o / NR_, k = o % NR_, px = p % gp, py = p / gp;
            float a[4];
#pragma unroll
            for (int c = 0; c < 4; c++)
                a[c] = blk_apply<NR_, NE_>(T + c * OSZ, child + ((2 * py + (c >> 1)) * gc + 2 * px + (c & 1)) * NR_, k);
            const float v = (a[0] + a[1]) + (a[2] + a[3]);
            par[o] = v;
            Mall[(lev_off[l] + (long long)(py0 + py) * n + px0 + px) * NR_ + k] = v;
        }
        __syncthreads();
        child = par;
        par += gp * gp * NR_;
        gc = gp;
    }
    // levels above cb: the last of four siblings to finish forms the parent
    int bxl = cbx, byl = cby;
    for (int l = cb - 1; l >= 2; l--) {
        __threadfence();  // this CTA's multipoles are visible before it arrives
        __syncthreads();
        const int px = bxl >> 1, py = byl >> 1, n = 1 << l, nc = 2 * n;
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(&ctr[lev_off[l] + (long long)py * n + px], 1u);
            s_last = t == 3;
        }
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        float *sib = mb;  // the four children, read through L2
        for (int i = threadIdx.x; i < 4 * NR_; i += blockDim.x) {
            const int c = i / NR_, k = i % NR_;
            sib[i] = __ldcg(&Mall[(lev_off[l + 1] + (long long)(2 * py + (c >> 1)) * nc + 2 * px + (c & 1)) * NR_ + k]);
        }
        __syncthreads();
        const float *T = Ts + (tls ? (l - 2) : 0) * 4 * OSZ;
        for (int k = threadIdx.x; k < NR_; k += blockDim.x) {
            float a[4];
#pragma unroll
            for (int c = 0; c < 4; c++) a[c] = blk_apply<NR_, NE_>(T + c * OSZ, sib + c * NR_, k);
            Mall[(lev_off[l] + (long long)py * n + px) * NR_ + k] = (a[0] + a[1]) + (a[2] + a[3]);
        }
        if (threadIdx.x == 0) ctr[lev_off[l] + (long long)py * n + px] = 0u;  // ready for the next launch
        bxl = px;
        byl = py;
    }
}

int up_level(int L) { return std::max(2, L - 2); }

// dynamic shared memory of k_up at L levels (ntab M2M tables)
size_t up_smem(int L, int NR, int NE, int ntab)
{
    const int cb = up_level(L), gs = 1 << (L - cb), G = gs * gs;
    const size_t osz = (size_t)NE * NE + (size_t)(NR - NE) * (NR - NE);
    int nm = 0;
    for (int g = G; g >= 1; g /= 4) nm += g;
    return ((size_t)NR * UP_WP + (size_t)ntab * 4 * osz + (size_t)G * UP_C + (size_t)std::max(nm, 4) * NR) *
           sizeof(float);
}


__global__ void __launch_bounds__(128) k_top_l2l(float *__restrict__ Lfin, const float *__restrict__ Lpart,
                                                 const float *__restrict__ Tb, long long off2, long long off3,
                                                 long long part_stride, int nsplit, FmmDev f)
{
    pdl_begin();
    extern __shared__ __align__(16) float smb[];
    const int NE = f.NE, NO = f.NR - f.NE;
    const int tsz = 4 * (NE * NE + NO * NO);
    const int KT = blockDim.x / 4;
    float *Ts = smb, *Lp = smb + tsz;
    stage_async(Ts, Tb, tsz);
    const int P = blockIdx.x;
    l2l_top_box(Lfin, Lpart, off2 + P, part_stride, nsplit, f, threadIdx.x, blockDim.x);
    __syncthreads();
    l2l_item(Lfin, Lpart, Ts, Lp, off2, off3, 8, 4, P, part_stride, nsplit, f, threadIdx.x, KT);
}

// Downward pass of one level: L(child) = sum of the NSPLIT M2L partials of the
// child (fixed order) + L2L of the final parent local.  CTA per parent box,
// thread per (child c, coefficient k); operator blocks and the parent local
// staged in shared memory.  np == 0 is level 2 (CTA per box).
__global__ void k_l2l_c(float *__restrict__ Lfin, const float *__restrict__ Lpart, const float *__restrict__ Tb,
                        long long off_p, long long off_c, int nc, int np, long long part_stride, int nsplit, FmmDev f)
{
    pdl_begin();
    extern __shared__ __align__(16) float smb[];
    const int NE = f.NE, NO = f.NR - f.NE;
    if (np == 0) {
        l2l_top_box(Lfin, Lpart, off_c + blockIdx.x, part_stride, nsplit, f, threadIdx.x, blockDim.x);
        return;
    }
    const int tsz = 4 * (NE * NE + NO * NO);
    const int KT = blockDim.x / 4;
    float *Ts = smb;          // [4][blocks]
    float *Lp = smb + tsz;    // [NR]
    stage_async(Ts, Tb, tsz);
    l2l_item(Lfin, Lpart, Ts, Lp, off_p, off_c, nc, np, blockIdx.x, part_stride, nsplit, f, threadIdx.x, KT);
}

// Fused far field (P <= 4, solver far_mode 1): ONE cooperative launch (one
// CTA per SM, all co-resident) runs P2M, the M2M levels L-1 .. 2, the
// resident M2L of every level and the L2L levels 2 .. L-1, with a grid
// barrier between dependent phases, instead of 2 L - 1 short launches.  At
// 256 x 256 x 3 it measured slower than the per-stage launches (9 barriers
// and thinly filled upper-level phases cost more than the launches they
// save, and its shared memory keeps the concurrent near field off the SMs),
// so it is an option, not the default.  Each CTA keeps the M2M, L2L and
// all 49 M2L operator slots in shared memory; the M2L table streams in with
// cp.async while the upward pass runs.  Every item runs the same code (and
// summation order) as the per-stage kernels, so both paths give identical
// bits.  Data written inside the launch is read with ordinary loads after the
// barrier's gpu-scope acquire, never through the non-coherent (ld.global.nc)
// path.
}  // namespace

struct FarSync {
    unsigned count;  // CTAs arrived at the current barrier (returns to 0)
    unsigned gen;    // barrier generation
    int err;         // 1: a barrier wait timed out
    int pad;
};

namespace {

constexpr long long BARRIER_CYCLES = 2000000000LL;  // ~1 s

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// all CTAs of the (cooperative) grid; bounded: a wait longer than ~1 s sets
// sy->err and returns
__device__ void grid_barrier(FarSync *sy)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned g = ld_acquire_u32(&sy->gen);
        __threadfence();
        if (atomicAdd(&sy->count, 1u) == gridDim.x - 1) {
            atomicExch(&sy->count, 0u);
            __threadfence();
            atomicAdd(&sy->gen, 1u);
        } else {
            const long long t0 = clock64();
            while (ld_acquire_u32(&sy->gen) == g) {
                if (clock64() - t0 > BARRIER_CYCLES) {
                    atomicExch(&sy->err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <int NR_>
__host__ __device__ constexpr int far_kt() { return ((NR_ + 31) / 32) * 32; }

template <int NR_, int NE_>
constexpr int far_scratch(int C)
{
    constexpr int KT = far_kt<NR_>();
    constexpr int G = (32 * RES_WARPS) / (4 * KT);
    const int a = C * BB, b = RES_WARPS * RES_TPI * (NR_ + 1), c = G * (4 * NR_ + 4 * KT + NR_);
    return a > b ? (a > c ? a : c) : (b > c ? b : c);
}

template <int NR_, int NE_>
__global__ void __launch_bounds__(32 * RES_WARPS) k_far(const float *__restrict__ rho, const float *__restrict__ Wg,
                                                        float *__restrict__ Mall, float *__restrict__ Lpart,
                                                        float *__restrict__ Lall, const float *__restrict__ Tm2m,
                                                        const float *__restrict__ Tm2lc,
                                                        const float *__restrict__ Tl2l, const int4 *__restrict__ items,
                                                        int nitems, const long long *__restrict__ lev_off, FmmDev f,
                                                        int nbx, int nby, int lend, FarSync *sy)
{
    constexpr int NO_ = NR_ - NE_;
    constexpr int OSZ = NE_ * NE_ + NO_ * NO_;
    constexpr int KT = far_kt<NR_>();
    constexpr int G = (32 * RES_WARPS) / (4 * KT);  // parent boxes per pass in M2M / L2L
    static_assert((49 * OSZ) % 4 == 0 && G >= 1, "operator table must be whole float4s");
    extern __shared__ __align__(16) float sf[];
    float *Tl = sf;                 // [49][OSZ] M2L
    float *Tu = Tl + 49 * OSZ;      // [4 OSZ]  M2M
    float *Td = Tu + 4 * OSZ;       // [4 OSZ]  L2L
    float *scr = Td + 4 * OSZ;      // P2M charges | M2L reduction | per-group M2M/L2L scratch
    const int tid = threadIdx.x;
    for (int i = tid * 4; i < 49 * OSZ; i += blockDim.x * 4)
        umma::cp_async16(umma::smem_u32(Tl + i), Tm2lc + i, true);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    // synchronous: the M2L table's asynchronous copies stay in flight meanwhile
    for (int i = tid * 4; i < 4 * OSZ; i += blockDim.x * 4) {
        *reinterpret_cast<float4 *>(&Tu[i]) = __ldg(reinterpret_cast<const float4 *>(&Tm2m[i]));
        *reinterpret_cast<float4 *>(&Td[i]) = __ldg(reinterpret_cast<const float4 *>(&Tl2l[i]));
    }
    __syncthreads();
    const int grp = tid / (4 * KT), t = tid % (4 * KT);
    float *Mc = scr + grp * (4 * NR_ + 4 * KT + NR_);  // group scratch: [4 NR] children, [4 KT] partials
    float *red = Mc + 4 * NR_;
    float *Lp = red + 4 * KT;                           // [NR] parent local (L2L)

    // P2M: items of BB leaf boxes along a row
    const int rowitems = (nbx + BB - 1) / BB;
    for (int it = blockIdx.x; it < rowitems * nby; it += gridDim.x)
        p2m_item(rho, Wg, scr, Mall + lev_off[f.L] * NR_, f, it / rowitems, (it % rowitems) * BB);
    grid_barrier(sy);
    // M2M: level L-1 .. 2
    for (int l = f.L - 1; l >= 2; l--) {
        const int np = 1 << l;
        for (int base = blockIdx.x * G; base < np * np; base += gridDim.x * G) {
            const int box = base + grp;
            m2m_item(Mall, Tu, Mc, red, lev_off[l], lev_off[l + 1], np, box, f, t, KT, grp < G && box < np * np);
        }
        grid_barrier(sy);
    }
    // M2L, every level
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) m2l_res_item<NR_, NE_, false>(Mall, Lpart, Tl, scr, items[it], lev_off);
    // L2L: level 2 from its partials, then 3 .. lend
    if (lend >= 2) {
        grid_barrier(sy);
        for (int b = blockIdx.x; b < 16; b += gridDim.x) l2l_top_box(Lall, Lpart, lev_off[2] + b, 0, 1, f, tid, blockDim.x);
        for (int l = 3; l <= lend; l++) {
            grid_barrier(sy);
            const int nc = 1 << l, np = nc / 2;
            for (int base = blockIdx.x * G; base < np * np; base += gridDim.x * G) {
                const int pb = base + grp;
                l2l_item(Lall, Lpart, Td, Lp, lev_off[l - 1], lev_off[l], nc, np, pb, 0, 1, f, t, KT,
                         grp < G && pb < np * np);
            }
        }
    }
}

// Leaf kernels.  The near field (P2P) needs only the charges, so it runs on a
// side stream concurrently with the far-field chain (P2M .. L2L); the L2P
// kernel joins the two.
//
// k_p2p: exact near field.  CTA = BB leaf boxes of one row; G thread groups,
// each thread = (group, box, target row y, layer z) holding the S targets of
// its row in registers.  Group g takes the g-th third of the neighbourhood's
// source rows (G = 3: one source box row each); for every source row the
// thread loads the 3S charges and the 2S-entry near-field row G[|dz|][|dy|][.]
// into registers and does 3S x S FMAs with compile-time indices |S + i - j|.
// The groups' partial sums are added in group order through shared memory.
template <int S, int BB, int G>
__global__ void __launch_bounds__(512) k_p2p(const float *__restrict__ rho, const float *__restrict__ Gn,
                                              float *__restrict__ out, FmmDev f)
{
    extern __shared__ __align__(16) float sl[];
    const int Z = f.Z;
    constexpr int W = (BB + 2) * S;        // charges per staged row
    float *qn = sl;                        // [Z][3S][W]
    float *g = qn + Z * 3 * S * W;         // [Z][2S][2S]
    __shared__ int nzr[384];               // staged source row (z, y) holds charge; Z 3S <= 384 whenever BB S Z <= 512
    static_assert(W % 4 == 0, "staged rows are scanned as float4");
    const int by = blockIdx.y, bx0 = blockIdx.x * BB;
    const int xs0 = bx0 * S - S, ys0 = by * S - S;
    // charges (zero-filled off the grid) and the near-field table all in
    // flight at once, then one scan per staged row for charge
    for (int i = threadIdx.x; i < Z * 3 * S * W; i += blockDim.x) {
        const int xx = xs0 + i % W, yy = ys0 + (i / W) % (3 * S), zz = i / (W * 3 * S);
        const bool ok = xx >= 0 && yy >= 0 && xx < f.X && yy < f.Y;
        cp_async4(qn + i, ok ? rho + ((long long)zz * f.Y + yy) * f.X + xx : rho, ok);
    }
    for (int i = threadIdx.x * 4; i < Z * 4 * S * S; i += blockDim.x * 4)
        umma::cp_async16(umma::smem_u32(g + i), Gn + i, true);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    for (int i = threadIdx.x; i < Z * 3 * S; i += blockDim.x) {
        const float4 *rw = reinterpret_cast<const float4 *>(qn + i * W);
        bool nz = false;
#pragma unroll
        for (int v = 0; v < W / 4; v++) {
            const float4 u = rw[v];
            nz |= (u.x != 0.f) | (u.y != 0.f) | (u.z != 0.f) | (u.w != 0.f);
        }
        nzr[i] = nz;
    }
    __syncthreads();
    const int nt = BB * S * Z;
    const int grp = threadIdx.x / nt, t = threadIdx.x % nt;
    const int b = t / (S * Z), r = t % (S * Z);
    const int ly = r % S, lz = r / S;
    float acc[S];
#pragma unroll
    for (int i = 0; i < S; i++) acc[i] = 0.f;
    constexpr int RG = 3 * S / G;  // source rows per group
    for (int zs = 0; zs < Z; zs++) {
        const int dz = abs(zs - lz);
        for (int ys = grp * RG; ys < (grp + 1) * RG; ys++) {
            if (!nzr[zs * 3 * S + ys]) continue;  // no charge in this source row (uniform per warp)
            const int dy = abs(ys - ly - S);
            const float *grow = g + (dz * 2 * S + dy) * 2 * S;
            const float *qrow = qn + (zs * 3 * S + ys) * W + b * S;
            float gr[2 * S], qr[3 * S];
            if constexpr (S % 4 == 0) {
#pragma unroll
                for (int v = 0; v < 2 * S / 4; v++) {
                    const float4 u = reinterpret_cast<const float4 *>(grow)[v];
                    gr[4 * v] = u.x; gr[4 * v + 1] = u.y; gr[4 * v + 2] = u.z; gr[4 * v + 3] = u.w;
                }
#pragma unroll
                for (int v = 0; v < 3 * S / 4; v++) {
                    const float4 u = reinterpret_cast<const float4 *>(qrow)[v];
                    qr[4 * v] = u.x; qr[4 * v + 1] = u.y; qr[4 * v + 2] = u.z; qr[4 * v + 3] = u.w;
                }
            } else {
#pragma unroll
                for (int v = 0; v < 2 * S; v++) gr[v] = grow[v];
#pragma unroll
                for (int v = 0; v < 3 * S; v++) qr[v] = qrow[v];
            }
#pragma unroll
            for (int j = 0; j < 3 * S; j++)
#pragma unroll
                for (int i = 0; i < S; i++) {
                    const int d = (S + i - j) < 0 ? (j - S - i) : (S + i - j);
                    acc[i] = fmaf(qr[j], gr[d], acc[i]);
                }
        }
    }
    if constexpr (G > 1) {
        float *red = g + Z * 4 * S * S;  // [G-1][S][nt]
        if (grp > 0)
#pragma unroll
            for (int i = 0; i < S; i++) red[((grp - 1) * S + i) * nt + t] = acc[i];
        __syncthreads();
        if (grp > 0) return;
        for (int gg = 1; gg < G; gg++)
#pragma unroll
            for (int i = 0; i < S; i++) acc[i] += red[((gg - 1) * S + i) * nt + t];
    }
    const int y = by * S + ly;
    if (bx0 + b >= f.nb || y >= f.Y) return;
    float *o = out + ((long long)lz * f.Y + y) * f.X + (long long)(bx0 + b) * S;
    if (S % 4 == 0 && (f.X & 3) == 0 && (bx0 + b) * S + S <= f.X) {  // 16-byte stores
#pragma unroll
        for (int v4 = 0; v4 < S / 4; v4++)
            reinterpret_cast<float4 *>(o)[v4] = make_float4(acc[4 * v4], acc[4 * v4 + 1], acc[4 * v4 + 2], acc[4 * v4 + 3]);
        return;
    }
#pragma unroll
    for (int i = 0; i < S; i++)
        if ((bx0 + b) * S + i < f.X) o[i] = acc[i];
}

// k_l2p: leaf locals (the leaf level's L2L: NSPLIT-summed M2L partials plus
// the L2L of the parent's final local, none when the leaf level is 2), then
// phi = near field + sum_k V[k][cell] L[k].  Same thread layout as k_p2p.
// The parents' final locals (level L-1) come, by pmode:
//   0  none (leaf level 2)
//   1  ready in Lpar (an L2L pass formed them)
//   2  formed here: L2L of the grandparents' final locals (Lgp, level L-2)
//      plus the parents' M2L partials (Lpp), the order of the L2L pass
//   3  formed here from the parents' partials alone (parent level 2)
//   4  as 2, with the grandparents' final locals formed here too: levels
//      2 .. L-2 of the CTA's ancestors from their M2L partials (Lpart_all,
//      lev_off), in the order of l2l_top_box / l2l_item, so no L2L launch
//      precedes L2P
template <int S, int BB, int G>
__global__ void __launch_bounds__(512) k_l2p(const float *__restrict__ near, const float *__restrict__ Lpart_leaf,
                                              const float *__restrict__ Lpar, const float *__restrict__ Tl2l,
                                              const float *__restrict__ Vt, float *__restrict__ phi, FmmDev f,
                                              long long part_stride, int nsplit, int pmode,
                                              const float *__restrict__ Lgp, const float *__restrict__ Lpp,
                                              int nnear, long long near_stride, const float *__restrict__ Lpart_all,
                                              const long long *__restrict__ lev_off)
{
    extern __shared__ __align__(16) float sl[];
    const int Z = f.Z;
    const int NE = f.NE, NO = f.NR - f.NE;
    constexpr int GB = BB >= 4 ? BB / 4 : 1;          // grandparents under the CTA's BB leaves
    float *Ts = sl;                                   // L2L operator blocks
    float *Lb = Ts + 4 * (NE * NE + NO * NO);         // [BB][NR] leaf locals
    float *Lp = Lb + BB * f.NR;                       // [BB/2][NR] parent locals
    float *Lg = Lp + (BB / 2) * f.NR;                 // [GB][NR] grandparent locals
    const int by = blockIdx.y, bx0 = blockIdx.x * BB;
    const int haspar = pmode != 0;
    const int np = f.nb >> 1, prow = by >> 1;
    // every global read that does not depend on another goes out first: the
    // L2L operators (cp.async), the grandparents' locals, partial 0 of this
    // thread's first parent and leaf M2L partials and its near-field values
    // (registers); the sums below keep their order (operator term, then
    // partial 0, 1, ..)
    if (haspar) {
        const int tsz = 4 * (NE * NE + NO * NO);
        for (int i = threadIdx.x * 4; i < tsz; i += blockDim.x * 4)
            umma::cp_async16(umma::smem_u32(Ts + i), Tl2l + i, true);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    pdl_begin();  // the operators above are constant; what follows is the predecessors' output
    float ppre, lpre;  // partial 0 of this thread's first parent and leaf item
    // pmode 4: partial 0 of this thread's ancestor item at levels 2 .. 4 (the
    // item the level loop below gives it when GB NR <= blockDim)
    constexpr int NPF = 3;
    float apre[NPF];
#pragma unroll
    for (int u = 0; u < NPF; u++) {
        apre[u] = 0.f;
        const int l = 2 + u, i = threadIdx.x;
        if (pmode == 4 && l <= f.L - 2 && i < GB * f.NR && nsplit > 0) {
            const int sh = f.L - l, ax = (bx0 >> sh) + i / f.NR;
            if (ax <= (min(bx0 + BB, f.nb) - 1) >> sh)
                apre[u] = Lpart_all[(lev_off[l] + (long long)(by >> sh) * (1 << l) + ax) * f.NR + i % f.NR];
        }
    }
    {
        const int i = threadIdx.x;
        const int pc = (bx0 >> 1) + i / f.NR, k = i % f.NR;
        const bool okp = pmode >= 2 && i < (BB / 2) * f.NR && pc < np && nsplit > 0;
        const bool okl = i < BB * f.NR && bx0 + i / f.NR < f.nb && nsplit > 0;
        ppre = okp ? Lpp[((long long)prow * np + pc) * f.NR + k] : 0.f;
        lpre = okl ? Lpart_leaf[((long long)by * f.nb + bx0 + i / f.NR) * f.NR + k] : 0.f;
    }
    const int nt = BB * S * Z;
    const int grp = threadIdx.x / nt, t = threadIdx.x % nt;
    const int b = t / (S * Z), r = t % (S * Z);
    const int ly = r % S, lz = r / S;
    const int y = by * S + ly;
    const bool valid = bx0 + b < f.nb && y < f.Y;
    const long long row = ((long long)lz * f.Y + y) * f.X + (long long)(bx0 + b) * S;
    float acc[S];
    // 16-byte accesses where the row of S cells lies inside the grid on a 16-byte boundary
    const bool vec = S % 4 == 0 && (f.X & 3) == 0 && (bx0 + b) * S + S <= f.X;
    // near field, in parts for k_p2p_tc (one per source box row) added in order
    for (int q = 0; q < nnear; q++) {
        const float *nq = near + q * near_stride + row;
        if (vec) {
#pragma unroll
            for (int v4 = 0; v4 < S / 4; v4++) {
                const float4 u = (valid && grp == 0) ? reinterpret_cast<const float4 *>(nq)[v4] : make_float4(0.f, 0.f, 0.f, 0.f);
                if (q == 0) {
                    acc[4 * v4] = u.x; acc[4 * v4 + 1] = u.y; acc[4 * v4 + 2] = u.z; acc[4 * v4 + 3] = u.w;
                } else {
                    acc[4 * v4] += u.x; acc[4 * v4 + 1] += u.y; acc[4 * v4 + 2] += u.z; acc[4 * v4 + 3] += u.w;
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < S; i++) {
                const float u = (valid && grp == 0 && (bx0 + b) * S + i < f.X) ? nq[i] : 0.f;
                acc[i] = q == 0 ? u : acc[i] + u;
            }
        }
    }
    if (pmode == 1) {
        for (int i = threadIdx.x; i < (BB / 2) * f.NR; i += blockDim.x) {
            const int pb = (bx0 >> 1) + i / f.NR;
            Lp[i] = (pb < np) ? Lpar[((long long)prow * np + pb) * f.NR + i % f.NR] : 0.f;
        }
    } else if (pmode == 2) {
        const int ng = np >> 1, g0 = bx0 >> 2;
        for (int i = threadIdx.x; i < GB * f.NR; i += blockDim.x) {
            const int gc = g0 + i / f.NR;
            Lg[i] = (gc < ng) ? Lgp[((long long)(prow >> 1) * ng + gc) * f.NR + i % f.NR] : 0.f;
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    if (pmode == 4) {
        // ancestors of the CTA's leaves at levels 2 .. L-2 (at most GB per
        // level), each level from the one above; Lb is free until the leaf
        // locals and holds the intermediate levels, level L-2 ends in Lg
        float *cur = Lb, *nxt = Lb + GB * f.NR;
        int ax0p = 0;
        for (int l = 2; l <= f.L - 2; l++) {
            const int sh = f.L - l, n = 1 << l;
            const int ax0 = bx0 >> sh, ax1 = (min(bx0 + BB, f.nb) - 1) >> sh, ay = by >> sh;
            float *dst = (l == f.L - 2) ? Lg : nxt;
            for (int i = threadIdx.x; i < GB * f.NR; i += blockDim.x) {
                const int ax = ax0 + i / f.NR, k = i % f.NR;
                float v = 0.f;
                if (ax <= ax1) {
                    const long long box = lev_off[l] + (long long)ay * n + ax;
                    if (l > 2) {
                        const int c = (ax & 1) | ((ay & 1) << 1);
                        const int blk = k >= NE, NB = blk ? NO : NE, kk = blk ? k - NE : k, boff = blk ? NE : 0;
                        const float *T = Ts + blk_base(c, NE, NO, blk);
                        const float *lp = cur + ((ax >> 1) - ax0p) * f.NR + boff;
                        float a2 = 0.f;
#pragma unroll 8
                        for (int j = 0; j < NB; j++) a2 = fmaf(T[j * NB + kk], lp[j], a2);
                        v = a2;
                    }
                    for (int q = 0; q < nsplit; q++) {
                        float pq;
                        if (q == 0 && i == (int)threadIdx.x && l - 2 < NPF) {
                            pq = apre[0];
#pragma unroll
                            for (int u = 1; u < NPF; u++)
                                if (l - 2 == u) pq = apre[u];
                        } else {
                            pq = Lpart_all[q * part_stride + box * f.NR + k];
                        }
                        v += pq;
                    }
                }
                dst[i] = v;
            }
            __syncthreads();
            nxt = cur;
            cur = dst;
            ax0p = ax0;
        }
    }
    if (pmode >= 2) {
        const int g0 = bx0 >> 2;
        for (int i = threadIdx.x; i < (BB / 2) * f.NR; i += blockDim.x) {
            const int pc = (bx0 >> 1) + i / f.NR, k = i % f.NR;
            float v = 0.f;
            if (pc < np) {
                if (pmode == 2 || pmode == 4) {
                    const int c = (pc & 1) | ((prow & 1) << 1);
                    const int blk = k >= NE, NB = blk ? NO : NE, kk = blk ? k - NE : k, boff = blk ? NE : 0;
                    const float *T = Ts + blk_base(c, NE, NO, blk);
                    const float *lg = Lg + ((pc >> 1) - g0) * f.NR + boff;
                    float a2 = 0.f;
#pragma unroll 8
                    for (int j = 0; j < NB; j++) a2 = fmaf(T[j * NB + kk], lg[j], a2);
                    v = a2;
                }
                const long long pbox = (long long)prow * np + pc;
                for (int q = 0; q < nsplit; q++)
                    v += (q == 0 && i == (int)threadIdx.x) ? ppre : Lpp[q * part_stride + pbox * f.NR + k];
            }
            Lp[i] = v;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < BB * f.NR; i += blockDim.x) {
        const int bb = i / f.NR, k = i % f.NR;
        float v = 0.f;
        if (bx0 + bb < f.nb) {
            const long long box = (long long)by * f.nb + bx0 + bb;
            if (haspar) {
                const int c = ((bx0 + bb) & 1) | ((by & 1) << 1);
                const int blk = k >= NE, NB = blk ? NO : NE, kk = blk ? k - NE : k, boff = blk ? NE : 0;
                const float *T = Ts + blk_base(c, NE, NO, blk);
                const float *lp = Lp + (bb >> 1) * f.NR + boff;
                for (int j = 0; j < NB; j++) v = fmaf(T[j * NB + kk], lp[j], v);
            }
            for (int q = 0; q < nsplit; q++)
                v += (q == 0 && i == (int)threadIdx.x) ? lpre : Lpart_leaf[q * part_stride + box * f.NR + k];
        }
        Lb[i] = v;
    }
    __syncthreads();
    // G thread groups: group g evaluates coefficients [k0, k1) of every target
    const float *Lbb = Lb + b * f.NR;
    const int c0 = lz * S * S + ly * S;
    const int k0 = grp * f.NR / G, k1 = valid ? (grp + 1) * f.NR / G : k0;
#pragma unroll 4
    for (int k = k0; k < k1; k++) {
        const float lk = Lbb[k];
        const float *vrow = Vt + (long long)k * f.C + c0;
        if constexpr (S % 4 == 0) {
#pragma unroll
            for (int v = 0; v < S / 4; v++) {
                const float4 u = __ldg(reinterpret_cast<const float4 *>(vrow) + v);
                acc[4 * v + 0] = fmaf(u.x, lk, acc[4 * v + 0]);
                acc[4 * v + 1] = fmaf(u.y, lk, acc[4 * v + 1]);
                acc[4 * v + 2] = fmaf(u.z, lk, acc[4 * v + 2]);
                acc[4 * v + 3] = fmaf(u.w, lk, acc[4 * v + 3]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < S; i++) acc[i] = fmaf(__ldg(&vrow[i]), lk, acc[i]);
        }
    }
    if constexpr (G > 1) {
        __syncthreads();  // the leaf locals are no longer read: Lb .. becomes [G-1][S][nt]
        float *red = Lb;
        if (grp > 0)
#pragma unroll
            for (int i = 0; i < S; i++) red[((grp - 1) * S + i) * nt + t] = acc[i];
        __syncthreads();
        if (grp > 0) return;
        for (int gg = 1; gg < G; gg++)
#pragma unroll
            for (int i = 0; i < S; i++) acc[i] += red[((gg - 1) * S + i) * nt + t];
    }
    if (!valid) return;
    if (vec) {
#pragma unroll
        for (int v4 = 0; v4 < S / 4; v4++)
            reinterpret_cast<float4 *>(phi + row)[v4] = make_float4(acc[4 * v4], acc[4 * v4 + 1], acc[4 * v4 + 2], acc[4 * v4 + 3]);
        return;
    }
#pragma unroll
    for (int i = 0; i < S; i++)
        if ((bx0 + b) * S + i < f.X) phi[row + i] = acc[i];
}

// ---- tensor-core M2L ------------------------------------------------------
// Gather: row r (a target box of one parity class at one level) of A'_b gets,
// for each of the class's 27 offsets q, the source multipole block b
// (NB floats, zero when the source is off the grid) split into BF16 hi and
// lo, laid out [hi | hi | lo] over K = 3 * 27 * NBp.  A grouped tcgen05 GEMM
// then forms sum_q S_q T_q^T from hi*hi + hi*lo + lo*hi in one K sweep
// (relative error ~2^-16 of each product: the split recovers far more than
// BF16 alone, below the FMM truncation error for P <= 6).
__global__ void k_m2l_gather(const float *__restrict__ Mall, __nv_bfloat16 *__restrict__ A0,
                             __nv_bfloat16 *__restrict__ A1, const int4 *__restrict__ rowinfo,
                             const long long *__restrict__ lev_off, FmmDev f, int rows, int K0, int K1, int NBp0,
                             int NBp1)
{
    // the 27 offsets of each parity class in the order the operators were
    // packed (6 x 6 around the parity position minus the 3 x 3 near block)
    __shared__ int sox[4][27], soy[4][27];
    if (threadIdx.x < 4) {
        const int px = threadIdx.x & 1, py = threadIdx.x >> 1;
        int cnt = 0;
        for (int yy = 0; yy < 6; yy++)
            for (int xx = 0; xx < 6; xx++) {
                const int dx = px - 3 + xx, dy = py - 3 + yy;
                if (max(abs(dx), abs(dy)) < 2) continue;
                sox[threadIdx.x][cnt] = dx;
                soy[threadIdx.x][cnt] = dy;
                cnt++;
            }
    }
    __syncthreads();
    const int blk = blockIdx.y;
    const int NB = blk ? f.NR - f.NE : f.NE, NBp = blk ? NBp1 : NBp0, K = blk ? K1 : K0;
    const int boff = blk ? f.NE : 0;
    __nv_bfloat16 *A = blk ? A1 : A0;
    // one thread per run of 8 coefficients of one offset: 16-byte stores of
    // hi, hi and lo (NBp and K are multiples of 8, rows start 16-B aligned)
    const int cpq = NBp >> 3, per_row = 27 * cpq;
    const long long total = (long long)rows * per_row;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e / per_row), c = (int)(e % per_row);
        const int q = c / cpq, j0 = (c % cpq) * 8;
        const int4 ri = rowinfo[r];
        const int lev = ri.x, par = ri.y & 3, t = ri.z;
        const int n = 1 << lev, nh = n >> 1;
        const int tx = 2 * (t % nh) + (par & 1), ty = 2 * (t / nh) + (par >> 1);
        const int sx = tx - sox[par][q], sy = ty - soy[par][q];
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = 0.f;
        if (sx >= 0 && sy >= 0 && sx < n && sy < n) {
            const float *src = Mall + (lev_off[lev] + (long long)sy * n + sx) * f.NR + boff + j0;
#pragma unroll
            for (int i = 0; i < 8; i++)
                if (j0 + i < NB) v[i] = __ldg(src + i);
        }
        __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            hi[i] = __float2bfloat16_rn(v[i]);
            lo[i] = __float2bfloat16_rn(v[i] - __bfloat162float(hi[i]));
        }
        __nv_bfloat16 *row = A + (long long)r * 3 * K + q * NBp + j0;
        *reinterpret_cast<uint4 *>(row) = *reinterpret_cast<const uint4 *>(hi);
        *reinterpret_cast<uint4 *>(row + K) = *reinterpret_cast<const uint4 *>(hi);
        *reinterpret_cast<uint4 *>(row + 2 * K) = *reinterpret_cast<const uint4 *>(lo);
    }
}

// ---- tensor-core near field (leaf side 8) ----------------------------------
// Translation invariance: for a source box offset (dx, dy) in {-1, 0, 1}^2 the
// near-field coupling of a leaf box's C = 64 Z cells to its neighbour's is one
// fixed C x C matrix T_(dx,dy), built from the near-field table Gn.  For one
// offset the near field of every leaf box is a GEMM:
//   phi_(dx,dy)[box][t] = sum_s R[box + (dx, dy)][s] T_(dx,dy)[t][s].
// Both operands are split into BF16 hi + lo and the tensor cores add
// R_hi T_hi + R_lo T_hi + R_hi T_lo in FP32 (relative error ~2^-16 per
// product).  CTA = 4 x 32 boxes x one source box row dy x half of the target
// cells: M = 128 boxes, N = C / 2 target cells (<= 128), K = 3 C in steps of
// one (dx, source layer); each operand tile is one TMA copy in the
// 128-byte-swizzled layout the MMA reads: the charges from box-major BF16
// hi / lo copies of rho (one leaf box layer = one 128-byte row), the operator
// rows from T.  The three source box rows' partials go to separate buffers
// that L2P adds in a fixed order.  Few CTAs (six per 128 boxes), so the
// far-field chain that runs beside it keeps most SMs.
// pipeline stages: four (one more step in flight per SM) where 4 x (A + B
// tiles) fits in shared memory, three at C = 256
template <int BN>
__host__ __device__ constexpr int ntc_stages() { return BN <= 192 ? 4 : 3; }

// BN = C target cells of a box; a CTA takes half of them (N = BN / 2)
template <int BN>
struct NtcSmem {
    alignas(1024) uint8_t ahi[ntc_stages<BN>()][umma::BM * 128];
    alignas(1024) uint8_t alo[ntc_stages<BN>()][umma::BM * 128];
    alignas(1024) uint8_t bhi[ntc_stages<BN>()][(BN / 2) * 128];
    alignas(1024) uint8_t blo[ntc_stages<BN>()][(BN / 2) * 128];
    uint64_t full[ntc_stages<BN>()];  // the stage's four TMA copies landed
    uint64_t done[ntc_stages<BN>()];  // the MMAs reading the stage finished
    uint32_t tmem;
    int err;
    int last;                   // last step whose MMAs were committed (-1: none)
};

__device__ int g_p2p_tc_err;

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(umma::smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// TMA tile loads into this CTA's shared memory, completing on an mbarrier
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, int c0, int c1, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            umma::smem_u32(dst)),
        "l"((uint64_t)tm), "r"(c0), "r"(c1), "r"(umma::smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2, int c3,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(umma::smem_u32(dst)),
        "l"((uint64_t)tm), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(umma::smem_u32(bar))
        : "memory");
}

// zero-padded BF16 hi / lo copies of rho, box-major: [Z][nby][nbx][8 y][8 x],
// so that one layer of one leaf box is one 128-byte row of a TMA tile
__global__ void k_rho_split(const float *__restrict__ rho, __nv_bfloat16 *__restrict__ hi,
                            __nv_bfloat16 *__restrict__ lo, FmmDev f, int nbx, int nby)
{
    pdl_begin();
    const int n = f.Z * nby * nbx * 64;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int bz = i >> 6, box = bz % (nbx * nby), z = bz / (nbx * nby);
        const int x = (box % nbx) * 8 + (i & 7), y = (box / nbx) * 8 + ((i >> 3) & 7);
        const float v = (x < f.X && y < f.Y) ? rho[((long long)z * f.Y + y) * f.X + x] : 0.f;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        hi[i] = h;
        lo[i] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

// T'[dy][t][k'] for t < C, k' = part * 3C + dx * C + cell; part 0 hi, 1 lo
__global__ void k_build_ntc(const float *__restrict__ Gn, __nv_bfloat16 *__restrict__ T, int Z)
{
    const int C = 64 * Z, K3 = 3 * C, Kp = 2 * K3;
    const long long n = 3LL * C * Kp;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int kp = (int)(i % Kp), t = (int)((i / Kp) % C), dy = (int)(i / ((long long)Kp * C)) - 1;
        const int rem = kp % K3, dxo = rem / C - 1, sc = rem % C;
        const int tz = t >> 6, ty = (t >> 3) & 7, tx = t & 7;
        const int sz = sc >> 6, sy = (sc >> 3) & 7, sx = sc & 7;
        const int ax = abs(tx - sx - 8 * dxo), ay = abs(ty - sy - 8 * dy), az = abs(tz - sz);
        const float g = Gn[(az * 16 + ay) * 16 + ax];
        const __nv_bfloat16 hi = __float2bfloat16_rn(g);
        T[i] = (kp / K3 == 1) ? __float2bfloat16_rn(g - __bfloat162float(hi)) : hi;
    }
}

template <int BN>
size_t ntc_smem() { return 1024 + sizeof(NtcSmem<BN>); }

constexpr int NTC_TW = 32, NTC_TH = 4;  // CTA tile: 4 box rows x 32 boxes = the MMA's 128 rows

// grid (ceil(nbx / 32) x ceil(nby / 4), 3 dy, 2 halves of the target cells); 128 threads; BN = C = 64 Z.
// Each CTA sums, for its 4 x 32 boxes, the source boxes in box row dy: one
// step per (dx, source layer sz) brings in four TMA tiles (the source boxes'
// layer-sz charges hi and lo, from the box-major copies, off-grid boxes read
// as zero; the operator columns hi and lo of (dx, sz)) and issues R_hi T_hi
// + R_lo T_hi + R_hi T_lo.  Its partial goes to [3 dy][N].  Thread 0 keeps
// ntc_stages<BN>() steps in flight and issues the MMAs.
template <int BN>
__global__ void __launch_bounds__(128) k_p2p_tc(const __grid_constant__ CUtensorMap tm_hi,
                                                const __grid_constant__ CUtensorMap tm_lo,
                                                const __grid_constant__ CUtensorMap tm_T, float *__restrict__ near3,
                                                FmmDev f, int nbx, int nby, long long ncell)
{
    pdl_begin();
    extern __shared__ uint8_t raw_ntc[];
    uint8_t *base = (uint8_t *)(((uintptr_t)raw_ntc + 1023) & ~(uintptr_t)1023);
    NtcSmem<BN> &s = *reinterpret_cast<NtcSmem<BN> *>(base);
    constexpr int C = BN, K3 = 3 * C, NH = BN / 2;     // NH target cells per CTA
    constexpr int NS = ntc_stages<BN>();
    constexpr int TCOLS = NH <= 32 ? 32 : NH <= 64 ? 64 : NH <= 128 ? 128 : 256;  // allocation: a power of two
    constexpr uint32_t TX = 2 * (umma::BM + NH) * 128;  // bytes per step
    const int nk = 3 * f.Z;                             // steps: (dx, source layer)
    const int colt = (nbx + NTC_TW - 1) / NTC_TW;
    const int bx0 = (blockIdx.x % colt) * NTC_TW, by0 = (blockIdx.x / colt) * NTC_TH;
    const int dyi = blockIdx.y, t0 = blockIdx.z * NH;  // target cells t0 .. t0 + NH - 1
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float *out = near3 + (long long)dyi * ncell;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(umma::smem_u32(&s.tmem)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < NS; i++) {
            umma::mbar_init(&s.full[i]);
            umma::mbar_init(&s.done[i]);
        }
        s.err = 0;
        s.last = -1;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = s.tmem;
    if (tid == 0) {
        const uint32_t idesc = umma::idesc_bf16(NH);
        auto issue = [&](int kt) {
            const int st = kt % NS, dxi = kt / f.Z, sz = kt % f.Z, kc = dxi * C + sz * 64;
            mbar_expect_tx(&s.full[st], TX);
            tma_load_4d(s.ahi[st], &tm_hi, 0, bx0 + dxi - 1, by0 + dyi - 1, sz, &s.full[st]);
            tma_load_4d(s.alo[st], &tm_lo, 0, bx0 + dxi - 1, by0 + dyi - 1, sz, &s.full[st]);
            tma_load_2d(s.bhi[st], &tm_T, kc, dyi * C + t0, &s.full[st]);
            tma_load_2d(s.blo[st], &tm_T, K3 + kc, dyi * C + t0, &s.full[st]);
        };
        bool ok = true;
        int issued = 0, landed = 0;
        for (; issued < NS && issued < nk; issued++) issue(issued);
        for (int kt = 0; kt < nk && ok; kt++) {
            const int st = kt % NS;
            ok = umma::mbar_wait(&s.full[st], (uint32_t)((kt / NS) & 1));
            if (!ok) break;
            landed = kt + 1;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t ah = umma::smem_u32(s.ahi[st]), al = umma::smem_u32(s.alo[st]);
            const uint32_t bh = umma::smem_u32(s.bhi[st]), bl = umma::smem_u32(s.blo[st]);
#pragma unroll
            for (int kk = 0; kk < umma::BK / 16; kk++) {
                umma::mma_bf16(tmem, umma::desc_sw128(ah + kk * 32), umma::desc_sw128(bh + kk * 32), idesc,
                               (kt > 0 || kk > 0) ? 1u : 0u);
                umma::mma_bf16(tmem, umma::desc_sw128(al + kk * 32), umma::desc_sw128(bh + kk * 32), idesc, 1u);
                umma::mma_bf16(tmem, umma::desc_sw128(ah + kk * 32), umma::desc_sw128(bl + kk * 32), idesc, 1u);
            }
            umma::mma_commit(&s.done[st]);
            s.last = kt;
            // refill the stage of step kt - 1 once its MMAs are done (step kt's run meanwhile)
            const int prev = kt - 1, nxt = prev + NS;
            if (prev >= 0 && nxt < nk) {
                ok = umma::mbar_wait(&s.done[prev % NS], (uint32_t)((prev / NS) & 1));
                if (ok) issue(issued++);
            }
        }
        // after a timeout: let every copy still in flight land before the CTA's memory goes away
        for (int kt = landed; kt < issued; kt++) umma::mbar_wait(&s.full[kt % NS], (uint32_t)((kt / NS) & 1));
        if (!ok) s.err = 1;
    }
    __syncthreads();
    bool ok = s.err == 0;
    const int last = s.last;
    // the last commit covers every earlier MMA
    if (last >= 0) {
        const bool fin = umma::mbar_wait(&s.done[last % NS], (uint32_t)((last / NS) & 1));
        ok = ok && fin;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (!ok || last != nk - 1) {
        if (lane == 0) atomicExch(&g_p2p_tc_err, 1);
    } else {
        // warp w holds accumulator rows 32 w .. 32 w + 31 = boxes (bx0 + lane, by0 + w);
        // 16 columns = two cell rows of one layer: 16-byte stores where the
        // box's 8 cells lie inside the grid on a 16-byte boundary
        const int bx = bx0 + lane, by = by0 + warp;
        const bool okb = bx < nbx && by < nby;
        const bool vec = (f.X & 3) == 0 && bx * 8 + 8 <= f.X;
        for (int c0 = 0; c0 < NH; c0 += 16) {
            float v[16];
            umma::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (!okb) continue;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int t = t0 + c0 + 8 * h, tz = t >> 6, y = by * 8 + ((t >> 3) & 7);
                if (y >= f.Y) continue;
                float *o = out + ((long long)tz * f.Y + y) * f.X + bx * 8;
                if (vec) {
                    reinterpret_cast<float4 *>(o)[0] = make_float4(v[8 * h], v[8 * h + 1], v[8 * h + 2], v[8 * h + 3]);
                    reinterpret_cast<float4 *>(o)[1] = make_float4(v[8 * h + 4], v[8 * h + 5], v[8 * h + 6], v[8 * h + 7]);
                } else {
#pragma unroll
                    for (int i = 0; i < 8; i++)
                        if (bx * 8 + i < f.X) o[i] = v[8 * h + i];
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS) : "memory");
}

// out[i] = sum of n parts of stride ns, in order
__global__ void k_sum_parts(const float *__restrict__ parts, int n, long long ns, float *__restrict__ out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    float v = parts[i];
    for (int q = 1; q < n; q++) v += parts[q * ns + i];
    out[i] = v;
}

// TMA descriptor of a BF16 tensor (dims / box innermost first, byte strides of dims 1..)
int ntc_tensor_map(CUtensorMap *tm, void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
                   const cuuint32_t *box)
{
    static PFN_cuTensorMapEncodeTiled encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            mms_set_error("tensor-core near field: cuTensorMapEncodeTiled unavailable");
            return MMS_ERR_CUDA;
        }
        encode = (PFN_cuTensorMapEncodeTiled)fn;
    }
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, base, dims, strides, box, es,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        mms_set_error("tensor-core near field: tensor map encoding failed (%d)", (int)r);
        return MMS_ERR_ARG;
    }
    return MMS_OK;
}

#define MMS_NTC_CASES(X) X(64) X(128) X(192) X(256)

__device__ int g_m2l_tc_err;

constexpr int TC_STAGES = 4;

// grouped tensor-core M2L: blockIdx.z = (parity class, parity block), x = 128
// target rows, y = a share of K written to its own partial-local buffer
__global__ void __launch_bounds__(128) k_m2l_gemm(const TcGroup *__restrict__ groups, int ksplit,
                                                  long long part_stride)
{
    extern __shared__ uint8_t raw[];
    const TcGroup g = groups[blockIdx.z];
    const int m0 = blockIdx.x * umma::BM;
    if (m0 >= g.M) return;  // before any tensor-memory allocation
    const int ktiles = (g.K + umma::BK - 1) / umma::BK, per = (ktiles + ksplit - 1) / ksplit;
    const int k0 = blockIdx.y * per * umma::BK;
    const int kl = max(0, min(g.K - k0, per * umma::BK));
    uint8_t *base = (uint8_t *)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
    umma::Smem<64, TC_STAGES> &s = *reinterpret_cast<umma::Smem<64, TC_STAGES> *>(base);
    umma::gemm_tile<64, TC_STAGES>(g.A + (kl > 0 ? k0 : 0), g.lda, g.B + (kl > 0 ? k0 : 0), g.ldb,
                                   g.C + blockIdx.y * part_stride, g.ldc, g.M, g.N, kl, m0, 0, 0, &g_m2l_tc_err, s,
                                   g.rowmap);
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


// leaf-kernel specialisations: boxes per CTA, threads per CTA (0 = none)
int leaf_bb(int S) { return S >= 8 ? 4 : 8; }

int leaf_threads(const FmmDev &f)
{
    const int S = f.s;
    if (S != 2 && S != 4 && S != 8 && S != 16) return 0;
    const int t = leaf_bb(S) * S * f.Z;
    return t <= 512 ? t : 0;
}

// thread groups per leaf box in k_l2p (on the critical path after the join):
// 3 while the CTA stays <= 512 threads
int leaf_groups(const FmmDev &f) { return 3 * leaf_threads(f) <= 512 ? 3 : 1; }
// in k_p2p, which runs beside the far-field chain: the same three groups (once
// the far chain was shortened, the near field became the longer branch at
// leaf 8 and the wider CTAs paid off there too: 3980 -> 4126 steps/s)
int p2p_groups(const FmmDev &f) { return leaf_groups(f); }

size_t p2p_smem(const FmmDev &f)
{
    const int S = f.s, B = leaf_bb(S), W = (B + 2) * S;
    return ((size_t)f.Z * 3 * S * W + (size_t)f.Z * 4 * S * S +
            (size_t)(p2p_groups(f) - 1) * S * leaf_threads(f)) * sizeof(float);
}

size_t l2p_smem(const FmmDev &f)
{
    const int B = leaf_bb(f.s);
    const size_t tsz = 4 * ((size_t)f.NE * f.NE + (size_t)(f.NR - f.NE) * (f.NR - f.NE));
    const int GB = B >= 4 ? B / 4 : 1;
    // after the leaf locals are consumed, the area from Lb on holds the groups' partial sums
    const size_t locals = (size_t)B * f.NR + (size_t)(B / 2) * f.NR + (size_t)GB * f.NR;
    const size_t partial = (size_t)(leaf_groups(f) - 1) * f.s * leaf_threads(f);
    return (tsz + std::max(locals, partial)) * sizeof(float);
}

#define MMS_LEAF_CASES(X) X(2, 8) X(4, 8) X(8, 4) X(16, 4)

int leaf_set_smem(const FmmDev &f)
{
    const int a = (int)p2p_smem(f), b = (int)l2p_smem(f);
    cudaError_t e = cudaSuccess;
#define X(S_, B_)                                                                                    \
    if (f.s == S_ && a > 48 * 1024) {                                                                \
        e = cudaFuncSetAttribute(k_p2p<S_, B_, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, a);   \
        if (e == cudaSuccess)                                                                        \
            e = cudaFuncSetAttribute(k_p2p<S_, B_, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, a); \
    }                                                                                                \
    if (f.s == S_ && e == cudaSuccess && b > 48 * 1024) {                                            \
        e = cudaFuncSetAttribute(k_l2p<S_, B_, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);   \
        if (e == cudaSuccess)                                                                        \
            e = cudaFuncSetAttribute(k_l2p<S_, B_, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, b); \
    }
    MMS_LEAF_CASES(X)
#undef X
    if (e != cudaSuccess) {
        mms_set_error("leaf kernel shared memory (%d / %d B): %s", a, b, cudaGetErrorString(e));
        return MMS_ERR_ARG;
    }
    return MMS_OK;
}

int p2p_launch(const FmmDev &f, int nbx, int nby, const float *rho, const float *Gn, float *out, cudaStream_t st)
{
    const dim3 grid(div_up(nbx, leaf_bb(f.s)), nby);
#define X(S_, B_)                                                                                              \
    if (f.s == S_) {                                                                                           \
        if (p2p_groups(f) == 3)                                                                                \
            MMS_CUDA_TRY(launch_k(k_p2p<S_, B_, 3>, grid, dim3(3 * leaf_threads(f)), p2p_smem(f), st, rho, Gn, out, f)); \
        else                                                                                                   \
            MMS_CUDA_TRY(launch_k(k_p2p<S_, B_, 1>, grid, dim3(leaf_threads(f)), p2p_smem(f), st, rho, Gn, out, f)); \
        return MMS_OK;                                                                                         \
    }
    MMS_LEAF_CASES(X)
#undef X
    mms_set_error("no leaf kernel for side %d", f.s);
    return MMS_ERR_ARG;
}

int l2p_launch(const FmmDev &f, int nbx, int nby, const float *near, const float *Lpart_leaf, const float *Lpar,
               const float *Tl2l, const float *Vt, float *phi, long long part_stride, int nsplit, int pmode,
               const float *Lgp, const float *Lpp, int nnear, long long near_stride, const float *Lpart_all,
               const long long *lev_off, cudaStream_t st)
{
    const dim3 grid(div_up(nbx, leaf_bb(f.s)), nby);
#define X(S_, B_)                                                                                              \
    if (f.s == S_) {                                                                                           \
        if (leaf_groups(f) == 3)                                                                               \
            MMS_CUDA_TRY(launch_k(k_l2p<S_, B_, 3>, grid, dim3(3 * leaf_threads(f)), l2p_smem(f), st, near,      \
                                  Lpart_leaf, Lpar, Tl2l, Vt, phi, f, part_stride, nsplit, pmode, Lgp, Lpp, nnear, \
                                  near_stride, Lpart_all, lev_off));                                       \
        else                                                                                                   \
            MMS_CUDA_TRY(launch_k(k_l2p<S_, B_, 1>, grid, dim3(leaf_threads(f)), l2p_smem(f), st, near, Lpart_leaf, \
                                  Lpar, Tl2l, Vt, phi, f, part_stride, nsplit, pmode, Lgp, Lpp, nnear,        \
                                  near_stride, Lpart_all, lev_off));                                       \
        return MMS_OK;                                                                                         \
    }
    MMS_LEAF_CASES(X)
#undef X
    mms_set_error("no leaf kernel for side %d", f.s);
    return MMS_ERR_ARG;
}

// resident-operator M2L specialisations: (NR, NE) for P = 1 .. 5 and the two network widths
#define MMS_M2L_RES_CASES(X) X(6, 4) X(12, 8) X(20, 12) X(24, 16) X(30, 18) X(40, 24) X(42, 24)

int m2l_res_supported(int NR, int NE)
{
#define X(a, b) if (NR == a && NE == b) return 1;
    MMS_M2L_RES_CASES(X)
#undef X
    return 0;
}

size_t m2l_res_smem(int NR, int NE)
{
    const int NO = NR - NE;
    return std::max((size_t)49 * (NE * NE + NO * NO), (size_t)RES_WARPS * RES_TPI * (NR + 1)) * sizeof(float);
}

int m2l_res_prepare(int NR, int NE)
{
    const int b = (int)m2l_res_smem(NR, NE);
    cudaError_t e = cudaSuccess;
#define X(a, c) if (NR == a && NE == c) e = cudaFuncSetAttribute(k_m2l_res<a, c>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    MMS_M2L_RES_CASES(X)
#undef X
    if (e != cudaSuccess) {
        mms_set_error("M2L shared memory (%d B): %s", b, cudaGetErrorString(e));
        return MMS_ERR_ARG;
    }
    return MMS_OK;
}

int m2l_res_launch(const FmmDev &f, int nitems, const float *Mall, float *Lout, const float *Tc, const int4 *items,
                   const long long *lev, cudaStream_t st, long long lstride = 0)
{
    const size_t sm = m2l_res_smem(f.NR, f.NE);
#define X(a, c) if (f.NR == a && f.NE == c) { MMS_CUDA_TRY(launch_k(k_m2l_res<a, c>, dim3(nitems), dim3(32 * RES_WARPS), sm, st, Mall, Lout, Tc, items, lev, f, lstride)); return MMS_OK; }
    MMS_M2L_RES_CASES(X)
#undef X
    mms_set_error("no resident M2L kernel for NR=%d", f.NR);
    return MMS_ERR_ARG;
}

// One shared-memory carveout (the largest) for every kernel of the potential.
// An SM changes its L1 / shared-memory split only when idle, so kernels with
// different splits cannot share it: the near field, which runs beside the
// far-field chain, and the chain's kernels would otherwise take turns on the
// SMs, and a programmatic early launch could not overlap its predecessor.
int fmm_set_carveout()
{
    const int c = cudaSharedmemCarveoutMaxShared;
    const void *k[] = {(const void *)k_p2m_row<4, false>, (const void *)k_p2m_row<BB, false>,
                       (const void *)k_p2m_row<4, true>, (const void *)k_p2m_row<BB, true>, (const void *)k_m2m_c,
                       (const void *)k_top_m2m,    (const void *)k_top_l2l,     (const void *)k_l2l_c,
                       (const void *)k_m2l_split,  (const void *)k_m2l_gather,  (const void *)k_m2l_gemm};
    for (const void *fn : k) MMS_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, c));
#define X(a, b) MMS_CUDA_TRY(cudaFuncSetAttribute(k_m2l_res<a, b>, cudaFuncAttributePreferredSharedMemoryCarveout, c));
    MMS_M2L_RES_CASES(X)
#undef X
#define X(S_, B_)                                                                                            \
    MMS_CUDA_TRY(cudaFuncSetAttribute(k_p2p<S_, B_, 1>, cudaFuncAttributePreferredSharedMemoryCarveout, c)); \
    MMS_CUDA_TRY(cudaFuncSetAttribute(k_p2p<S_, B_, 3>, cudaFuncAttributePreferredSharedMemoryCarveout, c)); \
    MMS_CUDA_TRY(cudaFuncSetAttribute(k_l2p<S_, B_, 1>, cudaFuncAttributePreferredSharedMemoryCarveout, c)); \
    MMS_CUDA_TRY(cudaFuncSetAttribute(k_l2p<S_, B_, 3>, cudaFuncAttributePreferredSharedMemoryCarveout, c));
    MMS_LEAF_CASES(X)
#undef X
    return MMS_OK;
}
}  // namespace

int fmm_default_leaf(int P, int X, int Y);
int far_prepare(mms_ctx *ctx, FmmPlan *pl);
static int l2p_up(const FmmPlan *pl);
static int l2p_top(const FmmPlan *pl);
static int p2m_up(const FmmPlan *pl);

int fmm_plan_create(mms_ctx *ctx)
{
    const int P = ctx->s.fmm_order;
    if (P < 1 || P > 9) {
        mms_set_error("FMM order P must be 1..9 (got %d)", P);
        return MMS_ERR_ARG;
    }
    int s = ctx->s.fmm_leaf;
    if (s == 0) s = ctx->s.kind == MMS_SOLVER_SURROGATE ? FN_S : fmm_default_leaf(P, ctx->g.xdim, ctx->g.ydim);
    if (ctx->s.kind == MMS_SOLVER_SURROGATE && (s != FN_S || ctx->g.zdim != FN_Z)) {
        mms_set_error("the surrogate solver works on %d x %d x %d leaf boxes (leaf side %d, %d layers given)", FN_S,
                      FN_S, FN_Z, s, ctx->g.zdim);
        return MMS_ERR_ARG;
    }
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
            Vt[(size_t)k * f.C + c] = (float)(V[(size_t)c * f.NR + k] / w);
        }
    // M2M / L2L, transposed to [j][k]
    const int NR = f.NR;
    // M2M / L2L parity blocks, [c][blk][j][k]
    const int NEb = f.NE, NOb = NR - f.NE;
    const size_t cstride = (size_t)NEb * NEb + (size_t)NOb * NOb;
    std::vector<float> Tm2m(4 * cstride), Tl2l(4 * cstride);
    for (int c = 0; c < 4; c++) {
        const double dxv = ((c & 1) - 0.5) / 2, dyv = ((c >> 1) - 0.5) / 2 * ay;
        const std::vector<double> a = fmmops::m2m(lay, dxv, dyv, 0.0);
        const std::vector<double> b = fmmops::l2l(lay, -dxv, -dyv, 0.0);
        for (int blk = 0; blk < 2; blk++) {
            const int b0 = blk ? NEb : 0, NB = blk ? NOb : NEb;
            const size_t base = c * cstride + (blk ? (size_t)NEb * NEb : 0);
            for (int j = 0; j < NB; j++)
                for (int k = 0; k < NB; k++) {
                    Tm2m[base + (size_t)j * NB + k] = (float)a[(size_t)(b0 + k) * NR + (b0 + j)];
                    Tl2l[base + (size_t)j * NB + k] = (float)b[(size_t)(b0 + k) * NR + (b0 + j)];
                }
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
    std::vector<float> Tm2lc((size_t)49 * ((size_t)NB0 * NB0 + (size_t)NB1 * NB1), 0.f);
    for (int o = 0; o < 49; o++)
        for (int blk = 0; blk < 2; blk++) {
            const int NB = blk ? NB1 : NB0, KP = pl->KPb[blk];
            const float *src = &Tm2l[((size_t)o * 2 + blk) * NBmax * KPmax];
            float *dst = &Tm2lc[(size_t)o * ((size_t)NB0 * NB0 + (size_t)NB1 * NB1) + (blk ? (size_t)NB0 * NB0 : 0)];
            for (int j = 0; j < NB; j++)
                for (int k = 0; k < NB; k++) dst[(size_t)j * NB + k] = src[(size_t)j * KP + k];
        }
    const int m2l_mode = ctx->s.m2l_mode;
    // auto: the tensor-core path from P = 6 at leaf <= 4 and from P = 8 at any
    // leaf, where it measured faster than the FP32 kernels on a 256 x 256 x 3
    // film (M2L 49 vs 64 us at P = 6 leaf 4; 72 vs 110 and 29 vs 37 us at P = 8
    // leaf 4 and 8) at little cost in accuracy (phi rel-L2 vs exact 3.35e-5 vs
    // 3.34e-5 at P = 6, 3.9e-6 vs 3.5e-6 at P = 8); below, the FP32 kernels
    pl->m2l_tc = m2l_mode == 2 || (m2l_mode == 0 && (P >= 8 || (P >= 6 && f.s <= 4)));
    pl->m2l_resident = !pl->m2l_tc && m2l_res_supported(NR, f.NE);
    // tensor-core M2L operands: B'_{p,b} rows k = [T_hi | T_lo | T_hi] over the
    // class's 27 offsets (q-major, NBp-padded), matching k_m2l_gather's order
    std::vector<__nv_bfloat16> tcB;
    std::vector<long long> tcBoff(8, 0);
    if (pl->m2l_tc) {
        for (int blk = 0; blk < 2; blk++) {
            const int NB = blk ? NB1 : NB0;
            pl->tcNBp[blk] = (NB + 7) & ~7;
            pl->tcK[blk] = 27 * pl->tcNBp[blk];
        }
        for (int par = 0; par < 4; par++) {
            const int px = par & 1, py = par >> 1;
            for (int blk = 0; blk < 2; blk++) {
                const int NB = blk ? NB1 : NB0, NBp = pl->tcNBp[blk], K = pl->tcK[blk], KP = pl->KPb[blk];
                tcBoff[par * 2 + blk] = (long long)tcB.size();
                std::vector<__nv_bfloat16> Bg((size_t)NB * 3 * K, __float2bfloat16_rn(0.f));
                int q = 0;
                for (int yy = 0; yy < 6; yy++)
                    for (int xx = 0; xx < 6; xx++) {
                        const int ox = px - 3 + xx, oy = py - 3 + yy;
                        if (std::max(abs(ox), abs(oy)) < 2) continue;
                        const int o = (oy + 3) * 7 + (ox + 3);
                        const float *src = &Tm2l[((size_t)o * 2 + blk) * NBmax * KPmax];
                        for (int k = 0; k < NB; k++)
                            for (int j = 0; j < NB; j++) {
                                const float v = src[(size_t)j * KP + k];
                                const __nv_bfloat16 hi = __float2bfloat16_rn(v);
                                const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
                                const size_t base = (size_t)k * 3 * K + (size_t)q * NBp + j;
                                Bg[base] = hi;
                                Bg[base + K] = lo;
                                Bg[base + 2 * K] = hi;
                            }
                        q++;
                    }
                tcB.insert(tcB.end(), Bg.begin(), Bg.end());
            }
        }
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
    std::vector<int4> ritems;
    for (int l = 2; l <= f.L; l++) {
        const int nh = (1 << l) / 2;
        for (int par = 0; par < 4; par++)
            for (int t0 = 0; t0 < nh * nh; t0 += RES_TPI) ritems.push_back(make_int4(l, par, t0, 0));
    }
    pl->n_res_items = (int)ritems.size();

    // tensor-core M2L rows: every box of levels >= 2, grouped by parity class
    std::vector<int> tc_rowmap;
    std::vector<int4> tc_rowinfo;
    int tc_base[5] = {0, 0, 0, 0, 0};
    if (pl->m2l_tc) {
        for (int par = 0; par < 4; par++) {
            tc_base[par] = (int)tc_rowmap.size();
            for (int l = 2; l <= f.L; l++) {
                const int nh = (1 << l) / 2;
                for (int t = 0; t < nh * nh; t++) {
                    const int bx = 2 * (t % nh) + (par & 1), by = 2 * (t / nh) + (par >> 1);
                    tc_rowmap.push_back((int)(pl->lev_off[l] + (long long)by * (1 << l) + bx));
                    tc_rowinfo.push_back(make_int4(l, par, t, 0));
                }
            }
        }
        tc_base[4] = (int)tc_rowmap.size();
        pl->tc_rows = tc_base[4];
        pl->tc_maxm = 0;
        int tiles = 0;
        for (int par = 0; par < 4; par++) {
            pl->tc_maxm = std::max(pl->tc_maxm, tc_base[par + 1] - tc_base[par]);
            tiles += 2 * ((tc_base[par + 1] - tc_base[par] + umma::BM - 1) / umma::BM);
        }
        // enough CTAs for two per SM, at least 4 K tiles each, at most NSPLIT partials
        const int ktiles = (3 * std::max(pl->tcK[0], pl->tcK[1]) + umma::BK - 1) / umma::BK;
        pl->tc_ksplit = std::max(1, std::min({NSPLIT, (296 + tiles - 1) / std::max(1, tiles), ktiles / 4}));
    }
    int st = MMS_OK;
    if (!st) st = upload(ctx, pl, &pl->Wt, Wt);
    if (!st) st = upload(ctx, pl, &pl->Vt, Vt);
    if (!st) st = upload(ctx, pl, &pl->Tm2m, Tm2m);
    if (!st) st = upload(ctx, pl, &pl->Tl2l, Tl2l);
    if (!st) st = upload(ctx, pl, &pl->Tm2l, Tm2l);
    if (!st) st = upload(ctx, pl, &pl->Tm2lc, Tm2lc);
    if (!st && pl->m2l_tc) {
        st = upload(ctx, pl, &pl->tcB, tcB);
        if (!st) st = upload(ctx, pl, &pl->tc_rowmap, tc_rowmap);
        if (!st) st = upload(ctx, pl, &pl->tc_rowinfo, tc_rowinfo);
        for (int blk = 0; blk < 2 && !st; blk++) {
            std::vector<__nv_bfloat16> z((size_t)pl->tc_rows * 3 * pl->tcK[blk]);
            st = upload(ctx, pl, &pl->tcA[blk], z);
        }
        if (!st) {
            std::vector<TcGroup> grp(8);
            for (int par = 0; par < 4; par++)
                for (int blk = 0; blk < 2; blk++) {
                    TcGroup &g = grp[par * 2 + blk];
                    g.A = pl->tcA[blk] + (size_t)tc_base[par] * 3 * pl->tcK[blk];
                    g.B = pl->tcB + tcBoff[par * 2 + blk];
                    g.C = nullptr;  // set at launch: Lpart + block offset
                    g.rowmap = pl->tc_rowmap + tc_base[par];
                    g.lda = g.ldb = 3 * pl->tcK[blk];
                    g.ldc = NR;
                    g.M = tc_base[par + 1] - tc_base[par];
                    g.N = blk ? NB1 : NB0;
                    g.K = 3 * pl->tcK[blk];
                    g.pad[0] = g.pad[1] = 0;
                }
            pl->tc_group_host = grp;  // uploaded once Lpart exists (C pointers)
        }
    }
    if (!st) st = upload(ctx, pl, &pl->m2l_items, items);
    if (!st) st = upload(ctx, pl, &pl->res_items, ritems);
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
            cudaMalloc((void **)&pl->Lpart, NSPLIT * ncoef * sizeof(float)) != cudaSuccess ||
            cudaMalloc((void **)&pl->Gn, (size_t)Z * 4 * s * s * sizeof(float)) != cudaSuccess) {
            cudaFree(lev_dev);
            fmm_plan_destroy(ctx);
            mms_set_error("FMM plan: device allocation failed");
            return MMS_ERR_NOMEM;
        }
        if (cudaMalloc((void **)&pl->near, (size_t)ctx->N * sizeof(float)) != cudaSuccess ||
            cudaStreamCreateWithFlags(&pl->side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&pl->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&pl->ev_join, cudaEventDisableTiming) != cudaSuccess) {
            fmm_plan_destroy(ctx);
            mms_set_error("FMM plan: stream/event/buffer creation failed");
            return MMS_ERR_NOMEM;
        }
        pl->bytes += (2 + NSPLIT) * ncoef * sizeof(float) + (size_t)Z * 4 * s * s * sizeof(float) +
                     (size_t)ctx->N * sizeof(float);
        MMS_CUDA_TRY(cudaMemsetAsync(pl->Lpart, 0, NSPLIT * ncoef * sizeof(float), ctx->stream));
        if (pl->m2l_tc) {
            for (int i = 0; i < 8; i++) pl->tc_group_host[i].C = pl->Lpart + ((i & 1) ? f.NE : 0);
            if (cudaMalloc((void **)&pl->tc_groups, 8 * sizeof(TcGroup)) != cudaSuccess) {
                fmm_plan_destroy(ctx);
                mms_set_error("FMM plan: device allocation failed");
                return MMS_ERR_NOMEM;
            }
            pl->bytes += 8 * sizeof(TcGroup);
            MMS_CUDA_TRY(cudaMemcpyAsync(pl->tc_groups, pl->tc_group_host.data(), 8 * sizeof(TcGroup),
                                         cudaMemcpyHostToDevice, ctx->stream));
            MMS_CUDA_TRY(cudaFuncSetAttribute(k_m2l_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)(sizeof(umma::Smem<64, TC_STAGES>) + 1024)));
        }
        MMS_CUDA_TRY(cudaMemsetAsync(pl->Mall, 0, ncoef * sizeof(float), ctx->stream));
        MMS_CUDA_TRY(cudaMemsetAsync(pl->Lall, 0, ncoef * sizeof(float), ctx->stream));
    }
    k_build_gn<<<div_up((long long)Z * 4 * s * s, 128), 128, 0, ctx->stream>>>(pl->Gn, Z, s, ctx->g.dx, ctx->g.dy,
                                                                            ctx->g.dz);
    MMS_LAUNCH_CHECK(ctx);
    pl->lev_dev = lev_dev;
    const size_t m2ls_smem = ((size_t)NBmax * KPmax + 32 * (size_t)(NBmax | 1)) * sizeof(float);
    if (m2ls_smem > 48 * 1024)
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_m2l_split, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m2ls_smem));
    if (pl->m2l_resident) MMS_TRY(m2l_res_prepare(NR, f.NE));
    if (pl->m2l_resident && NR <= 30 && leaf_threads(f) > 0 && f.L >= 2 && ctx->s.far_mode == 1)
        MMS_TRY(far_prepare(ctx, pl));
    {
        // P2M with W staged and the fused parent M2M: at most 160 KB
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_p2m_row<BB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_p2m_row<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_p2m_row<BB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_p2m_row<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    }
    {
        const size_t tsz = 4 * cstride;
        const int KT = ((NR + 31) / 32) * 32;
        const size_t a1 = (tsz + 4 * (size_t)NR + 4 * (size_t)KT) * sizeof(float), a2 = (tsz + (size_t)NR) * sizeof(float);
        if (a1 > 48 * 1024)
            MMS_CUDA_TRY(cudaFuncSetAttribute(k_m2m_c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a1));
        if (a2 > 48 * 1024)
            MMS_CUDA_TRY(cudaFuncSetAttribute(k_l2l_c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a2));

    }
    if (leaf_threads(f) > 0) MMS_TRY(leaf_set_smem(f));
    MMS_TRY(fmm_set_carveout());

    // algorithmic work of one evaluation (FMA = 2 flops), per stage
    const long long nleafb = (long long)f.nb * f.nb;
    double fl = 0;
    pl->stage_flops[0] = 2.0 * nleafb * f.C * NR;  // P2M
    pl->stage_flops[4] = 2.0 * nleafb * f.C * NR;  // L2P (P2P added below)
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
    pl->stage_flops[2] = 2.0 * m2l_pairs * blk2;
    pl->stage_flops[1] = 0;
    for (int l = 2; l < f.L; l++) pl->stage_flops[1] += 2.0 * 4.0 * (double)(1 << l) * (1 << l) * blk2;
    pl->stage_flops[3] = 0;
    for (int l = 3; l <= f.L; l++) pl->stage_flops[3] += 2.0 * (double)(1 << l) * (1 << l) * blk2;
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
    pl->stage_flops[4] += 2.0 * pairs;
    // attribute the levels the leaf kernels form to the stage that runs them:
    // the leaf-level L2L (and level L-1's, l2p_up) to L2P, level L-1's M2M
    // (p2m_up) to P2M
    if (leaf_threads(f) > 0 && f.L >= 2) {
        const double leafl2l = 2.0 * (double)(1 << f.L) * (1 << f.L) * blk2;
        if (f.L >= 3) {
            pl->stage_flops[3] -= leafl2l;
            pl->stage_flops[4] += leafl2l;
        }
        if (l2p_up(pl) && f.L - 1 >= 3) {
            const double m = 2.0 * (double)(1 << (f.L - 1)) * (1 << (f.L - 1)) * blk2;
            pl->stage_flops[3] -= m;
            pl->stage_flops[4] += m;
        }
        if (l2p_top(pl)) {  // every remaining level of the downward pass
            pl->stage_flops[4] += pl->stage_flops[3];
            pl->stage_flops[3] = 0;
        }
        if (p2m_up(pl)) {
            const double m = 2.0 * 4.0 * (double)(1 << (f.L - 1)) * (1 << (f.L - 1)) * blk2;
            pl->stage_flops[1] -= m;
            pl->stage_flops[0] += m;
        }
    }
    if (f.L < 2)
        for (int i = 0; i < 4; i++) pl->stage_flops[i] = 0;
    if (f.L < 2) pl->stage_flops[4] = 2.0 * pairs;
    for (int i = 0; i < 5; i++) fl += pl->stage_flops[i];
    pl->flops = fl;
    pl->p2p_pairs = pairs;
    pl->m2l_pairs = m2l_pairs;
    // near field on the tensor cores (k_p2p_tc) at leaf side 8 with a far field
    // and Z <= 4, by default (near_mode 0) or on request (2); FP32 k_p2p
    // otherwise.  At 256 x 256 x 3 (P = 4) it took the RK4 step from 224 to
    // 191 us (174 us with the later changes): its few CTAs (24, now 48) leave
    // the SMs' FMA and load pipes to the far-field chain that runs beside it,
    // where k_p2p's 256 CTAs competed with it.
    const int nmode = ctx->s.near_mode;
    const bool ntc_ok = s == 8 && leaf_threads(f) > 0 && f.L >= 2 && Z <= 4;
    if (nmode < 0 || nmode > 2 || (nmode == 2 && !ntc_ok)) {
        fmm_plan_destroy(ctx);
        if (nmode < 0 || nmode > 2)
            mms_set_error("near_mode must be 0 (auto), 1 (FP32) or 2 (tensor cores), got %d", nmode);
        else
            mms_set_error("tensor-core near field needs leaf side 8, at least 2 levels and Z <= 4");
        return MMS_ERR_ARG;
    }
    if (ntc_ok && nmode != 1) {
        const int C = 64 * Z;
        const int nbx = std::min(f.nb, (f.X + s - 1) / s), nby = std::min(f.nb, (f.Y + s - 1) / s);
        const size_t nT = 3 * (size_t)C * 6 * C, nR = 2 * (size_t)Z * 64 * nbx * nby;
        if (cudaMalloc((void **)&pl->ntcT, nT * sizeof(__nv_bfloat16)) != cudaSuccess ||
            cudaMalloc((void **)&pl->ntcR, nR * sizeof(__nv_bfloat16)) != cudaSuccess ||
            cudaMalloc((void **)&pl->near3, 3 * (size_t)ctx->N * sizeof(float)) != cudaSuccess) {
            fmm_plan_destroy(ctx);
            mms_set_error("FMM plan: device allocation failed");
            return MMS_ERR_NOMEM;
        }
        pl->bytes += (nT + nR) * sizeof(__nv_bfloat16) + 3 * (size_t)ctx->N * sizeof(float);
        MMS_CUDA_TRY(cudaMemsetAsync(pl->ntcR, 0, nR * sizeof(__nv_bfloat16), ctx->stream));
        k_build_ntc<<<296, 256, 0, ctx->stream>>>(pl->Gn, pl->ntcT, Z);
        MMS_LAUNCH_CHECK(ctx);
        {
            // charges: [Z][nby][nbx][64] BF16 (hi, then lo), tiles of 1 x 4 x 32 x 64;
            // operators: [3 C][9 C] BF16, tiles of C x 64
            const cuuint64_t dR[4] = {64, (cuuint64_t)nbx, (cuuint64_t)nby, (cuuint64_t)Z};
            const cuuint64_t sR[3] = {128, (cuuint64_t)nbx * 128, (cuuint64_t)nbx * nby * 128};
            const cuuint32_t bR[4] = {64, NTC_TW, NTC_TH, 1};
            const cuuint64_t dT[2] = {(cuuint64_t)6 * C, (cuuint64_t)3 * C};
            const cuuint64_t sT[1] = {(cuuint64_t)6 * C * 2};
            const cuuint32_t bT[2] = {64, (cuuint32_t)C / 2};
            int e = ntc_tensor_map(&pl->ntc_map[0], pl->ntcR, 4, dR, sR, bR);
            if (e == MMS_OK) e = ntc_tensor_map(&pl->ntc_map[1], pl->ntcR + nR / 2, 4, dR, sR, bR);
            if (e == MMS_OK) e = ntc_tensor_map(&pl->ntc_map[2], pl->ntcT, 2, dT, sT, bT);
            if (e != MMS_OK) {
                char keep[512];
                strncpy(keep, mms_last_error(), sizeof keep - 1);
                keep[sizeof keep - 1] = 0;
                fmm_plan_destroy(ctx);
                mms_set_error("%s", keep);
                return e;
            }
        }
#define X(BN_)                                                                                                   \
    if (C == BN_) {                                                                                              \
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_p2p_tc<BN_>, cudaFuncAttributeMaxDynamicSharedMemorySize,            \
                                          (int)ntc_smem<BN_>()));                                                \
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_p2p_tc<BN_>, cudaFuncAttributePreferredSharedMemoryCarveout,         \
                                          cudaSharedmemCarveoutMaxShared));                                      \
    }
        MMS_NTC_CASES(X)
#undef X
        pl->p2p_tc = 1;
    }
    if (pl->p2p_tc || pl->m2l_tc) {  // wait-timeout flags of the tensor-core kernels
        const int zero = 0;
        MMS_CUDA_TRY(cudaMemcpyToSymbolAsync(g_p2p_tc_err, &zero, sizeof zero, 0, cudaMemcpyHostToDevice, ctx->stream));
        MMS_CUDA_TRY(cudaMemcpyToSymbolAsync(g_m2l_tc_err, &zero, sizeof zero, 0, cudaMemcpyHostToDevice, ctx->stream));
    }
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return MMS_OK;
}

void fmm_plan_destroy(mms_ctx *ctx)
{
    FmmPlan *pl = ctx->fmm;
    if (!pl) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    void *b[] = {pl->Wt, pl->Vt, pl->Tm2m, pl->Tl2l, pl->Tm2l, pl->Tm2lc, pl->Gn, pl->Mall, pl->Lall, pl->Lpart,
                 pl->m2l_items, pl->res_items, pl->lev_dev, pl->near, pl->tcA[0], pl->tcA[1], pl->tcB, pl->tc_rowmap,
                 pl->tc_rowinfo, pl->tc_groups, pl->far_sync, pl->ntcT, pl->ntcR, pl->near3, pl->fnW, pl->fnV,
                 pl->fnM2L, pl->fnM2M, pl->fnL2L, pl->fnM, pl->fnLp, pl->fnCtr};
    for (void *p : b)
        if (p) cudaFree(p);
    if (pl->side) cudaStreamSynchronize(pl->side);
    if (pl->ev_fork) cudaEventDestroy(pl->ev_fork);
    if (pl->ev_join) cudaEventDestroy(pl->ev_join);
    if (pl->side) cudaStreamDestroy(pl->side);
    delete pl;
    ctx->fmm = nullptr;
}

size_t fmm_plan_bytes(const mms_ctx *ctx) { return ctx->fmm ? ctx->fmm->bytes : 0; }

// the per-stage path forms level L-1's locals inside L2P (one launch fewer
// after the M2L) when the tree has a level L-1 >= 2 and the leaf kernels
// exist, and level L-1's multipoles inside P2M when also NR <= 32 (P <= 4:
// one 128-thread group per parent, 512 threads)
static int l2p_up(const FmmPlan *pl) { return pl->d.L >= 3 && leaf_threads(pl->d) > 0 && !pl->far_fused; }
static int p2m_up(const FmmPlan *pl) { return l2p_up(pl) && pl->d.NR <= 32; }
// levels 2 and 3 share one launch each way (k_top_m2m / k_top_l2l: 16 KT <= 512 threads)
static int top_two(const FmmPlan *pl) { return pl->d.NR <= 32 && !pl->far_fused; }
// L2P also forms levels 2 .. L-2 of each CTA's ancestors (pmode 4): no L2L
// launch at all between the M2L and L2P
static int l2p_top(const FmmPlan *pl) { return l2p_up(pl) && pl->d.L >= 4; }

// L2P of the far field onto the near field already in pl->near
static int l2p_launch_far(mms_ctx *ctx, const float *rho, float *phi)
{
    (void)rho;
    FmmPlan *pl = ctx->fmm;
    const FmmDev &f = pl->d;
    const int nbx = std::min(f.nb, (f.X + f.s - 1) / f.s), nby = std::min(f.nb, (f.Y + f.s - 1) / f.s);
    const int nsplit = pl->m2l_tc ? pl->tc_ksplit : (pl->m2l_resident ? 1 : NSPLIT);
    const float *Lpar = f.L > 2 ? pl->Lall + pl->lev_off[f.L - 1] * f.NR : nullptr;
    // parents' locals: ready (an L2L pass made level L-1) or formed in the leaf kernel
    const int pmode = f.L <= 2 ? 0 : (!l2p_up(pl) ? 1 : (l2p_top(pl) ? 4 : (f.L - 1 >= 3 ? 2 : 3)));
    const float *Lgp = f.L >= 4 ? pl->Lall + pl->lev_off[f.L - 2] * f.NR : nullptr;
    const float *Lpp = f.L > 2 ? pl->Lpart + pl->lev_off[f.L - 1] * f.NR : nullptr;
    const float *near = pl->p2p_tc ? pl->near3 : pl->near;
    MMS_TRY(l2p_launch(f, nbx, nby, near, pl->Lpart + pl->lev_off[f.L] * f.NR, Lpar, pl->Tl2l, pl->Vt, phi,
                       pl->nbox_total * f.NR, nsplit, pmode, Lgp, Lpp, pl->p2p_tc ? 3 : 1, ctx->N, pl->Lpart,
                       pl->lev_dev, ctx->stream));
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}


// near field of the FMM potential into pl->near (k_p2p) or, on the tensor
// cores, into the three partials pl->near3 (k_p2p_tc)
static int near_launch(mms_ctx *ctx, const float *rho, cudaStream_t st)
{
    FmmPlan *pl = ctx->fmm;
    const FmmDev &f = pl->d;
    const int nbx = std::min(f.nb, (f.X + f.s - 1) / f.s), nby = std::min(f.nb, (f.Y + f.s - 1) / f.s);
    if (!pl->p2p_tc) return p2p_launch(f, nbx, nby, rho, pl->Gn, pl->near, st);
    const long long nR = (long long)f.Z * 64 * nbx * nby;
    __nv_bfloat16 *rhi = pl->ntcR, *rlo = pl->ntcR + nR;
    // the divergence that produced rho wrote its split already, or k_rho_split does it here
    if (pl->split_of != rho)
        MMS_CUDA_TRY(launch_k(k_rho_split, dim3((unsigned)div_up(nR, 256)), dim3(256), 0, st, rho, rhi, rlo, f, nbx,
                              nby));
    pl->split_of = nullptr;
    const dim3 grid((unsigned)(div_up(nbx, NTC_TW) * div_up(nby, NTC_TH)), 3, 2);
#define X(BN_)                                                                                                  \
    if (64 * f.Z == BN_) {                                                                                      \
        MMS_CUDA_TRY(launch_k(k_p2p_tc<BN_>, grid, dim3(128), ntc_smem<BN_>(), st, pl->ntc_map[0], pl->ntc_map[1], \
                              pl->ntc_map[2], pl->near3, f, nbx, nby, (long long)ctx->N));                     \
        return MMS_OK;                                                                                          \
    }
    MMS_NTC_CASES(X)
#undef X
    mms_set_error("tensor-core near field: no kernel for %d layers", f.Z);
    return MMS_ERR_ARG;
}

// P2M (with the level L-1 M2M when p2m_up) from rho, or, with dv, from the
// divergence of dv->M that the kernel forms and stores as it goes
static int p2m_launch(mms_ctx *ctx, const float *rho, const DivSrc *dv)
{
    FmmPlan *pl = ctx->fmm;
    const FmmDev &f = pl->d;
    const int nbx = std::min(f.nb, (f.X + f.s - 1) / f.s), nby = std::min(f.nb, (f.Y + f.s - 1) / f.s);
    const size_t tsz = 4 * ((size_t)f.NE * f.NE + (size_t)(f.NR - f.NE) * (f.NR - f.NE));
    const int KT = ((f.NR + 31) / 32) * 32;
    const long long leaf_off = pl->lev_off[f.L];
    const int up = p2m_up(pl);
    const int rows = up ? 2 : 1;
    // item width: 4 boxes where the boxes are large (leaf side >= 8) or
    // the expansions long (NR > 32), for twice the CTAs; else 8
    const int PB = (f.s >= 8 || f.NR > 32) ? 4 : BB;
    const size_t extra = up ? tsz + (PB / 2) * (4 * (size_t)f.NR + 4 * (size_t)KT) : 0;
    // without the parent step, long expansions read W through L1 as they
    // go instead of staging all of it first
    const int wsm = (f.C * f.NR) % 4 == 0 &&
                    ((size_t)f.C * (rows * PB + f.NR) + extra) * sizeof(float) <= 160 * 1024;
    const size_t smem = ((size_t)f.C * (rows * PB + (wsm ? f.NR : 0)) + extra) * sizeof(float);
    const dim3 grid(div_up(nbx, PB), up ? div_up(nby, 2) : nby),
        block(up ? (PB / 2) * 4 * KT : std::min(512, ((PB * f.NR + 31) / 32) * 32));
    const long long off_par = up ? pl->lev_off[f.L - 1] : 0LL;
    const DivSrc d0 = dv ? *dv : DivSrc{};
#define P2M_ARGS grid, block, smem, ctx->stream, rho, (const float *)pl->Wt, pl->Mall, leaf_off, f, wsm, up, \
                 (const float *)pl->Tm2m, off_par, d0
    if (PB == 4 && dv)
        MMS_CUDA_TRY(launch_k(k_p2m_row<4, true>, P2M_ARGS));
    else if (PB == 4)
        MMS_CUDA_TRY(launch_k(k_p2m_row<4, false>, P2M_ARGS));
    else if (dv)
        MMS_CUDA_TRY(launch_k(k_p2m_row<BB, true>, P2M_ARGS));
    else
        MMS_CUDA_TRY(launch_k(k_p2m_row<BB, false>, P2M_ARGS));
#undef P2M_ARGS
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

// the near field on the side stream, after the work queued on the main one so
// far; ev_join marks its end
static int near_fork(mms_ctx *ctx, const float *rho)
{
    FmmPlan *pl = ctx->fmm;
    MMS_CUDA_TRY(cudaEventRecord(pl->ev_fork, ctx->stream));
    MMS_CUDA_TRY(cudaStreamWaitEvent(pl->side, pl->ev_fork, 0));
    MMS_TRY(near_launch(ctx, rho, pl->side));
    MMS_LAUNCH_CHECK(ctx);
    MMS_CUDA_TRY(cudaEventRecord(pl->ev_join, pl->side));
    return MMS_OK;
}

// One stage of the FMM potential: 0 P2M, 1 M2M (all levels), 2 M2L (all
// levels), 3 L2L (all levels, with the M2L partial sums), 4 L2P + P2P.  Every
// stage only reads what earlier stages wrote, so re-running one stage on
// unchanged inputs reproduces its output (mms_fmm_stage_times relies on that).
static int launch_fmm_stage(mms_ctx *ctx, int stage, const float *rho, float *phi)
{
    FmmPlan *pl = ctx->fmm;
    const FmmDev &f = pl->d;
    const int far = f.L >= 2;
    const int nbx = std::min(f.nb, (f.X + f.s - 1) / f.s), nby = std::min(f.nb, (f.Y + f.s - 1) / f.s);
    const long long part_stride = pl->nbox_total * f.NR;
    const int thr = ((f.NR + 31) / 32) * 32;
    const size_t tsz = 4 * ((size_t)f.NE * f.NE + (size_t)(f.NR - f.NE) * (f.NR - f.NE));
    const int KT = ((f.NR + 31) / 32) * 32;
    const int nsplit = pl->m2l_tc ? pl->tc_ksplit : (pl->m2l_resident ? 1 : NSPLIT);
    if (stage < 4 && !far) return MMS_OK;
    switch (stage) {
    case 0:
        MMS_TRY(p2m_launch(ctx, rho, nullptr));
        break;
    case 1: {
        // level L-1 is formed inside P2M when p2m_up(); levels 3 and 2 in one
        // launch when top_two()
        const int lstart = f.L - 1 - p2m_up(pl);
        const int top = top_two(pl) && lstart >= 3;
        for (int l = lstart; l >= (top ? 4 : 2); l--) {
            const int np = 1 << l;
            MMS_CUDA_TRY(launch_k(k_m2m_c, dim3(np * np), dim3(4 * KT),
                                  (tsz + 4 * (size_t)f.NR + 4 * (size_t)KT) * sizeof(float), ctx->stream, pl->Mall,
                                  (const float *)pl->Tm2m, pl->lev_off[l], pl->lev_off[l + 1], np, f));
            MMS_LAUNCH_CHECK(ctx);
        }
        if (top) {
            MMS_CUDA_TRY(launch_k(k_top_m2m, dim3(16), dim3(16 * KT),
                                  (tsz + 4 * (4 * (size_t)f.NR + 4 * (size_t)KT) + 4 * (size_t)f.NR) * sizeof(float),
                                  ctx->stream,
                                  pl->Mall, (const float *)pl->Tm2m, pl->lev_off[2], pl->lev_off[3], pl->lev_off[4],
                                  f));
            MMS_LAUNCH_CHECK(ctx);
        }
        break;
    }
    case 2: {
        if (pl->m2l_tc) {
            const long long runs = (long long)pl->tc_rows * 27 * (std::max(pl->tcNBp[0], pl->tcNBp[1]) / 8);
            k_m2l_gather<<<dim3((unsigned)div_up(runs, 256), 2), 256, 0, ctx->stream>>>(
                pl->Mall, pl->tcA[0], pl->tcA[1], pl->tc_rowinfo, pl->lev_dev, f, pl->tc_rows, pl->tcK[0], pl->tcK[1],
                pl->tcNBp[0], pl->tcNBp[1]);
            MMS_LAUNCH_CHECK(ctx);
            k_m2l_gemm<<<dim3(div_up(pl->tc_maxm, umma::BM), pl->tc_ksplit, 8), 128,
                         sizeof(umma::Smem<64, TC_STAGES>) + 1024, ctx->stream>>>(pl->tc_groups, pl->tc_ksplit,
                                                                                 part_stride);
            MMS_LAUNCH_CHECK(ctx);
            break;
        }
        if (pl->m2l_resident) {
            MMS_TRY(m2l_res_launch(f, pl->n_res_items, pl->Mall, pl->Lpart, pl->Tm2lc, pl->res_items, pl->lev_dev,
                                   ctx->stream));
        } else {
            const int NBmax = std::max(f.NE, f.NR - f.NE);
            const int KPmax = std::max(pl->KPb[0], pl->KPb[1]);
            const size_t sm = ((size_t)NBmax * KPmax + 32 * (size_t)(NBmax | 1)) * sizeof(float);
            MMS_CUDA_TRY(launch_k(k_m2l_split, dim3(pl->n_m2l_items, 2, NSPLIT), dim3(32 * M2L_WARPS), sm,
                                  ctx->stream, (const float *)pl->Mall, pl->Lpart, (const float *)pl->Tm2l,
                                  (const int4 *)pl->m2l_items, (const long long *)pl->lev_dev, f, pl->KPb[0],
                                  pl->KPb[1], NBmax, part_stride));
        }
        MMS_LAUNCH_CHECK(ctx);
        break;
    }
    case 3: {
        // level 2 from its M2L partials, levels 3 .. L-1 one launch each; the
        // leaf level is formed inside the leaf kernel (or by k_l2l_c for the
        // generic leaf kernel); with l2p_top the leaf kernel forms them all
        if (l2p_top(pl)) break;
        const int lend = leaf_threads(f) > 0 ? f.L - 1 - l2p_up(pl) : f.L;
        const int top = top_two(pl) && lend >= 3;
        if (top) {
            MMS_CUDA_TRY(launch_k(k_top_l2l, dim3(16), dim3(4 * KT), (tsz + (size_t)f.NR) * sizeof(float),
                                  ctx->stream, pl->Lall, (const float *)pl->Lpart, (const float *)pl->Tl2l,
                                  pl->lev_off[2], pl->lev_off[3], part_stride, nsplit, f));
            MMS_LAUNCH_CHECK(ctx);
        } else if (lend >= 2) {
            MMS_CUDA_TRY(launch_k(k_l2l_c, dim3(16), dim3(thr), 0, ctx->stream, pl->Lall,
                                  (const float *)pl->Lpart, (const float *)pl->Tl2l, 0LL, pl->lev_off[2], 4, 0,
                                  part_stride, nsplit, f));
            MMS_LAUNCH_CHECK(ctx);
        }
        for (int l = top ? 4 : 3; l <= lend; l++) {
            const int nc = 1 << l, np = nc / 2;
            MMS_CUDA_TRY(launch_k(k_l2l_c, dim3(np * np), dim3(4 * KT), (tsz + (size_t)f.NR) * sizeof(float),
                                  ctx->stream, pl->Lall, (const float *)pl->Lpart, (const float *)pl->Tl2l,
                                  pl->lev_off[l - 1], pl->lev_off[l], nc, np, part_stride, nsplit, f));
            MMS_LAUNCH_CHECK(ctx);
        }
        break;
    }
    case 4:
        // (timing path) near field then far field, both on the main stream
        if (leaf_threads(f) > 0) {
            if (!far) {
                MMS_TRY(p2p_launch(f, nbx, nby, rho, pl->Gn, phi, ctx->stream));
                MMS_LAUNCH_CHECK(ctx);
            } else {
                MMS_TRY(near_launch(ctx, rho, ctx->stream));
                MMS_LAUNCH_CHECK(ctx);
                MMS_TRY(l2p_launch_far(ctx, rho, phi));
            }
        } else {
            const size_t smem = ((size_t)f.Z * 9 * f.s * f.s + (size_t)f.Z * 4 * f.s * f.s + f.NR) * sizeof(float);
            const int threads = ((f.C + 31) / 32) * 32;
            k_l2p_p2p<<<f.nb * f.nb, threads, smem, ctx->stream>>>(rho, pl->Lall + pl->lev_off[f.L] * f.NR, pl->Vt,
                                                                  pl->Gn, phi, f, far);
            MMS_LAUNCH_CHECK(ctx);
        }
        break;
    default:
        break;
    }
    return MMS_OK;
}

#define MMS_FAR_CASES(X) X(6, 4) X(12, 8) X(20, 12) X(30, 18)

// sizes and enables the fused far-field kernel; leaves it off (per-stage
// kernels) when the device cannot co-schedule one CTA per SM
int far_prepare(mms_ctx *ctx, FmmPlan *pl)
{
    const FmmDev &f = pl->d;
    int coop = 0, sms = 0;
    MMS_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device));
    MMS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    if (!coop) return MMS_OK;
    const int NO = f.NR - f.NE, OSZ = f.NE * f.NE + NO * NO;
    int scratch = 0, occ = 0;
#define X(a, c)                                                                                      \
    if (f.NR == a && f.NE == c) {                                                                    \
        scratch = far_scratch<a, c>(f.C);                                                            \
        pl->far_smem = (size_t)(57 * OSZ + scratch) * sizeof(float);                                 \
        if (pl->far_smem > 227 * 1024) return MMS_OK;                                                \
        MMS_CUDA_TRY(cudaFuncSetAttribute(k_far<a, c>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                                          (int)pl->far_smem));                                      \
        MMS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_far<a, c>, 32 * RES_WARPS, \
                                                                   pl->far_smem));                   \
    }
    MMS_FAR_CASES(X)
#undef X
    if (occ < 1) return MMS_OK;
    if (cudaMalloc((void **)&pl->far_sync, sizeof(FarSync)) != cudaSuccess) {
        mms_set_error("FMM plan: device allocation failed");
        return MMS_ERR_NOMEM;
    }
    MMS_CUDA_TRY(cudaMemset(pl->far_sync, 0, sizeof(FarSync)));
    pl->far_grid = sms;  // one CTA per SM: co-resident with room to spare
    pl->far_fused = 1;
    return MMS_OK;
}

int far_launch(mms_ctx *ctx, const float *rho)
{
    FmmPlan *pl = ctx->fmm;
    const FmmDev &f = pl->d;
    const int nbx = std::min(f.nb, (f.X + f.s - 1) / f.s), nby = std::min(f.nb, (f.Y + f.s - 1) / f.s);
    const int lend = f.L - 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(pl->far_grid);
    cfg.blockDim = dim3(32 * RES_WARPS);
    cfg.dynamicSmemBytes = pl->far_smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
#define X(a, c)                                                                                                   \
    if (f.NR == a && f.NE == c) {                                                                                 \
        MMS_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_far<a, c>, rho, (const float *)pl->Wt, pl->Mall, pl->Lpart,        \
                                        pl->Lall, (const float *)pl->Tm2m, (const float *)pl->Tm2lc,                \
                                        (const float *)pl->Tl2l, (const int4 *)pl->res_items, pl->n_res_items,      \
                                        (const long long *)pl->lev_dev, f, nbx, nby, lend, pl->far_sync));         \
        MMS_LAUNCH_CHECK(ctx);                                                                                    \
        return MMS_OK;                                                                                            \
    }
    MMS_FAR_CASES(X)
#undef X
    mms_set_error("no fused far-field kernel for NR=%d", f.NR);
    return MMS_ERR_ARG;
}

// The potential of an RK4 stage's state.  With the resident M2L, k_p2m_row
// forms rho = div M as it stages the charges and stores rho and its BF16
// split; the near field, which reads the split, forks after it and runs
// beside M2M and M2L.  That saves the divergence launch on the chain (P = 4
// and 5 at leaf 8: 4 % and 10 % more RK4 steps/s at 256 x 256 x 3).  The
// longer M2L kernels (split FP32 at P = 6: 8 % fewer steps/s; tensor cores at
// P = 8: no change) lose more from sharing the SMs with the near field, so
// those plans, like the ones without the row P2M (generic leaf kernel, one
// level, the fused far field), run the divergence kernel first and fork the
// near field before the P2M.
int launch_potential_fmm_state(mms_ctx *ctx, const double *M, float *rho, float *phi)
{
    MmsRange nvtx_("mms/fmm_potential");
    FmmPlan *pl = ctx->fmm;
    if (!pl) {
        mms_set_error("FMM plan missing");
        return MMS_ERR_ARG;
    }
    const FmmDev &f = pl->d;
    if (leaf_threads(f) == 0 || f.L < 2 || pl->far_fused || !pl->m2l_resident) {
        MMS_TRY(launch_divergence_soa(ctx, M, rho));
        return launch_potential_fmm(ctx, rho, phi);
    }
    DivSrc dv{};
    dv.M = M;
    dv.rho = rho;
    dv.g = ctx->gk();
    dv.h = mmsdev::div_scale(ctx->g.dx, ctx->g.dy, ctx->g.dz);
    void *hi = nullptr, *lo = nullptr;
    if (fmm_split_target(ctx, &hi, &lo, &dv.nbx, &dv.nby)) {
        dv.hi = (__nv_bfloat16 *)hi;
        dv.lo = (__nv_bfloat16 *)lo;
    }
    MMS_TRY(p2m_launch(ctx, rho, &dv));
    pl->split_of = dv.hi ? rho : nullptr;
    MMS_TRY(near_fork(ctx, rho));
    for (int st = 1; st < 4; st++) MMS_TRY(launch_fmm_stage(ctx, st, rho, phi));
    MMS_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, pl->ev_join, 0));
    return l2p_launch_far(ctx, rho, phi);
}

// 1 when a bounded wait gave up since the plan was made: a grid barrier of the
// fused far-field kernel, or an mbarrier wait of the tensor-core near field or
// M2L (their flags are per device and cleared when such a plan is made)
int fmm_far_error(mms_ctx *ctx)
{
    if (!ctx->fmm) return 0;
    int err = 0;
    if (ctx->fmm->far_sync) {
        FarSync h{};
        if (cudaMemcpy(&h, ctx->fmm->far_sync, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
        err |= h.err != 0;
    }
    if (ctx->fmm->p2p_tc || ctx->fmm->m2l_tc) {
        int a = 0, b = 0;
        if (cudaMemcpyFromSymbol(&a, g_p2p_tc_err, sizeof a) != cudaSuccess ||
            cudaMemcpyFromSymbol(&b, g_m2l_tc_err, sizeof b) != cudaSuccess)
            return 1;
        err |= (ctx->fmm->p2p_tc && a) || (ctx->fmm->m2l_tc && b);
    }
    return err;
}

int launch_potential_fmm(mms_ctx *ctx, const float *rho, float *phi)
{
    MmsRange nvtx_("mms/fmm_potential");
    FmmPlan *pl = ctx->fmm;
    if (!pl) {
        mms_set_error("FMM plan missing");
        return MMS_ERR_ARG;
    }
    const FmmDev &f = pl->d;
    if (leaf_threads(f) == 0 || f.L < 2) {
        for (int st = 0; st < 5; st++) MMS_TRY(launch_fmm_stage(ctx, st, rho, phi));
        return MMS_OK;
    }
    // fork: the near field on the side stream, the far-field chain on the main one
    MMS_TRY(near_fork(ctx, rho));
    if (pl->far_fused)
        MMS_TRY(far_launch(ctx, rho));
    else
        for (int st = 0; st < 4; st++) MMS_TRY(launch_fmm_stage(ctx, st, rho, phi));
    MMS_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, pl->ev_join, 0));
    return l2p_launch_far(ctx, rho, phi);
}

// ===========================================================================
// Learned far-field network (solver MMS_SOLVER_SURROGATE).
//
// A linear multilevel convolutional operator over the quadtree of 8 x 8 x 3
// leaf boxes, with the FMM's data flow and its own per-level weights:
//   encoder  m_leaf = W^T q                      (replaces P2M)
//   down     m_par  = sum_child M2M_l m_child     (replaces M2M)
//   lateral  l_t   += sum_{o in IL(t)} M2L_l m_{t-o}  (replaces M2L; the
//                     reference's interaction lists, Box.cu:171-195)
//   up       l_chd += L2L_l l_par                (replaces L2L)
//   decoder  phi    = V^T l_leaf + exact near field (replaces L2P; the near
//                     field is the FMM's own P2P over the 3 x 3 leaf
//                     neighbourhood)
// Widths: FN_NE channels even and FN_NO odd under z -> -z, every table block
// diagonal (the layout of the FMM's parity blocks).  The weights come from
// mms_ctx_set_surrogate (trained by the mms_farnet_* kernels); they are
// indexed by depth (0 = leaf), the tables here by level of this grid.
//
// Three launches on the main stream beside the near field on the side
// stream: k_up<24,16> (encoder and the whole upward pass), the resident M2L with
// per-level tables, and k_fn_down (the whole downward pass, decoder, and the
// join with the near field).
constexpr int FN_DOWN_THREADS = 256;
constexpr int FN_DN_CELLS = (FN_Z * 16 * 16 + FN_DOWN_THREADS - 1) / FN_DOWN_THREADS;  // cells per thread in k_fn_down

namespace {

// stage n floats (n % 4 == 0, 16-byte aligned) into shared memory with
// asynchronous copies; commit only (the caller waits)
__device__ __forceinline__ void fn_stage(float *dst, const float *src, int n)
{
    for (int i = threadIdx.x * 4; i < n; i += blockDim.x * 4) umma::cp_async16(umma::smem_u32(dst + i), src + i, true);
}

// Downward pass, decoder and the join with the near field.  CTA = one box of
// level L - 1 (its 4 leaf boxes; one leaf box when L = 2): the locals of its
// ancestors from level 2 down (L2L of the parent's final local plus the
// box's interaction-list local, one box per level), its leaves' locals, then
// phi = near field (nnear partials, added in order) + V^T l_leaf at every
// cell of the 16 x 16 x 3 region.
template <int NR_, int NE_>
__global__ void __launch_bounds__(FN_DOWN_THREADS) k_fn_down(const float *__restrict__ Lp,
                                                             const float *__restrict__ Tl2l,
                                                             const float *__restrict__ V,
                                                             const float *__restrict__ near, int nnear,
                                                             long long near_stride, float *__restrict__ phi,
                                                             const long long *__restrict__ lev_off, FmmDev f)
{
    constexpr int OSZ_ = FnShape<NR_, NE_>::OSZ;
    __shared__ float cur[NR_], nxt[NR_], leaf[4][NR_];
    extern __shared__ __align__(16) float dsm[];
    const int L = f.L;
    float *Vs = dsm;                  // [NR][C]
    // L2L tables the chain uses: for levels 3 .. L-1 the one of the CTA's
    // ancestor's child position, then the 4 of level L-1 (the leaves'); they
    // and the decoder are constant, so they stream in while the predecessors
    // finish (group 0: tables, group 1: decoder)
    float *Ts = Vs + NR_ * FN_C;
    float *Lc = Ts + (L > 2 ? (L + 1) * OSZ_ : 0);  // interaction-list locals: ancestors 2..L-1, 4 leaves
    if (L > 2) {
        const int np = 1 << (L - 1), pbx = blockIdx.x % np, pby = blockIdx.x / np;
        for (int l = 3; l <= L - 1; l++) {
            const int sh = L - 1 - l, bx = pbx >> sh, by = pby >> sh;
            const int c = (by & 1) * 2 + (bx & 1);
            fn_stage(Ts + (l - 3) * OSZ_, Tl2l + ((long long)(l - 1 - 2) * 4 + c) * OSZ_, OSZ_);
        }
        fn_stage(Ts + (L - 3) * OSZ_, Tl2l + (long long)(L - 1 - 2) * 4 * OSZ_, 4 * OSZ_);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    fn_stage(Vs, V, NR_ * FN_C);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    pdl_begin();
    // the near field of this CTA's cells, every load issued before anything waits
    int nlx0, nly0, nrw;
    if (L <= 2) {
        nlx0 = blockIdx.x % (1 << L);
        nly0 = blockIdx.x / (1 << L);
        nrw = FN_S;
    } else {
        nlx0 = 2 * (blockIdx.x % (1 << (L - 1)));
        nly0 = 2 * (blockIdx.x / (1 << (L - 1)));
        nrw = 2 * FN_S;
    }
    float nv[FN_DN_CELLS];
#pragma unroll
    for (int r = 0; r < FN_DN_CELLS; r++) {
        const int e = threadIdx.x + r * FN_DOWN_THREADS;
        const int rx = e % nrw, ry = (e / nrw) % nrw, lz = e / (nrw * nrw);
        const int x = nlx0 * FN_S + rx, y = nly0 * FN_S + ry;
        float v = 0.f;
        if (e < FN_Z * nrw * nrw && x < f.X && y < f.Y) {
            const long long cell = ((long long)lz * f.Y + y) * f.X + x;
            v = __ldg(&near[cell]);
            for (int qn = 1; qn < nnear; qn++) v += __ldg(&near[qn * near_stride + cell]);
        }
        nv[r] = v;
    }
    if (L > 2) {
        const int np = 1 << (L - 1), pbx = blockIdx.x % np, pby = blockIdx.x / np;
        // the CTA's chain, every load in flight at once: level l (2..L-1) ancestor, then the 4 leaves
        for (int i = threadIdx.x; i < (L + 2) * (NR_ / 4); i += blockDim.x) {
            const int r = i / (NR_ / 4), k4 = i % (NR_ / 4);
            long long box;
            if (r < L - 2) {
                const int l = r + 2, sh = L - 1 - l;
                box = lev_off[l] + (long long)(pby >> sh) * (1 << l) + (pbx >> sh);
            } else {
                const int c = r - (L - 2);
                box = lev_off[L] + (long long)(2 * pby + (c >> 1)) * (1 << L) + 2 * pbx + (c & 1);
            }
            umma::cp_async16(umma::smem_u32(Lc + r * NR_ + 4 * k4), Lp + box * NR_ + 4 * k4, true);
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");  // group 2: the chain
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    int nlf, lx0, ly0;  // leaves handled and the first one
    if (L <= 2) {
        // one leaf box per CTA, its local is its interaction-list local
        const int n = 1 << L;
        lx0 = blockIdx.x % n;
        ly0 = blockIdx.x / n;
        nlf = 1;
        for (int k = threadIdx.x; k < NR_; k += blockDim.x)
            leaf[0][k] = Lp[(lev_off[L] + (long long)ly0 * n + lx0) * NR_ + k];
    } else {
        const int np = 1 << (L - 1);
        const int pbx = blockIdx.x % np, pby = blockIdx.x / np;
        for (int k = threadIdx.x; k < NR_; k += blockDim.x) cur[k] = Lc[k];
        __syncthreads();
        for (int l = 3; l <= L - 1; l++) {
            const float *T = Ts + (l - 3) * OSZ_;
            for (int k = threadIdx.x; k < NR_; k += blockDim.x) nxt[k] = Lc[(l - 2) * NR_ + k] + blk_apply<NR_, NE_>(T, cur, k);
            __syncthreads();
            for (int k = threadIdx.x; k < NR_; k += blockDim.x) cur[k] = nxt[k];
            __syncthreads();
        }
        lx0 = 2 * pbx;
        ly0 = 2 * pby;
        nlf = 4;
        for (int i = threadIdx.x; i < 4 * NR_; i += blockDim.x) {
            const int c = i / NR_, k = i % NR_;
            const float *T = Ts + (L - 3 + c) * OSZ_;
            leaf[c][k] = Lc[(L - 2 + c) * NR_ + k] + blk_apply<NR_, NE_>(T, cur, k);
        }
    }
    __syncthreads();
    // decoder + near field over the region, a row at a time; the near field
    // (complete before the launch) was read into registers at the start
    const int gw = nlf == 4 ? 2 : 1, rw = gw * FN_S;
#pragma unroll
    for (int r = 0; r < FN_DN_CELLS; r++) {
        const int e = threadIdx.x + r * FN_DOWN_THREADS;
        if (e >= FN_Z * rw * rw) break;
        const int rx = e % rw, ry = (e / rw) % rw, lz = e / (rw * rw);
        const int x = lx0 * FN_S + rx, y = ly0 * FN_S + ry;
        if (x >= f.X || y >= f.Y) continue;
        const long long cell = ((long long)lz * f.Y + y) * f.X + x;
        const int b = (ry / FN_S) * gw + rx / FN_S, c = lz * FN_S * FN_S + (ry % FN_S) * FN_S + rx % FN_S;
        float acc = nv[r];
        const float *lb = leaf[b];
#pragma unroll 8
        for (int k = 0; k < NR_; k++) acc = fmaf(Vs[k * FN_C + c], lb[k], acc);
        phi[cell] = acc;
    }
}

size_t fn_down_smem(int L, int NR, int OSZ)
{
    return ((size_t)NR * FN_C + (size_t)(L > 2 ? L + 1 : 0) * OSZ + (size_t)(L + 2) * NR) * sizeof(float);
}

// the widths the solver runs: X(NR, NE)
#define MMS_FN_WIDTHS(X) X(24, 16) X(40, 24)

}  // namespace

// tables per level of this grid from a weight vector of width Sh (encoder
// scaled to physical units: phi = dx^2 net(rho) for cubic cells), into the
// plan's buffers (sized for the widest network)
template <class Sh>
int farnet_tables(mms_ctx *ctx, const float *w)
{
    FmmPlan *pl = ctx->fmm;
    const FmmDev &f = pl->d;
    constexpr int NR = Sh::NR, OSZ = Sh::OSZ;
    const int L = std::max(f.L, 2);
    const int nlev = L - 1;  // levels 2..L
    const double sc = ctx->g.dx * ctx->g.dx;
    std::vector<float> W((size_t)FN_C * NR), V((size_t)NR * FN_C);
    for (int c = 0; c < FN_C; c++)  // [c][k] -> [k][c]
        for (int k = 0; k < NR; k++) W[(size_t)k * FN_C + c] = (float)(w[Sh::off_W() + c * NR + k] * sc);
    for (size_t i = 0; i < V.size(); i++) V[i] = w[Sh::off_V() + i];
    std::vector<float> M2L((size_t)nlev * 49 * OSZ), M2M((size_t)std::max(1, nlev - 1) * 4 * OSZ, 0.f),
        L2L(M2M.size(), 0.f);
    for (int l = 2; l <= L; l++) {
        const int d = L - l;
        memcpy(&M2L[(size_t)(l - 2) * 49 * OSZ], w + Sh::off_M2L(d), 49 * OSZ * sizeof(float));
        if (l < L) {  // parent level l, depth d >= 1
            memcpy(&M2M[(size_t)(l - 2) * 4 * OSZ], w + Sh::off_M2M(d), 4 * OSZ * sizeof(float));
            memcpy(&L2L[(size_t)(l - 2) * 4 * OSZ], w + Sh::off_L2L(d), 4 * OSZ * sizeof(float));
        }
    }
    // buffer sizes of the widest network, so that either width fits
    constexpr int OSZ_MAX = FnWide::OSZ;
    const size_t cap[5] = {(size_t)FN_C * FN_NR_MAX, (size_t)FN_NR_MAX * FN_C, (size_t)nlev * 49 * OSZ_MAX,
                           (size_t)std::max(1, nlev - 1) * 4 * OSZ_MAX, (size_t)std::max(1, nlev - 1) * 4 * OSZ_MAX};
    float **dst[5] = {&pl->fnW, &pl->fnV, &pl->fnM2L, &pl->fnM2M, &pl->fnL2L};
    const std::vector<float> *src[5] = {&W, &V, &M2L, &M2M, &L2L};
    for (int i = 0; i < 5; i++) {
        if (!*dst[i]) {
            if (cudaMalloc((void **)dst[i], cap[i] * sizeof(float)) != cudaSuccess) {
                mms_set_error("surrogate: device allocation failed");
                return MMS_ERR_NOMEM;
            }
            pl->bytes += cap[i] * sizeof(float);
        }
        MMS_CUDA_TRY(cudaMemcpyAsync(*dst[i], src[i]->data(), src[i]->size() * sizeof(float),
                                     cudaMemcpyHostToDevice, ctx->stream));
    }
    pl->fn_nr = NR;
    pl->fn_ne = Sh::NE;
    return MMS_OK;
}

// Binds a weight vector (indexed by depth) to the context's plan.  Its length
// picks the width: FnTrain (24 channels) or FnWide (32).  Leaf side 8 and 3
// layers only.
int farnet_bind(mms_ctx *ctx, const float *w, long long count)
{
    FmmPlan *pl = ctx->fmm;
    if (!pl) {
        mms_set_error("surrogate: no FMM plan");
        return MMS_ERR_ARG;
    }
    const FmmDev &f = pl->d;
    if (f.s != FN_S || f.Z != FN_Z) {
        mms_set_error("surrogate: the network works on 8 x 8 x 3 leaf boxes (leaf side %d, %d layers given)", f.s,
                      f.Z);
        return MMS_ERR_ARG;
    }
    if (f.L > FN_DEPTHS + 1) {
        mms_set_error("surrogate: a grid of %d quadtree levels exceeds the network's %d depths", f.L, FN_DEPTHS);
        return MMS_ERR_ARG;
    }
    if (count == FnTrain::num_params()) {
        MMS_TRY(farnet_tables<FnTrain>(ctx, w));
    } else if (count == FnWide::num_params()) {
        MMS_TRY(farnet_tables<FnWide>(ctx, w));
    } else {
        mms_set_error("surrogate: %lld weights given; the networks have %lld (width %d) or %lld (width %d)", count,
                      FnTrain::num_params(), FnTrain::NR, FnWide::num_params(), FnWide::NR);
        return MMS_ERR_ARG;
    }
    if (!pl->fnM) {
        const size_t nb = (size_t)std::max(pl->nbox_total, 1LL);
        if (cudaMalloc((void **)&pl->fnM, nb * FN_NR_MAX * sizeof(float)) != cudaSuccess ||
            cudaMalloc((void **)&pl->fnLp, nb * FN_NR_MAX * sizeof(float)) != cudaSuccess ||
            cudaMalloc((void **)&pl->fnCtr, nb * sizeof(unsigned)) != cudaSuccess) {
            mms_set_error("surrogate: device allocation failed");
            return MMS_ERR_NOMEM;
        }
        pl->bytes += nb * (2 * FN_NR_MAX * sizeof(float) + sizeof(unsigned));
        MMS_CUDA_TRY(cudaMemsetAsync(pl->fnM, 0, nb * FN_NR_MAX * sizeof(float), ctx->stream));
        MMS_CUDA_TRY(cudaMemsetAsync(pl->fnLp, 0, nb * FN_NR_MAX * sizeof(float), ctx->stream));
        MMS_CUDA_TRY(cudaMemsetAsync(pl->fnCtr, 0, nb * sizeof(unsigned), ctx->stream));
#define X(NR_, NE_)                                                                                              \
    MMS_TRY(m2l_res_prepare(NR_, NE_));                                                                          \
    MMS_CUDA_TRY(cudaFuncSetAttribute(k_up<NR_, NE_>, cudaFuncAttributeMaxDynamicSharedMemorySize,              \
                                      (int)up_smem(FN_DEPTHS + 1, NR_, NE_, FN_DEPTHS - 1)));                   \
    MMS_CUDA_TRY(cudaFuncSetAttribute(k_up<NR_, NE_>, cudaFuncAttributePreferredSharedMemoryCarveout,           \
                                      cudaSharedmemCarveoutMaxShared));                                         \
    MMS_CUDA_TRY(cudaFuncSetAttribute(k_fn_down<NR_, NE_>, cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                                      (int)fn_down_smem(FN_DEPTHS + 1, NR_, FnShape<NR_, NE_>::OSZ)));         \
    MMS_CUDA_TRY(cudaFuncSetAttribute(k_fn_down<NR_, NE_>, cudaFuncAttributePreferredSharedMemoryCarveout,      \
                                      cudaSharedmemCarveoutMaxShared));
        MMS_FN_WIDTHS(X)
#undef X
    }
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    pl->fn_ready = 1;
    return MMS_OK;
}

// the network's three launches at width Sh: upward pass, interaction lists,
// downward pass + decoder + the join with the near field
template <class Sh>
int farnet_launch(mms_ctx *ctx, const float *rho, float *phi)
{
    FmmPlan *pl = ctx->fmm;
    const FmmDev &f = pl->d;
    constexpr int NR = Sh::NR, NE = Sh::NE, OSZ = Sh::OSZ;
    const int cb = up_level(f.L);
    MMS_CUDA_TRY(launch_k(k_up<NR, NE>, dim3(1u << (2 * cb)), dim3(UP_THREADS), up_smem(f.L, NR, NE, f.L - 2),
                          ctx->stream, rho, (const float *)pl->fnW, (const float *)pl->fnM2M, 4LL * OSZ, pl->fnM,
                          (const long long *)pl->lev_dev, pl->fnCtr, f, cb));
    MMS_LAUNCH_CHECK(ctx);
    const float *near = pl->p2p_tc ? pl->near3 : pl->near;
    const int nnear = pl->p2p_tc ? 3 : 1;
    FmmDev fn = f;
    fn.NR = NR;
    fn.NE = NE;
    MMS_TRY(m2l_res_launch(fn, pl->n_res_items, pl->fnM, pl->fnLp, pl->fnM2L, pl->res_items, pl->lev_dev, ctx->stream,
                           49LL * OSZ));
    MMS_LAUNCH_CHECK(ctx);
    MMS_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, pl->ev_join, 0));
    const unsigned ndown = f.L > 2 ? 1u << (2 * (f.L - 1)) : 1u << (2 * f.L);
    MMS_CUDA_TRY(launch_k(k_fn_down<NR, NE>, dim3(ndown), dim3(FN_DOWN_THREADS), fn_down_smem(f.L, NR, OSZ),
                          ctx->stream, (const float *)pl->fnLp, (const float *)pl->fnL2L, (const float *)pl->fnV, near,
                          nnear, (long long)ctx->N, phi, (const long long *)pl->lev_dev, f));
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

// surrogate potential: the exact near field on the side stream; the network's
// three launches on the main one; the last adds the two
int launch_potential_surrogate(mms_ctx *ctx, const float *rho, float *phi)
{
    MmsRange nvtx_("mms/surrogate_potential");
    FmmPlan *pl = ctx->fmm;
    if (!pl || !pl->fn_ready) {
        mms_set_error("surrogate solver: no weights bound (mms_ctx_set_surrogate)");
        return MMS_ERR_NOT_READY;
    }
    const FmmDev &f = pl->d;
    MMS_TRY(near_fork(ctx, rho));
    if (f.L < 2) {
        // no far field: every box is in every other's near zone
        MMS_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, pl->ev_join, 0));
        k_sum_parts<<<(unsigned)div_up(ctx->N, 256), 256, 0, ctx->stream>>>(pl->p2p_tc ? pl->near3 : pl->near,
                                                                            pl->p2p_tc ? 3 : 1, ctx->N, phi);
        MMS_LAUNCH_CHECK(ctx);
        return MMS_OK;
    }
    if (pl->fn_nr == FnWide::NR) return farnet_launch<FnWide>(ctx, rho, phi);
    return farnet_launch<FnTrain>(ctx, rho, phi);
}

int fmm_split_target(const mms_ctx *ctx, void **hi, void **lo, int *nbx, int *nby)
{
    const FmmPlan *pl = ctx->fmm;
    if (!pl || !pl->p2p_tc) return 0;
    const FmmDev &f = pl->d;
    *nbx = std::min(f.nb, (f.X + f.s - 1) / f.s);
    *nby = std::min(f.nb, (f.Y + f.s - 1) / f.s);
    *hi = pl->ntcR;
    *lo = pl->ntcR + (size_t)f.Z * 64 * *nbx * *nby;
    return 1;
}

void fmm_split_written(mms_ctx *ctx, const float *rho)
{
    if (ctx->fmm) ctx->fmm->split_of = rho;
}

// FMM potential and its exact near-field part (for the surrogate's targets)
int launch_potential_split(mms_ctx *ctx, const float *rho, float *phi, float *near)
{
    FmmPlan *pl = ctx->fmm;
    if (!pl || leaf_threads(pl->d) == 0) {
        mms_set_error("potential split: needs an FMM plan with a power-of-two leaf side");
        return MMS_ERR_ARG;
    }
    MMS_TRY(launch_potential_fmm(ctx, rho, phi));
    const FmmDev &f = pl->d;
    if (pl->p2p_tc) {
        // the near field the potential used: its three partials, added in L2P's order
        k_sum_parts<<<(unsigned)div_up((long long)ctx->N, 256), 256, 0, ctx->stream>>>(pl->near3, 3, ctx->N, near);
    } else {
        const int nbx = std::min(f.nb, (f.X + f.s - 1) / f.s), nby = std::min(f.nb, (f.Y + f.s - 1) / f.s);
        MMS_TRY(p2p_launch(f, nbx, nby, rho, pl->Gn, near, ctx->stream));
    }
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

extern "C" int mms_fmm_info(const mms_ctx *ctx, int *levels, int *leaf, int *order, double stage_flops[5],
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
    if (stage_flops)
        for (int i = 0; i < 5; i++) stage_flops[i] = pl->stage_flops[i];
    if (p2p_pairs) *p2p_pairs = pl->p2p_pairs;
    if (m2l_pairs) *m2l_pairs = pl->m2l_pairs;
    return MMS_OK;
}

extern "C" int mms_fmm_kernels(const mms_ctx *ctx, int *near_tc, int *m2l_tc)
{
    if (!ctx || !ctx->fmm) {
        mms_set_error("context has no FMM plan");
        return MMS_ERR_ARG;
    }
    if (near_tc) *near_tc = ctx->fmm->p2p_tc;
    if (m2l_tc) *m2l_tc = ctx->fmm->m2l_tc;
    return MMS_OK;
}

extern "C" int mms_fmm_stage_times(mms_ctx *ctx, const float *rho, float *phi, int reps, double ms[5])
{
    if (!ctx || !ctx->fmm || !rho || !phi || reps < 1 || !ms) {
        mms_set_error("mms_fmm_stage_times: bad argument or no FMM plan");
        return MMS_ERR_ARG;
    }
    cudaEvent_t e0, e1;
    MMS_CUDA_TRY(cudaEventCreate(&e0));
    MMS_CUDA_TRY(cudaEventCreate(&e1));
    int st = launch_potential_fmm(ctx, rho, phi);  // valid inputs for every stage
    for (int s = 0; s < 5 && st == MMS_OK; s++) {
        st = launch_fmm_stage(ctx, s, rho, phi);  // warm
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < reps && st == MMS_OK; r++) st = launch_fmm_stage(ctx, s, rho, phi);
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        ms[s] = (double)t / reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}
