// Training of the learned far-field network (mms_farnet_*): forward pass,
// relative-L2 loss against far-field targets, adjoint passes, weight
// gradients on the tensor cores, Adam.
//
// The network (farnet.cuh) is the FMM's data flow with its own weights per
// level: encoder (P2M), down (M2M), interaction-list lateral (M2L), up (L2L),
// decoder (L2P); the exact near field is not part of it.  Activations are
// FP32, one [batch][box][NR] tensor per kind over the boxes of every level
// (levels 2..L, level-major, box row-major inside a level):
//   M   multipoles           Lf  final locals (M2L + L2L of the parent's)
//   dM  dloss/dM             dL  dloss/dLf
// Every forward and adjoint kernel gives each output element to one thread
// (no atomics: fixed summation order, reproducible bits).  The weight
// gradients are sums of outer products over boxes and samples, each family
// one GEMM: the operands are gathered into K-major BF16 hi/lo planes
// ([hi | lo | hi] against [hi | hi | lo], relative error ~2^-16 per product)
// and multiplied by the tcgen05 core (umma_gemm_bf16_splitk: the long K
// range, boxes x samples, split over CTAs, the partials summed in a fixed
// order); the block-diagonal entries are then added into the gradient vector.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include <cuda_bf16.h>

#include "farnet.cuh"
#include "mms_internal.cuh"

using bf16 = __nv_bfloat16;

struct mms_farnet {
    int X = 0, Y = 0, L = 0, nb = 0, batch = 0;
    long long N = 0;     // cells per sample (FN_Z * Y * X)
    long long nbox = 0;  // boxes of levels 2..L
    long long lev_off[FN_DEPTHS + 3] = {};
    long long *lev_dev = nullptr;
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // weights, gradient, Adam moments
    float *sc = nullptr;  // per-weight step scale (1 unless set)
    float *M = nullptr, *Lf = nullptr, *dM = nullptr, *dL = nullptr;
    float *out = nullptr, *dout = nullptr;
    double *lsum = nullptr;
    bf16 *A = nullptr, *B = nullptr;
    float *Cm = nullptr, *Cp = nullptr;  // GEMM result, split-K partials
    size_t a_elems = 0, b_elems = 0, c_elems = 0, p_elems = 0;
    long long step = 0;
    size_t bytes = 0;
};

namespace {

enum Fam { FAM_W = 0, FAM_V = 1, FAM_M2L = 2, FAM_M2M = 3, FAM_L2L = 4 };

struct NetK {
    int X, Y, L, nb, batch;
    long long N, nbox;
    long long lev[FN_DEPTHS + 3];
};

// out_k = sum_j T[blk][j][k] x_j (x: NR floats of global memory)
__device__ __forceinline__ float t_apply(const float *__restrict__ T, const float *__restrict__ x, int k)
{
    float acc = 0.f;
    if (k < FN_NE) {
        for (int j = 0; j < FN_NE; j++) acc = fmaf(T[j * FN_NE + k], x[j], acc);
    } else {
        const float *To = T + FN_NE * FN_NE;
        const int kk = k - FN_NE;
        for (int j = 0; j < FN_NO; j++) acc = fmaf(To[j * FN_NO + kk], x[FN_NE + j], acc);
    }
    return acc;
}

// out_j = sum_k T[blk][j][k] x_k (the adjoint of t_apply)
__device__ __forceinline__ float t_apply_adj(const float *__restrict__ T, const float *__restrict__ x, int j)
{
    float acc = 0.f;
    if (j < FN_NE) {
        const float *row = T + j * FN_NE;
        for (int k = 0; k < FN_NE; k++) acc = fmaf(row[k], x[k], acc);
    } else {
        const float *row = T + FN_NE * FN_NE + (j - FN_NE) * FN_NO;
        for (int k = 0; k < FN_NO; k++) acc = fmaf(row[k], x[FN_NE + k], acc);
    }
    return acc;
}

// o = (ox, oy) lies in the interaction list of the box at (tx, ty)
__device__ __forceinline__ bool in_list(int ox, int oy, int tx, int ty)
{
    const int px = tx & 1, py = ty & 1;
    return max(abs(ox), abs(oy)) >= 2 && ox >= px - 3 && ox <= px + 2 && oy >= py - 3 && oy <= py + 2;
}

__device__ __forceinline__ long long cell_of(const NetK &k, int bx, int by, int c, bool *ok)
{
    const int x = bx * FN_S + c % FN_S, y = by * FN_S + (c / FN_S) % FN_S, z = c / (FN_S * FN_S);
    *ok = x < k.X && y < k.Y;
    return ((long long)z * k.Y + y) * k.X + x;
}

// encoder: M[b][leaf][k] = sum_c W[c][k] u[b][cell(leaf, c)]
__global__ void k_t_p2m(const float *__restrict__ u, const float *__restrict__ w, float *__restrict__ M, NetK k)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nl = (long long)k.nb * k.nb;
    if (i >= k.batch * nl * FN_NR) return;
    const int ch = (int)(i % FN_NR);
    const long long bl = i / FN_NR;
    const int b = (int)(bl / nl), box = (int)(bl % nl), bx = box % k.nb, by = box / k.nb;
    const float *W = w + fn_off_W();
    const float *ub = u + (long long)b * k.N;
    float acc = 0.f;
    for (int c = 0; c < FN_C; c++) {
        bool ok;
        const long long cell = cell_of(k, bx, by, c, &ok);
        if (ok) acc = fmaf(W[c * FN_NR + ch], ub[cell], acc);
    }
    M[((long long)b * k.nbox + k.lev[k.L] + box) * FN_NR + ch] = acc;
}

// down: level l from level l + 1
__global__ void k_t_m2m(const float *__restrict__ w, float *__restrict__ M, NetK k, int l)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = 1 << l;
    if (i >= (long long)k.batch * n * n * FN_NR) return;
    const int ch = (int)(i % FN_NR);
    const long long bp = i / FN_NR;
    const int b = (int)(bp / ((long long)n * n)), p = (int)(bp % ((long long)n * n)), px = p % n, py = p / n;
    const float *A = w + fn_off_M2M(k.L - l);
    const float *Mb = M + (long long)b * k.nbox * FN_NR;
    float acc = 0.f;
    for (int c = 0; c < 4; c++) {
        const int cx = 2 * px + (c & 1), cy = 2 * py + (c >> 1);
        acc += t_apply(A + c * FN_OSZ, Mb + (k.lev[l + 1] + (long long)cy * 2 * n + cx) * FN_NR, ch);
    }
    M[((long long)b * k.nbox + k.lev[l] + p) * FN_NR + ch] = acc;
}

// lateral + up: Lf_l[t] = sum_{o in IL(t)} M2L_l[o] M_l[t - o] + L2L(Lf_{l-1}[parent])
__global__ void k_t_local(const float *__restrict__ w, const float *__restrict__ M, float *__restrict__ Lf, NetK k,
                          int l)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = 1 << l;
    if (i >= (long long)k.batch * n * n * FN_NR) return;
    const int ch = (int)(i % FN_NR);
    const long long bt = i / FN_NR;
    const int b = (int)(bt / ((long long)n * n)), t = (int)(bt % ((long long)n * n)), tx = t % n, ty = t / n;
    const float *T = w + fn_off_M2L(k.L - l);
    const float *Mb = M + ((long long)b * k.nbox + k.lev[l]) * FN_NR;
    float acc = 0.f;
    const int px = tx & 1, py = ty & 1;
    for (int oy = py - 3; oy <= py + 2; oy++)
        for (int ox = px - 3; ox <= px + 2; ox++) {
            if (max(abs(ox), abs(oy)) < 2) continue;
            const int sx = tx - ox, sy = ty - oy;
            if (sx < 0 || sy < 0 || sx >= n || sy >= n) continue;
            acc += t_apply(T + ((oy + 3) * 7 + ox + 3) * FN_OSZ, Mb + ((long long)sy * n + sx) * FN_NR, ch);
        }
    if (l > 2) {
        const float *Bt = w + fn_off_L2L(k.L - (l - 1));
        const int c = (ty & 1) * 2 + (tx & 1);
        acc += t_apply(Bt + c * FN_OSZ,
                       Lf + ((long long)b * k.nbox + k.lev[l - 1] + (long long)(ty >> 1) * (n >> 1) + (tx >> 1)) * FN_NR,
                       ch);
    }
    Lf[((long long)b * k.nbox + k.lev[l] + t) * FN_NR + ch] = acc;
}

// decoder: out[b][cell] = sum_k V[k][c] Lf_L[b][leaf][k]
__global__ void k_t_l2p(const float *__restrict__ w, const float *__restrict__ Lf, float *__restrict__ out, NetK k)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k.batch * k.N) return;
    const int b = (int)(i / k.N);
    const long long cell = i % k.N;
    const int x = (int)(cell % k.X), y = (int)((cell / k.X) % k.Y), z = (int)(cell / ((long long)k.X * k.Y));
    const int bx = x / FN_S, by = y / FN_S, c = z * FN_S * FN_S + (y % FN_S) * FN_S + x % FN_S;
    const float *V = w + fn_off_V();
    const float *lb = Lf + ((long long)b * k.nbox + k.lev[k.L] + (long long)by * k.nb + bx) * FN_NR;
    float acc = 0.f;
    for (int ch = 0; ch < FN_NR; ch++) acc = fmaf(V[ch * FN_C + c], lb[ch], acc);
    out[i] = acc;
}

// loss sums and the output adjoint: dout = 2 (out - far) / (nrm_b batch)
__global__ void k_t_loss(const float *__restrict__ out, const float *__restrict__ far, const float *__restrict__ nrm,
                         float *__restrict__ dout, double *__restrict__ lsum, NetK k, int nbatch)
{
    const int b = blockIdx.y;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double r2 = 0.0;
    if (i < k.N) {
        const long long e = (long long)b * k.N + i;
        const float r = out[e] - far[e];
        dout[e] = 2.f * r / (nrm[b] * (float)nbatch);
        r2 = (double)r * r;
    }
    for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = r2;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += red[q];
        atomicAdd(&lsum[b], s);
    }
}

// adjoint of the decoder: dL_L[b][leaf][k] = sum_c V[k][c] dout[b][cell(leaf, c)]
__global__ void k_t_l2p_adj(const float *__restrict__ w, const float *__restrict__ dout, float *__restrict__ dL, NetK k)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nl = (long long)k.nb * k.nb;
    if (i >= k.batch * nl * FN_NR) return;
    const int ch = (int)(i % FN_NR);
    const long long bl = i / FN_NR;
    const int b = (int)(bl / nl), box = (int)(bl % nl), bx = box % k.nb, by = box / k.nb;
    const float *V = w + fn_off_V() + (long long)ch * FN_C;
    const float *db = dout + (long long)b * k.N;
    float acc = 0.f;
    for (int c = 0; c < FN_C; c++) {
        bool ok;
        const long long cell = cell_of(k, bx, by, c, &ok);
        if (ok) acc = fmaf(V[c], db[cell], acc);
    }
    dL[((long long)b * k.nbox + k.lev[k.L] + box) * FN_NR + ch] = acc;
}

// adjoint of the up pass into level l - 1: dL_{l-1}[p] = sum_c L2L[c]^T dL_l[child c]
__global__ void k_t_l2l_adj(const float *__restrict__ w, float *__restrict__ dL, NetK k, int l)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int np = 1 << (l - 1), nc = 1 << l;
    if (i >= (long long)k.batch * np * np * FN_NR) return;
    const int j = (int)(i % FN_NR);
    const long long bp = i / FN_NR;
    const int b = (int)(bp / ((long long)np * np)), p = (int)(bp % ((long long)np * np)), px = p % np, py = p / np;
    const float *Bt = w + fn_off_L2L(k.L - (l - 1));
    const float *db = dL + ((long long)b * k.nbox + k.lev[l]) * FN_NR;
    float acc = 0.f;
    for (int c = 0; c < 4; c++) {
        const int cx = 2 * px + (c & 1), cy = 2 * py + (c >> 1);
        acc += t_apply_adj(Bt + c * FN_OSZ, db + ((long long)cy * nc + cx) * FN_NR, j);
    }
    dL[((long long)b * k.nbox + k.lev[l - 1] + p) * FN_NR + j] = acc;
}

// adjoint into the multipoles of level l: dM_l[s] = sum over targets t = s + o
// whose list holds o of M2L[o]^T dL_l[t], plus M2M[c]^T dM_{l-1}[parent]
__global__ void k_t_dm(const float *__restrict__ w, const float *__restrict__ dL, float *__restrict__ dM, NetK k, int l)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = 1 << l;
    if (i >= (long long)k.batch * n * n * FN_NR) return;
    const int j = (int)(i % FN_NR);
    const long long bs = i / FN_NR;
    const int b = (int)(bs / ((long long)n * n)), s = (int)(bs % ((long long)n * n)), sx = s % n, sy = s / n;
    const float *T = w + fn_off_M2L(k.L - l);
    const float *db = dL + ((long long)b * k.nbox + k.lev[l]) * FN_NR;
    float acc = 0.f;
    for (int oy = -3; oy <= 3; oy++)
        for (int ox = -3; ox <= 3; ox++) {
            const int tx = sx + ox, ty = sy + oy;
            if (tx < 0 || ty < 0 || tx >= n || ty >= n || !in_list(ox, oy, tx, ty)) continue;
            acc += t_apply_adj(T + ((oy + 3) * 7 + ox + 3) * FN_OSZ, db + ((long long)ty * n + tx) * FN_NR, j);
        }
    if (l > 2) {
        const float *A = w + fn_off_M2M(k.L - (l - 1));
        const int c = (sy & 1) * 2 + (sx & 1);
        acc += t_apply_adj(A + c * FN_OSZ,
                           dM + ((long long)b * k.nbox + k.lev[l - 1] + (long long)(sy >> 1) * (n >> 1) + (sx >> 1)) *
                                    FN_NR,
                           j);
    }
    dM[((long long)b * k.nbox + k.lev[l] + s) * FN_NR + j] = acc;
}

// ---- weight gradients ---------------------------------------------------------
// One family = one GEMM C[fa][fb] = sum_r A[fa][r] B[fb][r] over the rows r =
// (sample, box of the family's level).  feature value of side 0 (A) / 1 (B):
//   W    A: c -> u at cell c of the leaf         B: k -> dM_L
//   V    A: k -> Lf_L                            B: c -> dout at cell c
//   M2L  A: (slot, j) -> M_l[t - o] (0 unless o in IL(t) and on the level)
//                                                B: k -> dL_l[t]
//   M2M  A: (c, j) -> M_{l+1}[child c]           B: k -> dM_l
//   L2L  A: j -> Lf_l                            B: (c, k) -> dL_{l+1}[child c]
struct GatherP {
    int fam, side, l, nfeat, n;  // n: boxes a side at the row level
    long long rows, Kp;
    const float *u, *dout, *M, *Lf, *dM, *dL;
};

__device__ float feat_value(const GatherP &p, const NetK &k, int f, long long r)
{
    const long long nn = (long long)p.n * p.n;
    const int b = (int)(r / nn), box = (int)(r % nn), bx = box % p.n, by = box / p.n;
    const long long base = (long long)b * k.nbox;
    switch (p.fam) {
    case FAM_W:
        if (p.side == 0) {
            bool ok;
            const long long cell = cell_of(k, bx, by, f, &ok);
            return ok ? p.u[(long long)b * k.N + cell] : 0.f;
        }
        return p.dM[(base + k.lev[k.L] + box) * FN_NR + f];
    case FAM_V:
        if (p.side == 0) return p.Lf[(base + k.lev[k.L] + box) * FN_NR + f];
        {
            bool ok;
            const long long cell = cell_of(k, bx, by, f, &ok);
            return ok ? p.dout[(long long)b * k.N + cell] : 0.f;
        }
    case FAM_M2L:
        if (p.side == 0) {
            const int slot = f / FN_NR, j = f % FN_NR;
            const int ox = slot % 7 - 3, oy = slot / 7 - 3;
            if (!in_list(ox, oy, bx, by)) return 0.f;
            const int sx = bx - ox, sy = by - oy;
            if (sx < 0 || sy < 0 || sx >= p.n || sy >= p.n) return 0.f;
            return p.M[(base + k.lev[p.l] + (long long)sy * p.n + sx) * FN_NR + j];
        }
        return p.dL[(base + k.lev[p.l] + box) * FN_NR + f];
    case FAM_M2M:
        if (p.side == 0) {
            const int c = f / FN_NR, j = f % FN_NR;
            const int cx = 2 * bx + (c & 1), cy = 2 * by + (c >> 1);
            return p.M[(base + k.lev[p.l + 1] + (long long)cy * 2 * p.n + cx) * FN_NR + j];
        }
        return p.dM[(base + k.lev[p.l] + box) * FN_NR + f];
    default:  // FAM_L2L
        if (p.side == 0) return p.Lf[(base + k.lev[p.l] + box) * FN_NR + f];
        {
            const int c = f / FN_NR, kk = f % FN_NR;
            const int cx = 2 * bx + (c & 1), cy = 2 * by + (c >> 1);
            return p.dL[(base + k.lev[p.l + 1] + (long long)cy * 2 * p.n + cx) * FN_NR + kk];
        }
    }
}

// K-major operand [feat][3 Kp]: side 0 [hi | lo | hi], side 1 [hi | hi | lo];
// rows r >= rows (padding to Kp) are zero
__global__ void k_t_gather(GatherP p, NetK k, bf16 *__restrict__ out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)p.nfeat * p.Kp) return;
    const int f = (int)(i / p.Kp);
    const long long r = i % p.Kp;
    const float v = r < p.rows ? feat_value(p, k, f, r) : 0.f;
    const bf16 hi = __float2bfloat16_rn(v);
    const bf16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
    bf16 *row = out + (long long)f * 3 * p.Kp;
    row[r] = hi;
    row[p.Kp + r] = p.side == 0 ? lo : hi;
    row[2 * p.Kp + r] = p.side == 0 ? hi : lo;
}

// add the block-diagonal entries of C into the gradient vector
__global__ void k_t_scatter(const float *__restrict__ C, int fam, int d, int nb_, float *__restrict__ g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    switch (fam) {
    case FAM_W:
        if (i < FN_C * FN_NR) g[fn_off_W() + i] += C[i];  // C[c][k]
        return;
    case FAM_V:
        if (i < FN_NR * FN_C) g[fn_off_V() + i] += C[i];  // C[k][c]
        return;
    default: {
        // entry e of nb_ operators of OSZ each
        if (i >= nb_ * FN_OSZ) return;
        const int op = i / FN_OSZ, e = i % FN_OSZ;
        int j, kk;
        if (e < FN_NE * FN_NE) {
            j = e / FN_NE;
            kk = e % FN_NE;
        } else {
            j = FN_NE + (e - FN_NE * FN_NE) / FN_NO;
            kk = FN_NE + (e - FN_NE * FN_NE) % FN_NO;
        }
        float v;
        long long dst;
        if (fam == FAM_M2L) {
            v = C[(long long)(op * FN_NR + j) * FN_NR + kk];
            dst = fn_off_M2L(d) + (long long)op * FN_OSZ + e;
        } else if (fam == FAM_M2M) {
            v = C[(long long)(op * FN_NR + j) * FN_NR + kk];
            dst = fn_off_M2M(d) + (long long)op * FN_OSZ + e;
        } else {
            v = C[(long long)j * (4 * FN_NR) + op * FN_NR + kk];
            dst = fn_off_L2L(d) + (long long)op * FN_OSZ + e;
        }
        g[dst] += v;
    }
    }
}

// Adam with a per-weight step scale: a weight moves by lr * sc_i per unit of
// normalised gradient, so tables whose entries span many orders of magnitude
// take relative steps
__global__ void k_t_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                         float *__restrict__ v, const float *__restrict__ sc, long long n, float lr, float b1,
                         float b2, float eps, float c1, float c2)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * sc[i] * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_t_fill(float *__restrict__ a, long long n, float v)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

NetK netk(const mms_farnet *n, int nbatch)
{
    NetK k;
    k.X = n->X;
    k.Y = n->Y;
    k.L = n->L;
    k.nb = n->nb;
    k.batch = nbatch;
    k.N = n->N;
    k.nbox = n->nbox;
    for (int i = 0; i < FN_DEPTHS + 3; i++) k.lev[i] = n->lev_off[i];
    return k;
}

constexpr int TB = 256;
inline unsigned nblk(long long n) { return (unsigned)((n + TB - 1) / TB); }

int forward(mms_farnet *n, const float *u, int nbatch)
{
    const NetK k = netk(n, nbatch);
    cudaStream_t st = 0;
    const long long nl = (long long)n->nb * n->nb;
    k_t_p2m<<<nblk(nbatch * nl * FN_NR), TB, 0, st>>>(u, n->w, n->M, k);
    for (int l = n->L - 1; l >= 2; l--)
        k_t_m2m<<<nblk((long long)nbatch * (1LL << (2 * l)) * FN_NR), TB, 0, st>>>(n->w, n->M, k, l);
    for (int l = 2; l <= n->L; l++)
        k_t_local<<<nblk((long long)nbatch * (1LL << (2 * l)) * FN_NR), TB, 0, st>>>(n->w, n->M, n->Lf, k, l);
    k_t_l2p<<<nblk(nbatch * n->N), TB, 0, st>>>(n->w, n->Lf, n->out, k);
    MMS_CUDA_TRY(cudaGetLastError());
    return MMS_OK;
}

int gemm_family(mms_farnet *n, const NetK &k, GatherP p, int fa, int fb, int d)
{
    p.Kp = (p.rows + 7) / 8 * 8;
    GatherP pa = p, pb = p;
    pa.side = 0;
    pa.nfeat = fa;
    pb.side = 1;
    pb.nfeat = fb;
    if ((size_t)fa * 3 * p.Kp > n->a_elems || (size_t)fb * 3 * p.Kp > n->b_elems || (size_t)fa * fb > n->c_elems) {
        mms_set_error("farnet: gradient operand buffers too small");
        return MMS_ERR_ARG;
    }
    k_t_gather<<<nblk((long long)fa * p.Kp), TB>>>(pa, k, n->A);
    k_t_gather<<<nblk((long long)fb * p.Kp), TB>>>(pb, k, n->B);
    MMS_CUDA_TRY(cudaGetLastError());
    const int K3 = (int)(3 * p.Kp), bn = fb <= 64 ? 64 : 128;
    int splits = 1, kchunk = K3;
    MMS_TRY(umma_gemm_bf16_splitk_plan(fa, fb, K3, bn, &splits, &kchunk));
    if ((size_t)splits * fa * fb > n->p_elems) {
        mms_set_error("farnet: split-K partial buffer too small");
        return MMS_ERR_ARG;
    }
    MMS_TRY(umma_gemm_bf16_splitk(n->A, K3, n->B, K3, n->Cm, n->Cp, fa, fb, K3, bn, splits, kchunk, 0));
    const int ops = p.fam == FAM_M2L ? 49 : 4;
    const int cnt = (p.fam == FAM_W || p.fam == FAM_V) ? FN_C * FN_NR : ops * FN_OSZ;
    k_t_scatter<<<nblk(cnt), TB>>>(n->Cm, p.fam, d, ops, n->g);
    MMS_CUDA_TRY(cudaGetLastError());
    return MMS_OK;
}

// loss (host value) and the gradient into n->g
int gradient(mms_farnet *n, const float *u, const float *far, const float *nrm2, int nbatch, double *loss)
{
    MMS_TRY(forward(n, u, nbatch));
    const NetK k = netk(n, nbatch);
    MMS_CUDA_TRY(cudaMemsetAsync(n->lsum, 0, (size_t)nbatch * sizeof(double), 0));
    k_t_loss<<<dim3(nblk(n->N), nbatch), TB>>>(n->out, far, nrm2, n->dout, n->lsum, k, nbatch);
    const long long nl = (long long)n->nb * n->nb;
    k_t_l2p_adj<<<nblk(nbatch * nl * FN_NR), TB>>>(n->w, n->dout, n->dL, k);
    for (int l = n->L; l >= 3; l--)
        k_t_l2l_adj<<<nblk((long long)nbatch * (1LL << (2 * (l - 1))) * FN_NR), TB>>>(n->w, n->dL, k, l);
    for (int l = 2; l <= n->L; l++)
        k_t_dm<<<nblk((long long)nbatch * (1LL << (2 * l)) * FN_NR), TB>>>(n->w, n->dL, n->dM, k, l);
    MMS_CUDA_TRY(cudaGetLastError());
    MMS_CUDA_TRY(cudaMemsetAsync(n->g, 0, (size_t)fn_num_params() * sizeof(float), 0));
    GatherP p{};
    p.u = u;
    p.dout = n->dout;
    p.M = n->M;
    p.Lf = n->Lf;
    p.dM = n->dM;
    p.dL = n->dL;
    // encoder and decoder (leaf level)
    p.n = n->nb;
    p.l = n->L;
    p.rows = (long long)nbatch * nl;
    p.fam = FAM_W;
    MMS_TRY(gemm_family(n, k, p, FN_C, FN_NR, 0));
    p.fam = FAM_V;
    MMS_TRY(gemm_family(n, k, p, FN_NR, FN_C, 0));
    for (int l = 2; l <= n->L; l++) {
        p.l = l;
        p.n = 1 << l;
        p.rows = (long long)nbatch * p.n * p.n;
        p.fam = FAM_M2L;
        MMS_TRY(gemm_family(n, k, p, 49 * FN_NR, FN_NR, n->L - l));
        if (l < n->L) {
            p.fam = FAM_M2M;
            MMS_TRY(gemm_family(n, k, p, 4 * FN_NR, FN_NR, n->L - l));
            p.fam = FAM_L2L;
            MMS_TRY(gemm_family(n, k, p, FN_NR, 4 * FN_NR, n->L - l));
        }
    }
    std::vector<double> ls(nbatch), nh(nbatch);
    std::vector<float> nf(nbatch);
    MMS_CUDA_TRY(cudaMemcpy(ls.data(), n->lsum, (size_t)nbatch * sizeof(double), cudaMemcpyDeviceToHost));
    MMS_CUDA_TRY(cudaMemcpy(nf.data(), nrm2, (size_t)nbatch * sizeof(float), cudaMemcpyDeviceToHost));
    MMS_TRY(umma_check_error());
    double L = 0;
    for (int b = 0; b < nbatch; b++) L += ls[b] / nf[b];
    if (loss) *loss = L / nbatch;
    return MMS_OK;
}

int check_batch(const mms_farnet *n, int nbatch)
{
    if (!n || nbatch < 1 || nbatch > n->batch) {
        mms_set_error("farnet: bad network or batch size %d", nbatch);
        return MMS_ERR_ARG;
    }
    return MMS_OK;
}

}  // namespace

extern "C" {

long long mms_farnet_num_params(void) { return fn_num_params(); }

long long mms_surrogate_num_params(int width)
{
    if (width == FnTrain::NR) return FnTrain::num_params();
    if (width == FnWide::NR) return FnWide::num_params();
    return 0;
}

int mms_farnet_create(int xdim, int ydim, int batch, mms_farnet **out)
{
    if (!out || xdim < 1 || ydim < 1 || batch < 1) {
        mms_set_error("mms_farnet_create: bad argument");
        return MMS_ERR_ARG;
    }
    *out = nullptr;
    const int nleaf = std::max(1, (std::max(xdim, ydim) + FN_S - 1) / FN_S);
    int L = 0;
    while ((1 << L) < nleaf) L++;
    if (L < 2 || L > FN_DEPTHS + 1) {
        mms_set_error("mms_farnet_create: a %d x %d grid has %d quadtree levels; the network needs 2..%d", xdim, ydim,
                      L, FN_DEPTHS + 1);
        return MMS_ERR_ARG;
    }
    mms_farnet *n = new mms_farnet();
    n->X = xdim;
    n->Y = ydim;
    n->L = L;
    n->nb = 1 << L;
    n->batch = batch;
    n->N = (long long)FN_Z * xdim * ydim;
    long long tot = 0;
    for (int l = 2; l <= L; l++) {
        n->lev_off[l] = tot;
        tot += 1LL << (2 * l);
    }
    n->lev_off[L + 1] = tot;
    n->nbox = tot;
    const long long P = fn_num_params();
    const size_t act = (size_t)batch * tot * FN_NR;
    const long long rows_max = (long long)batch * n->nb * n->nb;
    const long long Kp = (rows_max + 7) / 8 * 8;
    n->a_elems = (size_t)(49 * FN_NR * 3 * Kp);  // A: up to max(49 NR, C) features
    n->b_elems = (size_t)(4 * FN_NR * 3 * Kp);
    n->c_elems = (size_t)49 * FN_NR * FN_NR + (size_t)FN_C * FN_NR;
    n->p_elems = n->c_elems * 148;  // up to one split per SM
    struct {
        void **p;
        size_t bytes;
    } a[] = {{(void **)&n->w, P * sizeof(float)},
             {(void **)&n->sc, P * sizeof(float)},
             {(void **)&n->g, P * sizeof(float)},
             {(void **)&n->m, P * sizeof(float)},
             {(void **)&n->v, P * sizeof(float)},
             {(void **)&n->M, act * sizeof(float)},
             {(void **)&n->Lf, act * sizeof(float)},
             {(void **)&n->dM, act * sizeof(float)},
             {(void **)&n->dL, act * sizeof(float)},
             {(void **)&n->out, (size_t)batch * n->N * sizeof(float)},
             {(void **)&n->dout, (size_t)batch * n->N * sizeof(float)},
             {(void **)&n->lsum, (size_t)batch * sizeof(double)},
             {(void **)&n->A, n->a_elems * sizeof(bf16)},
             {(void **)&n->B, std::max(n->b_elems, (size_t)(FN_C * 3 * Kp)) * sizeof(bf16)},
             {(void **)&n->Cm, n->c_elems * sizeof(float)},
             {(void **)&n->Cp, n->c_elems * 148 * sizeof(float)},
             {(void **)&n->lev_dev, (FN_DEPTHS + 3) * sizeof(long long)}};
    n->b_elems = std::max(n->b_elems, (size_t)(FN_C * 3 * Kp));  // B: up to max(4 NR, C) features
    for (auto &e : a) {
        if (cudaMalloc(e.p, e.bytes) != cudaSuccess) {
            mms_farnet_destroy(n);
            mms_set_error("mms_farnet_create: device allocation of %zu bytes failed", e.bytes);
            return MMS_ERR_NOMEM;
        }
        n->bytes += e.bytes;
    }
    cudaMemset(n->w, 0, P * sizeof(float));
    k_t_fill<<<nblk(P), TB>>>(n->sc, P, 1.f);
    cudaMemset(n->m, 0, P * sizeof(float));
    cudaMemset(n->v, 0, P * sizeof(float));
    if (cudaMemcpy(n->lev_dev, n->lev_off, sizeof(n->lev_off), cudaMemcpyHostToDevice) != cudaSuccess) {
        mms_farnet_destroy(n);
        mms_set_error("mms_farnet_create: copy failed");
        return MMS_ERR_CUDA;
    }
    *out = n;
    return MMS_OK;
}

void mms_farnet_destroy(mms_farnet *n)
{
    if (!n) return;
    cudaDeviceSynchronize();
    void *b[] = {n->w, n->sc, n->g, n->m, n->v, n->M, n->Lf, n->dM, n->dL, n->out, n->dout, n->lsum, n->A, n->B, n->Cm, n->Cp,
                 n->lev_dev};
    for (void *p : b)
        if (p) cudaFree(p);
    delete n;
}

int mms_farnet_set_weights(mms_farnet *n, const float *w, long long count)
{
    if (!n || !w || count != fn_num_params()) {
        mms_set_error("mms_farnet_set_weights: need %lld weights", fn_num_params());
        return MMS_ERR_ARG;
    }
    MMS_CUDA_TRY(cudaMemcpy(n->w, w, count * sizeof(float), cudaMemcpyHostToDevice));
    MMS_CUDA_TRY(cudaMemset(n->m, 0, count * sizeof(float)));
    MMS_CUDA_TRY(cudaMemset(n->v, 0, count * sizeof(float)));
    n->step = 0;
    return MMS_OK;
}

int mms_farnet_set_step_scale(mms_farnet *n, const float *scale, long long count)
{
    if (!n || !scale || count != fn_num_params()) {
        mms_set_error("mms_farnet_set_step_scale: need %lld scales", fn_num_params());
        return MMS_ERR_ARG;
    }
    MMS_CUDA_TRY(cudaMemcpy(n->sc, scale, count * sizeof(float), cudaMemcpyHostToDevice));
    return MMS_OK;
}

int mms_farnet_get_weights(mms_farnet *n, float *w, long long count)
{
    if (!n || !w || count != fn_num_params()) {
        mms_set_error("mms_farnet_get_weights: need %lld weights", fn_num_params());
        return MMS_ERR_ARG;
    }
    MMS_CUDA_TRY(cudaMemcpy(w, n->w, count * sizeof(float), cudaMemcpyDeviceToHost));
    return MMS_OK;
}

int mms_farnet_forward_dev(mms_farnet *n, const float *u, float *out, int nbatch)
{
    MMS_TRY(check_batch(n, nbatch));
    if (!u || !out) {
        mms_set_error("mms_farnet_forward_dev: NULL argument");
        return MMS_ERR_ARG;
    }
    MMS_TRY(forward(n, u, nbatch));
    MMS_CUDA_TRY(cudaMemcpyAsync(out, n->out, (size_t)nbatch * n->N * sizeof(float), cudaMemcpyDeviceToDevice, 0));
    MMS_CUDA_TRY(cudaStreamSynchronize(0));
    return MMS_OK;
}

int mms_farnet_gradient(mms_farnet *n, const float *u, const float *far, const float *nrm2, int nbatch, float *grad,
                        double *loss)
{
    MMS_TRY(check_batch(n, nbatch));
    if (!u || !far || !nrm2) {
        mms_set_error("mms_farnet_gradient: NULL argument");
        return MMS_ERR_ARG;
    }
    MMS_TRY(gradient(n, u, far, nrm2, nbatch, loss));
    if (grad) MMS_CUDA_TRY(cudaMemcpy(grad, n->g, fn_num_params() * sizeof(float), cudaMemcpyDeviceToHost));
    return MMS_OK;
}

int mms_farnet_train_step(mms_farnet *n, const float *u, const float *far, const float *nrm2, int nbatch, float lr,
                          float beta1, float beta2, float eps, double *loss)
{
    MMS_TRY(check_batch(n, nbatch));
    if (!u || !far || !nrm2 || !(lr >= 0)) {
        mms_set_error("mms_farnet_train_step: bad argument");
        return MMS_ERR_ARG;
    }
    MMS_TRY(gradient(n, u, far, nrm2, nbatch, loss));
    n->step++;
    const float c1 = 1.f - powf(beta1, (float)n->step), c2 = 1.f - powf(beta2, (float)n->step);
    const long long P = fn_num_params();
    k_t_adam<<<nblk(P), TB>>>(n->w, n->g, n->m, n->v, n->sc, P, lr, beta1, beta2, eps, c1, c2);
    MMS_CUDA_TRY(cudaGetLastError());
    return MMS_OK;
}

long long mms_farnet_device_bytes(const mms_farnet *n) { return n ? (long long)n->bytes : 0; }

}  // extern "C"
