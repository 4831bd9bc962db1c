// Surrogate far field: a 3-D convolutional neural operator that maps the cell
// charge density to the far-field part of the demag potential, the part the
// FMM's M2M / M2L / L2L passes produce.  The exact near field (P2P over the
// 3 x 3 leaf neighbourhood, all layers) is not learned; it is added in the
// last layer's epilogue.
//
// Grid.  The cell grid is cut into 4 x 4 in-plane patches, one per FMM leaf
// box and layer: level 0 of the network is the (Z, ceil(Y/4), ceil(X/4)) patch
// grid with the 16 charges of a patch as its 16 input channels and the 16 far-
// field potentials as its 16 output channels.  Levels 1..3 halve the in-plane
// extent; z keeps its Z layers at every level, so every convolution is 3-D.
//
// Network (U-Net, 4 levels, 32 channels, 232,448 weights, no biases, no
// activations: the map rho -> phi_far is linear, and a linear network keeps
// phi(-rho) = -phi(rho) and the error independent of the charge's amplitude):
//   a0 = conv3(x)                                  level 0, 16 -> 32
//   a_l = conv3(down(a_{l-1}))                     l = 1..3
//   b3 = conv3(a3)
//   c_l = conv3(up(c_{l+1}) + a_l)                 l = 2..0 (c_3 = b3)
//   y = point(c0)                                  32 -> 16
// conv3: 3x3x3, stride 1, zero padding; down: 1x2x2 stride 2; up: its
// transpose (each fine cell takes its parent through the weight of its
// position in the parent); point: 1x1x1.
//
// Arithmetic.  Weights are BF16 (FP32 master copy for the optimiser);
// activations are carried as BF16 hi/lo pairs (hi = bf16(v), lo = bf16(v -
// hi)), so a GEMM over K' = [hi | lo] against [W | W] multiplies FP32-accurate
// activations by the BF16 weights with FP32 accumulation on the tensor cores.
//
// Kernels.  Every layer is one implicit-GEMM launch (k_conv): tcgen05.mma with
// the accumulator in tensor memory, A gathered per 16-byte chunk straight from
// the activation rows of the layer's input (the tap pattern decides the source
// row), 4-stage cp.async pipeline, bounded mbarrier waits.  Training adds the
// adjoint convolutions (same kernel, adjoint weights), the weight gradients
// (a transposed im2col + split-K tcgen05 GEMM, hi/lo products), a per-sample
// relative-L2 loss and Adam.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include <cuda_bf16.h>

#include "mms_internal.cuh"
#include "umma.cuh"

using bf16 = __nv_bfloat16;

namespace {

enum Pattern { PAT_CONV3 = 0, PAT_DOWN = 1, PAT_UP = 2, PAT_POINT = 3 };
enum Epilogue { EP_SPLIT = 0, EP_F32 = 1, EP_PHI = 2 };

constexpr int PATCH = 4;
constexpr int CH = 32;
constexpr int LEVELS = 4;
constexpr int CIN0 = PATCH * PATCH;
constexpr int CBN = 32;  // output channels per tile (N of the MMA)
// pipeline stages of k_conv: 4 for training (2 CTAs per SM over many tiles),
// 8 for the solver's batch-1 inference (few tiles: depth hides the latency)
constexpr int conv_smem(int stages) { return stages * (umma::BM * 128) + stages * (CBN * 128) + 1024 + 128; }

struct Layer {
    int pat, cin, cout, in, out, skip, taps;
    long long w_off, wf_off, wb_off;
};

void build_arch(std::vector<Layer> &L, std::vector<int> &lev, std::vector<int> &ch, long long &nparam,
                long long &nwf, long long &nwb)
{
    L.clear();
    lev.clear();
    ch.clear();
    nparam = nwf = nwb = 0;
    auto node = [&](int l, int c) {
        lev.push_back(l);
        ch.push_back(c);
        return (int)lev.size() - 1;
    };
    auto add = [&](int pat, int in, int out, int skip) {
        Layer y;
        y.pat = pat;
        y.cin = ch[in];
        y.cout = ch[out];
        y.in = in;
        y.out = out;
        y.skip = skip;
        y.taps = pat == PAT_CONV3 ? 27 : (pat == PAT_POINT ? 1 : 4);
        y.w_off = nparam;
        y.wf_off = nwf;
        y.wb_off = nwb;
        const long long n = (long long)y.cout * y.taps * y.cin;
        nparam += n;
        nwf += 2 * n;
        nwb += 2 * n;
        L.push_back(y);
    };
    const int x = node(0, CIN0);
    int a[LEVELS];
    a[0] = node(0, CH);
    add(PAT_CONV3, x, a[0], -1);
    for (int l = 1; l < LEVELS; l++) {
        const int d = node(l, CH);
        add(PAT_DOWN, a[l - 1], d, -1);
        a[l] = node(l, CH);
        add(PAT_CONV3, d, a[l], -1);
    }
    int cur = node(LEVELS - 1, CH);
    add(PAT_CONV3, a[LEVELS - 1], cur, -1);
    for (int l = LEVELS - 2; l >= 0; l--) {
        const int u = node(l, CH);
        add(PAT_UP, cur, u, a[l]);
        const int c = node(l, CH);
        add(PAT_CONV3, u, c, -1);
        cur = c;
    }
    const int y = node(0, CIN0);
    add(PAT_POINT, cur, y, -1);
}

// ---------------------------------------------------------------------------
// implicit-GEMM convolution on tcgen05

struct ConvP {
    const bf16 *ahi, *alo;  // input activations [rows][cin]
    int cin_log2, T, pat;
    int Z, Hin, Win, Hout, Wout;
    int P;                  // output rows
    const bf16 *w;          // [N][ldw], ldw = 2 T cin: [W | W] for the hi and lo halves
    int K, N, ldw;          // K = ldw (hi and lo) or T cin (hi only)
    int ep;
    const bf16 *shi, *slo;  // EP_SPLIT: skip tensor added before the split (may be NULL)
    bf16 *ohi, *olo;        // EP_SPLIT outputs [P][N]
    float *o32;             // EP_F32 output [P][N]
    int beta;               // EP_F32: accumulate
    float *phi;             // EP_PHI: cell potential [Z][Y][X] per sample
    const float *near;      // EP_PHI: near field added (may be NULL)
    float scale;            // EP_PHI: output scale
    int X, Y;               // EP_PHI: cell grid
    int *err;
};

__device__ __forceinline__ bool tap_src(const ConvP &p, int tap, int bz, int z, int y, int x, long long &row)
{
    switch (p.pat) {
    case PAT_CONV3: {
        const int zz = z + tap / 9 - 1, yy = y + (tap / 3) % 3 - 1, xx = x + tap % 3 - 1;
        if (zz < 0 || zz >= p.Z || yy < 0 || yy >= p.Hin || xx < 0 || xx >= p.Win) return false;
        row = ((long long)(bz - z + zz) * p.Hin + yy) * p.Win + xx;
        return true;
    }
    case PAT_DOWN: {
        const int yy = 2 * y + (tap >> 1), xx = 2 * x + (tap & 1);
        if (yy >= p.Hin || xx >= p.Win) return false;
        row = ((long long)bz * p.Hin + yy) * p.Win + xx;
        return true;
    }
    case PAT_UP:
        if (tap != (((y & 1) << 1) | (x & 1))) return false;
        row = ((long long)bz * p.Hin + (y >> 1)) * p.Win + (x >> 1);
        return true;
    default:
        row = ((long long)bz * p.Hout + y) * p.Wout + x;
        return true;
    }
}

template <int CS>
__global__ void __launch_bounds__(128) k_conv(ConvP p)
{
    extern __shared__ uint8_t smraw[];
    uint8_t *sm = (uint8_t *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    uint8_t *sa = sm;
    uint8_t *sb = sm + CS * (umma::BM * 128);
    uint64_t *done = (uint64_t *)(sb + CS * (CBN * 128));
    uint32_t *tslot = (uint32_t *)(done + CS);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * umma::BM;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         umma::smem_u32(tslot)),
                     "r"(CBN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < CS; i++) umma::mbar_init(&done[i]);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tslot;

    // this thread's 8 rows (chunk column c is fixed): decode the output position once
    const int c = tid & 7;
    int rz[8], ry[8], rx[8], rbz[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int r = (tid >> 3) + 16 * j;
        const int pr = min(m0 + r, p.P - 1);
        rx[j] = pr % p.Wout;
        const int q = pr / p.Wout;
        ry[j] = q % p.Hout;
        rbz[j] = q / p.Hout;
        rz[j] = rbz[j] % p.Z;
    }
    const int TC = p.T << p.cin_log2;
    const int nk = (p.K + umma::BK - 1) / umma::BK;

    auto load = [&](int st, int kt) {
        const int k = kt * umma::BK + c * 8;
        const bool kval = k < p.K;
        int half = 0, tap = 0, ci = 0;
        if (kval) {
            half = k >= TC;
            const int kk = k - half * TC;
            tap = kk >> p.cin_log2;
            ci = kk & ((1 << p.cin_log2) - 1);
        }
        const bf16 *src = half ? p.alo : p.ahi;
        const uint32_t sa_st = umma::smem_u32(sa + st * (umma::BM * 128));
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int r = (tid >> 3) + 16 * j;
            long long row = 0;
            bool ok = kval && m0 + r < p.P;
            if (ok) ok = tap_src(p, tap, rbz[j], rz[j], ry[j], rx[j], row);
            umma::cp_async16(sa_st + umma::sw128_off(r, c),
                             ok ? (const void *)(src + (row << p.cin_log2) + ci) : (const void *)p.ahi, ok);
        }
        const uint32_t sb_st = umma::smem_u32(sb + st * (CBN * 128));
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int i = tid + 128 * q;
            const int r = i >> 3, cc = i & 7;
            const int gk = kt * umma::BK + cc * 8;
            const bool ok = r < p.N && gk < p.K;
            umma::cp_async16(sb_st + umma::sw128_off(r, cc),
                             ok ? (const void *)(p.w + (long long)r * p.ldw + gk) : (const void *)p.w, ok);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    const uint32_t idesc = umma::idesc_bf16(CBN);
    bool ok = true;
    int issued = 0;
    for (; issued < CS - 1 && issued < nk; issued++) load(issued % CS, issued);
    for (int kt = 0; kt < nk && ok; kt++) {
        const int st = kt % CS;
        const int pending = issued - kt - 1;  // groups allowed to stay in flight
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
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t a0 = umma::smem_u32(sa + st * (umma::BM * 128));
            const uint32_t b0 = umma::smem_u32(sb + st * (CBN * 128));
#pragma unroll
            for (int kk = 0; kk < umma::BK / 16; kk++)
                umma::mma_bf16(tmem, umma::desc_sw128(a0 + kk * 32), umma::desc_sw128(b0 + kk * 32), idesc,
                               (kt > 0 || kk > 0) ? 1u : 0u);
            umma::mma_commit(&done[st]);
        }
        __syncwarp();
        if (issued < nk) {
            // the stage being refilled was read by tile kt-1: wait for its MMAs
            if (kt >= 1) ok = umma::mbar_wait(&done[(kt - 1) % CS], (uint32_t)(((kt - 1) / CS) & 1));
            if (ok) {
                load(issued % CS, issued);
                issued++;
            }
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    if (ok && nk > 0) ok = umma::mbar_wait(&done[(nk - 1) % CS], (uint32_t)(((nk - 1) / CS) & 1));
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (!ok) {
        if (lane == 0) atomicExch(p.err, 1);
    } else {
        float v[CBN];
        umma::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16), v);
        umma::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + 16u, v + 16);
        const int row = m0 + warp * 32 + lane;
        if (row < p.P) {
            if (p.ep == EP_SPLIT) {
                // N == 32: 4 x 16-byte chunks per output row
#pragma unroll
                for (int q = 0; q < CBN / 8; q++) {
                    float u[8];
#pragma unroll
                    for (int i = 0; i < 8; i++) u[i] = v[8 * q + i];
                    if (p.shi) {
                        const uint4 h4 = *(const uint4 *)(p.shi + (long long)row * CBN + 8 * q);
                        const uint4 l4 = *(const uint4 *)(p.slo + (long long)row * CBN + 8 * q);
                        const bf16 *h = (const bf16 *)&h4, *l = (const bf16 *)&l4;
#pragma unroll
                        for (int i = 0; i < 8; i++) u[i] += __bfloat162float(h[i]) + __bfloat162float(l[i]);
                    }
                    uint4 ho, lo;
                    bf16 *hb = (bf16 *)&ho, *lb = (bf16 *)&lo;
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        hb[i] = __float2bfloat16_rn(u[i]);
                        lb[i] = __float2bfloat16_rn(u[i] - __bfloat162float(hb[i]));
                    }
                    *(uint4 *)(p.ohi + (long long)row * CBN + 8 * q) = ho;
                    *(uint4 *)(p.olo + (long long)row * CBN + 8 * q) = lo;
                }
            } else if (p.ep == EP_F32) {
                float *o = p.o32 + (long long)row * p.N;
                for (int n = 0; n < p.N; n++) o[n] = p.beta ? o[n] + v[n] : v[n];
            } else {
                const int x = row % p.Wout, q = row / p.Wout, y = q % p.Hout, bz = q / p.Hout;
#pragma unroll
                for (int n = 0; n < CIN0; n++) {
                    const int cy = y * PATCH + (n >> 2), cx = x * PATCH + (n & 3);
                    if (cy < p.Y && cx < p.X) {
                        const long long idx = ((long long)bz * p.Y + cy) * p.X + cx;
                        p.phi[idx] = (p.near ? p.near[idx] : 0.f) + v[n] * p.scale;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(CBN) : "memory");
}

// ---------------------------------------------------------------------------
// layout kernels

// cells [B][Z][Y][X] * scale -> patch rows [B Z H W][16] as hi/lo BF16
__global__ void k_patchify(const float *__restrict__ u, float scale, int X, int Y, int H, int W, long long P,
                           bf16 *__restrict__ hi, bf16 *__restrict__ lo)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P * CIN0) return;
    const long long p = i >> 4;
    const int n = (int)(i & 15);
    const int x = (int)(p % W);
    const long long q = p / W;
    const int y = (int)(q % H);
    const long long bz = q / H;
    const int cy = y * PATCH + (n >> 2), cx = x * PATCH + (n & 3);
    const float v = (cy < Y && cx < X) ? u[(bz * Y + cy) * X + cx] * scale : 0.f;
    const bf16 h = __float2bfloat16_rn(v);
    hi[i] = h;
    lo[i] = __float2bfloat16_rn(v - __bfloat162float(h));
}

__global__ void k_patchify_f32(const float *__restrict__ u, float scale, int X, int Y, int H, int W, long long P,
                               float *__restrict__ out)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P * CIN0) return;
    const long long p = i >> 4;
    const int n = (int)(i & 15);
    const int x = (int)(p % W);
    const long long q = p / W;
    const int y = (int)(q % H);
    const long long bz = q / H;
    const int cy = y * PATCH + (n >> 2), cx = x * PATCH + (n & 3);
    out[i] = (cy < Y && cx < X) ? u[(bz * Y + cy) * X + cx] * scale : 0.f;
}

// patch rows [P][16] -> cells, for reading the network's output
__global__ void k_unpatchify(const float *__restrict__ y32, int X, int Y, int H, int W, long long P,
                             float *__restrict__ out)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= P * CIN0) return;
    const long long p = i >> 4;
    const int n = (int)(i & 15);
    const int x = (int)(p % W);
    const long long q = p / W;
    const int y = (int)(q % H);
    const long long bz = q / H;
    const int cy = y * PATCH + (n >> 2), cx = x * PATCH + (n & 3);
    if (cy < Y && cx < X) out[(bz * Y + cy) * X + cx] = y32[i];
}

// per-sample sums of |tgt|^2 and |pred - tgt|^2 (double, atomics)
__global__ void k_loss_sums(const float *__restrict__ pred, const float *__restrict__ tgt, long long per,
                            double *__restrict__ sums)
{
    const int b = blockIdx.y;
    const float *pp = pred + b * per, *tt = tgt + b * per;
    double t2 = 0, e2 = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < per; i += (long long)gridDim.x * blockDim.x) {
        const double t = tt[i], e = (double)pp[i] - t;
        t2 += t * t;
        e2 += e * e;
    }
    for (int o = 16; o > 0; o >>= 1) {
        t2 += __shfl_xor_sync(0xffffffffu, t2, o);
        e2 += __shfl_xor_sync(0xffffffffu, e2, o);
    }
    __shared__ double s[2][8];
    if ((threadIdx.x & 31) == 0) {
        s[0][threadIdx.x >> 5] = t2;
        s[1][threadIdx.x >> 5] = e2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, c = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            a += s[0][w];
            c += s[1][w];
        }
        atomicAdd(&sums[2 * b], a);
        atomicAdd(&sums[2 * b + 1], c);
    }
}

// d loss / d pred for loss = mean_b |pred_b - tgt_b|^2 / |tgt_b|^2
__global__ void k_loss_grad(const float *__restrict__ pred, const float *__restrict__ tgt, long long per, int nb,
                            const double *__restrict__ sums, float *__restrict__ d)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= per * nb) return;
    const int b = (int)(i / per);
    const double t2 = sums[2 * b] > 0 ? sums[2 * b] : 1.0;
    d[i] = (float)(2.0 * ((double)pred[i] - (double)tgt[i]) / (nb * t2));
}

// FP32 [P][C] -> hi/lo BF16 [P][C] and transposed hi/lo [C][Ppad] (zero for P <= p < Ppad)
__global__ void k_split_t(const float *__restrict__ d, long long P, int C, long long Ppad, bf16 *__restrict__ hi,
                          bf16 *__restrict__ lo, bf16 *__restrict__ hT, bf16 *__restrict__ lT)
{
    __shared__ float t[64][33];
    const long long p0 = blockIdx.x * 64LL;
    for (int i = threadIdx.x; i < 64 * C; i += blockDim.x) {
        const int r = i / C, c = i % C;
        const long long p = p0 + r;
        float v = 0.f;
        if (p < P) {
            v = d[p * C + c];
            const bf16 h = __float2bfloat16_rn(v);
            hi[p * C + c] = h;
            lo[p * C + c] = __float2bfloat16_rn(v - __bfloat162float(h));
        }
        t[r][c] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 64 * C; i += blockDim.x) {
        const int c = i / 64, r = i % 64;
        const long long p = p0 + r;
        if (p < Ppad) {
            const float v = t[r][c];
            const bf16 h = __float2bfloat16_rn(v);
            hT[(long long)c * Ppad + p] = h;
            lT[(long long)c * Ppad + p] = __float2bfloat16_rn(v - __bfloat162float(h));
        }
    }
}

// transposed im2col of a layer's input: cT[(tap, ci)][p] for the output rows p
__global__ void k_im2col_t(ConvP p, long long Ppad, bf16 *__restrict__ cThi, bf16 *__restrict__ cTlo)
{
    const long long pr = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int rowk = blockIdx.y;  // tap * cin + ci
    if (pr >= Ppad) return;
    const int cin = 1 << p.cin_log2;
    const int tap = rowk >> p.cin_log2, ci = rowk & (cin - 1);
    bf16 h = __float2bfloat16_rn(0.f), l = h;
    if (pr < p.P) {
        const int x = (int)(pr % p.Wout);
        const long long q = pr / p.Wout;
        const int y = (int)(q % p.Hout);
        const int bz = (int)(q / p.Hout);
        long long row;
        if (tap_src(p, tap, bz, bz % p.Z, y, x, row)) {
            h = p.ahi[(row << p.cin_log2) + ci];
            l = p.alo[(row << p.cin_log2) + ci];
        }
    }
    cThi[(long long)rowk * Ppad + pr] = h;
    cTlo[(long long)rowk * Ppad + pr] = l;
}

// weight gradient partials: part[(prod, split)][m][n] = sum over this split's
// positions of A[m][p] B[n][p]; prod 0: hi.hi, 1: lo.hi, 2: hi.lo
__global__ void __launch_bounds__(128) k_dw(const bf16 *__restrict__ cThi, const bf16 *__restrict__ cTlo,
                                            const bf16 *__restrict__ dThi, const bf16 *__restrict__ dTlo, int M,
                                            int N, long long Ppad, int kchunk, float *__restrict__ part,
                                            int *__restrict__ err)
{
    __shared__ umma::Smem<32> s;
    const int prod = blockIdx.z, split = blockIdx.y;
    const long long k0 = (long long)split * kchunk;
    const long long rem = Ppad - k0;
    const int K = rem <= 0 ? 0 : (rem < kchunk ? (int)rem : kchunk);
    const bf16 *A = (prod == 1 ? cTlo : cThi) + k0;
    const bf16 *B = (prod == 2 ? dTlo : dThi) + k0;
    float *C = part + ((long long)prod * gridDim.y + split) * M * N;
    umma::gemm_tile<32>(A, (int)Ppad, B, (int)Ppad, C, N, M, N, K, blockIdx.x * umma::BM, 0, 0, err, s);
}

// gW[co][tap][ci] = sum over partials of part[.][(tap, ci)][co]
__global__ void k_dw_reduce(const float *__restrict__ part, int nparts, int T, int cin, int cout,
                            float *__restrict__ gW)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int M = T * cin;
    if (i >= M * cout) return;
    const int co = i / M, m = i % M;
    double acc = 0;
    for (int q = 0; q < nparts; q++) acc += part[((long long)q * M + m) * cout + co];
    gW[i] = (float)acc;  // i = co * M + tap * cin + ci
}

__global__ void k_axpy(const float *__restrict__ x, float *__restrict__ y, long long n)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i];
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, long long n, float lr, float b1, float b2, float eps, float bc1,
                       float bc2)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// BF16 operand layouts of one layer from the FP32 master weights W[co][tap][ci]:
//   wf[co][h T cin + tap cin + ci]        forward, h = 0 (hi half), 1 (lo half)
//   wb[ci][h T cout + tap' cout + co]     adjoint, tap' = 26 - tap for conv3
__global__ void k_build_w(const float *__restrict__ w32, int pat, int T, int cin, int cout, bf16 *__restrict__ wf,
                          bf16 *__restrict__ wb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cout * T * cin) return;
    const int ci = i % cin, tap = (i / cin) % T, co = i / (cin * T);
    const bf16 b = __float2bfloat16_rn(w32[i]);
    const long long Kf = 2LL * T * cin, Kb = 2LL * T * cout;
    wf[co * Kf + tap * cin + ci] = b;
    wf[co * Kf + (long long)T * cin + tap * cin + ci] = b;
    const int tb = pat == PAT_CONV3 ? 26 - tap : tap;
    wb[ci * Kb + tb * cout + co] = b;
    wb[ci * Kb + (long long)T * cout + tb * cout + co] = b;
}

__global__ void k_round_bf16(const float *__restrict__ w32, float *__restrict__ out, long long n)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = __bfloat162float(__float2bfloat16_rn(w32[i]));
}

int ilog2(int v)
{
    int l = 0;
    while ((1 << l) < v) l++;
    return l;
}

}  // namespace

// ---------------------------------------------------------------------------
// the network object

struct mms_sno {
    int device = 0;
    int X = 0, Y = 0, Z = 0, B = 0;
    int H[LEVELS] = {}, W[LEVELS] = {};
    std::vector<Layer> L;
    std::vector<int> lev, ch;
    long long nparam = 0, nwf = 0, nwb = 0;
    float *w32 = nullptr;
    bf16 *wf = nullptr, *wb = nullptr;
    std::vector<bf16 *> ahi, alo;  // per node
    float *y32 = nullptr;          // head output [P0][16]
    // training
    bool train_ready = false;
    float *g32 = nullptr, *m32 = nullptr, *v32 = nullptr, *tgt32 = nullptr;
    std::vector<float *> dn;       // per node gradient
    bf16 *dhi = nullptr, *dlo = nullptr, *dThi = nullptr, *dTlo = nullptr, *cThi = nullptr, *cTlo = nullptr;
    float *part = nullptr;
    long long part_cap = 0;
    double *lsum = nullptr, *h_lsum = nullptr;
    int *err = nullptr;
    int adam_t = 0;
    bool fast = false;  // solver inference: BF16 activations (hi products only)
    size_t bytes = 0;
    std::vector<void *> allocs;

    long long rows(int level, int nb) const { return (long long)nb * Z * H[level] * W[level]; }
    long long rows_pad(int level, int nb) const { return (rows(level, nb) + 63) / 64 * 64; }
};

namespace {

template <class T>
int sno_alloc(mms_sno *n, T **p, size_t count)
{
    size_t bytes = std::max<size_t>(16, count * sizeof(T));
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        mms_set_error("cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        return MMS_ERR_NOMEM;
    }
    n->allocs.push_back(*p);
    n->bytes += bytes;
    return MMS_OK;
}

int conv_attr_once()
{
    static int dev_done = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev_done == dev) return MMS_OK;
    MMS_CUDA_TRY(cudaFuncSetAttribute(k_conv<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, conv_smem(4)));
    MMS_CUDA_TRY(cudaFuncSetAttribute(k_conv<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, conv_smem(8)));
    dev_done = dev;
    return MMS_OK;
}

ConvP conv_params(const mms_sno *n, const Layer &y, int nb, bool adjoint)
{
    ConvP p;
    memset(&p, 0, sizeof p);
    const int lin = n->lev[y.in], lout = n->lev[y.out];
    p.Z = n->Z;
    p.err = n->err;
    if (!adjoint) {
        p.ahi = n->ahi[y.in];
        p.alo = n->alo[y.in];
        p.cin_log2 = ilog2(y.cin);
        p.T = y.taps;
        p.pat = y.pat;
        p.Hin = n->H[lin];
        p.Win = n->W[lin];
        p.Hout = n->H[lout];
        p.Wout = n->W[lout];
        p.P = (int)n->rows(lout, nb);
        p.w = n->wf + y.wf_off;
        p.K = p.ldw = 2 * y.taps * y.cin;
        p.N = y.cout;
    } else {
        // gradient w.r.t. the layer input: the adjoint pattern over the input rows
        p.ahi = n->dhi;
        p.alo = n->dlo;
        p.cin_log2 = ilog2(y.cout);
        p.T = y.taps;
        p.pat = y.pat == PAT_DOWN ? PAT_UP : (y.pat == PAT_UP ? PAT_DOWN : y.pat);
        p.Hin = n->H[lout];
        p.Win = n->W[lout];
        p.Hout = n->H[lin];
        p.Wout = n->W[lin];
        p.P = (int)n->rows(lin, nb);
        p.w = n->wb + y.wb_off;
        p.K = p.ldw = 2 * y.taps * y.cout;
        p.N = y.cin;
    }
    return p;
}

// fast: batch-1 inference, hi products only (BF16 activations) and a deep pipeline
int launch_conv(ConvP p, cudaStream_t st, bool fast = false)
{
    MMS_TRY(conv_attr_once());
    if (fast) {
        p.K = p.ldw / 2;
        k_conv<8><<<div_up(p.P, umma::BM), 128, conv_smem(8), st>>>(p);
    } else {
        k_conv<4><<<div_up(p.P, umma::BM), 128, conv_smem(4), st>>>(p);
    }
    MMS_CUDA_TRY(cudaGetLastError());
    return MMS_OK;
}

// forward through every layer except the head; the head is issued by the caller
int forward_body(mms_sno *n, int nb, const float *u, float uscale, cudaStream_t st, bool fast = false)
{
    const long long P0 = n->rows(0, nb);
    k_patchify<<<div_up(P0 * CIN0, 256), 256, 0, st>>>(u, uscale, n->X, n->Y, n->H[0], n->W[0], P0, n->ahi[0],
                                                        n->alo[0]);
    MMS_CUDA_TRY(cudaGetLastError());
    for (size_t i = 0; i + 1 < n->L.size(); i++) {
        const Layer &y = n->L[i];
        ConvP p = conv_params(n, y, nb, false);
        p.ep = EP_SPLIT;
        p.ohi = n->ahi[y.out];
        p.olo = n->alo[y.out];
        if (y.skip >= 0) {
            p.shi = n->ahi[y.skip];
            p.slo = n->alo[y.skip];
        }
        MMS_TRY(launch_conv(p, st, fast));
    }
    return MMS_OK;
}

int check_err(mms_sno *n, cudaStream_t st)
{
    int h = 0;
    MMS_CUDA_TRY(cudaMemcpyAsync(&h, n->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    MMS_CUDA_TRY(cudaStreamSynchronize(st));
    if (h) {
        mms_set_error("surrogate kernel: tensor-core barrier wait timed out");
        MMS_CUDA_TRY(cudaMemsetAsync(n->err, 0, sizeof(int), st));
        return MMS_ERR_CUDA;
    }
    return MMS_OK;
}

int rebuild_bf16(mms_sno *n, cudaStream_t st)
{
    for (const Layer &y : n->L) {
        const int cnt = y.cout * y.taps * y.cin;
        k_build_w<<<div_up(cnt, 256), 256, 0, st>>>(n->w32 + y.w_off, y.pat, y.taps, y.cin, y.cout, n->wf + y.wf_off,
                                                     n->wb + y.wb_off);
        MMS_CUDA_TRY(cudaGetLastError());
    }
    return MMS_OK;
}

int train_alloc(mms_sno *n)
{
    if (n->train_ready) return MMS_OK;
    const int B = n->B;
    MMS_TRY(sno_alloc(n, &n->g32, n->nparam));
    MMS_TRY(sno_alloc(n, &n->m32, n->nparam));
    MMS_TRY(sno_alloc(n, &n->v32, n->nparam));
    MMS_CUDA_TRY(cudaMemset(n->m32, 0, n->nparam * sizeof(float)));
    MMS_CUDA_TRY(cudaMemset(n->v32, 0, n->nparam * sizeof(float)));
    const long long P0 = n->rows(0, B), P0p = n->rows_pad(0, B);
    MMS_TRY(sno_alloc(n, &n->tgt32, P0 * CIN0));
    n->dn.assign(n->lev.size(), nullptr);
    for (size_t i = 1; i < n->lev.size(); i++)  // no gradient for the input node
        MMS_TRY(sno_alloc(n, &n->dn[i], n->rows(n->lev[i], B) * n->ch[i]));
    MMS_TRY(sno_alloc(n, &n->dhi, P0 * CH));
    MMS_TRY(sno_alloc(n, &n->dlo, P0 * CH));
    MMS_TRY(sno_alloc(n, &n->dThi, P0p * CH));
    MMS_TRY(sno_alloc(n, &n->dTlo, P0p * CH));
    MMS_TRY(sno_alloc(n, &n->cThi, P0p * 27 * CH));
    MMS_TRY(sno_alloc(n, &n->cTlo, P0p * 27 * CH));
    n->part_cap = 3LL * 64 * 27 * CH * CH;
    MMS_TRY(sno_alloc(n, &n->part, n->part_cap));
    MMS_TRY(sno_alloc(n, &n->lsum, 2 * B));
    MMS_CUDA_TRY(cudaMallocHost((void **)&n->h_lsum, 2 * B * sizeof(double)));
    n->train_ready = true;
    return MMS_OK;
}

// loss and gradient of the loss w.r.t. every weight (into g32) for the batch
int loss_and_grad(mms_sno *n, int nb, const float *u, const float *far, float uscale, float fscale,
                  cudaStream_t st, double *loss)
{
    MMS_TRY(train_alloc(n));
    MMS_TRY(forward_body(n, nb, u, uscale, st));
    const Layer &hd = n->L.back();
    ConvP ph = conv_params(n, hd, nb, false);
    ph.ep = EP_F32;
    ph.o32 = n->y32;
    MMS_TRY(launch_conv(ph, st));
    const long long P0 = n->rows(0, nb);
    k_patchify_f32<<<div_up(P0 * CIN0, 256), 256, 0, st>>>(far, fscale, n->X, n->Y, n->H[0], n->W[0], P0, n->tgt32);
    MMS_CUDA_TRY(cudaGetLastError());
    const long long per = P0 / nb * CIN0;
    MMS_CUDA_TRY(cudaMemsetAsync(n->lsum, 0, 2 * nb * sizeof(double), st));
    k_loss_sums<<<dim3(64, nb), 256, 0, st>>>(n->y32, n->tgt32, per, n->lsum);
    MMS_CUDA_TRY(cudaGetLastError());
    // backward
    for (size_t i = 1; i < n->lev.size(); i++)
        MMS_CUDA_TRY(cudaMemsetAsync(n->dn[i], 0, n->rows(n->lev[i], nb) * n->ch[i] * sizeof(float), st));
    k_loss_grad<<<div_up(per * nb, 256), 256, 0, st>>>(n->y32, n->tgt32, per, nb, n->lsum, n->dn[hd.out]);
    MMS_CUDA_TRY(cudaGetLastError());
    for (int li = (int)n->L.size() - 1; li >= 0; li--) {
        const Layer &y = n->L[li];
        const int lout = n->lev[y.out];
        const long long Pout = n->rows(lout, nb), Ppad = n->rows_pad(lout, nb);
        k_split_t<<<div_up(Ppad, 64), 256, 0, st>>>(n->dn[y.out], Pout, y.cout, Ppad, n->dhi, n->dlo, n->dThi,
                                                    n->dTlo);
        MMS_CUDA_TRY(cudaGetLastError());
        if (y.skip >= 0) {
            const long long cnt = Pout * y.cout;
            k_axpy<<<div_up(cnt, 256), 256, 0, st>>>(n->dn[y.out], n->dn[y.skip], cnt);
            MMS_CUDA_TRY(cudaGetLastError());
        }
        // weight gradient
        ConvP pf = conv_params(n, y, nb, false);
        k_im2col_t<<<dim3(div_up(Ppad, 256), y.taps * y.cin), 256, 0, st>>>(pf, Ppad, n->cThi, n->cTlo);
        MMS_CUDA_TRY(cudaGetLastError());
        const int M = y.taps * y.cin;
        const int ktiles = (int)(Ppad / 64);
        int splits = std::max(1, std::min(64, ktiles / 16));
        const int kchunk = (int)((ktiles + splits - 1) / splits) * 64;
        splits = (int)((Ppad + kchunk - 1) / kchunk);
        if (3LL * splits * M * y.cout > n->part_cap) {
            mms_set_error("surrogate: partial buffer too small");
            return MMS_ERR_ARG;
        }
        k_dw<<<dim3(div_up(M, umma::BM), splits, 3), 128, 0, st>>>(n->cThi, n->cTlo, n->dThi, n->dTlo, M, y.cout,
                                                                    Ppad, kchunk, n->part, n->err);
        MMS_CUDA_TRY(cudaGetLastError());
        k_dw_reduce<<<div_up(M * y.cout, 256), 256, 0, st>>>(n->part, 3 * splits, y.taps, y.cin, y.cout,
                                                             n->g32 + y.w_off);
        MMS_CUDA_TRY(cudaGetLastError());
        // input gradient (not for the network input)
        if (y.in != 0) {
            ConvP pa = conv_params(n, y, nb, true);
            pa.ep = EP_F32;
            pa.o32 = n->dn[y.in];
            pa.beta = 1;
            MMS_TRY(launch_conv(pa, st));
        }
    }
    if (loss) {
        MMS_CUDA_TRY(cudaMemcpyAsync(n->h_lsum, n->lsum, 2 * nb * sizeof(double), cudaMemcpyDeviceToHost, st));
        MMS_TRY(check_err(n, st));
        double acc = 0;
        for (int b = 0; b < nb; b++) acc += n->h_lsum[2 * b + 1] / (n->h_lsum[2 * b] > 0 ? n->h_lsum[2 * b] : 1.0);
        *loss = acc / nb;
    }
    return MMS_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// internal entry used by the surrogate solver (fmm.cu)

int sno_launch_far(mms_sno *n, cudaStream_t st, const float *rho, float in_scale, float *phi, const float *near,
                   float out_scale, cudaEvent_t wait_before_head, int64_t *launches)
{
    MMS_TRY(forward_body(n, 1, rho, in_scale, st, n->fast));
    if (wait_before_head) MMS_CUDA_TRY(cudaStreamWaitEvent(st, wait_before_head, 0));
    ConvP ph = conv_params(n, n->L.back(), 1, false);
    ph.ep = EP_PHI;
    ph.phi = phi;
    ph.near = near;
    ph.scale = out_scale;
    ph.X = n->X;
    ph.Y = n->Y;
    MMS_TRY(launch_conv(ph, st, n->fast));
    if (launches) *launches += (int64_t)n->L.size() + 1;
    return MMS_OK;
}

int sno_error_flag(mms_sno *n, cudaStream_t st) { return check_err(n, st); }

void sno_set_fast(mms_sno *n, bool fast) { n->fast = fast; }

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

long long mms_sno_num_params(void)
{
    std::vector<Layer> L;
    std::vector<int> lev, ch;
    long long np, nf, nbk;
    build_arch(L, lev, ch, np, nf, nbk);
    return np;
}

int mms_sno_create(int xdim, int ydim, int zdim, int batch, mms_sno **out)
{
    if (!out || xdim < 1 || ydim < 1 || zdim < 1 || batch < 1) {
        mms_set_error("mms_sno_create: bad argument");
        return MMS_ERR_ARG;
    }
    *out = nullptr;
    mms_sno *n = new mms_sno();
    cudaGetDevice(&n->device);
    n->X = xdim;
    n->Y = ydim;
    n->Z = zdim;
    n->B = batch;
    n->H[0] = (ydim + PATCH - 1) / PATCH;
    n->W[0] = (xdim + PATCH - 1) / PATCH;
    for (int l = 1; l < LEVELS; l++) {
        n->H[l] = (n->H[l - 1] + 1) / 2;
        n->W[l] = (n->W[l - 1] + 1) / 2;
    }
    build_arch(n->L, n->lev, n->ch, n->nparam, n->nwf, n->nwb);
    int st = MMS_OK;
    do {
        if (n->rows(0, batch) * 27 * CH >= (1LL << 31) || n->rows_pad(0, batch) * 27 * CH >= (1LL << 40)) {
            mms_set_error("mms_sno_create: grid x batch too large");
            st = MMS_ERR_ARG;
            break;
        }
        if ((st = sno_alloc(n, &n->w32, n->nparam)) || (st = sno_alloc(n, &n->wf, n->nwf)) ||
            (st = sno_alloc(n, &n->wb, n->nwb)) || (st = sno_alloc(n, &n->err, 1)))
            break;
        cudaMemset(n->w32, 0, n->nparam * sizeof(float));
        cudaMemset(n->wf, 0, n->nwf * sizeof(bf16));
        cudaMemset(n->wb, 0, n->nwb * sizeof(bf16));
        cudaMemset(n->err, 0, sizeof(int));
        n->ahi.assign(n->lev.size(), nullptr);
        n->alo.assign(n->lev.size(), nullptr);
        for (size_t i = 0; i + 1 < n->lev.size() && st == MMS_OK; i++) {
            const long long cnt = n->rows(n->lev[i], batch) * n->ch[i];
            if ((st = sno_alloc(n, &n->ahi[i], cnt)) || (st = sno_alloc(n, &n->alo[i], cnt))) break;
        }
        if (st) break;
        st = sno_alloc(n, &n->y32, n->rows(0, batch) * CIN0);
    } while (0);
    if (st != MMS_OK) {
        for (void *p : n->allocs) cudaFree(p);
        delete n;
        return st;
    }
    *out = n;
    return MMS_OK;
}

void mms_sno_destroy(mms_sno *n)
{
    if (!n) return;
    cudaDeviceSynchronize();
    for (void *p : n->allocs) cudaFree(p);
    if (n->h_lsum) cudaFreeHost(n->h_lsum);
    delete n;
}

int mms_sno_set_weights(mms_sno *n, const float *w, long long count)
{
    if (!n || !w || count != n->nparam) {
        mms_set_error("mms_sno_set_weights: expected %lld weights", n ? n->nparam : 0LL);
        return MMS_ERR_ARG;
    }
    MMS_CUDA_TRY(cudaMemcpy(n->w32, w, count * sizeof(float), cudaMemcpyHostToDevice));
    MMS_TRY(rebuild_bf16(n, 0));
    if (n->train_ready) {
        MMS_CUDA_TRY(cudaMemset(n->m32, 0, n->nparam * sizeof(float)));
        MMS_CUDA_TRY(cudaMemset(n->v32, 0, n->nparam * sizeof(float)));
    }
    n->adam_t = 0;
    MMS_CUDA_TRY(cudaDeviceSynchronize());
    return MMS_OK;
}

int mms_sno_get_weights(mms_sno *n, float *w, long long count, int bf16_rounded)
{
    if (!n || !w || count != n->nparam) {
        mms_set_error("mms_sno_get_weights: expected %lld weights", n ? n->nparam : 0LL);
        return MMS_ERR_ARG;
    }
    MMS_CUDA_TRY(cudaDeviceSynchronize());
    if (bf16_rounded) {
        float *tmp = nullptr;
        MMS_CUDA_TRY(cudaMalloc(&tmp, count * sizeof(float)));
        k_round_bf16<<<div_up(count, 256), 256>>>(n->w32, tmp, count);
        cudaError_t e = cudaMemcpy(w, tmp, count * sizeof(float), cudaMemcpyDeviceToHost);
        cudaFree(tmp);
        MMS_CUDA_TRY(e);
    } else {
        MMS_CUDA_TRY(cudaMemcpy(w, n->w32, count * sizeof(float), cudaMemcpyDeviceToHost));
    }
    return MMS_OK;
}

int mms_sno_forward_dev(mms_sno *n, const float *u, float *out, int nbatch)
{
    if (!n || !u || !out || nbatch < 1 || nbatch > n->B) {
        mms_set_error("mms_sno_forward_dev: bad argument");
        return MMS_ERR_ARG;
    }
    MMS_TRY(forward_body(n, nbatch, u, 1.f, 0));
    ConvP ph = conv_params(n, n->L.back(), nbatch, false);
    ph.ep = EP_F32;
    ph.o32 = n->y32;
    MMS_TRY(launch_conv(ph, 0));
    const long long P0 = n->rows(0, nbatch);
    k_unpatchify<<<div_up(P0 * CIN0, 256), 256>>>(n->y32, n->X, n->Y, n->H[0], n->W[0], P0, out);
    MMS_CUDA_TRY(cudaGetLastError());
    return check_err(n, 0);
}

int mms_sno_gradient(mms_sno *n, const float *u, const float *far, int nbatch, float *grad, double *loss)
{
    if (!n || !u || !far || nbatch < 1 || nbatch > n->B) {
        mms_set_error("mms_sno_gradient: bad argument");
        return MMS_ERR_ARG;
    }
    MMS_TRY(loss_and_grad(n, nbatch, u, far, 1.f, 1.f, 0, loss));
    if (grad) MMS_CUDA_TRY(cudaMemcpy(grad, n->g32, n->nparam * sizeof(float), cudaMemcpyDeviceToHost));
    return MMS_OK;
}

int mms_sno_train_step(mms_sno *n, const float *u, const float *far, int nbatch, float lr, float beta1, float beta2,
                       float eps, double *loss)
{
    if (!n || !u || !far || nbatch < 1 || nbatch > n->B || !(lr >= 0)) {
        mms_set_error("mms_sno_train_step: bad argument");
        return MMS_ERR_ARG;
    }
    MMS_TRY(loss_and_grad(n, nbatch, u, far, 1.f, 1.f, 0, loss));
    n->adam_t++;
    const float bc1 = 1.f - powf(beta1, (float)n->adam_t), bc2 = 1.f - powf(beta2, (float)n->adam_t);
    k_adam<<<div_up(n->nparam, 256), 256>>>(n->w32, n->g32, n->m32, n->v32, n->nparam, lr, beta1, beta2, eps, bc1,
                                           bc2);
    MMS_CUDA_TRY(cudaGetLastError());
    return rebuild_bf16(n, 0);
}

long long mms_sno_device_bytes(const mms_sno *n) { return n ? (long long)n->bytes : 0; }

}  // extern "C"
