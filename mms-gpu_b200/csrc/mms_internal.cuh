// Internal declarations shared by the mms_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "mms_b200.h"
#include <nvtx3/nvToolsExt.h>

// NVTX range over a scope (host side): names the public entry points and the
// stages of a field evaluation in a profiler's timeline (nsys, or ncu
// --nvtx --nvtx-include "mms/..."); free when no profiler is attached.
struct MmsRange {
    explicit MmsRange(const char *name) { nvtxRangePushA(name); }
    ~MmsRange() { nvtxRangePop(); }
    MmsRange(const MmsRange &) = delete;
    MmsRange &operator=(const MmsRange &) = delete;
};

// ---------------------------------------------------------------------------
// error plumbing: every failure becomes a status code and a thread-local message
void mms_set_error(const char *fmt, ...);

#define MMS_CUDA_TRY(expr)                                                                  \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            mms_set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(e_)); \
            return MMS_ERR_CUDA;                                                            \
        }                                                                                   \
    } while (0)

#define MMS_TRY(expr)                  \
    do {                               \
        int s_ = (expr);               \
        if (s_ != MMS_OK) return s_;   \
    } while (0)

// after a launch: check the launch itself (asynchronous faults surface at sync)
#define MMS_LAUNCH_CHECK(ctx)                                                               \
    do {                                                                                    \
        (ctx)->launches++;                                                                  \
        cudaError_t e_ = cudaGetLastError();                                                \
        if (e_ != cudaSuccess) {                                                            \
            mms_set_error("%s:%d kernel launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            return MMS_ERR_CUDA;                                                            \
        }                                                                                   \
    } while (0)

// ---------------------------------------------------------------------------
// device-side constants of a grid / material, passed by value to kernels
struct GridK {
    int X, Y, Z;
    long long N;
    double dx, dy, dz;
};

constexpr int MMS_MAX_HEXT = 64;

struct PhysK {
    double Ms, alpha, gamma, mu0;
    double cexch;        // 2 A / (mu0 Ms^2)
    double cdemag;       // 1 / (4 pi)
    // the quotients of the per-cell field and LLG formed once on the host
    // (physk_derive), so that the kernels multiply instead of divide
    double hgx, hgy, hgz;  // cdemag / (2 d): the demag central difference
    double ecx, ecy, ecz;  // cexch / d^2: the exchange Laplacian
    double llg_a;          // alpha gamma / Ms
    double inv_mu0;        // 1 / mu0: B -> H
    int demag, exchange, external;
    int n_hext;          // 0 + external: the reference's built-in ramp
    int ref_stage_time;
};

inline void physk_derive(PhysK &k, double dx, double dy, double dz)
{
    k.hgx = k.cdemag / (2 * dx);
    k.hgy = k.cdemag / (2 * dy);
    k.hgz = k.cdemag / (2 * dz);
    k.ecx = k.cexch / (dx * dx);
    k.ecy = k.cexch / (dy * dy);
    k.ecz = k.cexch / (dz * dz);
    k.llg_a = k.alpha * k.gamma / k.Ms;
    k.inv_mu0 = 1.0 / k.mu0;
}

// time state kept on the device so a captured step graph stays valid:
//   [0] t      current time of the state M
//   [1] dt     step size
//   [2] t_k1   time at which H(M) (the k1 field) was evaluated; equals t
//              except in reference-stage-time mode (see mms_params)
constexpr int TIME_T = 0, TIME_DT = 1, TIME_TK1 = 2, TIME_SLOTS = 4;
//   [3] (low 32 bits) arrival counter of the last RK4 stage's CTAs: the last
//       to finish advances the time and resets it (k_rk4_stage)
constexpr int TIME_CTR = 3;

// statistics block: sums over material cells, finished on device
//   [0] sum M.H  [1] max |MxH|  [2..4] sum M  [5] sum |M|  [6] count  [7] nonfinite flag
constexpr int STAT_SLOTS = 8;

struct FmmPlan;  // fmm.cu

struct mms_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    mms_grid g{};
    mms_params p{};
    std::vector<double> hext_t, hext_b;
    mms_solver s{};
    long long N = 0;
    int64_t launches = 0;
    size_t dev_bytes = 0;

    // device buffers
    float *rho = nullptr, *phi = nullptr;       // N
    float *vecA = nullptr, *vecB = nullptr;     // 3N FP32 AoS scratch (host API)
    float *gtab = nullptr;                      // direct-sum kernel table X*Y*Z
    uint8_t *mat = nullptr;                     // N
    double *M = nullptr, *A = nullptr, *B = nullptr, *K = nullptr;  // 3N each, SoA planes
    double *Mbak = nullptr;                     // 3N, controller backup
    double *Mfull = nullptr;                    // 3N, step-doubling full-step result
    float *phibak = nullptr;                    // N, controller backup
    double *tstate = nullptr;                   // TIME_SLOTS
    double *hext = nullptr;                     // MMS_MAX_HEXT x 4 (t, Bx, By, Bz)
    double *stat_part = nullptr;                // per-block partial statistics
    double *stats = nullptr;                    // STAT_SLOTS
    int stat_blocks = 0;
    double *h_stats = nullptr;                  // pinned host mirror of stats + time

    FmmPlan *fmm = nullptr;

    // surrogate solver (MMS_SOLVER_SURROGATE): weights bound to the FMM plan
    bool sur_bound = false;
    int sur_every = 0;
    double sur_tol = 1e-3;
    bool sur_active = false;                    // false: the FMM took over
    long long sur_since = 0, sur_checks = 0, sur_fallbacks = 0;
    double sur_last_err = 0, sur_max_err = 0;

    bool state_ready = false;
    bool phi_valid = false;                     // phi holds the potential of M
    bool dt_known = false;                      // tstate's dt is dt_dev (set by mms_run_fixed)
    double dt_dev = 0.0;

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_kernels = 0;
    int graph_solver_kind = -1;
    bool graph_eval_first = false;              // the captured step evaluates phi(M) first

    GridK gk() const {
        GridK k;
        k.X = g.xdim; k.Y = g.ydim; k.Z = g.zdim; k.N = N;
        k.dx = g.dx; k.dy = g.dy; k.dz = g.dz;
        return k;
    }
    PhysK pk() const;
};

// ---------------------------------------------------------------------------
// kernel entry points (host-side launchers); all asynchronous on ctx->stream
int launch_divergence_soa(mms_ctx *ctx, const double *M, float *rho);
int launch_divergence_aos(mms_ctx *ctx, const float *M, float *rho);
int launch_gradient_aos(mms_ctx *ctx, const float *phi, double c, float *H);
int launch_exchange_aos(mms_ctx *ctx, const float *M, float *H);
int launch_hfield_aos(mms_ctx *ctx, const float *M, const float *phi, double t, float *H);
// stage 3 also advances the state's time (t_k1 = t, t += dt)
int launch_rk4_stage(mms_ctx *ctx, int stage, const double *Mst, double *Mnext);
int launch_stats(mms_ctx *ctx);

int direct_build_table(mms_ctx *ctx);
int launch_potential_direct(mms_ctx *ctx, const float *rho, float *phi);

int fmm_plan_create(mms_ctx *ctx);
int launch_potential_surrogate(mms_ctx *ctx, const float *rho, float *phi);
int launch_potential_split(mms_ctx *ctx, const float *rho, float *phi, float *near);
// binds the learned far-field network's weights (a vector indexed by depth,
// farnet.cuh) to the context's FMM plan (leaf 8, 3 layers)
int farnet_bind(mms_ctx *ctx, const float *w, long long count);
// rel-L2 |a - b| / |b| over n floats (tune.cu); synchronises ctx->stream
int rel_l2_dev(mms_ctx *ctx, const float *a, const float *b, long long n, double *out);
void fmm_plan_destroy(mms_ctx *ctx);
int launch_potential_fmm(mms_ctx *ctx, const float *rho, float *phi);
// FMM potential of the FP64 state M into phi, and rho = div M into rho: where
// the plan allows, the P2M forms rho itself (with the BF16 split of the
// tensor-core near field) instead of a divergence launch before it
int launch_potential_fmm_state(mms_ctx *ctx, const double *M, float *rho, float *phi);
// the tensor-core near field's box-major BF16 hi / lo charges, for a
// divergence kernel to write beside rho: returns 0 when the plan has no
// tensor-core near field; fmm_split_written(ctx, rho) records that they hold
// rho's split (a potential of that rho then skips k_rho_split), and
// fmm_split_written(ctx, nullptr) forgets it
int fmm_split_target(const mms_ctx *ctx, void **hi, void **lo, int *nbx, int *nby);
void fmm_split_written(mms_ctx *ctx, const float *rho);
int fmm_far_error(mms_ctx *ctx);  // 1: a bounded wait of an FMM kernel timed out
size_t fmm_plan_bytes(const mms_ctx *ctx);

// tcgen05 BF16 GEMM (gemm.cu): C (+)= A B^T, A M x K, B N x K, K-major
int umma_gemm_bf16(const void *A, int lda, const void *B, int ldb, float *C, int ldc, int M, int N, int K, int beta,
                   int bn, cudaStream_t st);
// split-K form for long K and few output tiles: `splits` CTAs per tile, each
// over kchunk (a multiple of 64) of K into Cpart[splits][M][N], then C = the
// fixed-order sum; umma_gemm_bf16_splitk_plan picks splits for ~one wave
int umma_gemm_bf16_splitk_plan(int M, int N, int K, int bn, int *splits, int *kchunk);
int umma_gemm_bf16_splitk(const void *A, int lda, const void *B, int ldb, float *C, float *Cpart, int M, int N,
                          int K, int bn, int splits, int kchunk, cudaStream_t st);
int umma_check_error();

// potential with the context's solver
int launch_potential(mms_ctx *ctx, const float *rho, float *phi);

// ---------------------------------------------------------------------------
// programmatic dependent launch: a kernel launched by launch_k may be scheduled
// while its stream predecessor is still running.  Every kernel launched this
// way starts with pdl_begin(): it waits for the predecessor grid's completion
// (and memory) before touching any input, then lets its own successor be
// scheduled.  The overlap hides launch and ramp-up latency between the many
// short kernels of a field evaluation.  MMS_PDL=0 in the environment turns the
// attribute off (plain stream order).
bool pdl_enabled();

__device__ __forceinline__ void pdl_begin()
{
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
#ifdef MMS_PDL_EARLY_TRIGGER
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
#endif
}

template <typename... KArgs, typename... Args>
cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// device allocation tracked in ctx->dev_bytes
template <class T>
int ctx_alloc(mms_ctx *ctx, T **p, size_t count)
{
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        mms_set_error("cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        return MMS_ERR_NOMEM;
    }
    ctx->dev_bytes += bytes;
    return MMS_OK;
}

static inline unsigned div_up(long long a, long long b) { return (unsigned)((a + b - 1) / b); }
