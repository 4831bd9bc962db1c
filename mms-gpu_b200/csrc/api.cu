// C ABI of mms_b200: contexts, the stateless field operators, the resident
// FP64 RK4 state, the fixed-step driver (optionally one CUDA graph per step)
// and the adaptive marching loop.
#include "mms_internal.cuh"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

static thread_local char g_err[1024] = "";

void mms_set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

namespace {

__global__ void k_set_dt(double *tstate, double dt) { tstate[TIME_DT] = dt; }

__global__ void k_set_time(double *tstate, double t, double tk1, double dt)
{
    tstate[TIME_T] = t;
    tstate[TIME_TK1] = tk1;
    tstate[TIME_DT] = dt;
}

// A new state in one launch: the material mask (mat_in -> mat, which may be
// the same buffer), M from AoS (x,y,z per cell; FP64, or FP32 in the
// reference's Vector3 layout, widened exactly) to the FP64 SoA planes with
// empty cells -> 0, the time (t, t_k1 = t, dt = 0) and the non-finite flag
// cleared
template <typename T>
__global__ void k_state_in(const T *__restrict__ in, const uint8_t *mat_in, uint8_t *mat, double *__restrict__ out,
                           long long N, double *__restrict__ tstate, double *__restrict__ stats, double t)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i == 0) {
        tstate[TIME_T] = t;
        tstate[TIME_TK1] = t;
        tstate[TIME_DT] = 0.0;
        stats[7] = 0.0;
    }
    if (i >= N) return;
    const uint8_t mv = mat_in[i];
    mat[i] = mv;
    const bool m = mv != 0;
    out[i] = m ? (double)in[3 * i + 0] : 0.0;
    out[i + N] = m ? (double)in[3 * i + 1] : 0.0;
    out[i + 2 * N] = m ? (double)in[3 * i + 2] : 0.0;
}

__global__ void k_soa_to_aos(const double *__restrict__ in, double *__restrict__ out, long long N)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= N) return;
    out[3 * i + 0] = in[i];
    out[3 * i + 1] = in[i + N];
    out[3 * i + 2] = in[i + 2 * N];
}

// FP64 SoA planes -> FP32 AoS, each component rounded to nearest
__global__ void k_soa_to_aos32(const double *__restrict__ in, float *__restrict__ out, long long N)
{
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= N) return;
    out[3 * i + 0] = (float)in[i];
    out[3 * i + 1] = (float)in[i + N];
    out[3 * i + 2] = (float)in[i + 2 * N];
}

// per-block max over material cells of max_c |a_c - b_c|, then a fixed-order finish
__global__ void k_maxdiff_part(const double *__restrict__ a, const double *__restrict__ b,
                               const uint8_t *__restrict__ mat, double *__restrict__ part, long long N)
{
    __shared__ double sh[8];
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < N && mat[i])
        for (int c = 0; c < 3; c++) v = fmax(v, fabs(a[i + c * N] - b[i + c * N]));
    if (!(v == v)) v = INFINITY;  // NaN counts as an infinite error
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = sh[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) r = fmax(r, sh[w]);
        part[blockIdx.x * 8] = r;
    }
}

__global__ void k_maxdiff_final(const double *__restrict__ part, int nb, double *__restrict__ out)
{
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += 32) v = fmax(v, part[(long long)b * 8]);
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) out[0] = v;
}

int check_grid(const mms_grid *g)
{
    if (!g || g->xdim < 1 || g->ydim < 1 || g->zdim < 1) {
        mms_set_error("grid dimensions must be positive");
        return MMS_ERR_ARG;
    }
    if (!(g->dx > 0 && g->dy > 0 && g->dz > 0)) {
        mms_set_error("cell sizes must be positive");
        return MMS_ERR_ARG;
    }
    if ((long long)g->xdim * g->ydim * g->zdim > (1LL << 31) / 4) {
        mms_set_error("grid too large (%d x %d x %d)", g->xdim, g->ydim, g->zdim);
        return MMS_ERR_ARG;
    }
    return MMS_OK;
}

int apply_params(mms_ctx *ctx, const mms_params *p)
{
    if (!p) {
        mms_set_error("params is NULL");
        return MMS_ERR_ARG;
    }
    if (!(p->Ms > 0) || !(p->mu0 > 0)) {
        mms_set_error("Ms and mu0 must be positive");
        return MMS_ERR_ARG;
    }
    if (p->n_hext < 0 || p->n_hext > MMS_MAX_HEXT || (p->n_hext > 0 && (!p->hext_t || !p->hext_b))) {
        mms_set_error("external field table: 0..%d entries with both arrays", MMS_MAX_HEXT);
        return MMS_ERR_ARG;
    }
    for (int k = 1; k < p->n_hext; k++)
        if (!(p->hext_t[k] > p->hext_t[k - 1])) {
            mms_set_error("external field table times must increase");
            return MMS_ERR_ARG;
        }
    ctx->p = *p;
    ctx->hext_t.assign(p->hext_t, p->hext_t + p->n_hext);
    ctx->hext_b.assign(p->hext_b, p->hext_b + 3 * p->n_hext);
    ctx->p.hext_t = nullptr;
    ctx->p.hext_b = nullptr;
    std::vector<double> tab(4 * MMS_MAX_HEXT, 0.0);
    for (int k = 0; k < p->n_hext; k++) {
        tab[4 * k] = p->hext_t[k];
        for (int c = 0; c < 3; c++) tab[4 * k + 1 + c] = p->hext_b[3 * k + c];
    }
    MMS_CUDA_TRY(cudaMemcpyAsync(ctx->hext, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice,
                                 ctx->stream));
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return MMS_OK;
}

void drop_graph(mms_ctx *ctx)
{
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    if (ctx->graph) cudaGraphDestroy(ctx->graph);
    ctx->graph_exec = nullptr;
    ctx->graph = nullptr;
    ctx->graph_kernels = 0;
}

// potential of the state M into ctx->phi (rho = div M into ctx->rho)
int eval_state_potential(mms_ctx *ctx, const double *Mst)
{
    MmsRange nvtx_("mms/field_evaluation");
    if (!ctx->p.demag) return MMS_OK;  // phi unused
    if (ctx->s.kind == MMS_SOLVER_FMM || (ctx->s.kind == MMS_SOLVER_SURROGATE && !ctx->sur_active))
        return launch_potential_fmm_state(ctx, Mst, ctx->rho, ctx->phi);
    MMS_TRY(launch_divergence_soa(ctx, Mst, ctx->rho));
    MMS_TRY(launch_potential(ctx, ctx->rho, ctx->phi));
    return MMS_OK;
}

// One RK4 step on the resident state, 4 field evaluations.  Normally phi holds
// the potential of M on entry and of the new M on exit (the k1 field of the
// next step).  With eval_first the step begins by evaluating the potential of
// M and leaves the new M's potential unevaluated: a state set from outside
// (which has no potential yet) then also costs 4 evaluations per step instead
// of 5.  Both orders evaluate the same potentials of the same states.
int rk4_step_kernels(mms_ctx *ctx, bool eval_first)
{
    MmsRange nvtx_("mms/rk4_step");
    if (eval_first) MMS_TRY(eval_state_potential(ctx, ctx->M));
    MMS_TRY(launch_rk4_stage(ctx, 0, ctx->M, ctx->A));
    MMS_TRY(eval_state_potential(ctx, ctx->A));
    MMS_TRY(launch_rk4_stage(ctx, 1, ctx->A, ctx->B));
    MMS_TRY(eval_state_potential(ctx, ctx->B));
    MMS_TRY(launch_rk4_stage(ctx, 2, ctx->B, ctx->A));
    MMS_TRY(eval_state_potential(ctx, ctx->A));
    MMS_TRY(launch_rk4_stage(ctx, 3, ctx->A, nullptr));
    if (!eval_first) MMS_TRY(eval_state_potential(ctx, ctx->M));
    return MMS_OK;
}

int ensure_phi(mms_ctx *ctx)
{
    if (!ctx->phi_valid) {
        MMS_TRY(eval_state_potential(ctx, ctx->M));
        ctx->phi_valid = true;
    }
    return MMS_OK;
}

// the solver a captured graph holds: the surrogate solver runs the FMM once it took over
int effective_kind(const mms_ctx *ctx)
{
    if (ctx->s.kind == MMS_SOLVER_SURROGATE && !ctx->sur_active) return MMS_SOLVER_FMM;
    return ctx->s.kind;
}

// Steps from a state without a potential (set from outside, or parameters
// changed) run in the evaluate-first order and leave phi invalid; steps from
// a state with its potential keep it valid.  Either way 4 evaluations a step.
int run_steps(mms_ctx *ctx, int nsteps, int use_graph)
{
    if (nsteps <= 0) return MMS_OK;
    const bool ef = !ctx->phi_valid;
    if (!use_graph) {
        for (int s = 0; s < nsteps; s++) MMS_TRY(rk4_step_kernels(ctx, ef));
        ctx->phi_valid = !ef;
        return MMS_OK;
    }
    const int kind = effective_kind(ctx);
    if (ctx->graph_exec && (ctx->graph_solver_kind != kind || ctx->graph_eval_first != ef)) drop_graph(ctx);
    if (!ctx->graph_exec) {
        const int64_t before = ctx->launches;
        MMS_CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int st = rk4_step_kernels(ctx, ef);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
        if (st != MMS_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) {
            mms_set_error("graph capture: %s", cudaGetErrorString(e));
            return MMS_ERR_CUDA;
        }
        ctx->graph = graph;
        MMS_CUDA_TRY(cudaGraphInstantiate(&ctx->graph_exec, graph, 0));
        ctx->graph_kernels = (int)(ctx->launches - before);
        ctx->launches = before;  // captured, not yet launched
        ctx->graph_solver_kind = kind;
        ctx->graph_eval_first = ef;
    }
    for (int s = 0; s < nsteps; s++) {
        MMS_CUDA_TRY(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
        ctx->launches += ctx->graph_kernels;
    }
    ctx->phi_valid = !ef;
    return MMS_OK;
}

// surrogate check on the current state: both potentials, rel-L2, fallback
int surrogate_check_now(mms_ctx *ctx, double *err_out)
{
    MmsRange nvtx_("mms/surrogate_check");
    MMS_TRY(launch_divergence_soa(ctx, ctx->M, ctx->rho));
    float *ps = ctx->vecA, *pf = ctx->vecB;
    MMS_TRY(launch_potential_surrogate(ctx, ctx->rho, ps));
    MMS_TRY(launch_potential_fmm(ctx, ctx->rho, pf));
    double err = 0;
    MMS_TRY(rel_l2_dev(ctx, ps, pf, ctx->N, &err));
    ctx->sur_checks++;
    ctx->sur_last_err = err;
    ctx->sur_max_err = std::max(ctx->sur_max_err, err);
    ctx->sur_since = 0;
    if (!(err <= ctx->sur_tol) && ctx->sur_active) {
        ctx->sur_active = false;
        ctx->sur_fallbacks++;
        // from here on phi is the FMM's potential of M
        MMS_CUDA_TRY(cudaMemcpyAsync(ctx->phi, pf, (size_t)ctx->N * sizeof(float), cudaMemcpyDeviceToDevice,
                                     ctx->stream));
        drop_graph(ctx);
    }
    if (err_out) *err_out = err;
    return MMS_OK;
}

bool surrogate_armed(const mms_ctx *ctx)
{
    return ctx->s.kind == MMS_SOLVER_SURROGATE && ctx->sur_bound && ctx->sur_active && ctx->sur_every > 0;
}

int read_stats(mms_ctx *ctx, double out[STAT_SLOTS])
{
    MMS_CUDA_TRY(cudaMemcpyAsync(ctx->h_stats, ctx->stats, STAT_SLOTS * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    memcpy(out, ctx->h_stats, STAT_SLOTS * sizeof(double));
    return MMS_OK;
}

int read_time(mms_ctx *ctx, double out[TIME_SLOTS])
{
    MMS_CUDA_TRY(cudaMemcpyAsync(ctx->h_stats + STAT_SLOTS, ctx->tstate, TIME_SLOTS * sizeof(double),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    memcpy(out, ctx->h_stats + STAT_SLOTS, TIME_SLOTS * sizeof(double));
    return MMS_OK;
}

int require_state(mms_ctx *ctx)
{
    if (!ctx) {
        mms_set_error("context is NULL");
        return MMS_ERR_ARG;
    }
    if (!ctx->state_ready) {
        mms_set_error("state not set (call mms_state_set first)");
        return MMS_ERR_NOT_READY;
    }
    return MMS_OK;
}

}  // namespace

bool pdl_enabled()
{
    static const bool on = [] {
        const char *e = getenv("MMS_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

int launch_potential(mms_ctx *ctx, const float *rho, float *phi)
{
    if (ctx->s.kind == MMS_SOLVER_SURROGATE)
        return ctx->sur_active ? launch_potential_surrogate(ctx, rho, phi) : launch_potential_fmm(ctx, rho, phi);
    if (ctx->s.kind == MMS_SOLVER_FMM) return launch_potential_fmm(ctx, rho, phi);
    return launch_potential_direct(ctx, rho, phi);
}

extern "C" {

int mms_abi_version(void) { return MMS_ABI_VERSION; }

const char *mms_last_error(void) { return g_err; }

int mms_ctx_create(const mms_grid *grid, const mms_params *params, const mms_solver *solver, void *stream,
                   mms_ctx **out)
{
    if (!out) {
        mms_set_error("out is NULL");
        return MMS_ERR_ARG;
    }
    *out = nullptr;
    MMS_TRY(check_grid(grid));
    mms_ctx *ctx = new (std::nothrow) mms_ctx();
    if (!ctx) {
        mms_set_error("host allocation failed");
        return MMS_ERR_NOMEM;
    }
    int st = MMS_OK;
    do {
        if (cudaGetDevice(&ctx->device) != cudaSuccess) {
            mms_set_error("no CUDA device");
            st = MMS_ERR_CUDA;
            break;
        }
        ctx->g = *grid;
        ctx->N = (long long)grid->xdim * grid->ydim * grid->zdim;
        if (stream) {
            ctx->stream = (cudaStream_t)stream;
        } else {
            // a blocking stream: ordered with the legacy default stream, so a
            // caller's default-stream copies and this context's kernels never race
            if (cudaStreamCreate(&ctx->stream) != cudaSuccess) {
                mms_set_error("cudaStreamCreate failed");
                st = MMS_ERR_CUDA;
                break;
            }
            ctx->own_stream = true;
        }
        const size_t N = (size_t)ctx->N;
        if ((st = ctx_alloc(ctx, &ctx->rho, N))) break;
        if ((st = ctx_alloc(ctx, &ctx->phi, N))) break;
        if ((st = ctx_alloc(ctx, &ctx->phibak, N))) break;
        if ((st = ctx_alloc(ctx, &ctx->vecA, 3 * N))) break;
        if ((st = ctx_alloc(ctx, &ctx->vecB, 3 * N))) break;
        if ((st = ctx_alloc(ctx, &ctx->mat, N))) break;
        if ((st = ctx_alloc(ctx, &ctx->M, 3 * N))) break;
        if ((st = ctx_alloc(ctx, &ctx->A, 3 * N))) break;
        if ((st = ctx_alloc(ctx, &ctx->B, 3 * N))) break;
        if ((st = ctx_alloc(ctx, &ctx->K, 3 * N))) break;
        if ((st = ctx_alloc(ctx, &ctx->Mbak, 3 * N))) break;
        if ((st = ctx_alloc(ctx, &ctx->Mfull, 3 * N))) break;
        if ((st = ctx_alloc(ctx, &ctx->tstate, TIME_SLOTS))) break;
        if ((st = ctx_alloc(ctx, &ctx->hext, 4 * MMS_MAX_HEXT))) break;
        ctx->stat_blocks = (int)div_up(ctx->N, 256);
        if ((st = ctx_alloc(ctx, &ctx->stat_part, (size_t)ctx->stat_blocks * 8))) break;
        if ((st = ctx_alloc(ctx, &ctx->stats, STAT_SLOTS))) break;
        if (cudaMallocHost((void **)&ctx->h_stats, (STAT_SLOTS + TIME_SLOTS) * sizeof(double)) != cudaSuccess) {
            mms_set_error("cudaMallocHost failed");
            st = MMS_ERR_NOMEM;
            break;
        }
        if (cudaMemsetAsync(ctx->stats, 0, STAT_SLOTS * sizeof(double), ctx->stream) != cudaSuccess ||
            cudaMemsetAsync(ctx->tstate, 0, TIME_SLOTS * sizeof(double), ctx->stream) != cudaSuccess ||
            cudaMemsetAsync(ctx->mat, 0, N, ctx->stream) != cudaSuccess) {
            mms_set_error("cudaMemset failed");
            st = MMS_ERR_CUDA;
            break;
        }
        if ((st = apply_params(ctx, params))) break;
        mms_solver def{};
        def.kind = MMS_SOLVER_DIRECT;
        def.fmm_order = 4;
        ctx->s = solver ? *solver : def;
        if (ctx->s.kind == MMS_SOLVER_FMM || ctx->s.kind == MMS_SOLVER_SURROGATE) {
            if ((st = fmm_plan_create(ctx))) break;
        } else if (ctx->s.kind == MMS_SOLVER_DIRECT) {
            if ((st = direct_build_table(ctx))) break;
        } else {
            mms_set_error("unknown solver kind %d", ctx->s.kind);
            st = MMS_ERR_ARG;
            break;
        }
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            mms_set_error("context set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
            st = MMS_ERR_CUDA;
            break;
        }
    } while (0);
    if (st != MMS_OK) {
        char keep[1024];
        strncpy(keep, g_err, sizeof keep - 1);
        keep[sizeof keep - 1] = 0;
        mms_ctx_destroy(ctx);
        mms_set_error("%s", keep);
        return st;
    }
    *out = ctx;
    return MMS_OK;
}

int mms_ctx_destroy(mms_ctx *ctx)
{
    if (!ctx) return MMS_OK;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drop_graph(ctx);
    fmm_plan_destroy(ctx);
    void *bufs[] = {ctx->rho, ctx->phi, ctx->phibak, ctx->vecA, ctx->vecB, ctx->gtab, ctx->mat, ctx->M, ctx->A,
                    ctx->B, ctx->K, ctx->Mbak, ctx->Mfull, ctx->tstate, ctx->hext, ctx->stat_part, ctx->stats};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (ctx->h_stats) cudaFreeHost(ctx->h_stats);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MMS_OK;
}

int mms_ctx_set_params(mms_ctx *ctx, const mms_params *params)
{
    if (!ctx) {
        mms_set_error("context is NULL");
        return MMS_ERR_ARG;
    }
    MMS_TRY(apply_params(ctx, params));
    drop_graph(ctx);  // captured kernels hold the old constants
    ctx->phi_valid = false;
    return MMS_OK;
}

int mms_ctx_set_solver(mms_ctx *ctx, const mms_solver *solver)
{
    if (!ctx || !solver) {
        mms_set_error("context or solver is NULL");
        return MMS_ERR_ARG;
    }
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    drop_graph(ctx);
    fmm_plan_destroy(ctx);
    ctx->sur_bound = false;  // the network's tables lived in the plan
    ctx->s = *solver;
    if (ctx->s.kind == MMS_SOLVER_FMM || ctx->s.kind == MMS_SOLVER_SURROGATE) {
        MMS_TRY(fmm_plan_create(ctx));
    } else if (ctx->s.kind == MMS_SOLVER_DIRECT) {
        if (!ctx->gtab) MMS_TRY(direct_build_table(ctx));
    } else {
        mms_set_error("unknown solver kind %d", ctx->s.kind);
        return MMS_ERR_ARG;
    }
    ctx->phi_valid = false;
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return MMS_OK;
}

int mms_ctx_sync(mms_ctx *ctx)
{
    if (!ctx) {
        mms_set_error("context is NULL");
        return MMS_ERR_ARG;
    }
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (fmm_far_error(ctx)) {
        mms_set_error("FMM: a bounded wait timed out (fused far-field barrier or tensor-core pipeline)");
        return MMS_ERR_CUDA;
    }
    return MMS_OK;
}

int64_t mms_ctx_kernel_launches(const mms_ctx *ctx) { return ctx ? ctx->launches : 0; }

size_t mms_ctx_device_bytes(const mms_ctx *ctx) { return ctx ? ctx->dev_bytes + fmm_plan_bytes(ctx) : 0; }

// ---- stateless operators ----------------------------------------------------

int mms_divergence_dev(mms_ctx *ctx, const float *M, float *rho)
{
    if (!ctx || !M || !rho) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    return launch_divergence_aos(ctx, M, rho);
}

int mms_potential_dev(mms_ctx *ctx, const float *rho, float *phi)
{
    MmsRange nvtx_("mms/potential");
    if (!ctx || !rho || !phi) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    return launch_potential(ctx, rho, phi);
}

int mms_gradient_dev(mms_ctx *ctx, const float *phi, double c, float *H)
{
    if (!ctx || !phi || !H) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    return launch_gradient_aos(ctx, phi, c, H);
}

int mms_exchange_dev(mms_ctx *ctx, const float *M, float *H)
{
    if (!ctx || !M || !H) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    return launch_exchange_aos(ctx, M, H);
}

int mms_hfield_dev(mms_ctx *ctx, const float *M, float *H, float *charge, float *potential, double t)
{
    MmsRange nvtx_("mms/hfield");
    if (!ctx || !M || !H) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    float *rho = charge ? charge : ctx->rho;
    float *phi = potential ? potential : ctx->phi;
    if (ctx->p.demag) {
        MMS_TRY(launch_divergence_aos(ctx, M, rho));
        MMS_TRY(launch_potential(ctx, rho, phi));
    }
    MMS_TRY(launch_hfield_aos(ctx, M, phi, t, H));
    if (!potential) ctx->phi_valid = false;  // ctx->phi no longer holds the state's potential
    return MMS_OK;
}

int mms_potential_host(mms_ctx *ctx, const float *rho, float *phi)
{
    if (!ctx || !rho || !phi) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    const size_t bytes = (size_t)ctx->N * sizeof(float);
    MMS_CUDA_TRY(cudaMemcpyAsync(ctx->vecA, rho, bytes, cudaMemcpyHostToDevice, ctx->stream));
    MMS_TRY(launch_potential(ctx, ctx->vecA, ctx->vecB));
    MMS_CUDA_TRY(cudaMemcpyAsync(phi, ctx->vecB, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return MMS_OK;
}

int mms_hfield_host(mms_ctx *ctx, const float *M, float *H, float *charge, float *potential, double t)
{
    if (!ctx || !M || !H) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    const size_t n = (size_t)ctx->N;
    MMS_CUDA_TRY(cudaMemcpyAsync(ctx->vecA, M, 3 * n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->p.demag) {
        MMS_TRY(launch_divergence_aos(ctx, ctx->vecA, ctx->rho));
        MMS_TRY(launch_potential(ctx, ctx->rho, ctx->phi));
    }
    MMS_TRY(launch_hfield_aos(ctx, ctx->vecA, ctx->phi, t, ctx->vecB));
    ctx->phi_valid = false;
    MMS_CUDA_TRY(cudaMemcpyAsync(H, ctx->vecB, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (charge)
        MMS_CUDA_TRY(cudaMemcpyAsync(charge, ctx->rho, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (potential)
        MMS_CUDA_TRY(cudaMemcpyAsync(potential, ctx->phi, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return MMS_OK;
}

// ---- resident state ------------------------------------------------------------

int mms_state_set_dev(mms_ctx *ctx, const uint8_t *material, const double *M, double t)
{
    MmsRange nvtx_("mms/state_set_dev");
    if (!ctx || !material || !M) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    k_state_in<double><<<div_up(ctx->N, 256), 256, 0, ctx->stream>>>(M, material, ctx->mat, ctx->M, ctx->N,
                                                                     ctx->tstate, ctx->stats, t);
    MMS_LAUNCH_CHECK(ctx);
    ctx->dt_known = false;
    ctx->state_ready = true;
    ctx->phi_valid = false;
    return MMS_OK;
}

int mms_state_set(mms_ctx *ctx, const uint8_t *material, const double *M, double t)
{
    if (!ctx || !material || !M) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    const size_t n = (size_t)ctx->N;
    MMS_CUDA_TRY(cudaMemcpyAsync(ctx->mat, material, n, cudaMemcpyHostToDevice, ctx->stream));
    MMS_CUDA_TRY(cudaMemcpyAsync(ctx->K, M, 3 * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    k_state_in<double><<<div_up(ctx->N, 256), 256, 0, ctx->stream>>>(ctx->K, ctx->mat, ctx->mat, ctx->M, ctx->N,
                                                                     ctx->tstate, ctx->stats, t);
    MMS_LAUNCH_CHECK(ctx);
    ctx->dt_known = false;
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->state_ready = true;
    ctx->phi_valid = false;
    return MMS_OK;
}

int mms_state_get_dev(mms_ctx *ctx, double *M)
{
    MmsRange nvtx_("mms/state_get_dev");
    MMS_TRY(require_state(ctx));
    if (!M) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    k_soa_to_aos<<<div_up(ctx->N, 256), 256, 0, ctx->stream>>>(ctx->M, M, ctx->N);
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

int mms_state_get(mms_ctx *ctx, double *M, double *t)
{
    MMS_TRY(require_state(ctx));
    if (M) {
        k_soa_to_aos<<<div_up(ctx->N, 256), 256, 0, ctx->stream>>>(ctx->M, ctx->K, ctx->N);
        MMS_LAUNCH_CHECK(ctx);
        MMS_CUDA_TRY(cudaMemcpyAsync(M, ctx->K, 3 * (size_t)ctx->N * sizeof(double), cudaMemcpyDeviceToHost,
                                     ctx->stream));
    }
    double ts[TIME_SLOTS];
    MMS_TRY(read_time(ctx, ts));
    if (t) *t = ts[TIME_T];
    double st[STAT_SLOTS];
    MMS_TRY(read_stats(ctx, st));
    if (st[7] != 0.0) {
        mms_set_error("non-finite magnetisation produced by a step");
        return MMS_ERR_NUMERIC;
    }
    return MMS_OK;
}

// ---- resident state in the reference's FP32 Vector3 layout ---------------------

int mms_state_set_f32_dev(mms_ctx *ctx, const uint8_t *material, const float *M, double t)
{
    MmsRange nvtx_("mms/state_set_f32_dev");
    if (!ctx || !material || !M) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    k_state_in<float><<<div_up(ctx->N, 256), 256, 0, ctx->stream>>>(M, material, ctx->mat, ctx->M, ctx->N,
                                                                    ctx->tstate, ctx->stats, t);
    MMS_LAUNCH_CHECK(ctx);
    ctx->dt_known = false;
    ctx->state_ready = true;
    ctx->phi_valid = false;
    return MMS_OK;
}

int mms_state_get_f32_dev(mms_ctx *ctx, float *M)
{
    MmsRange nvtx_("mms/state_get_f32_dev");
    MMS_TRY(require_state(ctx));
    if (!M) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    k_soa_to_aos32<<<div_up(ctx->N, 256), 256, 0, ctx->stream>>>(ctx->M, M, ctx->N);
    MMS_LAUNCH_CHECK(ctx);
    return MMS_OK;
}

// host FP32 I/O stages through the slope buffer K (3 N doubles, free between
// steps): the floats travel as floats, half the bytes of the FP64 path
int mms_state_set_f32(mms_ctx *ctx, const uint8_t *material, const float *M, double t)
{
    if (!ctx || !material || !M) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    const size_t n = (size_t)ctx->N;
    float *stage = reinterpret_cast<float *>(ctx->K);
    MMS_CUDA_TRY(cudaMemcpyAsync(ctx->mat, material, n, cudaMemcpyHostToDevice, ctx->stream));
    MMS_CUDA_TRY(cudaMemcpyAsync(stage, M, 3 * n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    k_state_in<float><<<div_up(ctx->N, 256), 256, 0, ctx->stream>>>(stage, ctx->mat, ctx->mat, ctx->M, ctx->N,
                                                                    ctx->tstate, ctx->stats, t);
    MMS_LAUNCH_CHECK(ctx);
    ctx->dt_known = false;
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->state_ready = true;
    ctx->phi_valid = false;
    return MMS_OK;
}

int mms_state_get_f32(mms_ctx *ctx, float *M, double *t)
{
    MMS_TRY(require_state(ctx));
    if (M) {
        float *stage = reinterpret_cast<float *>(ctx->K);
        k_soa_to_aos32<<<div_up(ctx->N, 256), 256, 0, ctx->stream>>>(ctx->M, stage, ctx->N);
        MMS_LAUNCH_CHECK(ctx);
        MMS_CUDA_TRY(cudaMemcpyAsync(M, stage, 3 * (size_t)ctx->N * sizeof(float), cudaMemcpyDeviceToHost,
                                     ctx->stream));
    }
    double ts[TIME_SLOTS];
    MMS_TRY(read_time(ctx, ts));
    if (t) *t = ts[TIME_T];
    double st[STAT_SLOTS];
    MMS_TRY(read_stats(ctx, st));
    if (st[7] != 0.0) {
        mms_set_error("non-finite magnetisation produced by a step");
        return MMS_ERR_NUMERIC;
    }
    return MMS_OK;
}

int mms_run_fixed(mms_ctx *ctx, double dt, int nsteps, int use_graph)
{
    MmsRange nvtx_("mms/run_fixed");
    MMS_TRY(require_state(ctx));
    if (nsteps < 0 || !(dt > 0) || !isfinite(dt)) {
        mms_set_error("dt must be positive and nsteps >= 0");
        return MMS_ERR_ARG;
    }
    // the device keeps dt between calls: a caller stepping with one dt
    // launches the step graph alone
    if (!ctx->dt_known || ctx->dt_dev != dt) {
        k_set_dt<<<1, 1, 0, ctx->stream>>>(ctx->tstate, dt);
        MMS_LAUNCH_CHECK(ctx);
        ctx->dt_known = true;
        ctx->dt_dev = dt;
    }
    int left = nsteps;
    while (left > 0 && surrogate_armed(ctx)) {
        const int chunk = (int)std::min<long long>(left, ctx->sur_every - ctx->sur_since);
        MMS_TRY(run_steps(ctx, chunk, use_graph));
        left -= chunk;
        ctx->sur_since += chunk;
        if (ctx->sur_since >= ctx->sur_every) MMS_TRY(surrogate_check_now(ctx, nullptr));
    }
    return (left > 0 || nsteps == 0) ? run_steps(ctx, left, use_graph) : MMS_OK;
}

int mms_state_stats(mms_ctx *ctx, double *E_eV, double *torque, double Mavg[3], double *Mmag_avg)
{
    MMS_TRY(require_state(ctx));
    MMS_TRY(ensure_phi(ctx));
    MMS_TRY(launch_stats(ctx));
    double st[STAT_SLOTS];
    MMS_TRY(read_stats(ctx, st));
    const double dV = ctx->g.dx * ctx->g.dy * ctx->g.dz;
    const double Ms = ctx->p.Ms, cnt = st[6] > 0 ? st[6] : 1.0;
    if (E_eV) *E_eV = st[0] * (-0.5 * ctx->p.mu0 * dV / 1.6e-19);
    if (torque) *torque = st[1] / Ms / Ms;
    if (Mavg)
        for (int c = 0; c < 3; c++) Mavg[c] = st[2 + c] / cnt / Ms;
    if (Mmag_avg) *Mmag_avg = st[5] / cnt / Ms;
    if (st[7] != 0.0) {
        mms_set_error("non-finite magnetisation produced by a step");
        return MMS_ERR_NUMERIC;
    }
    return MMS_OK;
}

// ---- adaptive marching --------------------------------------------------------

int mms_march(mms_ctx *ctx, const mms_controller *ctl, double finaltime, double dt0, mms_record *records,
              int max_records, int *n_records, mms_march_cb cb, void *user)
{
    MmsRange nvtx_("mms/march");
    MMS_TRY(require_state(ctx));
    if (!ctl || !(dt0 > 0)) {
        mms_set_error("controller NULL or dt0 <= 0");
        return MMS_ERR_ARG;
    }
    if (n_records) *n_records = 0;
    const double Ms = ctx->p.Ms, dV = ctx->g.dx * ctx->g.dy * ctx->g.dz;
    const double Ecoef = -0.5 * ctx->p.mu0 * dV / 1.6e-19;
    const size_t n3 = 3 * (size_t)ctx->N;
    double ts[TIME_SLOTS];
    MMS_TRY(read_time(ctx, ts));
    double t = ts[TIME_T];
    double dt = dt0;
    int tindex = 0, nrec = 0, rejects = 0;
    const int max_rejects = ctl->max_rejects > 0 ? ctl->max_rejects : 50;
    MMS_TRY(ensure_phi(ctx));
    MMS_TRY(launch_stats(ctx));
    double st[STAT_SLOTS];
    MMS_TRY(read_stats(ctx, st));
    double E = st[0] * Ecoef;

    auto backup = [&]() -> int {
        MMS_CUDA_TRY(cudaMemcpyAsync(ctx->Mbak, ctx->M, n3 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        MMS_CUDA_TRY(cudaMemcpyAsync(ctx->phibak, ctx->phi, (size_t)ctx->N * sizeof(float), cudaMemcpyDeviceToDevice,
                                     ctx->stream));
        return MMS_OK;
    };
    auto restore = [&](double t_, double tk1_) -> int {
        MMS_CUDA_TRY(cudaMemcpyAsync(ctx->M, ctx->Mbak, n3 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        MMS_CUDA_TRY(cudaMemcpyAsync(ctx->phi, ctx->phibak, (size_t)ctx->N * sizeof(float), cudaMemcpyDeviceToDevice,
                                     ctx->stream));
        k_set_time<<<1, 1, 0, ctx->stream>>>(ctx->tstate, t_, tk1_, 0.0);
        MMS_LAUNCH_CHECK(ctx);
        ctx->dt_known = false;
        ctx->phi_valid = true;
        return MMS_OK;
    };
    auto make_record = [&](double dtlog, double E2, double torque) {
        mms_record r;
        r.tindex = tindex;
        r.t = t;
        r.dt = dtlog;
        r.E_eV = E2;
        const double cnt = st[6] > 0 ? st[6] : 1.0;
        r.Mx = st[2] / cnt / Ms;
        r.My = st[3] / cnt / Ms;
        r.Mz = st[4] / cnt / Ms;
        r.Mmag = st[5] / cnt / Ms;
        r.torque = torque;
        return r;
    };
    // returns non-zero when the callback asks to stop
    auto record = [&](double dtlog, double E2, double torque) -> int {
        const mms_record r = make_record(dtlog, E2, torque);
        if (records && nrec < max_records) records[nrec] = r;
        nrec++;
        return cb ? cb(user, 0, &r) : 0;
    };
    auto report_reject = [&](double dtnew, double E2, double torque) -> int {
        if (!cb) return 0;
        const mms_record r = make_record(dtnew, E2, torque);
        return cb(user, 1, &r);
    };

    int status = MMS_OK;
    if (ctl->mode == 0) {
        // the reference's controller: ode_functions.cpp:226-341
        while (t <= finaltime) {
            MMS_TRY(read_time(ctx, ts));
            const double tk1 = ts[TIME_TK1];
            MMS_TRY(backup());
            k_set_dt<<<1, 1, 0, ctx->stream>>>(ctx->tstate, dt);
            MMS_LAUNCH_CHECK(ctx);
            ctx->dt_known = false;
            MMS_TRY(run_steps(ctx, 1, 0));
            MMS_TRY(launch_stats(ctx));
            MMS_TRY(read_stats(ctx, st));
            if (st[7] != 0.0) {
                mms_set_error("non-finite magnetisation at t = %g", t);
                return MMS_ERR_NUMERIC;
            }
            const double E2 = st[0] * Ecoef;
            const double torque = st[1] / Ms / Ms;
            if (E2 - E > 0.1) {  // reject: energy rose by more than 0.1 eV
                MMS_TRY(restore(t, tk1));
                if (surrogate_armed(ctx)) MMS_TRY(surrogate_check_now(ctx, nullptr));
                dt = dt / 2.5;
                if (report_reject(dt, E2, torque)) break;
                if (++rejects > max_rejects) {
                    status = MMS_ERR_REJECTED;
                    mms_set_error("step controller: %d consecutive rejections", rejects);
                    break;
                }
                continue;
            }
            rejects = 0;
            if (surrogate_armed(ctx) && ++ctx->sur_since >= ctx->sur_every) MMS_TRY(surrogate_check_now(ctx, nullptr));
            t = t + dt;                   // the step just taken
            dt = 1e-14 / torque / 2;      // ode_functions.cpp:298-299
            tindex++;
            E = E2;
            if (record(dt, E2, torque)) break;
            if (torque < (ctl->torque_stop > 0 ? ctl->torque_stop : 1e-3)) break;
        }
    } else {
        // RK4 step doubling: one full step vs two half steps, FP64 error
        // max_i |M_full - M_half|_inf / Ms; accept the two half steps
        const double rtol = ctl->rtol > 0 ? ctl->rtol : 1e-5;
        const double dtmin = ctl->dt_min > 0 ? ctl->dt_min : 0.0;
        const double dtmax = ctl->dt_max > 0 ? ctl->dt_max : 1e-11;
        double *errbuf = ctx->stats;  // slot 0 reused; stats recomputed before each record
        while (t < finaltime) {
            double h = std::min(dt, finaltime - t);
            if (h <= 0) break;
            MMS_TRY(read_time(ctx, ts));
            const double tk1 = ts[TIME_TK1];
            MMS_TRY(backup());
            k_set_dt<<<1, 1, 0, ctx->stream>>>(ctx->tstate, h);
            MMS_LAUNCH_CHECK(ctx);
            ctx->dt_known = false;
            MMS_TRY(run_steps(ctx, 1, 0));
            MMS_CUDA_TRY(cudaMemcpyAsync(ctx->Mfull, ctx->M, n3 * sizeof(double), cudaMemcpyDeviceToDevice,
                                         ctx->stream));
            MMS_TRY(restore(t, tk1));
            k_set_dt<<<1, 1, 0, ctx->stream>>>(ctx->tstate, 0.5 * h);
            MMS_LAUNCH_CHECK(ctx);
            ctx->dt_known = false;
            MMS_TRY(run_steps(ctx, 2, 0));
            const unsigned nb = div_up(ctx->N, 256);
            k_maxdiff_part<<<nb, 256, 0, ctx->stream>>>(ctx->Mfull, ctx->M, ctx->mat, ctx->stat_part, ctx->N);
            MMS_LAUNCH_CHECK(ctx);
            k_maxdiff_final<<<1, 32, 0, ctx->stream>>>(ctx->stat_part, (int)nb, errbuf);
            MMS_LAUNCH_CHECK(ctx);
            MMS_TRY(read_stats(ctx, st));
            const double err = st[0] / Ms;
            const double fac = (err > 0) ? 0.9 * pow(rtol / err, 0.2) : 5.0;
            double hnew = h * std::min(5.0, std::max(0.2, fac));
            hnew = std::min(hnew, dtmax);
            if (dtmin > 0) hnew = std::max(hnew, dtmin);
            if (!(err <= rtol) && !(dtmin > 0 && h <= dtmin)) {
                MMS_TRY(restore(t, tk1));
                if (surrogate_armed(ctx)) MMS_TRY(surrogate_check_now(ctx, nullptr));
                dt = hnew;
                if (report_reject(dt, 0.0, 0.0)) break;
                if (++rejects > max_rejects) {
                    status = MMS_ERR_REJECTED;
                    mms_set_error("step controller: %d consecutive rejections", rejects);
                    break;
                }
                continue;
            }
            rejects = 0;
            if (surrogate_armed(ctx) && ++ctx->sur_since >= ctx->sur_every) MMS_TRY(surrogate_check_now(ctx, nullptr));
            t += h;
            tindex++;
            dt = hnew;
            MMS_TRY(launch_stats(ctx));
            MMS_TRY(read_stats(ctx, st));
            if (st[7] != 0.0) {
                mms_set_error("non-finite magnetisation at t = %g", t);
                return MMS_ERR_NUMERIC;
            }
            const double torque = st[1] / Ms / Ms;
            if (record(h, st[0] * Ecoef, torque)) break;
            if (ctl->torque_stop > 0 && torque < ctl->torque_stop) break;
        }
    }
    if (n_records) *n_records = nrec;
    return status;
}


// ---- surrogate solver ------------------------------------------------------------

int mms_ctx_set_surrogate(mms_ctx *ctx, const float *w, long long count, int check_every, double tol, int fast)
{
    MmsRange nvtx_("mms/set_surrogate");
    if (!ctx || !w || check_every < 0 || !(tol > 0)) {
        mms_set_error("mms_ctx_set_surrogate: bad argument");
        return MMS_ERR_ARG;
    }
    if (ctx->s.kind != MMS_SOLVER_SURROGATE) {
        mms_set_error("mms_ctx_set_surrogate: the context's solver is not MMS_SOLVER_SURROGATE");
        return MMS_ERR_ARG;
    }
    if (fabs(ctx->g.dy / ctx->g.dx - 1.0) > 1e-9 || fabs(ctx->g.dz / ctx->g.dx - 1.0) > 1e-9) {
        mms_set_error("mms_ctx_set_surrogate: the network is trained for cubic cells");
        return MMS_ERR_ARG;
    }
    if (fast != 0) {
        mms_set_error("mms_ctx_set_surrogate: `fast` is reserved and must be 0");
        return MMS_ERR_ARG;
    }
    MMS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    const size_t before = fmm_plan_bytes(ctx);
    MMS_TRY(farnet_bind(ctx, w, count));
    ctx->dev_bytes += fmm_plan_bytes(ctx) - before;
    ctx->sur_bound = true;
    ctx->sur_every = check_every;
    ctx->sur_tol = tol;
    ctx->sur_active = true;
    ctx->sur_since = ctx->sur_checks = ctx->sur_fallbacks = 0;
    ctx->sur_last_err = ctx->sur_max_err = 0;
    drop_graph(ctx);
    ctx->phi_valid = false;
    return MMS_OK;
}

int mms_surrogate_check(mms_ctx *ctx, double *err)
{
    MMS_TRY(require_state(ctx));
    if (ctx->s.kind != MMS_SOLVER_SURROGATE || !ctx->sur_bound) {
        mms_set_error("mms_surrogate_check: no surrogate bound to this context");
        return MMS_ERR_ARG;
    }
    return surrogate_check_now(ctx, err);
}

int mms_surrogate_stats(const mms_ctx *ctx, int *active, long long *checks, long long *fallbacks, double *last_err,
                        double *max_err)
{
    if (!ctx) {
        mms_set_error("context is NULL");
        return MMS_ERR_ARG;
    }
    if (active) *active = ctx->s.kind == MMS_SOLVER_SURROGATE && ctx->sur_bound && ctx->sur_active;
    if (checks) *checks = ctx->sur_checks;
    if (fallbacks) *fallbacks = ctx->sur_fallbacks;
    if (last_err) *last_err = ctx->sur_last_err;
    if (max_err) *max_err = ctx->sur_max_err;
    return MMS_OK;
}

int mms_potential_split_dev(mms_ctx *ctx, const float *rho, float *phi, float *near)
{
    if (!ctx || !rho || !phi || !near) {
        mms_set_error("NULL argument");
        return MMS_ERR_ARG;
    }
    if (ctx->s.kind != MMS_SOLVER_FMM && ctx->s.kind != MMS_SOLVER_SURROGATE) {
        mms_set_error("mms_potential_split_dev: needs an FMM plan");
        return MMS_ERR_ARG;
    }
    return launch_potential_split(ctx, rho, phi, near);
}

}  // extern "C"
