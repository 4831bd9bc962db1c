/*
 * mms_b200 — B200-native (sm_100a) demag / LLG hot path of mms-gpu.
 *
 * Plain C ABI: plain pointers and sizes, no C++ or torch types.  A context
 * owns everything sized by the grid (device buffers, the FMM plan, the kernel
 * table of the direct sum, CUDA graphs); the caller owns its input/output
 * arrays.  Every entry point returns an mms_status; on failure
 * mms_last_error() gives a message (thread-local).  Nothing here calls exit().
 *
 * Conventions shared with the reference (akhan3/mms-gpu):
 *   cell index i = z*ydim*xdim + y*xdim + x          (vector_functions.cpp:20-26)
 *   vector fields at the boundary are FP32 AoS {x,y,z} triples (Vector3.hpp:10-12)
 *   potential phi_i = sum_{j != i} rho_j dV / |r_i - r_j|, WITHOUT 1/(4 pi)
 *                                                   (fmm_calc.cu:412-461)
 *   H_demag = (1/(4 pi)) * central-difference grad(phi) (ode_functions.cpp:51)
 *
 * Entry points and the reference interface each one replaces:
 *   mms_potential_dev / mms_potential_host
 *        <- calc_potential_exact   helper_functions.hpp:31-35 (solver DIRECT)
 *        <- calc_potential_exact_gpu helper_functions.hpp:37-40
 *        <- fmm_calc               helper_functions.hpp:24-29 (solver FMM)
 *   mms_hfield_dev / mms_hfield_host
 *        <- Hfield                 ode_functions.hpp:8-15
 *   mms_divergence_dev, mms_gradient_dev, mms_exchange_dev
 *        <- divergence_3d / gradient_3d / add_exchange_field
 *                                  vector_functions.hpp:9-25
 *   mms_state_*, mms_rk4_step, mms_run_fixed
 *        <- rk4_step               ode_functions.cpp:76-87 (no header upstream)
 *   mms_march                      <- time_marching ode_functions.hpp:17-24
 * The C++ shim with the reference's exact signatures is include/mms_ref_api.hpp.
 */
#ifndef MMS_B200_H
#define MMS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MMS_ABI_VERSION 1

typedef enum {
    MMS_OK = 0,
    MMS_ERR_ARG = 1,         /* bad argument / unsupported size               */
    MMS_ERR_CUDA = 2,        /* a CUDA runtime call failed                    */
    MMS_ERR_NOMEM = 3,       /* device or host allocation failed              */
    MMS_ERR_NUMERIC = 4,     /* NaN/Inf detected in a field or the state      */
    MMS_ERR_NOT_READY = 5,   /* state not initialised                         */
    MMS_ERR_REJECTED = 6     /* step controller gave up (too many rejections) */
} mms_status;

typedef enum {
    MMS_SOLVER_DIRECT = 0,   /* exact O(N^2) sum, FP32 tiles, compensated      */
    MMS_SOLVER_FMM = 1,      /* spherical-harmonic FMM, exact near field       */
    MMS_SOLVER_SURROGATE = 2 /* exact near field (FMM P2P, leaf 8) + far field
                                from the learned operator (mms_farnet_*); the
                                FMM of the solver's order checks it and takes
                                over (mms_ctx_set_surrogate)                  */
} mms_solver_kind;

typedef struct {
    int xdim, ydim, zdim;    /* cells                                          */
    double dx, dy, dz;       /* cell size (m)                                  */
} mms_grid;

typedef struct {
    double Ms;               /* saturation magnetisation (A/m)                 */
    double Aexch;            /* exchange constant (J/m)                        */
    double alpha;            /* damping                                        */
    double gamma;            /* gyromagnetic ratio (m/(A s))                   */
    double mu0;              /* vacuum permeability                            */
    int demag, exchange, external;
    /* external B(t) (tesla) as a clamped piecewise-linear table; H_ext = B/mu0.
     * n_hext == 0 with external != 0 selects the reference's built-in ramp
     * B_x = 0.3 T -> 0 over 1 ns (ode_functions.cpp:61).  Copied at set time. */
    int n_hext;
    const double *hext_t;    /* n_hext times (s), increasing                  */
    const double *hext_b;    /* n_hext x 3 (T)                                */
    /* 1: all RK4 stages evaluate H_ext at the step start t and the post-step
     * field at the old t, as the reference does (ode_functions.cpp:109-133,
     * :267); 0: stage times t + c_s dt. */
    int ref_stage_time;
} mms_params;

typedef struct {
    int kind;                /* mms_solver_kind                                */
    int fmm_order;           /* expansion order P (FMM), 1..9                  */
    int fmm_leaf;            /* leaf box side in cells (FMM), 2..16, or 0=auto */
    int m2l_mode;            /* FMM M2L: 0 auto, 1 FP32 SIMT, 2 tensor cores
                                (tcgen05, split-BF16 hi/lo products)          */
    int far_mode;            /* FMM far field: 0 one launch per stage and
                                level (default, fastest measured), 1 P2M ..
                                L2L in one cooperative launch with grid
                                barriers (P <= 4, FP32 M2L); identical bits   */
    int near_mode;           /* FMM near field: 0 auto (tensor cores at leaf
                                side 8 and Z <= 4, else FP32), 1 FP32 SIMT,
                                2 tensor cores (tcgen05 + TMA, split-BF16
                                hi/lo products; leaf side 8, Z <= 4 only)     */
    int reserved[2];
} mms_solver;

typedef struct mms_ctx mms_ctx;

/* library / context ---------------------------------------------------------- */
int mms_abi_version(void);
const char *mms_last_error(void);
/* Creates a context on the CURRENT CUDA device.  Allocates every device buffer
 * the grid needs; no later call allocates device memory (except mms_march's
 * host logs).  stream: a cudaStream_t (as void*), or NULL for a private
 * blocking stream (ordered with the legacy default stream). */
int mms_ctx_create(const mms_grid *grid, const mms_params *params, const mms_solver *solver,
                   void *stream, mms_ctx **out);
int mms_ctx_destroy(mms_ctx *ctx);
int mms_ctx_set_params(mms_ctx *ctx, const mms_params *params);
int mms_ctx_set_solver(mms_ctx *ctx, const mms_solver *solver);
/* Waits for the context's stream; MMS_ERR_CUDA when a kernel's bounded wait
 * gave up since the solver was set (fused far-field grid barrier, or the
 * tensor-core near field / M2L pipeline): its results are then not valid. */
int mms_ctx_sync(mms_ctx *ctx);
/* number of kernels this library launched through ctx so far */
int64_t mms_ctx_kernel_launches(const mms_ctx *ctx);
/* device bytes held by ctx */
size_t mms_ctx_device_bytes(const mms_ctx *ctx);

/* stateless field operators (device pointers, asynchronous on ctx's stream) - */
/* rho = div M (vector_functions.cpp:8-28).  M: N x 3 FP32 AoS, rho: N FP32 */
int mms_divergence_dev(mms_ctx *ctx, const float *M, float *rho);
/* phi from rho with ctx's solver (fmm_calc.cu:295-461). N FP32 each */
int mms_potential_dev(mms_ctx *ctx, const float *rho, float *phi);
/* H = c * grad(phi) (vector_functions.cpp:31-54).  H: N x 3 FP32 AoS, overwritten */
int mms_gradient_dev(mms_ctx *ctx, const float *phi, double c, float *H);
/* H += exchange field of M (vector_functions.cpp:57-103) */
int mms_exchange_dev(mms_ctx *ctx, const float *M, float *H);
/* full effective field at time t (ode_functions.cpp:21-70).  charge/potential
 * may be NULL (then ctx scratch is used) or N-float device outputs. */
int mms_hfield_dev(mms_ctx *ctx, const float *M, float *H, float *charge, float *potential, double t);

/* same, HOST pointers: copies in, computes, copies out, synchronises */
int mms_potential_host(mms_ctx *ctx, const float *rho, float *phi);
int mms_hfield_host(mms_ctx *ctx, const float *M, float *H, float *charge, float *potential, double t);

/* resident FP64 state and RK4 (ode_functions.cpp:76-148) ---------------------- */
/* material: N bytes (non-zero = magnetic), M: N x 3 FP64 AoS; host pointers.
 * M is taken as zero at empty cells. */
int mms_state_set(mms_ctx *ctx, const uint8_t *material, const double *M, double t);
int mms_state_get(mms_ctx *ctx, double *M, double *t);
/* same with device pointers (material u8, M FP64 AoS) */
int mms_state_set_dev(mms_ctx *ctx, const uint8_t *material, const double *M, double t);
int mms_state_get_dev(mms_ctx *ctx, double *M);
/* the state in the reference's own layout: M as N Vector3 of FP32
 * (fptype = float, Vector3.h), the M and M2 arguments of rk4_step
 * (ode_functions.cpp:76).  Set widens to the FP64 state exactly; get rounds
 * each component to nearest.  The copies move half the bytes of the FP64
 * calls; the state between steps stays FP64 on the device.  Host pointers,
 * synchronous, like mms_state_set / mms_state_get: */
int mms_state_set_f32(mms_ctx *ctx, const uint8_t *material, const float *M, double t);
int mms_state_get_f32(mms_ctx *ctx, float *M, double *t);
/* and with device pointers, asynchronous on the context's stream: */
int mms_state_set_f32_dev(mms_ctx *ctx, const uint8_t *material, const float *M, double t);
int mms_state_get_f32_dev(mms_ctx *ctx, float *M);
/* nsteps classical RK4 steps of size dt, 4 field evaluations per step.  With
 * use_graph != 0 one step is captured once as a CUDA graph and replayed. */
int mms_run_fixed(mms_ctx *ctx, double dt, int nsteps, int use_graph);
/* energy (eV) and max |M x H|/Ms^2 of the current state, as time_marching logs
 * them (ode_functions.cpp:234-240, :268-278); also <M>/Ms and <|M|>/Ms */
int mms_state_stats(mms_ctx *ctx, double *E_eV, double *torque, double Mavg[3], double *Mmag_avg);

/* adaptive RK4 --------------------------------------------------------------- */
typedef struct {
    int mode;                /* 0: reference energy/torque controller
                                   (ode_functions.cpp:226-341);
                                1: RK4 step doubling, FP64 error estimate, rtol */
    double rtol;             /* mode 1: max |M_full - M_half2| / Ms per step  */
    double dt_min, dt_max;   /* mode 1 clamps (s)                             */
    double torque_stop;      /* stop when max torque < this (reference 1e-3)  */
    int max_rejects;         /* consecutive rejections before giving up (50)  */
    int reserved[3];
} mms_controller;

typedef struct {             /* one record per accepted step, the 9 columns of
                                dynamics.dat (ode_functions.cpp:330-333)       */
    int tindex;
    double t, dt, E_eV, Mx, My, Mz, Mmag, torque;
} mms_record;

/* Called after every accepted step (rejected = 0) and every rejected attempt
 * (rejected = 1; rec->dt is then the reduced step).  The state may be read
 * with mms_state_get inside the callback.  A non-zero return stops marching. */
typedef int (*mms_march_cb)(void *user, int rejected, const mms_record *rec);

/* March until t > finaltime, the torque stop, or controller failure.
 * records: caller array of max_records (may be NULL); *n_records receives the
 * number of accepted steps.  cb may be NULL.  Returns MMS_ERR_REJECTED after
 * max_rejects consecutive rejections. */
int mms_march(mms_ctx *ctx, const mms_controller *ctl, double finaltime, double dt0,
              mms_record *records, int max_records, int *n_records, mms_march_cb cb, void *user);

/* FMM plan of a context: tree levels L (leaf level), leaf side, order P, the
 * algorithmic flops of one potential evaluation per stage (P2M, M2M, M2L, L2L,
 * L2P+P2P; 2 per multiply-add on the parity blocks, 2 per near-field pair) and
 * the P2P pair and M2L box-pair counts.  MMS_ERR_ARG if the solver is not FMM. */
int mms_fmm_info(const mms_ctx *ctx, int *levels, int *leaf, int *order, double stage_flops[5],
                 long long *p2p_pairs, long long *m2l_pairs);

/* Which kernels the FMM plan runs: near_tc 1 when the near field is the
 * tensor-core GEMM (k_p2p_tc), m2l_tc 1 when the M2L is (k_m2l_gemm); 0 for
 * the FP32 kernels.  Either pointer may be NULL.  No counterpart in the
 * reference (its FMM has one kernel per stage). */
int mms_fmm_kernels(const mms_ctx *ctx, int *near_tc, int *m2l_tc);

/* Per-stage device time of the FMM potential (ms per stage, all its levels):
 * [0] P2M, [1] M2M, [2] M2L, [3] L2L, [4] L2P + P2P.  After one full
 * evaluation each stage is re-launched `reps` times back to back between two
 * CUDA events on ctx's stream (stages are idempotent on unchanged inputs);
 * rho/phi are device arrays and phi ends up holding the potential of rho. */
int mms_fmm_stage_times(mms_ctx *ctx, const float *rho, float *phi, int reps, double ms[5]);

/* batched ensemble ----------------------------------------------------------- */
/* Many independent simulations of uneven grid size (same cell size and
 * material) advance together: one kernel launch per RK4 stage for the whole
 * ensemble, driven by an instance offset table; exact direct-sum demag per
 * instance; one CUDA graph per step.  Each instance has its own constant
 * external field bext (T), applied when params->external != 0.  No reference
 * counterpart (the reference runs one simulation per process). */
typedef struct {
    int xdim, ydim, zdim;    /* 1 <= xdim <= 256                               */
    double bext[3];          /* constant external field (T)                    */
} mms_ens_instance;

typedef struct mms_ens mms_ens;

int mms_ens_create(const mms_ens_instance *inst, int n, double dx, double dy, double dz,
                   const mms_params *params, void *stream, mms_ens **out);
int mms_ens_destroy(mms_ens *ens);
/* total cells (sum over instances) */
long long mms_ens_cells(const mms_ens *ens);
int64_t mms_ens_kernel_launches(const mms_ens *ens);
/* material (u8) and M (FP64 AoS) of all instances concatenated in instance
 * order, each in the cell order z*Y*X + y*X + x; host pointers */
int mms_ens_state_set(mms_ens *ens, const uint8_t *material, const double *M);
int mms_ens_state_get(mms_ens *ens, double *M, double *t);
int mms_ens_run_fixed(mms_ens *ens, double dt, int nsteps, int use_graph);
/* Chooses the batched direct kernel's shape by measurement on the current
 * state's charges: warps per CTA (4, 8, 16) x source rows staged per batch
 * (8, 16, 32), `reps` timed launches each; keeps the fastest (the results do
 * not depend on the shape).  Needs mms_ens_state_set first. */
int mms_ens_autotune(mms_ens *ens, int reps, int *warps, int *rows, double *best_ms);
int mms_ens_sync(mms_ens *ens);

/* allocation-free exact potential -------------------------------------------- */
/* No counterpart in the reference.  The exact direct-sum potential for callers
 * that cannot allocate device memory (a host whose pool allocator owns the
 * device memory, code running during CUDA graph capture, a loop that must not
 * take the allocation lock): no context, and no cudaMalloc/cudaFree or other
 * allocating call.  The scratch table lives in a fixed 4 MiB array inside the
 * library that each GPU which loads the library holds until exit; grids are
 * limited to xdim*ydim*zdim <= 1,048,576 cells and xdim <= 2048 (MMS_ERR_ARG
 * beyond).  rho/phi are device arrays; the work is queued on `stream` (a
 * cudaStream_t, NULL = legacy default stream).  The first call on each device
 * performs a one-time set-up (it looks up the table's device address) with
 * that device current; make that first call before any stream capture.  Every
 * call also raises the sum kernel's shared-memory limit when its row length
 * needs it (a host-side attribute, no allocation).  A CUDA error left pending
 * by earlier work is reported as such (MMS_ERR_CUDA) before anything is queued.
 * All calls share the one table, which keeps the last call's contents: calls
 * that overlap on the GPU (different streams, or different host threads on one
 * device) race and must be serialised by the caller. */
int mms_potential_direct_noalloc(const float *rho, float *phi, int xdim, int ydim, int zdim,
                                 double dx, double dy, double dz, void *stream);

/* autotuner ------------------------------------------------------------------ */
/* Chooses the FMM order P (3..8), leaf side (4, 8) and M2L kernel for a grid by
 * measurement: each candidate evaluates the potential of rho_dev (a device
 * charge density of the grid), its rel-L2 error against the exact direct sum
 * (computed on the same device) must be <= max_rel_err, and the fastest such
 * candidate (mean of `reps` evaluations, CUDA events) is returned in *best.
 * Cached per process by (grid, cell size, target).  No reference
 * counterpart (the reference hard-codes P, main.cpp:31). */
int mms_autotune_fmm(const mms_grid *grid, const mms_params *params, const float *rho_dev, double max_rel_err,
                     int reps, mms_solver *best, double *best_ms, double *best_err);
/* Same search, timed on what a time-stepping caller runs: each candidate
 * within the error target starts from the host state (material, M as
 * mms_state_set takes them) and *best_ms is its mean graph-captured RK4 step
 * of size dt over `reps` steps.  rho_dev is the charge density of that state
 * (the error sample). */
int mms_autotune_fmm_steps(const mms_grid *grid, const mms_params *params, const uint8_t *material,
                           const double *M, double dt, const float *rho_dev, double max_rel_err, int reps,
                           mms_solver *best, double *best_ms, double *best_err);

/* surrogate far field ---------------------------------------------------------
 * A learned far-field operator for thin films of 3 layers on cubic cells: a
 * linear multilevel convolutional network over the quadtree of 8 x 8 x 3 leaf
 * boxes with the FMM's data flow and its own weights per level.  The encoder
 * (replacing P2M) maps a leaf box's 192 cell charges to 24 channels (16 even,
 * 8 odd under z -> -z); 2 x 2 stride-2 convolutions go down the tree (M2M);
 * at every level a parity-aware 7 x 7 convolution over the interaction list
 * (children of the parent's neighbours that are not neighbours, the
 * reference's Box.cu:171-195) couples boxes (M2L); transposed convolutions go
 * back up (L2L) and the decoder (L2P) gives the far field at every cell.  The
 * near field over each leaf box's 3 x 3 neighbourhood stays exact.  Weights:
 * FP32, mms_farnet_num_params() of them, indexed by depth below the leaves, so
 * one vector serves every grid of 2..6 quadtree levels (up to 512 cells a
 * side); they start from nested SVD bases of the 1/r interactions and are
 * trained on FMM-generated (charge, far field) pairs by the kernels below.  It
 * replaces the far-field pass of the reference's fmm_calc (fmm_calc.cu:
 * 186-222); the reference has no learned component.
 *
 * Units: u = rho dx / Ms (dimensionless cell charge) in, phi_far / (Ms dx) out;
 * arrays are [batch][3][ydim][xdim] FP32 on the device.  All calls below run
 * on the legacy default stream and return when their results are ready. */
typedef struct mms_farnet mms_farnet;
long long mms_farnet_num_params(void);
/* a network for batches of up to `batch` samples of an xdim x ydim x 3 grid
 * (17..512 cells a side: 2..6 quadtree levels of 8-cell leaves) */
int mms_farnet_create(int xdim, int ydim, int batch, mms_farnet **out);
void mms_farnet_destroy(mms_farnet *net);
/* host arrays of mms_farnet_num_params() FP32 weights; set also resets Adam */
int mms_farnet_set_weights(mms_farnet *net, const float *w, long long count);
int mms_farnet_get_weights(mms_farnet *net, float *w, long long count);
/* out = far field of u for nbatch <= batch samples */
int mms_farnet_forward_dev(mms_farnet *net, const float *u, float *out, int nbatch);
/* loss = mean_b |net(u_b) - far_b|^2 / nrm2_b (nrm2_b = |phi_b|^2 of the total
 * potential, so the loss is the squared relative error of phi) and its
 * gradient with respect to the weights (host array, may be NULL); u, far:
 * device [nbatch][3][Y][X]; nrm2: device [nbatch] */
int mms_farnet_gradient(mms_farnet *net, const float *u, const float *far, const float *nrm2, int nbatch,
                        float *grad, double *loss);
/* per-weight multipliers of the Adam step (host array of num_params; 1 each
 * at creation): a weight moves by lr * scale_i per unit of normalised
 * gradient, e.g. scale_i ~ |w_i| for relative steps */
int mms_farnet_set_step_scale(mms_farnet *net, const float *scale, long long count);
/* one Adam step on that loss; *loss is the loss before the step */
int mms_farnet_train_step(mms_farnet *net, const float *u, const float *far, const float *nrm2, int nbatch,
                          float lr, float beta1, float beta2, float eps, double *loss);
long long mms_farnet_device_bytes(const mms_farnet *net);

/* number of FP32 weights of the network of `width` channels the solver runs:
 * 24 (16 even + 8 odd: the default, trained by mms_farnet_*) or 40 (24 + 16:
 * the accurate one, 5-10x closer to the exact sum for a ~30 % longer
 * evaluation); 0 for any other width */
long long mms_surrogate_num_params(int width);

/* Binds network weights to a context whose solver is MMS_SOLVER_SURROGATE
 * (leaf side 8, zdim 3, cubic cells); `count` picks the width (see
 * mms_surrogate_num_params).  It arms the network's check: every `check_every`
 * steps (0: never) of mms_run_fixed, and every `check_every` accepted steps
 * plus every rejected step of mms_march, the potential of the current state
 * is computed by both the network and the FMM (the solver's order P, leaf 8);
 * when their rel-L2 difference exceeds `tol` the FMM replaces the network for
 * the rest of the run.  `fast` is reserved and must be 0. */
int mms_ctx_set_surrogate(mms_ctx *ctx, const float *w, long long count, int check_every, double tol, int fast);
/* runs that check now on the current state; *err = rel-L2(surrogate, FMM) */
int mms_surrogate_check(mms_ctx *ctx, double *err);
/* active: 1 while the surrogate is in use, 0 after the FMM took over */
int mms_surrogate_stats(const mms_ctx *ctx, int *active, long long *checks, long long *fallbacks,
                        double *last_err, double *max_err);
/* far-field split of the FMM potential: phi = FMM(rho) and near = its exact
 * near-field part (leaf-box neighbourhood P2P); context solver must be
 * MMS_SOLVER_FMM or MMS_SOLVER_SURROGATE (device arrays of N floats) */
int mms_potential_split_dev(mms_ctx *ctx, const float *rho, float *phi, float *near);

/* diagnostics ---------------------------------------------------------------- */
/* The library's tcgen05 tensor-core GEMM on BF16 operands: C = A B^T (beta 0)
 * or C += A B^T (beta 1); A M x K and B N x K row-major (K contiguous), C
 * M x N FP32 row-major; K, lda, ldb multiples of 8; bn = 64 or 128 (tile N).
 * Device pointers; synchronises `stream`.  No reference counterpart (used to
 * validate the core behind the tensor-core M2L and the network's weight
 * gradients). */
int mms_diag_gemm_bf16(const void *A, int lda, const void *B, int ldb, float *C, int ldc,
                       int M, int N, int K, int beta, int bn, void *stream);
/* FP32 FMA throughput of the current device in TFLOP/s (a microbenchmark of
 * `reps` launches, one wave of 8 CTAs per SM): the roofline denominator of the
 * FP32-pipe-bound kernels (direct sum, near field).  No reference counterpart. */
int mms_diag_fma_tflops(int reps, double *tflops);

#ifdef __cplusplus
}
#endif
#endif
