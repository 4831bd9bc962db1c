// Drop-in shim: the reference's own C++ signatures (include/mms_ref_api.hpp)
// implemented on the mms_b200 C ABI.  Host arrays in, host arrays out; the
// device work runs on the B200 through a per-process context cache keyed by
// grid and solver.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "mms_b200.h"
#include "mms_ref_api.hpp"

// the reference's value type: three packed floats (Vector3.hpp:10-12)
struct Vector3 {
    fptype x, y, z;
};
static_assert(sizeof(Vector3) == 3 * sizeof(float), "Vector3 must be three packed floats");

namespace {

struct CachedCtx {
    mms_ctx *ctx = nullptr;
    mms_grid g{};
    int kind = -1, P = -1;
};

// one cached context per solver kind; the reference keeps equivalent statics
// (fmm_calc.cu:303-365, potential_calc.cu:127-153)
CachedCtx g_cache[2];

mms_params ref_params(fptype mu_0, fptype Ms, fptype Aexch, fptype alfa, fptype gamma, int demag, int exchange,
                      int external)
{
    mms_params p;
    memset(&p, 0, sizeof p);
    p.Ms = Ms;
    p.Aexch = Aexch;
    p.alpha = alfa;
    p.gamma = gamma;
    p.mu0 = mu_0;
    p.demag = demag;
    p.exchange = exchange;
    p.external = external;
    p.n_hext = 0;            // the reference's built-in ramp (ode_functions.cpp:61)
    p.ref_stage_time = 1;    // stage times as the reference evaluates them
    return p;
}

mms_params default_params()
{
    // main.cpp:107-111; only the grid matters for a bare potential call
    return ref_params((fptype)(4 * M_PI * 1e-7), 8.6e5f, 1.3e-11f, 0.5f, 2.21e5f, 1, 1, 0);
}

mms_ctx *get_ctx(int use_fmm, int xdim, int ydim, int zdim, fptype dx, fptype dy, fptype dz, int P,
                 const mms_params &p, int verbosity)
{
    const int kind = use_fmm ? MMS_SOLVER_FMM : MMS_SOLVER_DIRECT;
    CachedCtx &c = g_cache[kind];
    mms_grid g;
    g.xdim = xdim;
    g.ydim = ydim;
    g.zdim = zdim;
    g.dx = dx;
    g.dy = dy;
    g.dz = dz;
    mms_solver s;
    memset(&s, 0, sizeof s);
    s.kind = kind;
    s.fmm_order = P;
    s.fmm_leaf = 0;
    const bool same_grid = c.ctx && c.g.xdim == xdim && c.g.ydim == ydim && c.g.zdim == zdim && c.g.dx == g.dx &&
                           c.g.dy == g.dy && c.g.dz == g.dz;
    if (!same_grid) {
        if (c.ctx) mms_ctx_destroy(c.ctx);
        c.ctx = nullptr;
        if (mms_ctx_create(&g, &p, &s, nullptr, &c.ctx) != MMS_OK) {
            fprintf(stderr, "mms_b200: context creation failed: %s\n", mms_last_error());
            c.ctx = nullptr;
            return nullptr;
        }
        c.g = g;
        c.kind = kind;
        c.P = P;
        if (verbosity >= 15)
            printf("mms_b200: context for %dx%dx%d (%s), %.1f MB on the device\n", xdim, ydim, zdim,
                   use_fmm ? "FMM" : "direct", mms_ctx_device_bytes(c.ctx) / 1048576.0);
        return c.ctx;
    }
    if (kind == MMS_SOLVER_FMM && c.P != P) {
        if (mms_ctx_set_solver(c.ctx, &s) != MMS_OK) {
            fprintf(stderr, "mms_b200: %s\n", mms_last_error());
            return nullptr;
        }
        c.P = P;
    }
    if (mms_ctx_set_params(c.ctx, &p) != MMS_OK) {
        fprintf(stderr, "mms_b200: %s\n", mms_last_error());
        return nullptr;
    }
    return c.ctx;
}

int fail(const char *what)
{
    fprintf(stderr, "mms_b200: %s: %s\n", what, mms_last_error());
    return EXIT_FAILURE;
}

}  // namespace

int fmm_calc(const fptype *charge, fptype *potential, const int xdim, const int ydim, const int zdim,
             const fptype dx, const fptype dy, const fptype dz, const int P, const int use_gpu, const int verbosity)
{
    (void)use_gpu;
    mms_ctx *ctx = get_ctx(1, xdim, ydim, zdim, dx, dy, dz, P, default_params(), verbosity);
    if (!ctx) return EXIT_FAILURE;
    if (mms_potential_host(ctx, charge, potential) != MMS_OK) return fail("fmm_calc");
    return EXIT_SUCCESS;
}

int calc_potential_exact(const fptype *charge, const int xdim, const int ydim, const int zdim, const fptype dx,
                         const fptype dy, const fptype dz, fptype *potential, int use_gpu, const int verbosity)
{
    (void)use_gpu;
    mms_ctx *ctx = get_ctx(0, xdim, ydim, zdim, dx, dy, dz, 0, default_params(), verbosity);
    if (!ctx) return EXIT_FAILURE;
    if (mms_potential_host(ctx, charge, potential) != MMS_OK) return fail("calc_potential_exact");
    return EXIT_SUCCESS;
}

int calc_potential_exact_gpu(const fptype *charge, const int xdim, const int ydim, const int zdim, const fptype dx,
                             const fptype dy, const fptype dz, fptype *potential)
{
    return calc_potential_exact(charge, xdim, ydim, zdim, dx, dy, dz, potential, 1, 0);
}

int Hfield(const Vector3 *M, Vector3 *H, fptype *charge, fptype *potential, const fptype t, const int xdim,
           const int ydim, const int zdim, const fptype dx, const fptype dy, const fptype dz, const int P,
           const fptype mu_0, const fptype Ms, const fptype Aexch, const int demag, const int exchange,
           const int external, const int use_fmm, const int use_gpu, const int verbosity)
{
    (void)use_gpu;
    const mms_params p = ref_params(mu_0, Ms, Aexch, 0.5f, 2.21e5f, demag, exchange, external);
    mms_ctx *ctx = get_ctx(use_fmm, xdim, ydim, zdim, dx, dy, dz, P, p, verbosity);
    if (!ctx) return EXIT_FAILURE;
    if (mms_hfield_host(ctx, &M[0].x, &H[0].x, charge, potential, t) != MMS_OK) return fail("Hfield");
    return EXIT_SUCCESS;
}

int rk4_step(const fptype t, const fptype dt, fptype *t2, const byte *material, const Vector3 *M, Vector3 *M2,
             Vector3 *H, Vector3 *slope, Vector3 *this_slope, fptype *charge, fptype *potential, const int xdim,
             const int ydim, const int zdim, const fptype dx, const fptype dy, const fptype dz, const int P,
             const fptype mu_0, const fptype Ms, const fptype Aexch, const fptype alfa, const fptype gamma,
             const int demag, const int exchange, const int external, const int use_fmm, const int normalize,
             const int use_gpu, const int verbosity)
{
    (void)H; (void)slope; (void)this_slope; (void)charge; (void)potential; (void)use_gpu;
    if (!normalize) {
        fprintf(stderr, "mms_b200: rk4_step without |M| = Ms renormalisation is not provided\n");
        return EXIT_FAILURE;
    }
    const mms_params p = ref_params(mu_0, Ms, Aexch, alfa, gamma, demag, exchange, external);
    mms_ctx *ctx = get_ctx(use_fmm, xdim, ydim, zdim, dx, dy, dz, P, p, verbosity);
    if (!ctx) return EXIT_FAILURE;
    // k1 is evaluated from M at t, which is what the caller's H holds in every
    // reference call site (ode_functions.cpp:230,267).  M and M2 travel in the
    // caller's FP32 Vector3 layout; the step runs on the FP64 state (one
    // captured graph, replayed on every later call).
    if (mms_state_set_f32(ctx, material, &M[0].x, t) != MMS_OK) return fail("rk4_step");
    if (mms_run_fixed(ctx, dt, 1, 1) != MMS_OK) return fail("rk4_step");
    double tt = 0;
    if (mms_state_get_f32(ctx, &M2[0].x, &tt) != MMS_OK) return fail("rk4_step");
    *t2 = t + dt;
    return EXIT_SUCCESS;
}

namespace {

// Mdynamics.dat: one snapshot of M per accepted step in the layout of
// helper_functions.cpp:107-123 (per z, x outer, y inner, "%g %g %g \n").
// Formatting a snapshot of a large grid takes far longer than the GPU step,
// so snapshots are formatted on worker threads (the (z, x) columns split into
// chunks that are written in order) by a writer thread while marching goes
// on.  At most kDepth snapshots wait; the caller then blocks until one is
// written, so every snapshot is written, in order, and memory stays bounded.
class SnapshotWriter {
public:
    static constexpr int kDepth = 3;

    SnapshotWriter(FILE *fh, int zdim, int ydim, int xdim) : fh_(fh), Z_(zdim), Y_(ydim), X_(xdim)
    {
        const unsigned hc = std::thread::hardware_concurrency();
        nthreads_ = (int)std::max(1u, std::min(8u, hc ? hc : 1u));
        bufs_.resize(kDepth);
        for (auto &b : bufs_) {
            b.resize(3 * (size_t)zdim * ydim * xdim);
            free_.push_back(b.data());
        }
        th_ = std::thread([this] { run(); });
    }
    ~SnapshotWriter() { finish(); }

    // a buffer of 3 N floats to fill (blocks while every buffer waits)
    float *acquire()
    {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return !free_.empty(); });
        float *b = free_.front();
        free_.pop_front();
        return b;
    }
    // queue a filled buffer; release an unfilled one
    void submit(float *b)
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            queue_.push_back(b);
        }
        cv_.notify_all();
    }
    void release(float *b)
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            free_.push_back(b);
        }
        cv_.notify_all();
    }
    // write everything queued and stop; false if a write failed
    bool finish()
    {
        if (th_.joinable()) {
            {
                std::lock_guard<std::mutex> lk(mu_);
                stop_ = true;
            }
            cv_.notify_all();
            th_.join();
        }
        return ok_;
    }

private:
    void run()
    {
        for (;;) {
            float *b;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this] { return stop_ || !queue_.empty(); });
                if (queue_.empty()) return;  // stop_ and nothing left
                b = queue_.front();
                queue_.pop_front();
            }
            write(b);
            release(b);
        }
    }

    void format(const float *m, long long o0, long long o1, std::string &out) const
    {
        char line[96];
        for (long long o = o0; o < o1; o++) {
            const int z = (int)(o / X_), x = (int)(o % X_);
            for (int y = 0; y < Y_; y++) {
                const size_t i = (size_t)z * Y_ * X_ + (size_t)y * X_ + x;
                const int n = snprintf(line, sizeof line, "%g %g %g \n", m[3 * i], m[3 * i + 1], m[3 * i + 2]);
                out.append(line, (size_t)n);
            }
        }
    }

    void write(const float *m)
    {
        const long long cols = (long long)Z_ * X_;
        const int T = (int)std::min<long long>(nthreads_, std::max<long long>(1, cols));
        std::vector<std::string> parts(T);
        std::vector<std::thread> workers;
        for (int k = 1; k < T; k++)
            workers.emplace_back([this, m, cols, T, k, &parts] { format(m, cols * k / T, cols * (k + 1) / T, parts[k]); });
        format(m, 0, cols / T, parts[0]);
        for (auto &w : workers) w.join();
        for (const auto &p : parts)
            if (!p.empty() && fwrite(p.data(), 1, p.size(), fh_) != p.size()) ok_ = false;
    }

    FILE *fh_;
    int Z_, Y_, X_;
    int nthreads_ = 1;
    std::vector<std::vector<float>> bufs_;
    std::deque<float *> free_, queue_;
    std::mutex mu_;
    std::condition_variable cv_;
    bool stop_ = false;
    bool ok_ = true;  // written only by the writer thread, read after join
    std::thread th_;
};

struct MarchLog {
    mms_ctx *ctx;
    FILE *fh, *fhM, *fhp;
    SnapshotWriter *snap;
    int status;
};

int march_cb(void *user, int rejected, const mms_record *r)
{
    MarchLog *L = (MarchLog *)user;
    if (rejected) {
        // ode_functions.cpp:285-287
        printf("PANIC!! energy is increasing, so halving the step.\n");
        fprintf(L->fhp, "PANIC!! energy is increasing, so halving the step. %d, %g, %g, %g, %g \n", r->tindex,
                (fptype)r->t, (fptype)r->dt, (fptype)r->E_eV, (fptype)r->torque);
        return 0;
    }
    double t;
    float *buf = L->snap->acquire();
    if (mms_state_get_f32(L->ctx, buf, &t) != MMS_OK) {
        L->snap->release(buf);
        L->status = EXIT_FAILURE;
        return 1;
    }
    L->snap->submit(buf);
    // ode_functions.cpp:330-333
    fprintf(L->fh, "%d, %g, %g, %g, %g, %g, %g, %g, %g \n", r->tindex, (fptype)r->t, (fptype)r->dt, (fptype)r->E_eV,
            (fptype)r->Mx, (fptype)r->My, (fptype)r->Mz, (fptype)r->Mmag, (fptype)r->torque);
    fprintf(stdout, "%d, %g, %g, %g, %g, %g, %g, %g, %g \n", r->tindex, (fptype)r->t, (fptype)r->dt,
            (fptype)r->E_eV, (fptype)r->Mx, (fptype)r->My, (fptype)r->Mz, (fptype)r->Mmag, (fptype)r->torque);
    fflush(NULL);
    return 0;
}

}  // namespace

int time_marching(byte *material, Vector3 *M, const fptype finaltime, const fptype timestep, const int xdim,
                  const int ydim, const int zdim, const fptype dx, const fptype dy, const fptype dz, const int P,
                  const fptype mu_0, const fptype Ms, const fptype Aexch, const fptype alfa, const fptype gamma,
                  const int coupling, const int exchange, const int external, const int use_fmm, const int use_gpu,
                  const char *sim_name, const int verbosity)
{
    (void)use_gpu;
    const mms_params p = ref_params(mu_0, Ms, Aexch, alfa, gamma, coupling, exchange, external);
    mms_ctx *ctx = get_ctx(use_fmm, xdim, ydim, zdim, dx, dy, dz, P, p, verbosity);
    if (!ctx) return EXIT_FAILURE;
    char fn[1100];
    MarchLog L;
    L.ctx = ctx;
    L.snap = nullptr;
    L.status = EXIT_SUCCESS;
    snprintf(fn, sizeof fn, "%s/%s", sim_name, "dynamics.dat");
    L.fh = fopen(fn, "w");
    snprintf(fn, sizeof fn, "%s/%s", sim_name, "Mdynamics.dat");
    L.fhM = fopen(fn, "w");
    snprintf(fn, sizeof fn, "%s/%s", sim_name, "panic.dat");
    L.fhp = fopen(fn, "w");
    if (!L.fh || !L.fhM || !L.fhp) {
        printf("FATAL ERROR: Error opening file in %s\n", sim_name);
        if (L.fh) fclose(L.fh);
        if (L.fhM) fclose(L.fhM);
        if (L.fhp) fclose(L.fhp);
        return EXIT_FAILURE;
    }
    SnapshotWriter snap(L.fhM, zdim, ydim, xdim);
    L.snap = &snap;
    int st = mms_state_set_f32(ctx, material, &M[0].x, 0.0);
    if (st == MMS_OK) {
        mms_controller c;
        memset(&c, 0, sizeof c);
        c.mode = 0;
        c.torque_stop = 1e-3;   // ode_functions.cpp:337
        c.max_rejects = 50;     // ode_functions.cpp:289
        int nrec = 0;
        st = mms_march(ctx, &c, finaltime, timestep, nullptr, 0, &nrec, march_cb, &L);
        if (st == MMS_ERR_REJECTED) {
            // ode_functions.cpp:290-292: the reference stops and still succeeds
            fprintf(stdout, "PANIC!! Stuck in energy violation errors. Terminating the simulation.\n");
            fprintf(L.fhp, "PANIC!! Stuck in energy violation errors. Terminating the simulation.\n");
            st = MMS_OK;
        }
    }
    if (st == MMS_OK) {
        double t;
        st = mms_state_get_f32(ctx, &M[0].x, &t);
    }
    if (!snap.finish()) {
        printf("FATAL ERROR: writing Mdynamics.dat in %s failed\n", sim_name);
        L.status = EXIT_FAILURE;
    }
    fclose(L.fh);
    fclose(L.fhM);
    fclose(L.fhp);
    if (st != MMS_OK) return fail("time_marching");
    return L.status;
}
