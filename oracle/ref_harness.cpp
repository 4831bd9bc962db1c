/*
 * Test infrastructure only (part of the oracle).
 *
 * A command-line harness linked against the reference's own CPU sources
 * (compiled from the read-only reference tree by oracle/Makefile into
 * oracle/_ref/).  Each invocation runs ONE reference entry point on binary
 * inputs and writes binary outputs, so the reference's first-call statics
 * (fmm_calc.cu:303-365, fmm_calc.cu:35-124) are always sized for the case at
 * hand.  Used to (1) generate the golden fixtures under tests/golden/ and
 * (2) time the reference CPU path as the baseline in bench.py.
 *
 * Reference entry points called:
 *   calc_potential_exact  fmm_calc.cu:412-461   (use_gpu = 0)
 *   fmm_calc              fmm_calc.cu:295-408   (use_gpu = 0)
 *   Hfield                ode_functions.cpp:21-70
 *   rk4_step              ode_functions.cpp:76-148 (external linkage, no header)
 *   time_marching         ode_functions.cpp:158-365
 *   divergence_3d / gradient_3d / add_exchange_field  vector_functions.cpp:8-103
 *
 * usage: mmsref_harness <op> key=value ...   (see main() for the ops)
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <map>
#include <vector>
#include <chrono>
#include <sys/stat.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "mydefs.hpp"
#include "Vector3.hpp"
#include "helper_functions.hpp"
#include "vector_functions.hpp"
#include "ode_functions.hpp"

/* rk4_step has external linkage but no header (ode_functions.cpp:76-87) */
int rk4_step(const fptype t, const fptype dt, fptype *t2,
             const byte *material, const Vector3 *M, Vector3 *M2,
             Vector3 *H, Vector3 *slope, Vector3 *this_slope,
             fptype *charge, fptype *potential,
             const int xdim, const int ydim, const int zdim,
             const fptype dx, const fptype dy, const fptype dz,
             const int P,
             const fptype mu_0, const fptype Ms, const fptype Aexch, const fptype alfa, const fptype gamma,
             const int demag, const int exchange, const int external, const int use_fmm,
             const int normalize, const int use_gpu, const int verbosity);

static std::map<std::string, std::string> g_args;

static const char *arg_s(const char *k, const char *def = nullptr)
{
    auto it = g_args.find(k);
    if (it != g_args.end()) return it->second.c_str();
    if (!def) { fprintf(stderr, "mmsref_harness: missing argument %s\n", k); exit(2); }
    return def;
}
static int arg_i(const char *k, int def = -999999)
{
    auto it = g_args.find(k);
    if (it != g_args.end()) return atoi(it->second.c_str());
    if (def == -999999) { fprintf(stderr, "mmsref_harness: missing argument %s\n", k); exit(2); }
    return def;
}
static float arg_f(const char *k, double def = NAN)
{
    auto it = g_args.find(k);
    if (it != g_args.end()) return (float)strtod(it->second.c_str(), nullptr);
    if (std::isnan(def)) { fprintf(stderr, "mmsref_harness: missing argument %s\n", k); exit(2); }
    return (float)def;
}

template <class T>
static std::vector<T> read_bin(const char *path, size_t n)
{
    std::vector<T> v(n);
    FILE *f = fopen(path, "rb");
    if (!f) { fprintf(stderr, "mmsref_harness: cannot open %s\n", path); exit(2); }
    size_t got = fread(v.data(), sizeof(T), n, f);
    fclose(f);
    if (got != n) { fprintf(stderr, "mmsref_harness: %s holds %zu of %zu items\n", path, got, n); exit(2); }
    return v;
}

template <class T>
static void write_bin(const std::string &path, const T *p, size_t n)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "mmsref_harness: cannot write %s\n", path.c_str()); exit(2); }
    fwrite(p, sizeof(T), n, f);
    fclose(f);
}

static double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int main(int argc, char **argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: mmsref_harness <potential|hfield|stencils|rk4|march|time_rk4|time_hfield> key=value...\n");
        return 2;
    }
    const std::string op = argv[1];
    for (int i = 2; i < argc; i++) {
        const char *eq = strchr(argv[i], '=');
        if (!eq) { fprintf(stderr, "mmsref_harness: bad argument %s\n", argv[i]); return 2; }
        g_args[std::string(argv[i], eq - argv[i])] = std::string(eq + 1);
    }
    const int xdim = arg_i("xdim"), ydim = arg_i("ydim"), zdim = arg_i("zdim");
    const fptype dx = arg_f("dx"), dy = arg_f("dy"), dz = arg_f("dz");
    const size_t N = (size_t)xdim * ydim * zdim;
    const int P = arg_i("P", 3);
    const int verbosity = arg_i("verbosity", 0);
    /* material constants as main.cpp:107-111 computes them (double -> fptype) */
    const fptype mu_0 = 4 * M_PI * 1e-7;
    const fptype Ms = arg_f("Ms", 8.6e5);
    const fptype Aexch = arg_f("Aexch", 1.3e-11);
    const fptype alfa = arg_f("alfa", 0.5);
    const fptype gamma = arg_f("gamma", 2.21e5);
    const int demag = arg_i("demag", 1), exchange = arg_i("exchange", 1);
    const int external = arg_i("external", 0), use_fmm = arg_i("use_fmm", 0);
    const std::string out = arg_s("out", "");

    if (op == "potential") {
        std::vector<fptype> charge = read_bin<fptype>(arg_s("charge"), N);
        std::vector<fptype> pot(N, 0.f);
        int st = use_fmm ? fmm_calc(charge.data(), pot.data(), xdim, ydim, zdim, dx, dy, dz, P, 0, verbosity)
                         : calc_potential_exact(charge.data(), xdim, ydim, zdim, dx, dy, dz, pot.data(), 0, verbosity);
        if (st) return 1;
        write_bin(out, pot.data(), N);
        return 0;
    }
    if (op == "stencils") {
        std::vector<Vector3> M = read_bin<Vector3>(arg_s("M"), N);
        std::vector<fptype> S = read_bin<fptype>(arg_s("S"), N);
        std::vector<fptype> div(N);
        std::vector<Vector3> grad(N), exch(N);
        divergence_3d(M.data(), xdim, ydim, zdim, dx, dy, dz, div.data());
        gradient_3d(S.data(), xdim, ydim, zdim, dx, dy, dz, 1 / (4.0 * M_PI), grad.data());
        add_exchange_field(M.data(), Ms, Aexch, mu_0, xdim, ydim, zdim, dx, dy, dz, exch.data());
        write_bin(out + ".div", div.data(), N);
        write_bin(out + ".grad", grad.data(), N);
        write_bin(out + ".exch", exch.data(), N);
        return 0;
    }
    if (op == "hfield") {
        std::vector<Vector3> M = read_bin<Vector3>(arg_s("M"), N);
        std::vector<Vector3> H(N);
        std::vector<fptype> charge(N), pot(N);
        const fptype t = arg_f("t", 0.0);
        int st = Hfield(M.data(), H.data(), charge.data(), pot.data(), t, xdim, ydim, zdim, dx, dy, dz, P,
                        mu_0, Ms, Aexch, demag, exchange, external, use_fmm, 0, verbosity);
        if (st) return 1;
        write_bin(out + ".H", H.data(), N);
        write_bin(out + ".charge", charge.data(), N);
        write_bin(out + ".potential", pot.data(), N);
        return 0;
    }
    if (op == "rk4") {
        /* fixed-step marching in exactly the order time_marching performs an
         * accepted step (ode_functions.cpp:230-308) without its controller,
         * files or getchar(): H(M, t) once; per step rk4_step at t, then
         * Hfield(M2, t) (old t, :267), then M = M2, H = H2, t = t2. */
        std::vector<byte> material = read_bin<byte>(arg_s("material"), N);
        std::vector<Vector3> M = read_bin<Vector3>(arg_s("M"), N);
        std::vector<Vector3> M2(N), H(N), H2(N), H3(N), slope(N), this_slope(N);
        std::vector<fptype> charge(N), pot(N);
        const fptype dt = arg_f("dt");
        const int nsteps = arg_i("nsteps");
        fptype t = 0, t2 = 0;
        int st = Hfield(M.data(), H.data(), charge.data(), pot.data(), t, xdim, ydim, zdim, dx, dy, dz, P,
                        mu_0, Ms, Aexch, demag, exchange, external, use_fmm, 0, verbosity);
        for (int s = 0; s < nsteps && !st; s++) {
            H3 = H;
            st |= rk4_step(t, dt, &t2, material.data(), M.data(), M2.data(), H3.data(), slope.data(),
                           this_slope.data(), charge.data(), pot.data(), xdim, ydim, zdim, dx, dy, dz, P,
                           mu_0, Ms, Aexch, alfa, gamma, demag, exchange, external, use_fmm, 1, 0, verbosity);
            st |= Hfield(M2.data(), H2.data(), charge.data(), pot.data(), t, xdim, ydim, zdim, dx, dy, dz, P,
                         mu_0, Ms, Aexch, demag, exchange, external, use_fmm, 0, verbosity);
            M.swap(M2);
            H.swap(H2);
            t = t2;
        }
        if (st) return 1;
        write_bin(out + ".M", M.data(), N);
        write_bin(out + ".H", H.data(), N);
        return 0;
    }
    if (op == "march") {
        /* the reference's own driver loop including its energy/torque step
         * controller; writes <sim>/dynamics.dat, Mdynamics.dat, panic.dat */
        std::vector<byte> material = read_bin<byte>(arg_s("material"), N);
        std::vector<Vector3> M = read_bin<Vector3>(arg_s("M"), N);
        const char *sim = arg_s("sim");
        mkdir(sim, 0755);
        int st = time_marching(material.data(), M.data(), arg_f("finaltime"), arg_f("timestep"),
                               xdim, ydim, zdim, dx, dy, dz, P, mu_0, Ms, Aexch, alfa, gamma,
                               demag, exchange, external, use_fmm, 0, sim, verbosity);
        write_bin(out + ".M", M.data(), N);
        return st ? 1 : 0;
    }
    if (op == "time_rk4") {
        /* CPU baseline: `warmup` untimed then `nsteps` timed fixed-dt steps in
         * time_marching's accepted-step order (ode_functions.cpp:230-308): per
         * step rk4_step at t (three Hfield calls inside, :109-133) then
         * Hfield(M2) at the old t (:267).  The initial Hfield(M) is untimed.
         * Stops early, after the step that passes `budget_s` seconds of timed
         * work.  Prints one line per timed step (its wall seconds), then
         * "total <steps> <seconds> <threads>". */
        std::vector<byte> material = read_bin<byte>(arg_s("material"), N);
        std::vector<Vector3> M = read_bin<Vector3>(arg_s("M"), N);
        std::vector<Vector3> M2(N), H(N), H2(N), H3(N), slope(N), this_slope(N);
        std::vector<fptype> charge(N), pot(N);
        const fptype dt = arg_f("dt");
        const int nsteps = arg_i("nsteps"), warmup = arg_i("warmup", 0);
        const double budget = arg_f("budget_s", 1e30);
        fptype t = 0, t2 = 0;
        int st = Hfield(M.data(), H.data(), charge.data(), pot.data(), t, xdim, ydim, zdim, dx, dy, dz, P,
                        mu_0, Ms, Aexch, demag, exchange, external, use_fmm, 0, verbosity);
        double timed = 0;
        int done = 0;
        for (int s = 0; s < warmup + nsteps && !st; s++) {
            const double t0 = now_s();
            H3 = H;
            st |= rk4_step(t, dt, &t2, material.data(), M.data(), M2.data(), H3.data(), slope.data(),
                           this_slope.data(), charge.data(), pot.data(), xdim, ydim, zdim, dx, dy, dz, P,
                           mu_0, Ms, Aexch, alfa, gamma, demag, exchange, external, use_fmm, 1, 0, verbosity);
            st |= Hfield(M2.data(), H2.data(), charge.data(), pot.data(), t, xdim, ydim, zdim, dx, dy, dz, P,
                         mu_0, Ms, Aexch, demag, exchange, external, use_fmm, 0, verbosity);
            M.swap(M2);
            H.swap(H2);
            t = t2;
            const double t1 = now_s();
            if (s >= warmup) {
                printf("%.9f\n", t1 - t0);
                timed += t1 - t0;
                done++;
                if (timed > budget) break;
            }
        }
        int threads = 1;
#ifdef _OPENMP
        threads = omp_get_max_threads();
#endif
        printf("total %d %.9f %d\n", done, timed, threads);
        if (!out.empty()) write_bin(out + ".M", M.data(), N);
        return st ? 1 : 0;
    }
    if (op == "time_hfield") {
        /* CPU baseline: wall time of `reps` reference Hfield evaluations on
         * the given M (the potential dominates, >90 %).  Prints one line:
         * seconds_per_hfield threads */
        std::vector<Vector3> M = read_bin<Vector3>(arg_s("M"), N);
        std::vector<Vector3> H(N);
        std::vector<fptype> charge(N), pot(N);
        const int reps = arg_i("reps", 1);
        double t0 = now_s();
        int st = 0;
        for (int r = 0; r < reps; r++)
            st |= Hfield(M.data(), H.data(), charge.data(), pot.data(), 0.f, xdim, ydim, zdim, dx, dy, dz, P,
                         mu_0, Ms, Aexch, demag, exchange, external, use_fmm, 0, verbosity);
        double t1 = now_s();
        int threads = 1;
#ifdef _OPENMP
        threads = omp_get_max_threads();
#endif
        printf("%.9f %d\n", (t1 - t0) / reps, threads);
        if (!out.empty()) write_bin(out + ".H", H.data(), N);
        return st ? 1 : 0;
    }
    fprintf(stderr, "mmsref_harness: unknown op %s\n", op.c_str());
    return 2;
}
