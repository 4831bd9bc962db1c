/*
 * Test infrastructure only: the CPU oracle for the demag / LLG hot path.
 *
 * A plain-C restatement of the reference's per-step arithmetic, in FP64 (the
 * ground truth every GPU result is checked against) and, where the reference's
 * own FP32 operation order matters for a tight pin, in FP32.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the
 * product library never does.
 *
 * Layouts follow the reference: cell index i = z*ydim*xdim + y*xdim + x
 * (vector_functions.cpp:20-26); vector fields are AoS triples (Vector3.hpp:10-12).
 */
#ifndef MMS_ORACLE_H
#define MMS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int xdim, ydim, zdim;
    double dx, dy, dz;
} mo_grid;

typedef struct {
    double Ms, Aexch, alpha, gamma, mu0;
    int demag, exchange, external;
    /* external field B(t) in tesla as a piecewise-linear table, clamped at both
     * ends; H_ext = B / mu0.  n_hext == 0 with external != 0 selects the
     * reference's hard-coded ramp (ode_functions.cpp:61). */
    int n_hext;
    const double *hext_t;   /* n_hext times (s), increasing            */
    const double *hext_b;   /* n_hext x 3 field values (T)             */
    /* 1: every RK4 stage sees the step's start time t, as the reference does
     * (ode_functions.cpp:109,121,133); 0: stages at t + c*dt. */
    int ref_stage_time;
} mo_params;

/* ---- FP64 restatement --------------------------------------------------- */
/* rho = div M, central differences, zero outside (vector_functions.cpp:8-28) */
void mo_divergence(const mo_grid *g, const double *M, double *rho);
/* H = c * grad S, central differences, zero outside (vector_functions.cpp:31-54); overwrites H */
void mo_gradient(const mo_grid *g, const double *S, double c, double *H);
/* H += 2A/(mu0 Ms^2) lap M, M = 0 outside (vector_functions.cpp:57-103) */
void mo_add_exchange(const mo_grid *g, const double *M, double Ms, double Aexch, double mu0, double *H);
/* phi_i = sum_{j != i, rho_j != 0} rho_j dV / |r_i - r_j| (fmm_calc.cu:412-461) */
void mo_potential_direct(const mo_grid *g, const double *rho, double *phi);
/* the potential only at the targets listed (for bounded baseline samples) */
void mo_potential_direct_targets(const mo_grid *g, const double *rho, const int *targets, int ntargets,
                                 double *phi_out);
/* external field at time t, A/m */
void mo_hext(const mo_params *p, double t, double H[3]);
/* H(M) as Hfield does (ode_functions.cpp:21-70); rho/phi are scratch outputs */
void mo_hfield(const mo_grid *g, const mo_params *p, const double *M, double t,
               double *H, double *rho, double *phi);
/* dM/dt = -gamma MxH - (alpha gamma / Ms) Mx(MxH) (ode_functions.cpp:11-18) */
void mo_llg(const double *M, const double *H, double alpha, double gamma, double Ms, double *dMdt);
/* one classical RK4 step over material cells with |M| = Ms renormalisation
 * (ode_functions.cpp:76-148).  H_in is H(M) at time t (k1 reuses it, as the
 * reference does).  Empty cells of M_out are set to zero. */
void mo_rk4_step(const mo_grid *g, const mo_params *p, const unsigned char *material,
                 const double *M, const double *H_in, double t, double dt, double *M_out);
/* nsteps fixed RK4 steps; M is updated in place.  Mirrors the accepted-step
 * sequence of time_marching (ode_functions.cpp:230-308): the field used as k1
 * for step n+1 is evaluated at the OLD time t_n when ref_stage_time is set. */
void mo_rk4_run(const mo_grid *g, const mo_params *p, const unsigned char *material,
                double *M, double dt, int nsteps);
/* energy (eV) and max normalised torque as time_marching logs them
 * (ode_functions.cpp:234-240, 268-278) */
void mo_energy_torque(const mo_grid *g, const mo_params *p, const unsigned char *material,
                      const double *M, const double *H, double *E_eV, double *torque);

/* ---- FP32 replicas of the reference's operation order --------------------- */
void mo_divergence_f32(const mo_grid *g, const float *M, float *rho);
void mo_potential_direct_f32(const mo_grid *g, const float *rho, float *phi);

#ifdef __cplusplus
}
#endif
#endif
