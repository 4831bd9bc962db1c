/*
 * Test infrastructure only: CPU oracle for the demag / LLG hot path.
 * See mms_oracle.h.  Every function cites the reference lines it restates.
 */
#include "mms_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(g, x, y, z) ((size_t)(z) * (g)->ydim * (g)->xdim + (size_t)(y) * (g)->xdim + (size_t)(x))

static size_t ncells(const mo_grid *g) { return (size_t)g->xdim * g->ydim * g->zdim; }

/* vector_functions.cpp:8-28 */
void mo_divergence(const mo_grid *g, const double *M, double *rho)
{
    const int X = g->xdim, Y = g->ydim, Z = g->zdim;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < Z; z++)
        for (int y = 0; y < Y; y++)
            for (int x = 0; x < X; x++) {
                double x2 = (x != X - 1) ? M[3 * IDX(g, x + 1, y, z) + 0] : 0;
                double x0 = (x != 0) ? M[3 * IDX(g, x - 1, y, z) + 0] : 0;
                double y2 = (y != Y - 1) ? M[3 * IDX(g, x, y + 1, z) + 1] : 0;
                double y0 = (y != 0) ? M[3 * IDX(g, x, y - 1, z) + 1] : 0;
                double z2 = (z != Z - 1) ? M[3 * IDX(g, x, y, z + 1) + 2] : 0;
                double z0 = (z != 0) ? M[3 * IDX(g, x, y, z - 1) + 2] : 0;
                rho[IDX(g, x, y, z)] = ((x2 - x0) / g->dx + (y2 - y0) / g->dy + (z2 - z0) / g->dz) / 2.0;
            }
}

/* vector_functions.cpp:31-54 */
void mo_gradient(const mo_grid *g, const double *S, double c, double *H)
{
    const int X = g->xdim, Y = g->ydim, Z = g->zdim;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < Z; z++)
        for (int y = 0; y < Y; y++)
            for (int x = 0; x < X; x++) {
                double x2 = (x != X - 1) ? S[IDX(g, x + 1, y, z)] : 0;
                double x0 = (x != 0) ? S[IDX(g, x - 1, y, z)] : 0;
                double y2 = (y != Y - 1) ? S[IDX(g, x, y + 1, z)] : 0;
                double y0 = (y != 0) ? S[IDX(g, x, y - 1, z)] : 0;
                double z2 = (z != Z - 1) ? S[IDX(g, x, y, z + 1)] : 0;
                double z0 = (z != 0) ? S[IDX(g, x, y, z - 1)] : 0;
                size_t i = IDX(g, x, y, z);
                H[3 * i + 0] = (x2 - x0) / (2 * g->dx) * c;
                H[3 * i + 1] = (y2 - y0) / (2 * g->dy) * c;
                H[3 * i + 2] = (z2 - z0) / (2 * g->dz) * c;
            }
}

/* vector_functions.cpp:57-103 */
void mo_add_exchange(const mo_grid *g, const double *M, double Ms, double Aexch, double mu0, double *H)
{
    const int X = g->xdim, Y = g->ydim, Z = g->zdim;
    const double cm = 2 * Aexch / (mu0 * Ms * Ms);
#pragma omp parallel for collapse(2)
    for (int z = 0; z < Z; z++)
        for (int y = 0; y < Y; y++)
            for (int x = 0; x < X; x++) {
                size_t i = IDX(g, x, y, z);
                for (int c = 0; c < 3; c++) {
                    double m0 = M[3 * i + c];
                    double xp = (x != X - 1) ? M[3 * IDX(g, x + 1, y, z) + c] : 0;
                    double xm = (x != 0) ? M[3 * IDX(g, x - 1, y, z) + c] : 0;
                    double yp = (y != Y - 1) ? M[3 * IDX(g, x, y + 1, z) + c] : 0;
                    double ym = (y != 0) ? M[3 * IDX(g, x, y - 1, z) + c] : 0;
                    double zp = (z != Z - 1) ? M[3 * IDX(g, x, y, z + 1) + c] : 0;
                    double zm = (z != 0) ? M[3 * IDX(g, x, y, z - 1) + c] : 0;
                    double L = (xp + xm - 2 * m0) / (g->dx * g->dx) + (yp + ym - 2 * m0) / (g->dy * g->dy) +
                               (zp + zm - 2 * m0) / (g->dz * g->dz);
                    H[3 * i + c] += cm * L;
                }
            }
}

/* fmm_calc.cu:433-453, restated target-major so it parallelises without races */
void mo_potential_direct(const mo_grid *g, const double *rho, double *phi)
{
    const int X = g->xdim, Y = g->ydim, Z = g->zdim;
    const double dV = g->dx * g->dy * g->dz;
    const long N = (long)ncells(g);
#pragma omp parallel for schedule(dynamic, 64)
    for (long i = 0; i < N; i++) {
        const int x = (int)(i % X), y = (int)((i / X) % Y), z = (int)(i / ((long)X * Y));
        double acc = 0, comp = 0; /* Kahan: the FP64 truth should not depend on N */
        for (int zs = 0; zs < Z; zs++)
            for (int ys = 0; ys < Y; ys++)
                for (int xs = 0; xs < X; xs++) {
                    const double r = rho[IDX(g, xs, ys, zs)];
                    if (r == 0) continue;
                    if (xs == x && ys == y && zs == z) continue;
                    const double Rx = (x - xs) * g->dx, Ry = (y - ys) * g->dy, Rz = (z - zs) * g->dz;
                    const double term = r * dV / sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
                    const double yk = term - comp;
                    const double tk = acc + yk;
                    comp = (tk - acc) - yk;
                    acc = tk;
                }
        phi[i] = acc;
    }
}

void mo_potential_direct_targets(const mo_grid *g, const double *rho, const int *targets, int ntargets,
                                 double *phi_out)
{
    const int X = g->xdim, Y = g->ydim, Z = g->zdim;
    const double dV = g->dx * g->dy * g->dz;
#pragma omp parallel for schedule(dynamic, 8)
    for (int k = 0; k < ntargets; k++) {
        const long i = targets[k];
        const int x = (int)(i % X), y = (int)((i / X) % Y), z = (int)(i / ((long)X * Y));
        double acc = 0, comp = 0;
        for (int zs = 0; zs < Z; zs++)
            for (int ys = 0; ys < Y; ys++)
                for (int xs = 0; xs < X; xs++) {
                    const double r = rho[IDX(g, xs, ys, zs)];
                    if (r == 0) continue;
                    if (xs == x && ys == y && zs == z) continue;
                    const double Rx = (x - xs) * g->dx, Ry = (y - ys) * g->dy, Rz = (z - zs) * g->dz;
                    const double term = r * dV / sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
                    const double yk = term - comp;
                    const double tk = acc + yk;
                    comp = (tk - acc) - yk;
                    acc = tk;
                }
        phi_out[k] = acc;
    }
}

/* ode_functions.cpp:59-67 for the built-in ramp; otherwise a clamped
 * piecewise-linear table of B (T) */
void mo_hext(const mo_params *p, double t, double H[3])
{
    H[0] = H[1] = H[2] = 0;
    if (!p->external) return;
    if (p->n_hext <= 0) {
        H[0] = (1 / p->mu0) * ((t < 1e-9) ? (-0.3 / 1e-9 * t + 0.3) : 0);
        return;
    }
    const int n = p->n_hext;
    double B[3];
    if (t <= p->hext_t[0]) {
        for (int c = 0; c < 3; c++) B[c] = p->hext_b[c];
    } else if (t >= p->hext_t[n - 1]) {
        for (int c = 0; c < 3; c++) B[c] = p->hext_b[3 * (n - 1) + c];
    } else {
        int k = 0;
        while (k + 1 < n && p->hext_t[k + 1] < t) k++;
        const double w = (t - p->hext_t[k]) / (p->hext_t[k + 1] - p->hext_t[k]);
        for (int c = 0; c < 3; c++) B[c] = (1 - w) * p->hext_b[3 * k + c] + w * p->hext_b[3 * (k + 1) + c];
    }
    for (int c = 0; c < 3; c++) H[c] = B[c] / p->mu0;
}

/* ode_functions.cpp:21-70 */
void mo_hfield(const mo_grid *g, const mo_params *p, const double *M, double t,
               double *H, double *rho, double *phi)
{
    const size_t N = ncells(g);
    memset(H, 0, 3 * N * sizeof(double));
    if (p->demag) {
        mo_divergence(g, M, rho);
        mo_potential_direct(g, rho, phi);
        mo_gradient(g, phi, 1 / (4.0 * M_PI), H);
    }
    if (p->exchange) mo_add_exchange(g, M, p->Ms, p->Aexch, p->mu0, H);
    if (p->external) {
        double he[3];
        mo_hext(p, t, he);
        for (size_t i = 0; i < N; i++)
            for (int c = 0; c < 3; c++) H[3 * i + c] += he[c];
    }
}

/* ode_functions.cpp:11-18 */
void mo_llg(const double *M, const double *H, double alpha, double gamma, double Ms, double *dMdt)
{
    const double cx = M[1] * H[2] - M[2] * H[1];
    const double cy = M[2] * H[0] - M[0] * H[2];
    const double cz = M[0] * H[1] - M[1] * H[0];
    const double dx = M[1] * cz - M[2] * cy;
    const double dy = M[2] * cx - M[0] * cz;
    const double dz = M[0] * cy - M[1] * cx;
    const double a = alpha * gamma / Ms;
    dMdt[0] = -gamma * cx - a * dx;
    dMdt[1] = -gamma * cy - a * dy;
    dMdt[2] = -gamma * cz - a * dz;
}

/* ode_functions.cpp:76-148 */
void mo_rk4_step(const mo_grid *g, const mo_params *p, const unsigned char *material,
                 const double *M, const double *H_in, double t, double dt, double *M_out)
{
    const size_t N = ncells(g);
    double *slope = (double *)calloc(3 * N, sizeof(double));
    double *Mst = (double *)calloc(3 * N, sizeof(double));
    double *H = (double *)malloc(3 * N * sizeof(double));
    double *rho = (double *)malloc(N * sizeof(double));
    double *phi = (double *)malloc(N * sizeof(double));
    static const double cstage[4] = {0.0, 0.5, 0.5, 1.0};
    static const double wstage[4] = {1.0, 2.0, 2.0, 1.0};
    static const double advance[4] = {0.5, 0.5, 1.0, 0.0};
    for (int s = 0; s < 4; s++) {
        const double *Hs = H_in;
        const double *Ms_ = M;
        if (s > 0) {
            const double ts = p->ref_stage_time ? t : t + cstage[s] * dt;
            mo_hfield(g, p, Mst, ts, H, rho, phi);
            Hs = H;
            Ms_ = Mst;
        }
        for (size_t i = 0; i < N; i++) {
            if (!material[i]) continue;
            double k[3];
            mo_llg(&Ms_[3 * i], &Hs[3 * i], p->alpha, p->gamma, p->Ms, k);
            for (int c = 0; c < 3; c++) slope[3 * i + c] += wstage[s] * k[c];
            if (s < 3)
                for (int c = 0; c < 3; c++) Mst[3 * i + c] = M[3 * i + c] + advance[s] * dt * k[c];
        }
    }
    for (size_t i = 0; i < N; i++) {
        if (!material[i]) {
            M_out[3 * i] = M_out[3 * i + 1] = M_out[3 * i + 2] = 0;
            continue;
        }
        double m[3];
        for (int c = 0; c < 3; c++) m[c] = M[3 * i + c] + dt * slope[3 * i + c] * (1 / 6.0);
        const double s = p->Ms / sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        for (int c = 0; c < 3; c++) M_out[3 * i + c] = m[c] * s;
    }
    free(slope);
    free(Mst);
    free(H);
    free(rho);
    free(phi);
}

/* ode_functions.cpp:230-308 (accepted-step sequence, fixed dt) */
void mo_rk4_run(const mo_grid *g, const mo_params *p, const unsigned char *material,
                double *M, double dt, int nsteps)
{
    const size_t N = ncells(g);
    double *H = (double *)malloc(3 * N * sizeof(double));
    double *rho = (double *)malloc(N * sizeof(double));
    double *phi = (double *)malloc(N * sizeof(double));
    double *M2 = (double *)malloc(3 * N * sizeof(double));
    double t = 0;
    mo_hfield(g, p, M, t, H, rho, phi);
    for (int s = 0; s < nsteps; s++) {
        mo_rk4_step(g, p, material, M, H, t, dt, M2);
        mo_hfield(g, p, M2, p->ref_stage_time ? t : t + dt, H, rho, phi);
        memcpy(M, M2, 3 * N * sizeof(double));
        t += dt;
    }
    free(H);
    free(rho);
    free(phi);
    free(M2);
}

/* ode_functions.cpp:234-240 and 268-278 */
void mo_energy_torque(const mo_grid *g, const mo_params *p, const unsigned char *material,
                      const double *M, const double *H, double *E_eV, double *torque)
{
    const size_t N = ncells(g);
    double E = 0, tq = 0;
    for (size_t i = 0; i < N; i++) {
        if (!material[i]) continue;
        const double *m = &M[3 * i], *h = &H[3 * i];
        E += m[0] * h[0] + m[1] * h[1] + m[2] * h[2];
        const double cx = m[1] * h[2] - m[2] * h[1];
        const double cy = m[2] * h[0] - m[0] * h[2];
        const double cz = m[0] * h[1] - m[1] * h[0];
        const double t = sqrt(cx * cx + cy * cy + cz * cz);
        if (t > tq) tq = t;
    }
    *E_eV = E * (-0.5 * p->mu0 * (g->dx * g->dy * g->dz) / 1.6e-19);
    *torque = tq / p->Ms / p->Ms;
}

/* ---- FP32 replicas -------------------------------------------------------- */

/* vector_functions.cpp:8-28 in float, same operation order */
void mo_divergence_f32(const mo_grid *g, const float *M, float *rho)
{
    const int X = g->xdim, Y = g->ydim, Z = g->zdim;
    const float dx = (float)g->dx, dy = (float)g->dy, dz = (float)g->dz;
    for (int z = 0; z < Z; z++)
        for (int y = 0; y < Y; y++)
            for (int x = 0; x < X; x++) {
                float x2 = (x != X - 1) ? M[3 * IDX(g, x + 1, y, z) + 0] : 0;
                float x0 = (x != 0) ? M[3 * IDX(g, x - 1, y, z) + 0] : 0;
                float y2 = (y != Y - 1) ? M[3 * IDX(g, x, y + 1, z) + 1] : 0;
                float y0 = (y != 0) ? M[3 * IDX(g, x, y - 1, z) + 1] : 0;
                float z2 = (z != Z - 1) ? M[3 * IDX(g, x, y, z + 1) + 2] : 0;
                float z0 = (z != 0) ? M[3 * IDX(g, x, y, z - 1) + 2] : 0;
                float s = (x2 - x0) / dx + (y2 - y0) / dy + (z2 - z0) / dz;
                rho[IDX(g, x, y, z)] = (float)(s / 2.0);
            }
}

/* fmm_calc.cu:433-453 in float: per target, sources accumulate in increasing
 * source index, exactly the order of the reference's source-outer loop */
void mo_potential_direct_f32(const mo_grid *g, const float *rho, float *phi)
{
    const int X = g->xdim, Y = g->ydim, Z = g->zdim;
    const float dx = (float)g->dx, dy = (float)g->dy, dz = (float)g->dz;
    const float dV = dx * dy * dz;
    const long N = (long)ncells(g);
#pragma omp parallel for schedule(dynamic, 64)
    for (long i = 0; i < N; i++) {
        const int x = (int)(i % X), y = (int)((i / X) % Y), z = (int)(i / ((long)X * Y));
        float acc = 0;
        for (int zs = 0; zs < Z; zs++)
            for (int ys = 0; ys < Y; ys++)
                for (int xs = 0; xs < X; xs++) {
                    const float q = rho[IDX(g, xs, ys, zs)] * dV;
                    if (q == 0) continue;
                    if (xs == x && ys == y && zs == z) continue;
                    const float Rx = (x - xs) * dx, Ry = (y - ys) * dy, Rz = (z - zs) * dz;
                    acc += q / sqrtf(Rx * Rx + Ry * Ry + Rz * Rz);
                }
        phi[i] = acc;
    }
}
