// Per-cell device math shared by the single-grid and the ensemble kernels:
// cell coordinates, the external field table, the effective field from the
// FP32 potential and the FP64 state, and the LLG right-hand side.
#pragma once

#include "mms_internal.cuh"

namespace mmsdev {

__device__ __forceinline__ void cell_xyz(long long i, const GridK &g, int &x, int &y, int &z)
{
    x = (int)(i % g.X);
    long long r = i / g.X;
    y = (int)(r % g.Y);
    z = (int)(r / g.Y);
}

// clamped piecewise-linear B(t) table, or the reference's ramp (ode_functions.cpp:61)
__device__ __forceinline__ void hext_at(const PhysK &p, const double *__restrict__ tab, double t, double H[3])
{
    H[0] = H[1] = H[2] = 0.0;
    if (!p.external) return;
    if (p.n_hext == 0) {
        H[0] = p.inv_mu0 * ((t < 1e-9) ? (-0.3 / 1e-9 * t + 0.3) : 0.0);
        return;
    }
    const int n = p.n_hext;
    double b0, b1, b2;
    if (t <= tab[0]) {
        b0 = tab[1]; b1 = tab[2]; b2 = tab[3];
    } else if (t >= tab[4 * (n - 1)]) {
        b0 = tab[4 * (n - 1) + 1]; b1 = tab[4 * (n - 1) + 2]; b2 = tab[4 * (n - 1) + 3];
    } else {
        int k = 0;
        while (k + 1 < n && tab[4 * (k + 1)] < t) k++;
        const double w = (t - tab[4 * k]) / (tab[4 * (k + 1)] - tab[4 * k]);
        b0 = (1 - w) * tab[4 * k + 1] + w * tab[4 * (k + 1) + 1];
        b1 = (1 - w) * tab[4 * k + 2] + w * tab[4 * (k + 1) + 2];
        b2 = (1 - w) * tab[4 * k + 3] + w * tab[4 * (k + 1) + 3];
    }
    H[0] = b0 * p.inv_mu0;
    H[1] = b1 * p.inv_mu0;
    H[2] = b2 * p.inv_mu0;
}

// half reciprocal cell sizes 1 / (2 dx), 1 / (2 dy), 1 / (2 dz): the central
// difference weights of div_soa_cell, formed once on the host
struct DivScale {
    double hx, hy, hz;
};
inline DivScale div_scale(double dx, double dy, double dz) { return DivScale{0.5 / dx, 0.5 / dy, 0.5 / dz}; }

// rho = div M at cell i = (x, y, z) of the FP64 SoA state (planes N apart):
// central differences, zero outside the grid (vector_functions.cpp:8-28, in
// FP64), as products with the half reciprocal sizes (no divide on the device)
// rounded one by one (no contraction).  Every kernel that forms rho from the
// state uses this expression, so they agree bit for bit.
__device__ __forceinline__ float div_soa_cell(const double *__restrict__ M, long long i, int x, int y, int z,
                                              const GridK &g, const DivScale &h)
{
    const double *Mx = M, *My = M + g.N, *Mz = M + 2 * g.N;
    const long long sy = g.X, sz = (long long)g.X * g.Y;
    const double x2 = (x != g.X - 1) ? Mx[i + 1] : 0.0;
    const double x0 = (x != 0) ? Mx[i - 1] : 0.0;
    const double y2 = (y != g.Y - 1) ? My[i + sy] : 0.0;
    const double y0 = (y != 0) ? My[i - sy] : 0.0;
    const double z2 = (z != g.Z - 1) ? Mz[i + sz] : 0.0;
    const double z0 = (z != 0) ? Mz[i - sz] : 0.0;
    const double a = __dmul_rn(__dsub_rn(x2, x0), h.hx);
    const double b = __dmul_rn(__dsub_rn(y2, y0), h.hy);
    const double c = __dmul_rn(__dsub_rn(z2, z0), h.hz);
    return (float)__dadd_rn(__dadd_rn(a, b), c);
}

// index of cell (x, y, z) in the box-major BF16 charge layout of the
// tensor-core near field, [Z][nby][nbx][8][8] (leaf side 8)
__device__ __forceinline__ long long ntc_index(int x, int y, int z, int nbx, int nby)
{
    return (((long long)z * nby + (y >> 3)) * nbx + (x >> 3)) * 64 + (y & 7) * 8 + (x & 7);
}

// effective field at cell i from phi (FP32) and the FP64 stage state
__device__ __forceinline__ void field_soa(const float *__restrict__ phi, const double *__restrict__ M, long long i,
                                          int x, int y, int z, const GridK &g, const PhysK &p, const double he[3],
                                          double H[3])
{
    const long long sy = g.X, sz = (long long)g.X * g.Y;
    H[0] = he[0];
    H[1] = he[1];
    H[2] = he[2];
    if (p.demag) {
        double x2 = (x != g.X - 1) ? (double)phi[i + 1] : 0.0;
        double x0 = (x != 0) ? (double)phi[i - 1] : 0.0;
        double y2 = (y != g.Y - 1) ? (double)phi[i + sy] : 0.0;
        double y0 = (y != 0) ? (double)phi[i - sy] : 0.0;
        double z2 = (z != g.Z - 1) ? (double)phi[i + sz] : 0.0;
        double z0 = (z != 0) ? (double)phi[i - sz] : 0.0;
        H[0] += p.hgx * (x2 - x0);
        H[1] += p.hgy * (y2 - y0);
        H[2] += p.hgz * (z2 - z0);
    }
    if (p.exchange) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const double *Mc = M + c * g.N;
            double m0 = Mc[i];
            double xp = (x != g.X - 1) ? Mc[i + 1] : 0.0;
            double xm = (x != 0) ? Mc[i - 1] : 0.0;
            double yp = (y != g.Y - 1) ? Mc[i + sy] : 0.0;
            double ym = (y != 0) ? Mc[i - sy] : 0.0;
            double zp = (z != g.Z - 1) ? Mc[i + sz] : 0.0;
            double zm = (z != 0) ? Mc[i - sz] : 0.0;
            H[c] += (xp + xm - 2 * m0) * p.ecx + (yp + ym - 2 * m0) * p.ecy + (zp + zm - 2 * m0) * p.ecz;
        }
    }
}

// ode_functions.cpp:11-18
__device__ __forceinline__ void llg(const double m[3], const double h[3], const PhysK &p, double k[3])
{
    const double cx = m[1] * h[2] - m[2] * h[1];
    const double cy = m[2] * h[0] - m[0] * h[2];
    const double cz = m[0] * h[1] - m[1] * h[0];
    const double ex = m[1] * cz - m[2] * cy;
    const double ey = m[2] * cx - m[0] * cz;
    const double ez = m[0] * cy - m[1] * cx;
    const double a = p.llg_a;
    k[0] = -p.gamma * cx - a * ex;
    k[1] = -p.gamma * cy - a * ey;
    k[2] = -p.gamma * cz - a * ez;
}

}  // namespace mmsdev
