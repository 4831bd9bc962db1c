// Host-side construction of the FMM translation operators (FP64, once per plan).
//
// Basis: 3-D solid harmonics with the Greengard-Rokhlin normalisation
//   Y_n^m(t, p) = sqrt((n-|m|)!/(n+|m|)!) P_n^|m|(cos t) e^{i m p}
// (P without the Condon-Shortley phase).  The reference expands in the same
// spherical harmonics, unnormalised and limited to l <= 4
// (numerics.cu:59-114); here any order P works because every length is in
// units of the box width of its level.
//
// Translation theorems (multipole-to-multipole, multipole-to-local,
// local-to-local) follow Greengard & Rokhlin's published formulas with the
// factors A_n^m = (-1)^n / sqrt((n-m)!(n+m)!) and J = i^(...) phases.  Each
// complex-linear map on conjugate-symmetric coefficient sets is turned into a
// real matrix on the (re, im) pairs of m >= 0, ordered by the parity of n + m:
// translations within the z = 0 plane never couple the two parities, so the
// kernels apply two half-size blocks.
#include "fmm_ops.hpp"

#include <math.h>

#include <complex>
#include <vector>

namespace fmmops {

using cd = std::complex<double>;

static double fact(int n)
{
    double f = 1.0;
    for (int i = 2; i <= n; i++) f *= i;
    return f;
}

static double Acoef(int n, int m) { return ((n & 1) ? -1.0 : 1.0) / sqrt(fact(n - m) * fact(n + m)); }

// i^e for integer e
static cd ipow(int e)
{
    switch (((e % 4) + 4) % 4) {
    case 0: return cd(1, 0);
    case 1: return cd(0, 1);
    case 2: return cd(-1, 0);
    default: return cd(0, -1);
    }
}

// Y_n^m for 0 <= m <= n <= nmax at (theta, phi); Y[n*(nmax+1)+m]
static void ylm(int nmax, double th, double ph, std::vector<cd> &Y)
{
    const int S = nmax + 1;
    std::vector<double> P((size_t)S * S, 0.0);
    const double x = cos(th), s = sin(th) < 0 ? 0 : sin(th);
    P[0] = 1.0;
    for (int m = 1; m <= nmax; m++) P[m * S + m] = (2 * m - 1) * s * P[(m - 1) * S + m - 1];
    for (int m = 0; m < nmax; m++) P[(m + 1) * S + m] = (2 * m + 1) * x * P[m * S + m];
    for (int m = 0; m <= nmax; m++)
        for (int n = m + 2; n <= nmax; n++)
            P[n * S + m] = ((2 * n - 1) * x * P[(n - 1) * S + m] - (n + m - 1) * P[(n - 2) * S + m]) / (n - m);
    Y.assign((size_t)S * S, cd(0, 0));
    for (int n = 0; n <= nmax; n++)
        for (int m = 0; m <= n; m++)
            Y[n * S + m] = sqrt(fact(n - m) / fact(n + m)) * P[n * S + m] * std::polar(1.0, m * ph);
}

static cd Yget(const std::vector<cd> &Y, int nmax, int n, int m)
{
    const int S = nmax + 1;
    return m >= 0 ? Y[n * S + m] : std::conj(Y[n * S - m]);
}

static void sph(double x, double y, double z, double &r, double &th, double &ph)
{
    r = sqrt(x * x + y * y + z * z);
    th = (r > 0) ? acos(std::max(-1.0, std::min(1.0, z / r))) : 0.0;
    ph = atan2(y, x);
}

Layout::Layout(int P_) : P(P_)
{
    for (int par = 0; par < 2; par++)
        for (int n = 0; n <= P; n++)
            for (int m = 0; m <= n; m++)
                if (((n + m) & 1) == par) {
                    pn.push_back(n);
                    pm.push_back(m);
                }
    NR = 2 * (int)pn.size();
    NE = 0;
    for (size_t i = 0; i < pn.size(); i++)
        if (((pn[i] + pm[i]) & 1) == 0) NE += 2;
    index.assign((size_t)(P + 1) * (P + 1), -1);
    for (size_t i = 0; i < pn.size(); i++) index[pn[i] * (P + 1) + pm[i]] = (int)i;
}

// complex coefficient (n, m), m may be negative, from a real vector
static cd coef(const Layout &L, const double *v, int n, int m)
{
    const int i = L.index[n * (L.P + 1) + (m < 0 ? -m : m)];
    cd z(v[2 * i], v[2 * i + 1]);
    return m < 0 ? std::conj(z) : z;
}

// column-by-column real matrix (row-major NR x NR) of a complex map given as
// out(j, k >= 0) = fn(in, j, k)
template <class F>
static std::vector<double> real_operator(const Layout &L, F fn)
{
    const int NR = L.NR;
    std::vector<double> T((size_t)NR * NR, 0.0), e(NR, 0.0);
    for (int col = 0; col < NR; col++) {
        std::fill(e.begin(), e.end(), 0.0);
        e[col] = 1.0;
        for (size_t i = 0; i < L.pn.size(); i++) {
            const cd o = fn(e.data(), L.pn[i], L.pm[i]);
            T[(size_t)(2 * i) * NR + col] = o.real();
            T[(size_t)(2 * i + 1) * NR + col] = o.imag();
        }
    }
    return T;
}

std::vector<double> m2m(const Layout &L, double dx, double dy, double dz)
{
    const int P = L.P;
    double rho, al, be;
    sph(dx, dy, dz, rho, al, be);
    std::vector<cd> Y;
    ylm(P, al, be, Y);
    return real_operator(L, [&](const double *v, int j, int k) {
        cd s(0, 0);
        for (int n = 0; n <= j; n++)
            for (int m = -n; m <= n; m++) {
                if (abs(k - m) > j - n) continue;
                // child coefficients are in child units (half width): M_n * 2^-n in parent units
                const cd Mc = coef(L, v, j - n, k - m) / pow(2.0, j - n);
                s += Mc * ipow(abs(k) - abs(m) - abs(k - m)) * Acoef(n, m) * Acoef(j - n, k - m) * pow(rho, n) *
                     Yget(Y, P, n, -m) / Acoef(j, k);
            }
        return s;
    });
}

std::vector<double> m2l(const Layout &L, double dx, double dy, double dz)
{
    const int P = L.P;
    double rho, al, be;
    sph(dx, dy, dz, rho, al, be);
    std::vector<cd> Y;
    ylm(2 * P, al, be, Y);
    return real_operator(L, [&](const double *v, int j, int k) {
        cd s(0, 0);
        for (int n = 0; n <= P; n++)
            for (int m = -n; m <= n; m++)
                s += coef(L, v, n, m) * ipow(abs(k - m) - abs(k) - abs(m)) * Acoef(n, m) * Acoef(j, k) *
                     Yget(Y, 2 * P, j + n, m - k) / (((n & 1) ? -1.0 : 1.0) * Acoef(j + n, m - k) * pow(rho, j + n + 1));
        return s;
    });
}

std::vector<double> l2l(const Layout &L, double dx, double dy, double dz)
{
    const int P = L.P;
    double rho, al, be;
    sph(dx, dy, dz, rho, al, be);
    std::vector<cd> Y;
    ylm(P, al, be, Y);
    return real_operator(L, [&](const double *v, int j, int k) {
        cd s(0, 0);
        for (int n = j; n <= P; n++)
            for (int m = -n; m <= n; m++) {
                if (abs(m - k) > n - j) continue;
                s += coef(L, v, n, m) * ipow(abs(m) - abs(m - k) - abs(k)) * Acoef(n - j, m - k) * Acoef(j, k) *
                     Yget(Y, P, n - j, m - k) * pow(rho, n - j) / ((((n + j) & 1) ? -1.0 : 1.0) * Acoef(n, m));
            }
        return s / pow(2.0, j + 1);  // parent units -> child units
    });
}

void p2m_l2p(const Layout &L, const std::vector<double> &rx, const std::vector<double> &ry,
             const std::vector<double> &rz, std::vector<double> &W, std::vector<double> &V)
{
    const int NR = L.NR, C = (int)rx.size(), P = L.P;
    W.assign((size_t)NR * C, 0.0);
    V.assign((size_t)C * NR, 0.0);
    std::vector<cd> Y;
    for (int c = 0; c < C; c++) {
        double r, th, ph;
        sph(rx[c], ry[c], rz[c], r, th, ph);
        ylm(P, th, ph, Y);
        for (size_t i = 0; i < L.pn.size(); i++) {
            const int n = L.pn[i], m = L.pm[i];
            const cd y = Y[n * (P + 1) + m] * pow(r, n);
            // M_n^m = sum q r^n conj(Y_n^m)
            W[(size_t)(2 * i) * C + c] = y.real();
            W[(size_t)(2 * i + 1) * C + c] = -y.imag();
            // phi = sum_n [Re(L_n^0 Y_n^0) + 2 sum_{m>0} Re(L_n^m Y_n^m)] r^n
            const double f = (m == 0) ? 1.0 : 2.0;
            V[(size_t)c * NR + 2 * i] = f * y.real();
            V[(size_t)c * NR + 2 * i + 1] = -f * y.imag();
        }
    }
}

}  // namespace fmmops
