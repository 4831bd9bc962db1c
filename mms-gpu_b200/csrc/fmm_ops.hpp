// FMM translation operators built on the host in FP64 (fmm_ops.cpp).
#pragma once

#include <vector>

namespace fmmops {

// Real coefficient layout: pairs (n, m >= 0), even n + m first, each as (re, im)
struct Layout {
    int P = 0;
    int NR = 0;          // reals per expansion
    int NE = 0;          // reals in the even-parity block (the odd block is NR - NE)
    std::vector<int> pn, pm;
    std::vector<int> index;  // (n, m) -> pair index
    explicit Layout(int P);
};

// row-major NR x NR real matrices
// child multipole (child units) -> parent multipole; (dx,dy,dz) = child - parent centre, parent units
std::vector<double> m2m(const Layout &L, double dx, double dy, double dz);
// source multipole -> target local, same level; (dx,dy,dz) = source - target centre
std::vector<double> m2l(const Layout &L, double dx, double dy, double dz);
// parent local -> child local (child units); (dx,dy,dz) = parent - child centre, parent units
std::vector<double> l2l(const Layout &L, double dx, double dy, double dz);
// P2M weights W (NR x C, row-major) and L2P weights V (C x NR) for C points at
// (rx, ry, rz) relative to the box centre in box-width units
void p2m_l2p(const Layout &L, const std::vector<double> &rx, const std::vector<double> &ry,
             const std::vector<double> &rz, std::vector<double> &W, std::vector<double> &V);

}  // namespace fmmops
