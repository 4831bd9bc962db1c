"""Test infrastructure only: FP64 numpy restatement of this project's FMM.

The reference's "FMM" (fmm_calc.cu:20-408) is a tree code: P2M straight from
the charges at every level, M2P into the cells of up to 27 interaction boxes,
leaf P2P to the 8 same-layer neighbours plus the same cell in other layers.
This project replaces it with a full FMM on the same quadtree (the one the
reference builds in Box.cu:14-234, made implicit): P2M at the leaves,
M2M up, M2L over the same interaction lists (children of the parent's
neighbours that are not neighbours, <= 27, Box.cu:171-195), L2L down, L2P at
the leaves, and an exact P2P over each leaf's 3x3 neighbourhood, all layers.

Expansions are 3-D solid harmonics (Greengard-Rokhlin normalisation,
Y_n^m = sqrt((n-|m|)!/(n+|m|)!) P_n^|m|(cos t) e^{i m p}); the reference uses
the same basis unnormalised with l <= 4 (numerics.cu:59-114).  Lengths are in
units of the box width of each level, which removes the FP32 overflow the
reference hits at P = 4 (fmm_calc.cu:203) and makes every translation
operator level independent.

This module is the checker for the GPU FMM: the same plan, in FP64, written
independently of the CUDA code.
"""
from __future__ import annotations

from math import factorial

import numpy as np


def _lpmv_nocs(nmax, x):
    """P_n^m(x) without the Condon-Shortley phase, n,m <= nmax, as [n][m]"""
    x = np.asarray(x, np.float64)
    P = np.zeros((nmax + 1, nmax + 1) + x.shape)
    s = np.sqrt(np.maximum(0.0, 1 - x * x))
    P[0, 0] = 1.0
    for m in range(1, nmax + 1):
        P[m, m] = (2 * m - 1) * s * P[m - 1, m - 1]
    for m in range(0, nmax):
        P[m + 1, m] = (2 * m + 1) * x * P[m, m]
    for m in range(0, nmax + 1):
        for n in range(m + 2, nmax + 1):
            P[n, m] = ((2 * n - 1) * x * P[n - 1, m] - (n + m - 1) * P[n - 2, m]) / (n - m)
    return P


def ylm_all(nmax, th, ph):
    """Y_n^m for m >= 0, shape [n][m] + shape(th)"""
    P = _lpmv_nocs(nmax, np.cos(th))
    Y = np.zeros(P.shape, np.complex128)
    for n in range(nmax + 1):
        for m in range(n + 1):
            Y[n, m] = np.sqrt(factorial(n - m) / factorial(n + m)) * P[n, m] * np.exp(1j * m * np.asarray(ph))
    return Y


def _Y(Yall, n, m):
    return Yall[n, m] if m >= 0 else np.conj(Yall[n, -m])


def _A(n, m):
    return (-1) ** n / np.sqrt(float(factorial(n - m)) * float(factorial(n + m)))


def _sph(v):
    x, y, z = v
    r = np.sqrt(x * x + y * y + z * z)
    th = np.arccos(np.clip(z / r, -1, 1)) if r > 0 else 0.0
    return r, th, np.arctan2(y, x)


class Layout:
    """real coefficient vector: (n, m >= 0) pairs split by the parity of n + m
    (even block first), each pair stored as (re, im).  In-plane translations
    never mix the two blocks."""

    def __init__(self, P):
        self.P = P
        pairs = [(n, m) for n in range(P + 1) for m in range(n + 1)]
        even = [p for p in pairs if (p[0] + p[1]) % 2 == 0]
        odd = [p for p in pairs if (p[0] + p[1]) % 2 == 1]
        self.pairs = even + odd
        self.n_even = 2 * len(even)
        self.NR = 2 * len(pairs)
        self.index = {p: i for i, p in enumerate(self.pairs)}

    def to_complex(self, v):
        """real vector -> dict (n, m) for all m (conjugate-completed)"""
        c = {}
        for i, (n, m) in enumerate(self.pairs):
            z = v[2 * i] + 1j * v[2 * i + 1]
            c[(n, m)] = z
            if m > 0:
                c[(n, -m)] = np.conj(z)
        return c

    def to_real(self, c):
        v = np.zeros(self.NR)
        for i, (n, m) in enumerate(self.pairs):
            v[2 * i] = c[(n, m)].real
            v[2 * i + 1] = c[(n, m)].imag
        return v


def _real_operator(lay: Layout, fn):
    """real matrix of a complex-linear map on conjugate-symmetric coefficient
    sets (built column by column)"""
    T = np.zeros((lay.NR, lay.NR))
    for col in range(lay.NR):
        e = np.zeros(lay.NR)
        e[col] = 1.0
        T[:, col] = lay.to_real(fn(lay.to_complex(e)))
    return T


def op_m2m(lay, d):
    """child multipole (child units: half width) -> parent multipole (parent
    units); d = child centre - parent centre in parent units"""
    P = lay.P
    rho, al, be = _sph(np.asarray(d, np.float64))
    Y = ylm_all(P, al, be)

    def fn(Mc):
        Mc = {k: v / 2.0 ** k[0] for k, v in Mc.items()}  # child units -> parent units
        out = {}
        for j in range(P + 1):
            for k in range(j + 1):
                s = 0j
                for n in range(j + 1):
                    for m in range(-n, n + 1):
                        if abs(k - m) > j - n:
                            continue
                        s += (Mc[(j - n, k - m)] * (1j) ** (abs(k) - abs(m) - abs(k - m)) * _A(n, m) *
                              _A(j - n, k - m) * rho ** n * _Y(Y, n, -m) / _A(j, k))
                out[(j, k)] = s
        return out
    return _real_operator(lay, fn)


def op_m2l(lay, d):
    """source multipole -> target local, same level; d = source centre -
    target centre in level units"""
    P = lay.P
    rho, al, be = _sph(np.asarray(d, np.float64))
    Y = ylm_all(2 * P, al, be)

    def fn(M):
        out = {}
        for j in range(P + 1):
            for k in range(j + 1):
                s = 0j
                for n in range(P + 1):
                    for m in range(-n, n + 1):
                        s += (M[(n, m)] * (1j) ** (abs(k - m) - abs(k) - abs(m)) * _A(n, m) * _A(j, k) *
                              _Y(Y, j + n, m - k) / ((-1) ** n * _A(j + n, m - k) * rho ** (j + n + 1)))
                out[(j, k)] = s
        return out
    return _real_operator(lay, fn)


def op_l2l(lay, d):
    """parent local (parent units) -> child local (child units); d = parent
    centre - child centre in parent units"""
    P = lay.P
    rho, al, be = _sph(np.asarray(d, np.float64))
    Y = ylm_all(P, al, be)

    def fn(L):
        out = {}
        for j in range(P + 1):
            for k in range(j + 1):
                s = 0j
                for n in range(j, P + 1):
                    for m in range(-n, n + 1):
                        if abs(m - k) > n - j:
                            continue
                        s += (L[(n, m)] * (1j) ** (abs(m) - abs(m - k) - abs(k)) * _A(n - j, m - k) * _A(j, k) *
                              _Y(Y, n - j, m - k) * rho ** (n - j) / ((-1) ** (n + j) * _A(n, m)))
                out[(j, k)] = s / 2.0 ** (j + 1)  # parent units -> child units
        return out
    return _real_operator(lay, fn)


class Plan:
    """FMM plan for an X x Y x Z grid of (dx, dy, dz) cells, order P, leaf side s."""

    def __init__(self, X, Y, Z, dx, dy, dz, P=6, s=4):
        self.X, self.Y, self.Z = X, Y, Z
        self.dx, self.dy, self.dz = dx, dy, dz
        self.P, self.s = P, s
        nleaf = max(1, -(-max(X, Y) // s))
        self.L = int(np.ceil(np.log2(nleaf))) if nleaf > 1 else 0
        self.nb = 2 ** self.L
        self.lay = Layout(P)
        self.ay = dy / dx  # y length of a box in x-width units
        self.az = dz / dx
        self.zc = (Z - 1) / 2.0
        lay = self.lay
        self.m2m = {}
        self.l2l = {}
        for cy in (0, 1):
            for cx in (0, 1):
                dvec = ((cx - 0.5) / 2, (cy - 0.5) / 2 * self.ay, 0.0)
                self.m2m[(cx, cy)] = op_m2m(lay, dvec)
                self.l2l[(cx, cy)] = op_l2l(lay, (-dvec[0], -dvec[1], 0.0))
        self.m2l = {}
        for oy in range(-3, 4):
            for ox in range(-3, 4):
                if max(abs(ox), abs(oy)) >= 2:
                    self.m2l[(ox, oy)] = op_m2l(lay, (-ox, -oy * self.ay, 0.0))
        # P2M / L2P matrices over the s x s x Z cells of a leaf (z, y, x order)
        zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(s), np.arange(s), indexing="ij")
        rel = np.stack([(xx - (s - 1) / 2) / s, (yy - (s - 1) / 2) / s * self.ay,
                        (zz - self.zc) / s * self.az], -1).reshape(-1, 3)
        r = np.linalg.norm(rel, axis=1)
        th = np.where(r > 0, np.arccos(np.clip(rel[:, 2] / np.where(r > 0, r, 1), -1, 1)), 0.0)
        ph = np.arctan2(rel[:, 1], rel[:, 0])
        Yc = ylm_all(P, th, ph)
        C = len(rel)
        self.W = np.zeros((lay.NR, C))   # multipole = W q
        self.V = np.zeros((C, lay.NR))   # phi = V local
        for i, (n, m) in enumerate(lay.pairs):
            # M_n^m = sum q r^n Y_n^{-m} = sum q r^n conj(Y_n^m)
            v = r ** n * np.conj(Yc[n, m])
            self.W[2 * i] = v.real
            self.W[2 * i + 1] = v.imag
            # phi = sum_{n, m} L_n^m Y_n^m r^n = Re(L_n^0 Y_n^0) r^n + 2 Re(L_n^m Y_n^m) r^n
            w = r ** n * Yc[n, m] * (1.0 if m == 0 else 2.0)
            self.V[:, 2 * i] = w.real
            self.V[:, 2 * i + 1] = -w.imag

    def interaction_offsets(self, bx, by):
        """offsets (ox, oy) = target - source of the M2L list of box (bx, by)"""
        px, py = bx & 1, by & 1
        out = []
        for oy in range(py - 3, py + 3):
            for ox in range(px - 3, px + 3):
                if max(abs(ox), abs(oy)) >= 2:
                    out.append((ox, oy))
        return out

    def potential(self, rho):
        """phi_i = sum_{j != i} rho_j dV / |r_i - r_j| via the FMM"""
        X, Y, Z, s, nb, L = self.X, self.Y, self.Z, self.s, self.nb, self.L
        NR = self.lay.NR
        dV = self.dx * self.dy * self.dz
        w_phys = s * self.dx
        q = np.zeros((Z, nb * s, nb * s))
        q[:, :Y, :X] = np.asarray(rho, np.float64).reshape(Z, Y, X) * dV
        # leaf charges per box: [by, bx, C]
        qb = q.reshape(Z, nb, s, nb, s).transpose(1, 3, 0, 2, 4).reshape(nb, nb, -1)
        M = {L: qb @ self.W.T}
        for l in range(L - 1, 1, -1):
            n = 2 ** l
            Ml = np.zeros((n, n, NR))
            ch = M[l + 1]
            for cy in (0, 1):
                for cx in (0, 1):
                    Ml += ch[cy::2, cx::2] @ self.m2m[(cx, cy)].T
            M[l] = Ml
        Lc = {}
        for l in range(2, L + 1):
            n = 2 ** l
            Ll = np.zeros((n, n, NR))
            for by in range(n):
                for bx in range(n):
                    acc = np.zeros(NR)
                    for (ox, oy) in self.interaction_offsets(bx, by):
                        sx, sy = bx - ox, by - oy
                        if 0 <= sx < n and 0 <= sy < n:
                            acc += self.m2l[(ox, oy)] @ M[l][sy, sx]
                    Ll[by, bx] = acc
            if l > 2:
                par = Lc[l - 1]
                for cy in (0, 1):
                    for cx in (0, 1):
                        Ll[cy::2, cx::2] += par @ self.l2l[(cx, cy)].T
            Lc[l] = Ll
        phi_b = np.zeros((nb, nb, Z * s * s))
        if L >= 2:
            phi_b = (Lc[L] @ self.V.T) / w_phys
        phi = phi_b.reshape(nb, nb, Z, s, s).transpose(2, 0, 3, 1, 4).reshape(Z, nb * s, nb * s)
        # exact near field: 3x3 leaf neighbourhood, all layers, self excluded
        near = np.zeros_like(phi)
        zz = np.arange(Z)
        for by in range(nb):
            for bx in range(nb):
                y0, x0 = by * s, bx * s
                ys0, ys1 = max(0, y0 - s), min(nb * s, y0 + 2 * s)
                xs0, xs1 = max(0, x0 - s), min(nb * s, x0 + 2 * s)
                src = q[:, ys0:ys1, xs0:xs1]
                if not src.any():
                    continue
                sz, sy, sx = np.meshgrid(zz, np.arange(ys0, ys1), np.arange(xs0, xs1), indexing="ij")
                for tz in range(Z):
                    for ty in range(y0, y0 + s):
                        for tx in range(x0, x0 + s):
                            R = np.sqrt(((sx - tx) * self.dx) ** 2 + ((sy - ty) * self.dy) ** 2 +
                                        ((sz - tz) * self.dz) ** 2)
                            R[R == 0] = np.inf
                            near[tz, ty, tx] = (src / R).sum()
        return (phi + near)[:, :Y, :X]
