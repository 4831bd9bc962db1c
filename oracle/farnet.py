"""Test infrastructure only: FP64 numpy restatement of the learned far-field
operator (the network of mms-gpu_b200/mmsb200/farnet.py and of the library's
mms_farnet_* kernels): its forward pass, its relative-L2 loss and the gradient
of that loss with respect to every weight, written out adjoint by adjoint, plus
the exact near field it is paired with.  It checks the GPU forward, gradient
and inference kernels.  Either network width (the default 16 + 8 channels or
the accurate 24 + 16) is read off the length of the weight vector.

The far field it replaces is the reference's far-field pass (fmm_calc.cu:
186-222, multipole-to-potential over the interaction lists of Box.cu:171-195);
the near field (fmm_calc.cu:230-257 in the reference, here the full 3 x 3
leaf-box neighbourhood over all layers) stays exact.
"""
from __future__ import annotations

import math

import numpy as np

S, Z = 8, 3
C = S * S * Z
NE, NO = 16, 8          # the default network's even / odd channels
NR = NE + NO
OSZ = NE * NE + NO * NO
WIDTHS = ((16, 8), (24, 16))  # the default and the accurate network
NSLOT = 49
CHILD = [(0, 0), (1, 0), (0, 1), (1, 1)]  # (cx, cy), index cy * 2 + cx


def _layout(depths, ne=NE, no=NO):
    nr, osz = ne + no, ne * ne + no * no
    off, o = {}, 0
    off["W"] = o; o += C * nr
    off["V"] = o; o += nr * C
    for d in range(depths):
        off[("M2L", d)] = o; o += NSLOT * osz
    for d in range(1, depths):
        off[("M2M", d)] = o; o += 4 * osz
        off[("L2L", d)] = o; o += 4 * osz
    off["total"] = o
    return off


def width_of(size, depths):
    """(ne, no) of a weight vector of `size` floats"""
    for ne, no in WIDTHS:
        if _layout(depths, ne, no)["total"] == size:
            return ne, no
    raise AssertionError(f"{size} weights match no network width")


def _full(v, ne, no):
    """one packed [even j][k] + [odd j][k] block pair -> full (ne + no)^2 [j][k]"""
    T = np.zeros((ne + no, ne + no))
    T[:ne, :ne] = v[:ne * ne].reshape(ne, ne)
    T[ne:, ne:] = v[ne * ne:].reshape(no, no)
    return T


def _pack(T, ne):
    return np.concatenate([T[:ne, :ne].ravel(), T[ne:, ne:].ravel()])


def unpack(w, depths):
    w = np.asarray(w, np.float64)
    ne, no = width_of(w.size, depths)
    nr, osz = ne + no, ne * ne + no * no
    off = _layout(depths, ne, no)
    t = {"W": w[off["W"]:off["W"] + C * nr].reshape(C, nr),
         "V": w[off["V"]:off["V"] + nr * C].reshape(nr, C), "ne": ne}
    for d in range(depths):
        blk = w[off[("M2L", d)]:off[("M2L", d)] + NSLOT * osz].reshape(NSLOT, osz)
        t[("M2L", d)] = np.stack([_full(b, ne, no) for b in blk])
    for d in range(1, depths):
        for name in ("M2M", "L2L"):
            blk = w[off[(name, d)]:off[(name, d)] + 4 * osz].reshape(4, osz)
            t[(name, d)] = np.stack([_full(b, ne, no) for b in blk])
    return t


def pack(g, depths):
    ne = g["ne"]
    no = g["W"].shape[1] - ne
    nr, osz = ne + no, ne * ne + no * no
    off = _layout(depths, ne, no)
    w = np.zeros(off["total"])
    w[off["W"]:off["W"] + C * nr] = g["W"].ravel()
    w[off["V"]:off["V"] + nr * C] = g["V"].ravel()
    for d in range(depths):
        w[off[("M2L", d)]:off[("M2L", d)] + NSLOT * osz] = np.concatenate([_pack(T, ne) for T in g[("M2L", d)]])
    for d in range(1, depths):
        for name in ("M2M", "L2L"):
            w[off[(name, d)]:off[(name, d)] + 4 * osz] = np.concatenate([_pack(T, ne) for T in g[(name, d)]])
    return w


def levels(X, Y):
    nleaf = max(1, -(-max(X, Y) // S))
    L = 0
    while (1 << L) < nleaf:
        L += 1
    return L


def boxes(u, L):
    """[Z][Y][X] -> [nb][nb][C] leaf boxes (zero padded), c = z*64 + y*8 + x"""
    Zz, Y, X = u.shape
    nb = 1 << L
    q = np.zeros((Z, nb * S, nb * S))
    q[:, :Y, :X] = u
    return q.reshape(Z, nb, S, nb, S).transpose(1, 3, 0, 2, 4).reshape(nb, nb, C)


def unboxes(b, Y, X):
    nb = b.shape[0]
    return b.reshape(nb, nb, Z, S, S).transpose(2, 0, 3, 1, 4).reshape(Z, nb * S, nb * S)[:, :Y, :X]


def _il_mask(n, ox, oy):
    """targets t of an n x n level whose interaction list holds o = (ox, oy)"""
    par = np.arange(n) & 1
    mx = (par - 3 <= ox) & (ox <= par + 2)
    my = (par - 3 <= oy) & (oy <= par + 2)
    return (my[:, None] & mx[None, :]).astype(np.float64)[:, :, None]


def _offsets():
    return [(ox, oy) for oy in range(-3, 4) for ox in range(-3, 4) if max(abs(ox), abs(oy)) >= 2]


def _shift(A, ox, oy):
    """B[t] = A[t - o], zero where t - o is off the level"""
    n = A.shape[0]
    P = np.pad(A, ((3, 3), (3, 3), (0, 0)))
    return P[3 - oy:3 - oy + n, 3 - ox:3 - ox + n]


def forward(w, u, depths=5):
    """far field of the dimensionless charge u [Z][Y][X] (cell units); returns
    (phi [Z][Y][X], activations for the gradient)"""
    u = np.asarray(u, np.float64)
    _, Y, X = u.shape
    L = levels(X, Y)
    assert 2 <= L <= depths + 1, "grid needs 2 .. depths + 1 quadtree levels"
    t = unpack(w, depths)
    q = boxes(u, L)
    M = {L: q @ t["W"]}
    for l in range(L - 1, 1, -1):
        A = t[("M2M", L - l)]
        M[l] = sum(M[l + 1][cy::2, cx::2] @ A[c] for c, (cx, cy) in enumerate(CHILD))
    Lp, Lf = {}, {}
    for l in range(2, L + 1):
        n = 1 << l
        T = t[("M2L", L - l)]
        acc = np.zeros((n, n, t["W"].shape[1]))
        for ox, oy in _offsets():
            acc += _il_mask(n, ox, oy) * (_shift(M[l], ox, oy) @ T[(oy + 3) * 7 + ox + 3])
        Lp[l] = acc
        f = acc.copy()
        if l > 2:
            B = t[("L2L", L - (l - 1))]
            for c, (cx, cy) in enumerate(CHILD):
                f[cy::2, cx::2] += Lf[l - 1] @ B[c]
        Lf[l] = f
    phi_b = Lf[L] @ t["V"]
    return unboxes(phi_b, Y, X), {"q": q, "M": M, "Lf": Lf, "L": L, "t": t}


def loss_and_gradient(w, batch, depths=5):
    """batch: list of (u, far, nrm2); loss = mean_b |net(u_b) - far_b|^2 / nrm2_b
    (nrm2_b: |phi_b|^2 of the total potential); returns (loss, gradient vector)"""
    g = None
    loss = 0.0
    nb_ = len(batch)
    for u, far, nrm2 in batch:
        phi, a = forward(w, u, depths)
        r = phi - far
        loss += float((r * r).sum() / nrm2) / nb_
        _, Y, X = r.shape
        L, t, M, Lf, q = a["L"], a["t"], a["M"], a["Lf"], a["q"]
        dphi = boxes(2.0 * r / nrm2 / nb_, L)
        gr = {k: np.zeros_like(v) for k, v in t.items() if k != "ne"}
        gr["ne"] = t["ne"]
        gr["V"] += np.einsum("abk,abc->kc", Lf[L], dphi)
        dLf = {L: dphi @ t["V"].T}
        for l in range(L, 2, -1):
            B = t[("L2L", L - (l - 1))]
            dp = np.zeros_like(Lf[l - 1])
            for c, (cx, cy) in enumerate(CHILD):
                dch = dLf[l][cy::2, cx::2]
                dp += dch @ B[c].T
                gr[("L2L", L - (l - 1))][c] += np.einsum("abj,abk->jk", Lf[l - 1], dch)
            dLf[l - 1] = dp
        dM = {l: np.zeros_like(M[l]) for l in M}
        for l in range(2, L + 1):
            n = 1 << l
            T = t[("M2L", L - l)]
            for ox, oy in _offsets():
                s = (oy + 3) * 7 + ox + 3
                dLm = _il_mask(n, ox, oy) * dLf[l]          # targets whose list holds o
                # dM[t - o] += T dL[t]  <=>  dM[s] += (shift by -o of dLm) T^T
                dM[l] += _shift(dLm @ T[s].T, -ox, -oy)
                gr[("M2L", L - l)][s] += np.einsum("abj,abk->jk", _shift(M[l], ox, oy), dLm)
        # upward adjoint: dM[l + 1] gets M2M^T dM[l], from the top down
        for l in range(2, L):
            A = t[("M2M", L - l)]
            for c, (cx, cy) in enumerate(CHILD):
                dM[l + 1][cy::2, cx::2] += dM[l] @ A[c].T
                gr[("M2M", L - l)][c] += np.einsum("abj,abk->jk", M[l + 1][cy::2, cx::2], dM[l])
        gr["W"] += np.einsum("abc,abk->ck", q, dM[L])
        # keep only what the block-diagonal layout stores
        gv = pack(gr, depths)
        g = gv if g is None else g + gv
    return loss, g


def near_field(u):
    """exact near field of u [Z][Y][X] (cell units, cubic cells): the sum of
    u_j / |r_ij| over the cells j of the 3 x 3 leaf-box neighbourhood of i's
    leaf box, all layers, j != i"""
    u = np.asarray(u, np.float64)
    _, Y, X = u.shape
    L = levels(X, Y)
    q = boxes(u, L)
    nb = q.shape[0]
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(S), np.arange(S), indexing="ij")
    cells = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1).astype(np.float64)
    P = np.pad(q, ((1, 1), (1, 1), (0, 0)))
    out = np.zeros_like(q)
    for oy in (-1, 0, 1):
        for ox in (-1, 0, 1):
            d = (cells[None, :, :] + np.array([ox * S, oy * S, 0.0])) - cells[:, None, :]
            r = np.sqrt((d * d).sum(-1))
            G = np.where(r > 0, 1.0 / np.where(r > 0, r, 1.0), 0.0)
            out += P[1 + oy:1 + oy + nb, 1 + ox:1 + ox + nb] @ G.T
    return unboxes(out, Y, X)
