"""The learned far-field operator: layout of its weights and their initial values.

The network maps the cell charge of a thin film (leaf boxes of 8 x 8 cells x 3
layers, cubic cells) to the far-field part of the demag potential, the part the
FMM's P2M / M2M / M2L / L2L / L2P passes produce (fmm_calc.cu:186-222 in the
reference evaluates it by M2P); the exact near field over each leaf box's 3 x 3
neighbourhood is not learned.  It is a linear multilevel convolutional network
over the quadtree of leaf boxes (a U-Net whose skip connections are the
interaction-list convolutions):

    m_leaf[k]  = sum_c W[c][k] q[c]                              encoder (stride-8 conv)
    m_par[k]   = sum_child sum_j M2M_d[child][j][k] m_child[j]    down (2x2 stride-2 conv)
    l_t[k]    += sum_{o in IL(t)} sum_j M2L_d[o][j][k] m_{t-o}[j] lateral (parity-aware 7x7 conv)
    l_child[k]+= sum_j L2L_d[child][j][k] l_par[j]                up (2x2 transposed conv)
    phi[c]     = sum_k V[k][c] l_leaf[k]                          decoder

with q the dimensionless cell charge and phi the dimensionless far field
(q = rho dx / Ms in, phi / (Ms dx) out; for a linear map any common scale of rho
works the same).  IL(t) is the reference's interaction list (children of the
parent's neighbours that are not neighbours, Box.cu:171-195): the offsets o =
target - source in [px-3, px+2] x [py-3, py+2] with max(|ox|, |oy|) >= 2, (px,
py) the target's parity.  d is the depth of the level (0 = leaf), so one set of
weights serves every grid up to 2^(DEPTHS+1) leaf boxes a side.

Channels come in two blocks that never mix: NE channels even and NO channels
odd under the reflection z -> -z of the 3-layer film (the Green's function is
symmetric under it).  Every table is block diagonal.

Initial values: nested (H^2-matrix style) bases from truncated SVDs of the
exact 1/r interactions.  The leaf basis spans the dominant left singular
vectors of a leaf box's interactions with every box outside its near zone; a
parent's basis is the dominant subspace of its children's bases under the
parent-level interactions, so M2M and L2L are the transfer matrices of that
nesting, and M2L is the 1/r kernel compressed into the bases.  At width
16 + 8 this start is about ten times more accurate than the spherical-
harmonic expansion at order 4 (width 30) on disc-lattice films; training on
FMM-generated pairs then fits the weights to the charge distributions of LLG
trajectories.
"""
from __future__ import annotations

import numpy as np

S = 8                 # leaf side (cells)
Z = 3                 # layers
C = S * S * Z         # cells per leaf box, index c = z*64 + y*8 + x
NE, NO = 16, 8        # even / odd channels of the default (trainable) network
NR = NE + NO
OSZ = NE * NE + NO * NO
WIDE = (24, 16)       # even / odd channels of the accurate network (its nested-SVD start)
DEPTHS = 5            # depths 0..4: quadtrees of up to 6 levels (grids up to 512 cells a side)
NSLOT = 49            # M2L offset slots (oy + 3) * 7 + (ox + 3); the 9 near ones stay zero


def layout(depths=DEPTHS, ne=None, no=None):
    """offsets (in floats) of each table in the weight vector of a network
    with ne even and no odd channels (default: NE, NO)"""
    ne = NE if ne is None else ne
    no = NO if no is None else no
    nr, osz = ne + no, ne * ne + no * no
    off = {}
    o = 0
    off["W"] = o; o += C * nr
    off["V"] = o; o += nr * C
    for d in range(depths):
        off[("M2L", d)] = o; o += NSLOT * osz
    for d in range(1, depths):
        off[("M2M", d)] = o; o += 4 * osz
        off[("L2L", d)] = o; o += 4 * osz
    off["total"] = o
    return off


def num_params(depths=DEPTHS, ne=None, no=None):
    return layout(depths, ne, no)["total"]


def width_of(count, depths=DEPTHS):
    """(ne, no) of a weight vector of `count` floats: the default or the wide network"""
    for ne, no in ((NE, NO), WIDE):
        if num_params(depths, ne, no) == count:
            return ne, no
    raise ValueError(f"{count} weights match no network width")


def slot(ox, oy):
    return (oy + 3) * 7 + (ox + 3)


def pack_block(Te, To):
    """[j][k] even block then odd block, flattened"""
    return np.concatenate([np.asarray(Te, np.float64).ravel(), np.asarray(To, np.float64).ravel()])


# ---------------------------------------------------------------- initial values
def _cells():
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(S), np.arange(S), indexing="ij")
    return np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1).astype(np.float64)


def _parity_frames():
    """orthonormal frames of the z-even (2 x 64 dims) and z-odd (64 dims) cell spaces"""
    n = S * S
    Pe = np.zeros((C, 2 * n))
    Po = np.zeros((C, n))
    for i in range(n):
        Pe[n + i, i] = 1.0                                  # middle layer
        Pe[i, n + i] = Pe[2 * n + i, n + i] = 1 / np.sqrt(2)  # (z0 + z2) / sqrt 2
        Po[i, i] = 1 / np.sqrt(2)
        Po[2 * n + i, i] = -1 / np.sqrt(2)                  # (z0 - z2) / sqrt 2
    return Pe, Po


def _leaf_kernels(cells, offsets):
    """1/r between the cells of a leaf box and those of the box at leaf offset
    (dx, dy) (source - target), [len(offsets)][target c][source c]"""
    out = np.empty((len(offsets), C, C))
    for i, (dx, dy) in enumerate(offsets):
        d = (cells[None, :, :] + np.array([dx * S, dy * S, 0.0])) - cells[:, None, :]
        out[i] = 1.0 / np.sqrt((d * d).sum(-1))
    return out


def h2_init(depths=DEPTHS, R=8, Rup=4, ne=None, no=None):
    """weight vector (float64) of the nested-SVD start with ne even and no odd
    channels (default: NE, NO; WIDE for the accurate network)"""
    ne = NE if ne is None else ne
    no = NO if no is None else no
    cells = _cells()
    Pe, Po = _parity_frames()
    width = (ne, no)
    # offsets each depth's compressed kernel is needed at: the M2L (|o| <= 3),
    # the next depth's basis (|2D + child| <= 2 Rup + 1) and its kernels
    need = {depths - 1: 3}
    for d in range(depths - 2, -1, -1):
        need[d] = max(3, 2 * Rup + 1, 2 * need[d + 1] + 1)
    # leaf basis: dominant left singular vectors of the leaf's far interactions
    far = [(dx, dy) for dy in range(-R, R + 1) for dx in range(-R, R + 1) if max(abs(dx), abs(dy)) >= 2]
    Gf = _leaf_kernels(cells, far)
    U = []
    for P, k in ((Pe, ne), (Po, no)):
        A = np.concatenate([P.T @ g @ P for g in Gf], 1)
        U.append(P @ np.linalg.svd(A, full_matrices=False)[0][:, :k])
    del Gf
    # leaf compressed kernels K0(D) = U^T G_D U per block
    D0 = need[0]
    offs = [(dx, dy) for dy in range(-D0, D0 + 1) for dx in range(-D0, D0 + 1) if max(abs(dx), abs(dy)) >= 2]
    K = {}
    for i in range(0, len(offs), 256):
        chunk = offs[i:i + 256]
        G = _leaf_kernels(cells, chunk)
        for o, g in zip(chunk, G):
            K[o] = tuple(U[b].T @ g @ U[b] for b in (0, 1))
    Ks = {0: K}
    E = {}
    child = [(0, 0), (1, 0), (0, 1), (1, 1)]  # index cy * 2 + cx

    def coupled(Kc, D, b):
        """children-basis coupling of two parent boxes at parent offset D (source - target)"""
        k = width[b]
        out = np.zeros((4 * k, 4 * k))
        for a, (tx, ty) in enumerate(child):
            for c, (sx, sy) in enumerate(child):
                out[a * k:(a + 1) * k, c * k:(c + 1) * k] = Kc[(2 * D[0] + sx - tx, 2 * D[1] + sy - ty)][b]
        return out

    for d in range(1, depths):
        Kc = Ks[d - 1]
        farl = [(dx, dy) for dy in range(-Rup, Rup + 1) for dx in range(-Rup, Rup + 1) if max(abs(dx), abs(dy)) >= 2]
        Ed = []
        for b in (0, 1):
            A = np.concatenate([coupled(Kc, D, b) for D in farl], 1)
            Ed.append(np.linalg.svd(A, full_matrices=False)[0][:, :width[b]])
        E[d] = Ed
        Kd = {}
        for dy in range(-need[d], need[d] + 1):
            for dx in range(-need[d], need[d] + 1):
                if max(abs(dx), abs(dy)) >= 2:
                    Kd[(dx, dy)] = tuple(Ed[b].T @ coupled(Kc, (dx, dy), b) @ Ed[b] for b in (0, 1))
        Ks[d] = Kd

    off = layout(depths, ne, no)
    osz = ne * ne + no * no
    w = np.zeros(off["total"])
    Ufull = np.concatenate(U, 1)  # C x NR, even channels first
    w[off["W"]:off["W"] + C * (ne + no)] = Ufull.ravel()          # W[c][k]
    w[off["V"]:off["V"] + (ne + no) * C] = Ufull.T.ravel()        # V[k][c]
    for d in range(depths):
        t = np.zeros((NSLOT, osz))
        for oy in range(-3, 4):
            for ox in range(-3, 4):
                if max(abs(ox), abs(oy)) < 2:
                    continue
                Kd = Ks[d][(-ox, -oy)]  # source - target = -o; rows target channel, cols source channel
                t[slot(ox, oy)] = pack_block(Kd[0].T, Kd[1].T)  # [j = source][k = target]
        w[off[("M2L", d)]:off[("M2L", d)] + NSLOT * osz] = t.ravel()
    for d in range(1, depths):
        m2m = np.zeros((4, osz))
        l2l = np.zeros((4, osz))
        for c in range(4):
            blocks = [E[d][b][c * width[b]:(c + 1) * width[b]] for b in (0, 1)]  # child channel x parent channel
            m2m[c] = pack_block(blocks[0], blocks[1])        # [j = child][k = parent]
            l2l[c] = pack_block(blocks[0].T, blocks[1].T)    # [j = parent][k = child]
        w[off[("M2M", d)]:off[("M2M", d)] + 4 * osz] = m2m.ravel()
        w[off[("L2L", d)]:off[("L2L", d)] + 4 * osz] = l2l.ravel()
    return w


def step_scale(w, floor=1e-3, depths=DEPTHS):
    """per-weight Adam step scale for relative updates: |w_i| plus a floor of
    `floor` x the largest magnitude of w_i's table, so that entries that are
    zero can still move (the near-field M2L slots get 0: they never enter)"""
    w = np.asarray(w, np.float64)
    off = layout(depths)
    s = np.abs(w)
    keys = ["W", "V"] + [("M2L", d) for d in range(depths)] + [(n, d) for d in range(1, depths)
                                                                 for n in ("M2M", "L2L")]
    starts = sorted(off[k] for k in keys) + [off["total"]]
    for a, b in zip(starts[:-1], starts[1:]):
        s[a:b] += floor * np.abs(w[a:b]).max()
    for d in range(depths):
        base = off[("M2L", d)]
        for oy in (-1, 0, 1):
            for ox in (-1, 0, 1):
                o = base + slot(ox, oy) * OSZ
                s[o:o + OSZ] = 0.0
    return s.astype(np.float32)
