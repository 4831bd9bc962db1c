"""Geometries (material masks) and initial magnetisation states.

Masks are uint8 arrays of shape (zdim, ydim, xdim), non-zero = magnetic.
States are float64 arrays of shape (zdim, ydim, xdim, 3) in A/m, zero at
empty cells.  Following the reference's driver (main.cpp:192-221), material
sits in the layers z = 1 .. zdim-2 (the outer layers are empty padding) unless
``layers="all"`` is asked for.

Random states use numpy's Philox generator seeded explicitly, so every run of
the same seed gives identical bits.
"""
from __future__ import annotations

import numpy as np

MS_PERMALLOY = 8.6e5


def _layers(Z, layers):
    if layers == "all":
        return slice(0, Z)
    if Z < 3:
        raise ValueError("middle-layer geometries need zdim >= 3 (main.cpp:192)")
    return slice(1, Z - 1)


def rng(seed):
    return np.random.Generator(np.random.Philox(seed))


def from_plane(plane, Z, layers="middle"):
    """extrude a (ydim, xdim) 0/1 plane into the material layers"""
    Y, X = plane.shape
    m = np.zeros((Z, Y, X), np.uint8)
    m[_layers(Z, layers)] = (plane != 0).astype(np.uint8)
    return m


def reference_default(X, Y, Z):
    """the reference's built-in mask: a rectangle with a 1-cell empty border
    (main.cpp:119-130)"""
    p = np.zeros((Y, X), np.uint8)
    p[1:Y - 1, 1:X - 1] = 1
    return from_plane(p, Z)


def rectangle(X, Y, Z, layers="middle"):
    return from_plane(np.ones((Y, X), np.uint8), Z, layers)


def ellipse_plane(X, Y, cx, cy, ax, ay):
    y, x = np.meshgrid(np.arange(Y), np.arange(X), indexing="ij")
    return (((x - cx) / ax) ** 2 + ((y - cy) / ay) ** 2 <= 1.0).astype(np.uint8)


def disc(X, Y, Z, r, cx=None, cy=None, layers="middle"):
    cx = (X - 1) / 2 if cx is None else cx
    cy = (Y - 1) / 2 if cy is None else cy
    return from_plane(ellipse_plane(X, Y, cx, cy, r, r), Z, layers)


def disc_lattice(X, Y, Z, r, pitch, layers="middle"):
    """an lattice of discs of radius r (cells) at the given pitch, the first
    centre half a pitch in from the corner"""
    p = np.zeros((Y, X), np.uint8)
    for cy in np.arange(pitch / 2 - 0.5, Y, pitch):
        for cx in np.arange(pitch / 2 - 0.5, X, pitch):
            p |= ellipse_plane(X, Y, cx, cy, r, r)
    return from_plane(p, Z, layers)


def random_blocks_mask(X, Y, Z, frac, block, seed, layers="middle"):
    """about `frac` of the cells removed in random block x block squares"""
    g = rng(seed)
    p = np.ones((Y, X), np.uint8)
    nb = int(round(frac * X * Y / (block * block)))
    removed = 0
    while removed < nb:
        bx = int(g.integers(0, max(1, X // block))) * block
        by = int(g.integers(0, max(1, Y // block))) * block
        if p[by:by + block, bx:bx + block].any():
            p[by:by + block, bx:bx + block] = 0
            removed += 1
    return from_plane(p, Z, layers)


# ---- initial states --------------------------------------------------------

def _place(mask, v, Ms):
    M = np.zeros(mask.shape + (3,))
    M[:] = v
    return M * Ms * (mask[..., None] != 0)


def single_domain(mask, Ms=MS_PERMALLOY, phi=0.0):
    """uniform in-plane state (main.cpp:204-205)"""
    return _place(mask, np.array([np.cos(phi), np.sin(phi), 0.0]), Ms)


def random_sphere(mask, seed, Ms=MS_PERMALLOY):
    """unit vectors uniform on the sphere (u ~ U(-1,1), phi ~ U(0, 2 pi))"""
    g = rng(seed)
    u = g.uniform(-1, 1, mask.shape)
    ph = g.uniform(0, 2 * np.pi, mask.shape)
    s = np.sqrt(1 - u * u)
    v = np.stack([s * np.cos(ph), s * np.sin(ph), u], -1)
    return v * Ms * (mask[..., None] != 0)


def random_inplane(mask, seed, Ms=MS_PERMALLOY):
    """random in-plane angle per cell (the reference's IC = 2, main.cpp:206-207)"""
    g = rng(seed)
    ph = g.uniform(0, 2 * np.pi, mask.shape)
    v = np.stack([np.cos(ph), np.sin(ph), np.zeros_like(ph)], -1)
    return v * Ms * (mask[..., None] != 0)


def vortex_quadrants(mask, Ms=MS_PERMALLOY):
    """the reference's 4-quadrant vortex (IC = 1, main.cpp:208-216)"""
    Z, Y, X = mask.shape
    y, x = np.meshgrid(np.arange(Y), np.arange(X), indexing="ij")
    ph = np.where((x - X // 2 > 0) & (y - Y // 2 > 0), -np.pi / 4,
                  np.where((x - X // 2 <= 0) & (y - Y // 2 > 0), np.pi / 4,
                           np.where((x - X // 2 <= 0) & (y - Y // 2 <= 0), 3 * np.pi / 4, -3 * np.pi / 4)))
    v = np.stack([np.cos(ph), np.sin(ph), np.zeros_like(ph)], -1)
    return v[None] * Ms * (mask[..., None] != 0)


def vortex(mask, core_r=2.0, jitter_deg=0.0, seed=0, Ms=MS_PERMALLOY, cx=None, cy=None):
    """in-plane circulation phi = atan2(y, x) + pi/2 about the centre, +z core
    within core_r cells, plus an optional seeded Gaussian angular jitter"""
    Z, Y, X = mask.shape
    cx = (X - 1) / 2 if cx is None else cx
    cy = (Y - 1) / 2 if cy is None else cy
    y, x = np.meshgrid(np.arange(Y) - cy, np.arange(X) - cx, indexing="ij")
    ph = np.arctan2(y, x) + np.pi / 2
    th = np.where(np.hypot(x, y) <= core_r, 0.0, np.pi / 2)
    th = np.broadcast_to(th, mask.shape).copy()
    ph = np.broadcast_to(ph, mask.shape).copy()
    if jitter_deg:
        g = rng(seed)
        th = th + np.radians(jitter_deg) * g.standard_normal(mask.shape)
        ph = ph + np.radians(jitter_deg) * g.standard_normal(mask.shape)
    v = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1)
    return v * Ms * (mask[..., None] != 0)


def per_dot_random_inplane(X, Y, Z, r, pitch, seed, Ms=MS_PERMALLOY):
    """disc lattice with one random in-plane direction per dot"""
    g = rng(seed)
    mask = disc_lattice(X, Y, Z, r, pitch)
    M = np.zeros(mask.shape + (3,))
    for cy in np.arange(pitch / 2 - 0.5, Y, pitch):
        for cx in np.arange(pitch / 2 - 0.5, X, pitch):
            dot = from_plane(ellipse_plane(X, Y, cx, cy, r, r), Z)
            ph = g.uniform(0, 2 * np.pi)
            M[dot != 0] = [np.cos(ph), np.sin(ph), 0.0]
    return mask, M * Ms


def ensemble_instances(n, seed=2010, sides=(16, 24, 32, 40, 48, 56, 64), Z=3, bmax=0.05):
    """The batched-ensemble workload: instance i (seed + i) gets sides drawn
    uniformly from `sides`, a rectangle, disc or ellipse mask (material in the
    middle layers), random M on the sphere and a random in-plane constant
    external field with |B| <= bmax tesla.  Returns (dims, masks, Ms, bext)."""
    dims, masks, Ms, bext = [], [], [], []
    for i in range(n):
        g = rng(seed + i)
        X = int(g.choice(sides))
        Y = int(g.choice(sides))
        kind = int(g.integers(0, 3))
        if kind == 0:
            mask = rectangle(X, Y, Z)
        elif kind == 1:
            mask = disc(X, Y, Z, (min(X, Y) - 2) / 2)
        else:
            mask = from_plane(ellipse_plane(X, Y, (X - 1) / 2, (Y - 1) / 2, (X - 2) / 2, (Y - 2) / 3), Z)
        M = random_sphere(mask, seed + 100000 + i)
        b = bmax * np.sqrt(g.uniform(0, 1))
        ph = g.uniform(0, 2 * np.pi)
        dims.append((X, Y, Z))
        masks.append(mask)
        Ms.append(M)
        bext.append((b * np.cos(ph), b * np.sin(ph), 0.0))
    return dims, masks, Ms, bext
