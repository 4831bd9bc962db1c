"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs the reference's own CPU code (oracle/_ref/mmsref_harness, built from the
reference sources by ``make -C oracle``) on small seeded inputs and stores
inputs and outputs as .npz.  The reference has no golden vectors or known-answer
tests of its own, so these fixtures are what pins the oracle.

    python tests/golden/make_golden.py

Every fixture records the grid, the cell sizes and the reference entry point.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from oracle import ref  # noqa: E402

MS = 8.6e5


def random_sphere(rng, shape):
    """unit vectors uniform on the sphere (u ~ U(-1,1), phi ~ U(0, 2pi))"""
    u = rng.uniform(-1, 1, shape)
    ph = rng.uniform(0, 2 * np.pi, shape)
    s = np.sqrt(1 - u * u)
    return np.stack([s * np.cos(ph), s * np.sin(ph), u], -1)


def reference_default_geometry(X, Y, Z):
    """main.cpp:119-130,192-221: material in z = 1..Z-2, 1-cell empty border"""
    mat = np.zeros((Z, Y, X), np.uint8)
    mat[1:Z - 1, 1:Y - 1, 1:X - 1] = 1
    return mat


def full_geometry(X, Y, Z):
    mat = np.zeros((Z, Y, X), np.uint8)
    mat[1:Z - 1] = 1
    return mat


def smooth_state(X, Y, Z, mat, rng):
    """a gently curling in-plane state with a small out-of-plane tilt: smooth
    enough that FP32 and FP64 trajectories stay close over a few steps"""
    y, x = np.meshgrid(np.arange(Y), np.arange(X), indexing="ij")
    ph = 0.3 * np.sin(2 * np.pi * x / X) + 0.2 * np.cos(2 * np.pi * y / Y) + rng.uniform(-0.05, 0.05, (Y, X))
    th = np.pi / 2 - 0.1 * np.sin(2 * np.pi * (x + y) / (X + Y))
    v = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1)
    M = np.zeros((Z, Y, X, 3))
    M[:] = v[None]
    return (M * mat[..., None] * MS).astype(np.float32)


def main():
    if not ref.available():
        raise SystemExit("build the reference harness first: make -C oracle")
    rng = np.random.default_rng(2010)
    out = {}

    # 1. stencils on random fields (16x16x3)
    X, Y, Z = 16, 16, 3
    d = (5e-9, 5e-9, 5e-9)
    M = (random_sphere(rng, (Z, Y, X)) * MS).astype(np.float32)
    S = rng.standard_normal((Z, Y, X)).astype(np.float32) * 1e3
    div, grad, exch = ref.stencils(M, S, (X, Y, Z), d)
    np.savez_compressed(os.path.join(HERE, "stencils_16x16x3.npz"), M=M, S=S, div=div, grad=grad, exch=exch,
                        dims=(X, Y, Z), d=d, entry="divergence_3d/gradient_3d/add_exchange_field")

    # 2. potentials: direct on odd, non-square grids; FMM (P=1..3) on 2^k squares
    for (X, Y, Z, d) in [(16, 16, 3, (5e-9, 5e-9, 5e-9)), (24, 10, 3, (5e-9, 4e-9, 1e-8)),
                         (32, 32, 3, (5e-9, 5e-9, 5e-9))]:
        mat = full_geometry(X, Y, Z)
        Mr = (random_sphere(rng, (Z, Y, X)) * MS * mat[..., None]).astype(np.float32)
        g = oracle.Grid(X, Y, Z, *d)
        rho = oracle.divergence_f32(g, Mr)
        phi = ref.potential(rho, (X, Y, Z), d, use_fmm=False)
        rec = dict(rho=rho, phi_direct=phi, dims=(X, Y, Z), d=d, entry="calc_potential_exact")
        if X == Y and (X & (X - 1)) == 0:
            for P in (1, 2, 3):
                rec[f"phi_fmm_P{P}"] = ref.potential(rho, (X, Y, Z), d, use_fmm=True, P=P)
            rec["entry"] = "calc_potential_exact,fmm_calc"
        np.savez_compressed(os.path.join(HERE, f"potential_{X}x{Y}x{Z}.npz"), **rec)

    # 3. Hfield on the reference default geometry, with and without the ramp
    X, Y, Z = 16, 16, 3
    d = (5e-9, 5e-9, 5e-9)
    mat = reference_default_geometry(X, Y, Z)
    M = (random_sphere(rng, (Z, Y, X)) * MS * mat[..., None]).astype(np.float32)
    rec = dict(M=M, material=mat, dims=(X, Y, Z), d=d, entry="Hfield")
    for ext, t in [(0, 0.0), (1, 2.5e-10)]:
        H, q, phi = ref.hfield(M, (X, Y, Z), d, t=t, external=ext)
        rec[f"H_ext{ext}"], rec[f"charge_ext{ext}"], rec[f"phi_ext{ext}"] = H, q, phi
        rec[f"t_ext{ext}"] = t
    H, q, phi = ref.hfield(M, (X, Y, Z), d, use_fmm=True, P=3)
    rec["H_fmm_P3"] = H
    np.savez_compressed(os.path.join(HERE, "hfield_16x16x3.npz"), **rec)

    # 4. fixed-step RK4 trajectory, smooth start, with the ramp field on
    X, Y, Z = 16, 16, 3
    mat = full_geometry(X, Y, Z)
    M = smooth_state(X, Y, Z, mat, rng)
    rec = dict(M0=M, material=mat, dims=(X, Y, Z), d=d, dt=1e-13, entry="rk4_step (time_marching order)")
    for n in (1, 10):
        Mn, Hn = ref.rk4(mat, M, (X, Y, Z), d, 1e-13, n, external=1)
        rec[f"M_{n}"] = Mn
        rec[f"H_{n}"] = Hn
    np.savez_compressed(os.path.join(HERE, "rk4_16x16x3.npz"), **rec)

    # 5. the reference driver with its energy/torque controller (a short run)
    X, Y, Z = 8, 8, 3
    mat = reference_default_geometry(X, Y, Z)
    M = smooth_state(X, Y, Z, mat, rng)
    Mf, rows = ref.march(mat, M, (X, Y, Z), d, finaltime=2e-12, timestep=1e-14)
    np.savez_compressed(os.path.join(HERE, "march_8x8x3.npz"), M0=M, material=mat, M_final=Mf, dynamics=rows,
                        dims=(X, Y, Z), d=d, finaltime=2e-12, timestep=1e-14, entry="time_marching")
    # 6. the reference's own driver main.cpp (CPU build, oracle/_ref/main_ref):
    #    its dynamics.dat for two short runs, for the drop-in test of main.cpp
    #    linked against libmms_refapi.so
    main_ref = os.path.join(os.path.dirname(ref.REF_HARNESS), "main_ref")
    if os.path.exists(main_ref):
        import subprocess
        import tempfile
        rec = {"entry": "main.cpp -> time_marching"}
        for name, args in DROPIN_RUNS.items():
            with tempfile.TemporaryDirectory() as td:
                subprocess.run([main_ref] + args, cwd=td, check=True, stdin=subprocess.DEVNULL,
                               stdout=subprocess.DEVNULL)
                rows = []
                with open(os.path.join(td, args[15], "dynamics.dat")) as f:
                    for line in f:
                        parts = line.replace(",", " ").split()
                        if len(parts) == 9:
                            rows.append([float(v) for v in parts])
                rec[name] = np.array(rows)
                rec[name + "_args"] = np.array(args)
        np.savez_compressed(os.path.join(HERE, "dropin_main_16x16x3.npz"), **rec)
    print("wrote fixtures to", HERE)


# main.cpp positional arguments (main.cpp:49-70): image P finaltime timestep
# width height depth xdim ydim zdim demag exchange external use_fmm use_gpu
# sim_name seed IC
DROPIN_RUNS = {
    "sd": ["dummy.png", "3", "3e-11", "1e-14", "80e-9", "80e-9", "15e-9", "16", "16", "3", "1", "1", "0", "0",
           "0", "sim", "2010", "0"],
    "vortex_ext": ["dummy.png", "3", "2e-11", "1e-14", "80e-9", "80e-9", "15e-9", "16", "16", "3", "1", "1", "1",
                   "0", "0", "sim", "2010", "1"],
}


if __name__ == "__main__":
    main()
