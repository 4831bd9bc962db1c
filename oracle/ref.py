"""Test infrastructure only: run the reference's own CPU code.

``oracle/_ref/mmsref_harness`` is the reference's unmodified CPU sources
(fmm_calc.cu, ode_functions.cpp, vector_functions.cpp, ...) compiled by
``oracle/Makefile`` plus ``oracle/ref_harness.cpp``.  Every call runs in a
fresh process, so the reference's first-call statics (tree, pinned buffers,
sized on the first call: fmm_calc.cu:303-365) never leak between cases.

Arrays follow the reference's FP32 ``Vector3`` AoS layout (mydefs.hpp:6).
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

from . import REF_HARNESS


def available() -> bool:
    return os.path.exists(REF_HARNESS) and os.access(REF_HARNESS, os.X_OK)


def _run(op, kw, env=None, timeout=3600):
    args = [REF_HARNESS, op] + [f"{k}={v}" for k, v in kw.items()]
    e = dict(os.environ)
    if env:
        e.update(env)
    r = subprocess.run(args, capture_output=True, text=True, timeout=timeout, env=e, stdin=subprocess.DEVNULL)
    if r.returncode != 0:
        raise RuntimeError(f"mmsref_harness {op} failed ({r.returncode}): {r.stderr[-2000:]}")
    return r.stdout


def _grid_kw(dims, d):
    X, Y, Z = dims
    dx, dy, dz = d
    return dict(xdim=X, ydim=Y, zdim=Z, dx=repr(float(dx)), dy=repr(float(dy)), dz=repr(float(dz)))


def potential(charge, dims, d, use_fmm=False, P=3):
    """calc_potential_exact (use_fmm=False) or fmm_calc (use_fmm=True), CPU."""
    X, Y, Z = dims
    with tempfile.TemporaryDirectory() as td:
        np.ascontiguousarray(charge, np.float32).tofile(os.path.join(td, "q"))
        kw = _grid_kw(dims, d)
        kw.update(use_fmm=int(use_fmm), P=P, charge=os.path.join(td, "q"), out=os.path.join(td, "phi"))
        _run("potential", kw)
        return np.fromfile(os.path.join(td, "phi"), np.float32).reshape(Z, Y, X)


def stencils(M, S, dims, d):
    """divergence_3d(M), gradient_3d(S, 1/4pi) and add_exchange_field(M) onto zero."""
    X, Y, Z = dims
    with tempfile.TemporaryDirectory() as td:
        np.ascontiguousarray(M, np.float32).tofile(os.path.join(td, "M"))
        np.ascontiguousarray(S, np.float32).tofile(os.path.join(td, "S"))
        kw = _grid_kw(dims, d)
        o = os.path.join(td, "o")
        kw.update(M=os.path.join(td, "M"), S=os.path.join(td, "S"), out=o)
        _run("stencils", kw)
        sh = (Z, Y, X)
        return (np.fromfile(o + ".div", np.float32).reshape(sh),
                np.fromfile(o + ".grad", np.float32).reshape(sh + (3,)),
                np.fromfile(o + ".exch", np.float32).reshape(sh + (3,)))


def hfield(M, dims, d, t=0.0, use_fmm=False, P=3, demag=1, exchange=1, external=0):
    X, Y, Z = dims
    with tempfile.TemporaryDirectory() as td:
        np.ascontiguousarray(M, np.float32).tofile(os.path.join(td, "M"))
        kw = _grid_kw(dims, d)
        o = os.path.join(td, "o")
        kw.update(M=os.path.join(td, "M"), out=o, t=repr(float(t)), use_fmm=int(use_fmm), P=P, demag=demag,
                  exchange=exchange, external=external)
        _run("hfield", kw)
        sh = (Z, Y, X)
        return (np.fromfile(o + ".H", np.float32).reshape(sh + (3,)),
                np.fromfile(o + ".charge", np.float32).reshape(sh),
                np.fromfile(o + ".potential", np.float32).reshape(sh))


def rk4(material, M, dims, d, dt, nsteps, use_fmm=False, P=3, demag=1, exchange=1, external=0):
    """nsteps fixed-dt RK4 steps in time_marching's accepted-step order."""
    X, Y, Z = dims
    with tempfile.TemporaryDirectory() as td:
        np.ascontiguousarray(material, np.uint8).tofile(os.path.join(td, "mat"))
        np.ascontiguousarray(M, np.float32).tofile(os.path.join(td, "M"))
        kw = _grid_kw(dims, d)
        o = os.path.join(td, "o")
        kw.update(material=os.path.join(td, "mat"), M=os.path.join(td, "M"), out=o, dt=repr(float(dt)),
                  nsteps=nsteps, use_fmm=int(use_fmm), P=P, demag=demag, exchange=exchange, external=external)
        _run("rk4", kw)
        sh = (Z, Y, X)
        return (np.fromfile(o + ".M", np.float32).reshape(sh + (3,)),
                np.fromfile(o + ".H", np.float32).reshape(sh + (3,)))


def march(material, M, dims, d, finaltime, timestep, use_fmm=False, P=3, demag=1, exchange=1, external=0):
    """The reference's time_marching with its energy/torque controller.
    Returns (final M, dynamics rows as an (n, 9) array)."""
    X, Y, Z = dims
    with tempfile.TemporaryDirectory() as td:
        np.ascontiguousarray(material, np.uint8).tofile(os.path.join(td, "mat"))
        np.ascontiguousarray(M, np.float32).tofile(os.path.join(td, "M"))
        kw = _grid_kw(dims, d)
        o = os.path.join(td, "o")
        sim = os.path.join(td, "sim")
        kw.update(material=os.path.join(td, "mat"), M=os.path.join(td, "M"), out=o, sim=sim,
                  finaltime=repr(float(finaltime)), timestep=repr(float(timestep)), use_fmm=int(use_fmm), P=P,
                  demag=demag, exchange=exchange, external=external)
        _run("march", kw)
        rows = []
        with open(os.path.join(sim, "dynamics.dat")) as f:
            for line in f:
                parts = [p for p in line.replace(",", " ").split()]
                if len(parts) == 9:
                    rows.append([float(v) for v in parts])
        return (np.fromfile(o + ".M", np.float32).reshape(Z, Y, X, 3), np.array(rows))


def time_hfield(M, dims, d, use_fmm=False, P=3, reps=1, threads=None):
    """Wall seconds per reference Hfield evaluation and the thread count used."""
    X, Y, Z = dims
    env = {"OMP_NUM_THREADS": str(threads)} if threads else None
    with tempfile.TemporaryDirectory() as td:
        np.ascontiguousarray(M, np.float32).tofile(os.path.join(td, "M"))
        kw = _grid_kw(dims, d)
        kw.update(M=os.path.join(td, "M"), use_fmm=int(use_fmm), P=P, reps=reps)
        out = _run("time_hfield", kw, env=env)
        s, th = out.split()
        return float(s), int(th)


def time_rk4(material, M, dims, d, dt, nsteps, warmup=0, use_fmm=False, P=3, threads=None, budget_s=None):
    """Wall seconds of each of `nsteps` real reference RK4 steps (rk4_step +
    the post-step Hfield, time_marching's accepted-step order) after `warmup`
    untimed ones.  Returns (per-step seconds, threads); fewer steps than asked
    when `budget_s` seconds of timed work ran out."""
    env = {"OMP_NUM_THREADS": str(threads)} if threads else None
    with tempfile.TemporaryDirectory() as td:
        np.ascontiguousarray(material, np.uint8).tofile(os.path.join(td, "mat"))
        np.ascontiguousarray(M, np.float32).tofile(os.path.join(td, "M"))
        kw = _grid_kw(dims, d)
        kw.update(material=os.path.join(td, "mat"), M=os.path.join(td, "M"), dt=repr(float(dt)), nsteps=nsteps,
                  warmup=warmup, use_fmm=int(use_fmm), P=P)
        if budget_s is not None:
            kw["budget_s"] = repr(float(budget_s))
        out = _run("time_rk4", kw, env=env)
        lines = out.strip().splitlines()
        tot = lines[-1].split()
        assert tot[0] == "total", out[-200:]
        steps = [float(v) for v in lines[:-1]]
        assert len(steps) == int(tot[1])
        return steps, int(tot[3])
