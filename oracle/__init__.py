"""Test infrastructure only: the CPU oracle for the demag / LLG hot path.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package.  It is the checker, never the thing measured or
shipped: the product library (``mms-gpu_b200``) has no CPU fallback and never
loads anything from here.

Contents
  * ``liboracle.so`` (``mms_oracle.c``): an FP64 restatement of the reference's
    per-step arithmetic (divergence_3d, gradient_3d, add_exchange_field,
    calc_potential_exact, Hfield, LLG_Mprime, rk4_step) plus FP32 replicas of
    the reference's own operation order for divergence and the direct sum.
  * ``ref``: runs the reference's OWN CPU code, compiled from its sources into
    ``oracle/_ref/mmsref_harness`` by ``oracle/Makefile``, one call per process.
  * ``fmm``: an FP64 numpy restatement of this project's FMM (solid-harmonic
    P2M/M2M/M2L/L2L/L2P + P2P) used to check the GPU FMM stage by stage.

Parity pin: the reference ships no golden vectors or known-answer tests, so
the oracle is pinned against outputs of the reference itself run here
(``tests/golden/make_golden.py`` writes them from ``oracle/_ref``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "mmsref_harness")

MU0_F32 = float(np.float32(4 * np.pi * 1e-7))  # main.cpp:107 stores mu_0 as fptype


class _Grid(ctypes.Structure):
    _fields_ = [("xdim", ctypes.c_int), ("ydim", ctypes.c_int), ("zdim", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double)]


class _Params(ctypes.Structure):
    _fields_ = [("Ms", ctypes.c_double), ("Aexch", ctypes.c_double), ("alpha", ctypes.c_double),
                ("gamma", ctypes.c_double), ("mu0", ctypes.c_double),
                ("demag", ctypes.c_int), ("exchange", ctypes.c_int), ("external", ctypes.c_int),
                ("n_hext", ctypes.c_int),
                ("hext_t", ctypes.POINTER(ctypes.c_double)), ("hext_b", ctypes.POINTER(ctypes.c_double)),
                ("ref_stage_time", ctypes.c_int)]


def build(quiet: bool = True) -> None:
    """Compile liboracle.so and, when the reference tree is present (its path
    in MMS_REFERENCE_TREE, else the reference's location in the build
    container), the reference harness (``make -C oracle REF=...``)."""
    ref = os.environ.get("MMS_REFERENCE_TREE", "/root/reference")
    out = subprocess.run(["make", "-C", HERE, "all", f"REF={ref}"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class Grid:
    """Cell grid: dims and cell sizes (m).  Arrays use the reference's index
    order i = z*ydim*xdim + y*xdim + x, i.e. numpy shape (zdim, ydim, xdim)."""

    def __init__(self, xdim, ydim, zdim, dx, dy, dz):
        self.xdim, self.ydim, self.zdim = int(xdim), int(ydim), int(zdim)
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)

    @property
    def n(self):
        return self.xdim * self.ydim * self.zdim

    def c(self):
        return _Grid(self.xdim, self.ydim, self.zdim, self.dx, self.dy, self.dz)


class Params:
    """Material and field switches.  Defaults are the reference's permalloy
    constants (main.cpp:107-111)."""

    def __init__(self, Ms=8.6e5, Aexch=1.3e-11, alpha=0.5, gamma=2.21e5, mu0=4e-7 * np.pi,
                 demag=True, exchange=True, external=False, hext_t=None, hext_b=None,
                 ref_stage_time=False):
        self.Ms, self.Aexch, self.alpha, self.gamma, self.mu0 = Ms, Aexch, alpha, gamma, mu0
        self.demag, self.exchange, self.external = demag, exchange, external
        self.hext_t = None if hext_t is None else np.ascontiguousarray(hext_t, np.float64)
        self.hext_b = None if hext_b is None else np.ascontiguousarray(hext_b, np.float64).reshape(-1, 3)
        self.ref_stage_time = ref_stage_time

    def c(self):
        n = 0 if self.hext_t is None else len(self.hext_t)
        tp = _dp(self.hext_t) if n else None
        bp = _dp(self.hext_b) if n else None
        return _Params(self.Ms, self.Aexch, self.alpha, self.gamma, self.mu0, int(self.demag),
                       int(self.exchange), int(self.external), n, tp, bp, int(self.ref_stage_time))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def divergence(g: Grid, M):
    M = _f64(M)
    rho = np.zeros(g.n)
    lib().mo_divergence(ctypes.byref(g.c()), _dp(M), _dp(rho))
    return rho.reshape(g.zdim, g.ydim, g.xdim)


def gradient(g: Grid, S, c=1 / (4 * np.pi)):
    S = _f64(S)
    H = np.zeros(3 * g.n)
    lib().mo_gradient(ctypes.byref(g.c()), _dp(S), ctypes.c_double(c), _dp(H))
    return H.reshape(g.zdim, g.ydim, g.xdim, 3)


def exchange(g: Grid, M, p: Params = None):
    p = p or Params()
    M = _f64(M)
    H = np.zeros(3 * g.n)
    lib().mo_add_exchange(ctypes.byref(g.c()), _dp(M), ctypes.c_double(p.Ms), ctypes.c_double(p.Aexch),
                          ctypes.c_double(p.mu0), _dp(H))
    return H.reshape(g.zdim, g.ydim, g.xdim, 3)


def potential_direct(g: Grid, rho):
    """FP64 direct sum phi_i = sum_{j!=i, rho_j != 0} rho_j dV/|r_ij| (no 1/4pi)."""
    rho = _f64(rho)
    phi = np.zeros(g.n)
    lib().mo_potential_direct(ctypes.byref(g.c()), _dp(rho), _dp(phi))
    return phi.reshape(g.zdim, g.ydim, g.xdim)


def potential_direct_targets(g: Grid, rho, targets):
    rho = _f64(rho)
    t = np.ascontiguousarray(targets, dtype=np.int32)
    out = np.zeros(len(t))
    lib().mo_potential_direct_targets(ctypes.byref(g.c()), _dp(rho),
                                      t.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.c_int(len(t)),
                                      _dp(out))
    return out


def potential_direct_f32(g: Grid, rho):
    """The reference's FP32 direct sum in its own accumulation order."""
    rho = np.ascontiguousarray(rho, dtype=np.float32)
    phi = np.zeros(g.n, np.float32)
    lib().mo_potential_direct_f32(ctypes.byref(g.c()), _fp(rho), _fp(phi))
    return phi.reshape(g.zdim, g.ydim, g.xdim)


def divergence_f32(g: Grid, M):
    M = np.ascontiguousarray(M, dtype=np.float32)
    rho = np.zeros(g.n, np.float32)
    lib().mo_divergence_f32(ctypes.byref(g.c()), _fp(M), _fp(rho))
    return rho.reshape(g.zdim, g.ydim, g.xdim)


def hext(p: Params, t):
    out = np.zeros(3)
    pc = p.c()
    lib().mo_hext(ctypes.byref(pc), ctypes.c_double(t), _dp(out))
    return out


def hfield(g: Grid, p: Params, M, t=0.0):
    M = _f64(M)
    H = np.zeros(3 * g.n)
    rho = np.zeros(g.n)
    phi = np.zeros(g.n)
    pc = p.c()
    lib().mo_hfield(ctypes.byref(g.c()), ctypes.byref(pc), _dp(M), ctypes.c_double(t), _dp(H), _dp(rho), _dp(phi))
    sh = (g.zdim, g.ydim, g.xdim)
    return H.reshape(sh + (3,)), rho.reshape(sh), phi.reshape(sh)


def llg(M, H, alpha=0.5, gamma=2.21e5, Ms=8.6e5):
    M = _f64(M).reshape(-1, 3)
    H = _f64(H).reshape(-1, 3)
    out = np.empty_like(M)
    for i in range(len(M)):
        lib().mo_llg(_dp(M[i]), _dp(H[i]), ctypes.c_double(alpha), ctypes.c_double(gamma), ctypes.c_double(Ms),
                     _dp(out[i]))
    return out


def rk4_step(g: Grid, p: Params, material, M, H, t, dt):
    mat = np.ascontiguousarray(material, dtype=np.uint8)
    M = _f64(M)
    H = _f64(H)
    out = np.zeros(3 * g.n)
    pc = p.c()
    lib().mo_rk4_step(ctypes.byref(g.c()), ctypes.byref(pc), mat.ctypes.data_as(ctypes.c_void_p), _dp(M), _dp(H),
                      ctypes.c_double(t), ctypes.c_double(dt), _dp(out))
    return out.reshape(g.zdim, g.ydim, g.xdim, 3)


def rk4_run(g: Grid, p: Params, material, M, dt, nsteps):
    mat = np.ascontiguousarray(material, dtype=np.uint8)
    M = _f64(M).copy()
    pc = p.c()
    lib().mo_rk4_run(ctypes.byref(g.c()), ctypes.byref(pc), mat.ctypes.data_as(ctypes.c_void_p), _dp(M),
                     ctypes.c_double(dt), ctypes.c_int(nsteps))
    return M.reshape(g.zdim, g.ydim, g.xdim, 3)


def energy_torque(g: Grid, p: Params, material, M, H):
    mat = np.ascontiguousarray(material, dtype=np.uint8)
    M = _f64(M)
    H = _f64(H)
    E = ctypes.c_double()
    T = ctypes.c_double()
    pc = p.c()
    lib().mo_energy_torque(ctypes.byref(g.c()), ctypes.byref(pc), mat.ctypes.data_as(ctypes.c_void_p), _dp(M),
                           _dp(H), ctypes.byref(E), ctypes.byref(T))
    return E.value, T.value
