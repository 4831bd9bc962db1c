"""Python binding of the mms_b200 C ABI (include/mms_b200.h) via ctypes.

This is a thin host-side mirror of the library for tests, the benchmark and
scripting: every call goes straight to the sm_100a library
``mms-gpu_b200/lib/libmms_b200.so``.  There is no CPU fallback: if the
library is missing, ``load()`` raises.

Device arrays are passed as raw pointers (``torch.Tensor.data_ptr()``);
host arrays as numpy arrays.  Array layouts follow the reference
(akhan3/mms-gpu): cell index ``z*ydim*xdim + y*xdim + x``, i.e. numpy shape
``(zdim, ydim, xdim)`` for scalars and ``(zdim, ydim, xdim, 3)`` for vectors.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(PKG_DIR, "lib")
CSRC_DIR = os.path.join(PKG_DIR, "csrc")
LIB_PATH = os.path.join(LIB_DIR, "libmms_b200.so")
REFAPI_PATH = os.path.join(LIB_DIR, "libmms_refapi.so")

MMS_OK, MMS_ERR_ARG, MMS_ERR_CUDA, MMS_ERR_NOMEM, MMS_ERR_NUMERIC, MMS_ERR_NOT_READY, MMS_ERR_REJECTED = range(7)
SOLVER_DIRECT, SOLVER_FMM, SOLVER_SURROGATE = 0, 1, 2


class MmsError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"mms_b200 status {status}: {msg}")
        self.status = status


class Grid(ctypes.Structure):
    _fields_ = [("xdim", ctypes.c_int), ("ydim", ctypes.c_int), ("zdim", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double)]

    @property
    def n(self):
        return self.xdim * self.ydim * self.zdim

    @property
    def shape(self):
        return (self.zdim, self.ydim, self.xdim)


class Params(ctypes.Structure):
    _fields_ = [("Ms", ctypes.c_double), ("Aexch", ctypes.c_double), ("alpha", ctypes.c_double),
                ("gamma", ctypes.c_double), ("mu0", ctypes.c_double),
                ("demag", ctypes.c_int), ("exchange", ctypes.c_int), ("external", ctypes.c_int),
                ("n_hext", ctypes.c_int),
                ("hext_t", ctypes.POINTER(ctypes.c_double)), ("hext_b", ctypes.POINTER(ctypes.c_double)),
                ("ref_stage_time", ctypes.c_int)]


class Solver(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("fmm_order", ctypes.c_int), ("fmm_leaf", ctypes.c_int),
                ("m2l_mode", ctypes.c_int), ("far_mode", ctypes.c_int), ("near_mode", ctypes.c_int),
                ("reserved", ctypes.c_int * 2)]


class Controller(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("rtol", ctypes.c_double), ("dt_min", ctypes.c_double),
                ("dt_max", ctypes.c_double), ("torque_stop", ctypes.c_double), ("max_rejects", ctypes.c_int),
                ("reserved", ctypes.c_int * 3)]


class Record(ctypes.Structure):
    _fields_ = [("tindex", ctypes.c_int), ("t", ctypes.c_double), ("dt", ctypes.c_double),
                ("E_eV", ctypes.c_double), ("Mx", ctypes.c_double), ("My", ctypes.c_double),
                ("Mz", ctypes.c_double), ("Mmag", ctypes.c_double), ("torque", ctypes.c_double)]


MARCH_CB = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Record))

# every exported symbol of include/mms_b200.h with its ctypes signature
_VP, _I, _D, _I64, _SZ = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64, ctypes.c_size_t
SIGNATURES = {
    "mms_abi_version": (_I, []),
    "mms_last_error": (ctypes.c_char_p, []),
    "mms_ctx_create": (_I, [ctypes.POINTER(Grid), ctypes.POINTER(Params), ctypes.POINTER(Solver), _VP,
                            ctypes.POINTER(_VP)]),
    "mms_ctx_destroy": (_I, [_VP]),
    "mms_ctx_set_params": (_I, [_VP, ctypes.POINTER(Params)]),
    "mms_ctx_set_solver": (_I, [_VP, ctypes.POINTER(Solver)]),
    "mms_ctx_sync": (_I, [_VP]),
    "mms_ctx_kernel_launches": (_I64, [_VP]),
    "mms_ctx_device_bytes": (_SZ, [_VP]),
    "mms_divergence_dev": (_I, [_VP, _VP, _VP]),
    "mms_potential_dev": (_I, [_VP, _VP, _VP]),
    "mms_gradient_dev": (_I, [_VP, _VP, _D, _VP]),
    "mms_exchange_dev": (_I, [_VP, _VP, _VP]),
    "mms_hfield_dev": (_I, [_VP, _VP, _VP, _VP, _VP, _D]),
    "mms_potential_host": (_I, [_VP, _VP, _VP]),
    "mms_hfield_host": (_I, [_VP, _VP, _VP, _VP, _VP, _D]),
    "mms_state_set": (_I, [_VP, _VP, _VP, _D]),
    "mms_state_get": (_I, [_VP, _VP, ctypes.POINTER(_D)]),
    "mms_state_set_dev": (_I, [_VP, _VP, _VP, _D]),
    "mms_state_get_dev": (_I, [_VP, _VP]),
    "mms_state_set_f32": (_I, [_VP, _VP, _VP, _D]),
    "mms_state_get_f32": (_I, [_VP, _VP, ctypes.POINTER(_D)]),
    "mms_state_set_f32_dev": (_I, [_VP, _VP, _VP, _D]),
    "mms_state_get_f32_dev": (_I, [_VP, _VP]),
    "mms_run_fixed": (_I, [_VP, _D, _I, _I]),
    "mms_state_stats": (_I, [_VP, ctypes.POINTER(_D), ctypes.POINTER(_D), ctypes.POINTER(_D),
                             ctypes.POINTER(_D)]),
    "mms_march": (_I, [_VP, ctypes.POINTER(Controller), _D, _D, ctypes.POINTER(Record), _I, ctypes.POINTER(_I),
                       MARCH_CB, _VP]),
    "mms_diag_fma_tflops": (_I, [_I, ctypes.POINTER(_D)]),
    "mms_autotune_fmm": (_I, [ctypes.POINTER(Grid), ctypes.POINTER(Params), _VP, _D, _I, ctypes.POINTER(Solver),
                              ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "mms_autotune_fmm_steps": (_I, [ctypes.POINTER(Grid), ctypes.POINTER(Params), _VP, _VP, _D, _VP, _D, _I,
                                    ctypes.POINTER(Solver), ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "mms_diag_gemm_bf16": (_I, [_VP, _I, _VP, _I, _VP, _I, _I, _I, _I, _I, _I, _VP]),
    "mms_potential_direct_noalloc": (_I, [_VP, _VP, _I, _I, _I, _D, _D, _D, _VP]),
    "mms_ens_create": (_I, [_VP, _I, _D, _D, _D, ctypes.POINTER(Params), _VP, ctypes.POINTER(_VP)]),
    "mms_ens_destroy": (_I, [_VP]),
    "mms_ens_cells": (ctypes.c_longlong, [_VP]),
    "mms_ens_kernel_launches": (_I64, [_VP]),
    "mms_ens_state_set": (_I, [_VP, _VP, _VP]),
    "mms_ens_state_get": (_I, [_VP, _VP, ctypes.POINTER(_D)]),
    "mms_ens_run_fixed": (_I, [_VP, _D, _I, _I]),
    "mms_ens_sync": (_I, [_VP]),
    "mms_ens_autotune": (_I, [_VP, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_D)]),
    "mms_fmm_stage_times": (_I, [_VP, _VP, _VP, _I, ctypes.POINTER(_D)]),
    "mms_farnet_num_params": (ctypes.c_longlong, []),
    "mms_surrogate_num_params": (ctypes.c_longlong, [_I]),
    "mms_farnet_create": (_I, [_I, _I, _I, ctypes.POINTER(_VP)]),
    "mms_farnet_destroy": (None, [_VP]),
    "mms_farnet_set_weights": (_I, [_VP, _VP, ctypes.c_longlong]),
    "mms_farnet_get_weights": (_I, [_VP, _VP, ctypes.c_longlong]),
    "mms_farnet_set_step_scale": (_I, [_VP, _VP, ctypes.c_longlong]),
    "mms_farnet_forward_dev": (_I, [_VP, _VP, _VP, _I]),
    "mms_farnet_gradient": (_I, [_VP, _VP, _VP, _VP, _I, _VP, ctypes.POINTER(_D)]),
    "mms_farnet_train_step": (_I, [_VP, _VP, _VP, _VP, _I, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                   ctypes.c_float, ctypes.POINTER(_D)]),
    "mms_farnet_device_bytes": (ctypes.c_longlong, [_VP]),
    "mms_ctx_set_surrogate": (_I, [_VP, _VP, ctypes.c_longlong, _I, _D, _I]),
    "mms_surrogate_check": (_I, [_VP, ctypes.POINTER(_D)]),
    "mms_surrogate_stats": (_I, [_VP, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_longlong),
                                 ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "mms_potential_split_dev": (_I, [_VP, _VP, _VP, _VP]),
    "mms_fmm_kernels": (_I, [_VP, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "mms_fmm_info": (_I, [_VP, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_D),
                          ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
}

_lib = None


def build(verbose: bool = False) -> None:
    """Compile the sm_100a library in-tree (make -C mms-gpu_b200/csrc)."""
    r = subprocess.run(["make", "-C", CSRC_DIR, "-j8", "all"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("mms_b200 build failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    if verbose:
        print(r.stdout)


def load():
    """Load libmms_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() or "
                               f"make -C {CSRC_DIR}")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def _check(status):
    if status != MMS_OK:
        raise MmsError(status, load().mms_last_error().decode(errors="replace"))


def fma_tflops(reps=20):
    """measured FP32 FMA throughput of the current device (TFLOP/s)"""
    v = ctypes.c_double()
    _check(load().mms_diag_fma_tflops(reps, ctypes.byref(v)))
    return v.value


def fmm_stats(ctx):
    """FMM plan of a context: levels, leaf, order, flops per evaluation, pair counts"""
    L, s, P = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    fl = (ctypes.c_double * 5)()
    pp, mp = ctypes.c_longlong(), ctypes.c_longlong()
    _check(load().mms_fmm_info(ctx.h, ctypes.byref(L), ctypes.byref(s), ctypes.byref(P), fl,
                               ctypes.byref(pp), ctypes.byref(mp)))
    stages = dict(zip(("p2m", "m2m", "m2l", "l2l", "l2p_p2p"), list(fl)))
    ntc, mtc = ctypes.c_int(), ctypes.c_int()
    _check(load().mms_fmm_kernels(ctx.h, ctypes.byref(ntc), ctypes.byref(mtc)))
    return dict(levels=L.value, leaf=s.value, order=P.value, flops=float(sum(fl)), stage_flops=stages,
                p2p_pairs=pp.value, m2l_pairs=mp.value, near_tc=bool(ntc.value), m2l_tc=bool(mtc.value))


def fmm_stage_times(ctx, rho, phi, reps=10):
    """per-stage device ms of the FMM potential: P2M, M2M, M2L, L2L, L2P+P2P"""
    out = (ctypes.c_double * 5)()
    _check(load().mms_fmm_stage_times(ctx.h, _ptr(rho), _ptr(phi), reps, out))
    return dict(zip(("p2m", "m2m", "m2l", "l2l", "l2p_p2p"), list(out)))


def autotune_fmm(grid, params, rho_dev, max_rel_err=5e-4, reps=5):
    """fastest FMM solver for `grid` within `max_rel_err` of the exact sum on
    the sample charge density `rho_dev` (device tensor); returns
    (Solver, ms per potential, rel-L2 error)"""
    p = params[0] if isinstance(params, tuple) else params
    best = Solver()
    ms, err = ctypes.c_double(), ctypes.c_double()
    _check(load().mms_autotune_fmm(ctypes.byref(grid), ctypes.byref(p), _ptr(rho_dev), max_rel_err, reps,
                                   ctypes.byref(best), ctypes.byref(ms), ctypes.byref(err)))
    return best, ms.value, err.value


def autotune_fmm_steps(grid, params, material, M, dt, rho_dev, max_rel_err=5e-4, reps=20):
    """as autotune_fmm, but each candidate is timed on graph-captured RK4 steps
    of size dt from the host state (material, M); returns (Solver, ms per step,
    rel-L2 error)"""
    p = params[0] if isinstance(params, tuple) else params
    mat = np.ascontiguousarray(material, np.uint8)
    Mh = np.ascontiguousarray(M, np.float64)
    best = Solver()
    ms, err = ctypes.c_double(), ctypes.c_double()
    _check(load().mms_autotune_fmm_steps(ctypes.byref(grid), ctypes.byref(p), _ptr(mat), _ptr(Mh), dt,
                                         _ptr(rho_dev), max_rel_err, reps, ctypes.byref(best), ctypes.byref(ms),
                                         ctypes.byref(err)))
    return best, ms.value, err.value


def make_params(Ms=8.6e5, Aexch=1.3e-11, alpha=0.5, gamma=2.21e5, mu0=4e-7 * np.pi, demag=True, exchange=True,
                external=False, hext_t=None, hext_b=None, ref_stage_time=False):
    """Material constants default to the reference's permalloy (main.cpp:107-111).
    Returns (Params, keepalive) - keep the second item alive while Params is used."""
    keep = []
    n = 0
    tp = bp = None
    if hext_t is not None:
        t = np.ascontiguousarray(hext_t, np.float64)
        b = np.ascontiguousarray(hext_b, np.float64).reshape(-1, 3)
        keep += [t, b]
        n = len(t)
        tp = t.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        bp = b.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    p = Params(Ms, Aexch, alpha, gamma, mu0, int(demag), int(exchange), int(external), n, tp, bp,
               int(ref_stage_time))
    return p, keep


M2L_AUTO, M2L_SIMT, M2L_TENSOR = 0, 1, 2
NEAR_AUTO, NEAR_SIMT, NEAR_TENSOR = 0, 1, 2
FAR_STAGES, FAR_FUSED = 0, 1


def make_solver(kind=SOLVER_DIRECT, order=4, leaf=0, m2l_mode=M2L_AUTO, far_mode=FAR_STAGES, near_mode=NEAR_AUTO):
    s = Solver()
    s.kind, s.fmm_order, s.fmm_leaf, s.m2l_mode, s.far_mode = kind, order, leaf, m2l_mode, far_mode
    s.near_mode = near_mode
    return s


def _ptr(a):
    """raw pointer of a torch tensor or numpy array"""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)


class Context:
    """One simulation grid on the current CUDA device (mms_ctx)."""

    def __init__(self, grid: Grid, params=None, solver: Solver = None, stream=None):
        lib = load()
        self.grid = grid
        if params is None:
            params = make_params()
        self._params, self._keep = params if isinstance(params, tuple) else (params, [])
        self.solver = solver or make_solver()
        h = ctypes.c_void_p()
        st = ctypes.c_void_p(stream) if stream is not None else None
        _check(lib.mms_ctx_create(ctypes.byref(grid), ctypes.byref(self._params), ctypes.byref(self.solver), st,
                                  ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            load().mms_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- configuration
    def set_params(self, params):
        self._params, self._keep = params if isinstance(params, tuple) else (params, [])
        _check(load().mms_ctx_set_params(self.h, ctypes.byref(self._params)))

    def set_solver(self, solver: Solver):
        self.solver = solver
        _check(load().mms_ctx_set_solver(self.h, ctypes.byref(solver)))

    def sync(self):
        _check(load().mms_ctx_sync(self.h))

    @property
    def kernel_launches(self):
        return int(load().mms_ctx_kernel_launches(self.h))

    @property
    def device_bytes(self):
        return int(load().mms_ctx_device_bytes(self.h))

    # -- stateless operators on device pointers (torch tensors)
    def divergence_dev(self, M, rho):
        _check(load().mms_divergence_dev(self.h, _ptr(M), _ptr(rho)))

    def potential_dev(self, rho, phi):
        _check(load().mms_potential_dev(self.h, _ptr(rho), _ptr(phi)))

    def potential_split_dev(self, rho, phi, near):
        """FMM potential and its exact near-field part (device arrays)"""
        _check(load().mms_potential_split_dev(self.h, _ptr(rho), _ptr(phi), _ptr(near)))

    def set_surrogate(self, weights, check_every=50, tol=1e-3, fast=False):
        w = np.ascontiguousarray(weights, np.float32)
        _check(load().mms_ctx_set_surrogate(self.h, _ptr(w), w.size, check_every, tol, int(fast)))

    def surrogate_check(self):
        e = ctypes.c_double()
        _check(load().mms_surrogate_check(self.h, ctypes.byref(e)))
        return e.value

    def surrogate_stats(self):
        a, c, f = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong()
        le, me = ctypes.c_double(), ctypes.c_double()
        _check(load().mms_surrogate_stats(self.h, ctypes.byref(a), ctypes.byref(c), ctypes.byref(f),
                                          ctypes.byref(le), ctypes.byref(me)))
        return dict(active=bool(a.value), checks=c.value, fallbacks=f.value, last_err=le.value, max_err=me.value)

    def gradient_dev(self, phi, c, H):
        _check(load().mms_gradient_dev(self.h, _ptr(phi), c, _ptr(H)))

    def exchange_dev(self, M, H):
        _check(load().mms_exchange_dev(self.h, _ptr(M), _ptr(H)))

    def hfield_dev(self, M, H, charge=None, potential=None, t=0.0):
        _check(load().mms_hfield_dev(self.h, _ptr(M), _ptr(H), _ptr(charge), _ptr(potential), t))

    # -- host-pointer calls (numpy in, numpy out)
    def potential_host(self, rho):
        rho = np.ascontiguousarray(rho, np.float32)
        phi = np.empty(self.grid.shape, np.float32)
        _check(load().mms_potential_host(self.h, _ptr(rho), _ptr(phi)))
        return phi

    def hfield_host(self, M, t=0.0):
        M = np.ascontiguousarray(M, np.float32)
        H = np.empty(self.grid.shape + (3,), np.float32)
        q = np.empty(self.grid.shape, np.float32)
        phi = np.empty(self.grid.shape, np.float32)
        _check(load().mms_hfield_host(self.h, _ptr(M), _ptr(H), _ptr(q), _ptr(phi), t))
        return H, q, phi

    # -- resident FP64 state
    def state_set(self, material, M, t=0.0):
        mat = np.ascontiguousarray(material, np.uint8)
        M = np.ascontiguousarray(M, np.float64)
        _check(load().mms_state_set(self.h, _ptr(mat), _ptr(M), t))

    def state_set_dev(self, material, M, t=0.0):
        _check(load().mms_state_set_dev(self.h, _ptr(material), _ptr(M), t))

    def state_get(self):
        M = np.empty(self.grid.shape + (3,), np.float64)
        t = ctypes.c_double()
        _check(load().mms_state_get(self.h, _ptr(M), ctypes.byref(t)))
        return M, t.value

    def state_get_dev(self, M):
        _check(load().mms_state_get_dev(self.h, _ptr(M)))

    # the reference's FP32 Vector3 layout (N x 3 float32): half the bytes of
    # the FP64 calls; the resident state stays FP64
    def state_set_f32(self, material, M, t=0.0):
        mat = np.ascontiguousarray(material, np.uint8)
        M = np.ascontiguousarray(M, np.float32)
        _check(load().mms_state_set_f32(self.h, _ptr(mat), _ptr(M), t))

    def state_get_f32(self):
        M = np.empty(self.grid.shape + (3,), np.float32)
        t = ctypes.c_double()
        _check(load().mms_state_get_f32(self.h, _ptr(M), ctypes.byref(t)))
        return M, t.value

    def state_set_f32_dev(self, material, M, t=0.0):
        _check(load().mms_state_set_f32_dev(self.h, _ptr(material), _ptr(M), t))

    def state_get_f32_dev(self, M):
        _check(load().mms_state_get_f32_dev(self.h, _ptr(M)))

    def run_fixed(self, dt, nsteps, use_graph=True):
        _check(load().mms_run_fixed(self.h, dt, nsteps, int(use_graph)))

    def stats(self):
        E, T, mh = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        mavg = (ctypes.c_double * 3)()
        _check(load().mms_state_stats(self.h, ctypes.byref(E), ctypes.byref(T), mavg, ctypes.byref(mh)))
        return dict(E_eV=E.value, torque=T.value, Mavg=tuple(mavg), Mmag=mh.value)

    def march(self, finaltime, dt0, mode=0, rtol=1e-5, dt_min=0.0, dt_max=0.0, torque_stop=1e-3, max_rejects=50,
              max_records=100000, callback=None):
        ctl = Controller(mode, rtol, dt_min, dt_max, torque_stop, max_rejects)
        recs = (Record * max_records)()
        n = ctypes.c_int()
        if callback is not None:
            def _cb(user, rejected, rec):
                return int(bool(callback(int(rejected), rec.contents)))
            cb = MARCH_CB(_cb)
        else:
            cb = MARCH_CB()
        st = load().mms_march(self.h, ctypes.byref(ctl), finaltime, dt0, recs, max_records, ctypes.byref(n), cb,
                              None)
        rows = np.array([[r.tindex, r.t, r.dt, r.E_eV, r.Mx, r.My, r.Mz, r.Mmag, r.torque]
                         for r in recs[:min(n.value, max_records)]])
        if st not in (MMS_OK, MMS_ERR_REJECTED):
            _check(st)
        return rows, st


class FarNet:
    """The learned far-field network (mms_farnet) for [batch][3][Y][X] cell
    arrays on the current CUDA device: dimensionless charge u = rho dx / Ms in,
    dimensionless far-field potential phi_far / (Ms dx) out (the near field
    over each 8 x 8 x 3 leaf box's 3 x 3 neighbourhood excluded)."""

    def __init__(self, xdim, ydim, batch=1):
        self.shape = (3, ydim, xdim)
        self.batch = batch
        h = _VP()
        _check(load().mms_farnet_create(xdim, ydim, batch, ctypes.byref(h)))
        self.h = h

    @staticmethod
    def num_params():
        return int(load().mms_farnet_num_params())

    def close(self):
        if self.h:
            load().mms_farnet_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        _check(load().mms_farnet_set_weights(self.h, _ptr(w), w.size))

    def get_weights(self):
        w = np.empty(self.num_params(), np.float32)
        _check(load().mms_farnet_get_weights(self.h, _ptr(w), w.size))
        return w

    def set_step_scale(self, scale):
        s = np.ascontiguousarray(scale, np.float32)
        _check(load().mms_farnet_set_step_scale(self.h, _ptr(s), s.size))

    def forward_dev(self, u, out, nbatch=1):
        _check(load().mms_farnet_forward_dev(self.h, _ptr(u), _ptr(out), nbatch))

    def gradient(self, u, far, nrm2, nbatch=1):
        g = np.empty(self.num_params(), np.float32)
        loss = ctypes.c_double()
        _check(load().mms_farnet_gradient(self.h, _ptr(u), _ptr(far), _ptr(nrm2), nbatch, _ptr(g),
                                          ctypes.byref(loss)))
        return loss.value, g

    def train_step(self, u, far, nrm2, nbatch, lr, beta1=0.9, beta2=0.999, eps=1e-12):
        loss = ctypes.c_double()
        _check(load().mms_farnet_train_step(self.h, _ptr(u), _ptr(far), _ptr(nrm2), nbatch, lr, beta1, beta2, eps,
                                            ctypes.byref(loss)))
        return loss.value

    def device_bytes(self):
        return int(load().mms_farnet_device_bytes(self.h))

