"""Batched ensembles of independent simulations (mms_ens_* in mms_b200.h) and
their partition across GPUs.

One simulation never shards (its far field couples every cell), but an
ensemble does: ranks take disjoint subsets of the instances, balanced by
estimated cost, and need no data-path collective; only the host gathers the
per-instance results.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import Params, _check, _ptr, load, make_params


class EnsInstance(ctypes.Structure):
    _fields_ = [("xdim", ctypes.c_int), ("ydim", ctypes.c_int), ("zdim", ctypes.c_int),
                ("bext", ctypes.c_double * 3)]


def cost(dims):
    """relative cost of one instance per step: the exact sum is N^2 pairs"""
    X, Y, Z = dims
    n = X * Y * Z
    return float(n) * float(n)


def partition(costs, world, rank=None):
    """Greedy longest-processing-time split of instances over `world` ranks.
    Returns a list of index lists (or the list of `rank` when given)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load_ = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load_[k], k))
        parts[r].append(i)
        load_[r] += costs[i]
    parts = [sorted(p) for p in parts]
    return parts if rank is None else parts[rank]


class Ensemble:
    """Many grids with one cell size and material, advanced together."""

    def __init__(self, dims, d, params=None, bext=None, stream=None):
        lib = load()
        self.dims = [tuple(int(v) for v in t) for t in dims]
        n = len(self.dims)
        arr = (EnsInstance * n)()
        for i, (X, Y, Z) in enumerate(self.dims):
            arr[i].xdim, arr[i].ydim, arr[i].zdim = X, Y, Z
            b = (0.0, 0.0, 0.0) if bext is None else bext[i]
            for c in range(3):
                arr[i].bext[c] = float(b[c])
        self._params, self._keep = params if isinstance(params, tuple) else (params or make_params(), [])
        if isinstance(self._params, tuple):
            self._params, self._keep = self._params
        h = ctypes.c_void_p()
        st = ctypes.c_void_p(stream) if stream is not None else None
        _check(lib.mms_ens_create(ctypes.cast(arr, ctypes.c_void_p), n, d[0], d[1], d[2],
                                  ctypes.byref(self._params), st, ctypes.byref(h)))
        self.h = h
        self.offsets = np.cumsum([0] + [X * Y * Z for X, Y, Z in self.dims])

    @property
    def cells(self):
        return int(load().mms_ens_cells(self.h))

    @property
    def kernel_launches(self):
        return int(load().mms_ens_kernel_launches(self.h))

    def close(self):
        if getattr(self, "h", None):
            load().mms_ens_destroy(self.h)
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

    def concat(self, per_instance, dtype):
        return np.concatenate([np.ascontiguousarray(a, dtype).reshape(-1) for a in per_instance])

    def split(self, flat, comps):
        out = []
        for i, (X, Y, Z) in enumerate(self.dims):
            a, b = self.offsets[i], self.offsets[i + 1]
            out.append(flat[a * comps:b * comps].reshape((Z, Y, X) + ((comps,) if comps > 1 else ())))
        return out

    def state_set(self, materials, Ms):
        mat = self.concat(materials, np.uint8)
        M = self.concat(Ms, np.float64)
        _check(load().mms_ens_state_set(self.h, _ptr(mat), _ptr(M)))

    def state_get(self):
        M = np.empty(3 * self.cells, np.float64)
        t = ctypes.c_double()
        _check(load().mms_ens_state_get(self.h, _ptr(M), ctypes.byref(t)))
        return self.split(M, 3), t.value

    def run_fixed(self, dt, nsteps, use_graph=True):
        _check(load().mms_ens_run_fixed(self.h, dt, nsteps, int(use_graph)))

    def sync(self):
        _check(load().mms_ens_sync(self.h))

    def autotune(self, reps=5):
        """measured shape of the batched direct kernel: (warps per CTA, source
        rows per batch, ms per potential)"""
        w, q, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _check(load().mms_ens_autotune(self.h, reps, ctypes.byref(w), ctypes.byref(q), ctypes.byref(ms)))
        return w.value, q.value, ms.value
