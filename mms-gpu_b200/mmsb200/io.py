"""Input and output around a simulation: PNG geometry masks, the reference's
ASCII field files, and checkpoints of the FP64 state.

* ``mask_from_png`` reads a mask the way the reference's driver does
  (helper_functions.cpp:174-218 with main.cpp:117-118, 192-197).  The image
  rows are taken bottom-up, as FreeImage scanlines are.  Each pixel's gray
  level is ``(BYTE)(.3 r + .59 g + .11 b)``, and a pixel of gray 0 is
  material, placed in the layers z = 1 .. zdim-2.  An RGBA image is refused,
  as the reference asserts.
* ``save_scalar3d``, ``save_vector3d`` and ``append_vector3d`` write the
  reference's text layouts (helper_functions.cpp:55-123): for each layer z
  and column x, the y values in order, "%g" formatted.  This is MATLAB's
  column-major order.  FP32 input gives the reference's text exactly.
  ``save_dynamics`` writes mms_march's records as the reference's
  dynamics.dat, ``save_npy`` a binary field, and ``AsyncWriter`` runs any of
  them on a background thread, after the device-to-host copy it waits for.
* ``save_checkpoint``, ``load_checkpoint`` and ``resume`` keep and restore
  everything a run needs: the FP64 state, its time, the mask, the grid, the
  material and field parameters, the solver and, when bound, the surrogate
  weights.  There is no counterpart in the reference.

Arrays follow the library's layout: scalars (zdim, ydim, xdim), vectors
(zdim, ydim, xdim, 3).
"""
from __future__ import annotations

import numpy as np

from . import geometry


# ---------------------------------------------------------------- PNG masks
def mask_from_png(path, zdim=3, layers="middle"):
    """(mask (zdim, ydim, xdim) uint8, gray (ydim, xdim) uint8) from a PNG;
    xdim, ydim = the image's width and height"""
    from PIL import Image

    img = Image.open(path)
    if img.mode in ("RGBA", "LA") or (img.mode == "P" and "transparency" in img.info):
        raise ValueError(f"{path}: images with an alpha channel are not masks (the reference asserts so)")
    rgb = np.asarray(img.convert("RGB"), np.float64)
    gray = np.floor(.3 * rgb[..., 0] + .59 * rgb[..., 1] + .11 * rgb[..., 2]).astype(np.uint8)
    gray = gray[::-1]  # FreeImage's scanline 0 is the image's bottom row
    return geometry.from_plane((gray == 0).astype(np.uint8), zdim, layers), np.ascontiguousarray(gray)


# ------------------------------------------------------- reference text files
def _g(v):
    return "%g" % v


def save_scalar3d(path, field):
    """one line per (z, x) holding the column's y values, and a blank line
    after each layer (helper_functions.cpp:55-76)"""
    f = np.asarray(field)
    Z, Y, X = f.shape
    with open(path, "w") as fh:
        for z in range(Z):
            for x in range(X):
                fh.write("".join(_g(v) + " " for v in f[z, :, x]) + "\n")
            fh.write("\n")


def append_vector3d(fh, field):
    """one line "x y z " per cell, z-major then x then y
    (helper_functions.cpp:103-123)"""
    f = np.asarray(field)
    Z, Y, X, _ = f.shape
    for z in range(Z):
        for x in range(X):
            for y in range(Y):
                v = f[z, y, x]
                fh.write(f"{_g(v[0])} {_g(v[1])} {_g(v[2])} \n")


def save_vector3d(path, field):
    """a whole vector field in the layout of append_vector3d
    (helper_functions.cpp:80-100)"""
    with open(path, "w") as fh:
        append_vector3d(fh, field)


def save_npy(path, field):
    """a field as binary .npy (exact values, any dtype)"""
    np.save(path, np.asarray(field))


def format_record(r):
    """one line of the reference's dynamics.dat (ode_functions.cpp:330-333):
    tindex, t, dt, E (eV), Mx, My, Mz, |M|, torque; each value rounded to FP32
    first, as the reference prints its fptype fields"""
    vals = (r.t, r.dt, r.E_eV, r.Mx, r.My, r.Mz, r.Mmag, r.torque)
    return "%d, " % r.tindex + ", ".join(_g(float(np.float32(v))) for v in vals) + " \n"


def save_dynamics(path, records):
    """the records of mms_march (Context.march) as dynamics.dat"""
    with open(path, "w") as fh:
        for r in records:
            fh.write(format_record(r))


class AsyncWriter:
    """Writes fields on a background thread, in submission order, while the
    caller's GPU work goes on.  ``submit(writer, path, array, event)`` queues
    ``writer(path, array)`` (save_scalar3d, save_vector3d or save_npy); when
    ``event`` is given (anything with ``synchronize()``, e.g. a torch CUDA
    event recorded after a non-blocking device-to-host copy into a pinned
    buffer), the thread waits for it first.  The array must stay untouched
    until ``pending()`` is 0 or ``flush()`` returns; ``flush()`` re-raises the
    first write error."""

    def __init__(self):
        import queue
        import threading
        self._q = queue.Queue()
        self._err = None
        self._n = 0
        self._lock = threading.Lock()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        while True:
            job = self._q.get()
            if job is None:
                self._q.task_done()
                return
            writer, path, array, event = job
            try:
                if event is not None:
                    event.synchronize()
                writer(path, array)
            except Exception as e:  # reported by flush()
                with self._lock:
                    if self._err is None:
                        self._err = e
            finally:
                with self._lock:
                    self._n -= 1
                self._q.task_done()

    def submit(self, writer, path, array, event=None):
        with self._lock:
            self._n += 1
        self._q.put((writer, path, array, event))

    def pending(self):
        with self._lock:
            return self._n

    def flush(self):
        self._q.join()
        with self._lock:
            err, self._err = self._err, None
        if err is not None:
            raise err

    def close(self):
        self.flush()
        self._q.put(None)
        self._t.join()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ------------------------------------------------------------- checkpoints
_GRID = ("xdim", "ydim", "zdim", "dx", "dy", "dz")
_PARAMS = ("Ms", "Aexch", "alpha", "gamma", "mu0", "demag", "exchange", "external", "ref_stage_time")
_SOLVER = ("kind", "fmm_order", "fmm_leaf", "m2l_mode", "far_mode", "near_mode")


def save_checkpoint(path, ctx, material, weights=None):
    """write the context's state (FP64 M and t), the mask it was given, its
    grid, parameters (with the external-field table) and solver, and the
    surrogate weights if given, to one .npz file"""
    M, t = ctx.state_get()
    rec = {"M": M, "t": np.float64(t), "material": np.ascontiguousarray(material, np.uint8)}
    rec.update({"grid_" + k: np.float64(getattr(ctx.grid, k)) for k in _GRID})
    rec.update({"params_" + k: np.float64(getattr(ctx._params, k)) for k in _PARAMS})
    rec.update({"solver_" + k: np.int64(getattr(ctx.solver, k)) for k in _SOLVER})
    if ctx._params.n_hext > 0:
        rec["hext_t"], rec["hext_b"] = ctx._keep[0], ctx._keep[1]
    if weights is not None:
        rec["surrogate_weights"] = np.asarray(weights, np.float32)
    np.savez(path, **rec)


def load_checkpoint(path):
    """the contents of a checkpoint: M, t, material, and the Grid, params
    tuple (make_params's (Params, keepalive)) and Solver to build a context
    with; "surrogate_weights" when saved"""
    import mmsb200

    d = np.load(path)
    g = {k: d["grid_" + k].item() for k in _GRID}
    grid = mmsb200.Grid(int(g["xdim"]), int(g["ydim"]), int(g["zdim"]), g["dx"], g["dy"], g["dz"])
    p = {k: d["params_" + k].item() for k in _PARAMS}
    params = mmsb200.make_params(p["Ms"], p["Aexch"], p["alpha"], p["gamma"], p["mu0"], bool(p["demag"]),
                                 bool(p["exchange"]), bool(p["external"]),
                                 d["hext_t"] if "hext_t" in d else None, d["hext_b"] if "hext_b" in d else None,
                                 bool(p["ref_stage_time"]))
    s = mmsb200.Solver()
    for k in _SOLVER:
        setattr(s, k, int(d["solver_" + k]))
    out = {"M": d["M"], "t": float(d["t"]), "material": d["material"], "grid": grid, "params": params, "solver": s}
    if "surrogate_weights" in d:
        out["surrogate_weights"] = d["surrogate_weights"]
    return out


def resume(ctx, ckpt):
    """put a loaded checkpoint's state into a context built for it"""
    ctx.state_set(ckpt["material"], ckpt["M"], ckpt["t"])
