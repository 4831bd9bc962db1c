"""Geometry input and field output in the reference's formats, and
checkpoints of the FP64 state (CPU; the bit-exact resume runs under -m gpu).

  * PNG masks (helper_functions.cpp:174-218, main.cpp:192-197): rows bottom-up
    as FreeImage's scanlines, gray = (BYTE)(.3 r + .59 g + .11 b), gray 0 =
    material in the layers 1 .. zdim-2; RGBA refused;
  * text fields (helper_functions.cpp:55-123): per layer z and column x the
    y values, "%g" formatted.
"""
import numpy as np
import pytest

import mmsb200
from mmsb200 import io as mio


def test_png_mask_follows_the_reference(tmp_path):
    from PIL import Image
    W, H = 5, 4
    rgb = np.full((H, W, 3), 255, np.uint8)
    rgb[0, 0] = (0, 0, 0)          # top-left: material, lands in the LAST mask row
    rgb[3, 4] = (0, 0, 0)          # bottom-right: material, mask row 0
    rgb[1, 2] = (1, 1, 1)          # .3 + .59 + .11 = 0.999...: truncates to gray 0, material
    rgb[2, 1] = (2, 0, 0)          # gray (BYTE)0.6 = 0: material
    rgb[2, 3] = (0, 2, 0)          # gray (BYTE)1.18 = 1: empty
    path = tmp_path / "m.png"
    Image.fromarray(rgb, "RGB").save(path)
    mask, gray = mio.mask_from_png(path, zdim=3)
    assert mask.shape == (3, H, W) and mask.dtype == np.uint8
    want = np.zeros((H, W), np.uint8)
    for r, c in [(0, 0), (3, 4), (1, 2), (2, 1)]:
        want[H - 1 - r, c] = 1
    assert np.array_equal(mask[1], want)
    assert not mask[0].any() and not mask[2].any()
    assert gray[H - 1 - 2, 3] == 1 and gray[H - 1 - 1, 2] == 0


def test_png_mask_grayscale_and_alpha(tmp_path):
    from PIL import Image
    g = np.full((3, 4), 200, np.uint8)
    g[1, 1] = 0
    Image.fromarray(g, "L").save(tmp_path / "g.png")
    mask, _ = mio.mask_from_png(tmp_path / "g.png", zdim=4)
    assert mask[1:3].sum() == 2 and mask[1, 1, 1] == 1 and mask[2, 1, 1] == 1
    Image.fromarray(np.zeros((3, 4, 4), np.uint8), "RGBA").save(tmp_path / "a.png")
    with pytest.raises(ValueError):
        mio.mask_from_png(tmp_path / "a.png")


def test_text_fields_in_the_reference_layout(tmp_path):
    s = np.arange(12, dtype=np.float32).reshape(2, 2, 3) * 0.5   # (z, y, x)
    mio.save_scalar3d(tmp_path / "s.dat", s)
    want = "0 1.5 \n0.5 2 \n1 2.5 \n\n3 4.5 \n3.5 5 \n4 5.5 \n\n"
    assert open(tmp_path / "s.dat").read() == want
    v = np.zeros((1, 2, 2, 3), np.float32)
    v[0, 0, 0] = (1, 2, 3)
    v[0, 1, 0] = (4, 5, 6)
    v[0, 0, 1] = (7e-9, 8e5, -9.5)
    mio.save_vector3d(tmp_path / "v.dat", v)
    assert open(tmp_path / "v.dat").read() == "1 2 3 \n4 5 6 \n7e-09 800000 -9.5 \n0 0 0 \n"


class _FakeCtx:
    """what save_checkpoint reads from a context"""

    def __init__(self, M, t, grid, params, solver):
        self._M, self._t, self.grid, self.solver = M, t, grid, solver
        self._params, self._keep = params

    def state_get(self):
        return self._M, self._t


def test_checkpoint_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    grid = mmsb200.Grid(6, 5, 3, 5e-9, 4e-9, 3e-9)
    M = rng.standard_normal((3, 5, 6, 3))
    mat = (rng.random((3, 5, 6)) < 0.5).astype(np.uint8)
    ht, hb = np.array([0.0, 1e-9, 2e-9]), rng.standard_normal((3, 3)) * 0.01
    params = mmsb200.make_params(Ms=8e5, alpha=0.02, external=True, hext_t=ht, hext_b=hb, ref_stage_time=True)
    solver = mmsb200.make_solver(mmsb200.SOLVER_FMM, 6, 8, mmsb200.M2L_TENSOR, mmsb200.FAR_STAGES,
                                 mmsb200.NEAR_SIMT)
    w = rng.standard_normal(100).astype(np.float32)
    mio.save_checkpoint(tmp_path / "c.npz", _FakeCtx(M, 1.25e-10, grid, params, solver), mat, weights=w)
    c = mio.load_checkpoint(tmp_path / "c.npz")
    assert np.array_equal(c["M"], M) and c["M"].dtype == np.float64 and c["t"] == 1.25e-10
    assert np.array_equal(c["material"], mat)
    for k in ("xdim", "ydim", "zdim", "dx", "dy", "dz"):
        assert getattr(c["grid"], k) == getattr(grid, k)
    p = c["params"][0]
    assert (p.Ms, p.alpha, p.external, p.n_hext, p.ref_stage_time) == (8e5, 0.02, 1, 3, 1)
    assert np.array_equal(c["params"][1][0], ht) and np.array_equal(c["params"][1][1], hb)
    for k in ("kind", "fmm_order", "fmm_leaf", "m2l_mode", "far_mode", "near_mode"):
        assert getattr(c["solver"], k) == getattr(solver, k)
    assert np.array_equal(c["surrogate_weights"], w)


def test_dynamics_record_line():
    r = mmsb200.Record(7, 1.5e-12, 1e-13, -1234.56789, 0.1, -0.2, 0.97, 8.6e5, 3.3e-7)
    assert mio.format_record(r) == "7, 1.5e-12, 1e-13, -1234.57, 0.1, -0.2, 0.97, 860000, 3.3e-07 \n"


class _Event:
    def __init__(self):
        self.waited = 0

    def synchronize(self):
        self.waited += 1


def test_async_writer_matches_the_synchronous_writers(tmp_path):
    rng = np.random.default_rng(5)
    s = rng.standard_normal((2, 3, 4)).astype(np.float32)
    v = rng.standard_normal((2, 3, 4, 3)).astype(np.float32)
    ev = _Event()
    with mio.AsyncWriter() as w:
        w.submit(mio.save_scalar3d, tmp_path / "s_async.dat", s, ev)
        w.submit(mio.save_vector3d, tmp_path / "v_async.dat", v)
        w.submit(mio.save_npy, tmp_path / "v.npy", v, ev)
        w.flush()
        assert w.pending() == 0 and ev.waited == 2
    mio.save_scalar3d(tmp_path / "s.dat", s)
    mio.save_vector3d(tmp_path / "v.dat", v)
    assert open(tmp_path / "s_async.dat").read() == open(tmp_path / "s.dat").read()
    assert open(tmp_path / "v_async.dat").read() == open(tmp_path / "v.dat").read()
    assert np.array_equal(np.load(tmp_path / "v.npy"), v)


def test_async_writer_reports_a_failed_write(tmp_path):
    w = mio.AsyncWriter()
    w.submit(mio.save_npy, tmp_path / "missing_dir" / "x.npy", np.zeros(3))
    with pytest.raises(OSError):
        w.flush()
    w.close()
