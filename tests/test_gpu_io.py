"""A run resumed from a checkpoint continues the uninterrupted run bit for
bit (FMM at leaf 8 with the tensor-core near field, CUDA-graph steps)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_resume_from_checkpoint_is_bitwise(cuda, lib, tmp_path):
    import mmsb200
    from mmsb200 import geometry
    from mmsb200 import io as mio
    X, Y, Z = 64, 48, 3
    mask = geometry.disc(X, Y, Z, 20)
    M = geometry.random_inplane(mask, 7)
    grid = mmsb200.Grid(X, Y, Z, 5e-9, 5e-9, 5e-9)
    params = mmsb200.make_params(external=True, hext_t=np.array([0.0, 1e-9]),
                                 hext_b=np.array([[0.0, 0.0, 0.0], [0.02, 0.01, 0.0]]))
    solver = mmsb200.make_solver(mmsb200.SOLVER_FMM, 4, 8)
    with mmsb200.Context(grid, params, solver) as a:
        a.state_set(mask, M)
        a.run_fixed(1e-13, 5)
        mio.save_checkpoint(tmp_path / "c.npz", a, mask)
        a.run_fixed(1e-13, 5)
        a.sync()
        Ma, ta = a.state_get()
    c = mio.load_checkpoint(tmp_path / "c.npz")
    with mmsb200.Context(c["grid"], c["params"], c["solver"]) as b:
        mio.resume(b, c)
        b.run_fixed(1e-13, 5)
        b.sync()
        Mb, tb = b.state_get()
    assert ta == tb
    assert np.array_equal(Ma, Mb)
