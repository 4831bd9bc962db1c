"""The reference's own driver, main.cpp, linked against libmms_refapi.so instead
of its fmm_kernel.o + ode_functions.o (oracle/_ref/main_dropin), runs the whole
demag / LLG path on the GPU and writes the reference's dynamics.dat; it tracks
the reference's CPU build of the same main.cpp (tests/golden/dropin_main_16x16x3.npz).

Tolerances: the reference keeps its state in FP32 and this library in FP64,
and the step controller feeds dt = 1e-14 / (2 torque) back into the
trajectory, so the first 100 records agree to 1e-3 relative (time, dt, energy,
<M>, torque) and the end of the run to 2 % in time and energy.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, golden

pytestmark = pytest.mark.gpu

DROPIN = os.path.join(ROOT, "oracle", "_ref", "main_dropin")


def read_dynamics(path):
    rows = []
    with open(path) as f:
        for line in f:
            parts = line.replace(",", " ").split()
            if len(parts) == 9:
                rows.append([float(v) for v in parts])
    return np.array(rows)


def read_snapshots(path, ncell=16 * 16 * 3):
    """Mdynamics.dat as [snapshot][line][3]: lines of exactly three numbers"""
    vals = []
    with open(path) as f:
        for line in f:
            parts = line.split()
            assert len(parts) == 3, line
            vals.append([float(v) for v in parts])
    a = np.array(vals)
    assert len(a) % ncell == 0
    return a.reshape(-1, ncell, 3)


@pytest.mark.parametrize("run", ["sd", "vortex_ext"])
def test_reference_main_runs_on_the_gpu(cuda, lib, run):
    if not os.path.exists(DROPIN):
        pytest.skip("oracle/_ref/main_dropin was not built (the reference tree was absent at build time)")
    z = golden("dropin_main_16x16x3.npz")
    ref_rows = z[run]
    args = [str(a) for a in z[run + "_args"]]
    with tempfile.TemporaryDirectory() as td:
        r = subprocess.run([DROPIN] + args, cwd=td, stdin=subprocess.DEVNULL, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        rows = read_dynamics(os.path.join(td, args[15], "dynamics.dat"))
        snaps = read_snapshots(os.path.join(td, args[15], "Mdynamics.dat"))
    # one snapshot of the 16 x 16 x 3 cells per accepted step, every one
    # written (the writer thread formats them while marching goes on), each
    # cell |M| = Ms or empty
    assert snaps.shape == (len(rows), 16 * 16 * 3, 3)
    mag = np.linalg.norm(snaps, axis=-1)
    assert np.all((np.abs(mag - 8.6e5) < 8.6e5 * 1e-5) | (mag == 0))
    n = min(100, len(rows), len(ref_rows))
    assert n >= 50
    assert np.array_equal(rows[:n, 0], ref_rows[:n, 0])
    for col in (1, 2, 3, 8):
        rel = np.abs(rows[:n, col] - ref_rows[:n, col]) / np.maximum(np.abs(ref_rows[:n, col]), 1e-12)
        assert rel.max() < 1e-3, (col, rel.max())
    for col in (4, 5, 6):
        assert np.abs(rows[:n, col] - ref_rows[:n, col]).max() < 1e-3, col
    # end of the run: same final time window and energy
    assert abs(rows[-1, 1] - ref_rows[-1, 1]) / ref_rows[-1, 1] < 0.02
    assert abs(rows[-1, 3] - ref_rows[-1, 3]) / abs(ref_rows[-1, 3]) < 0.02
    assert abs(len(rows) - len(ref_rows)) / len(ref_rows) < 0.05
