"""GPU parity: the resident FP64 RK4 state (fixed step, CUDA graph, controller)
vs the FP64 oracle and the reference's trajectories.

Tolerances (max angle between magnetisation vectors over material cells):
  * vs the FP64 oracle on the same seeded input: 1e-4 deg after 10 steps
    (the only differences are the FP32 potential and FP32 field rounding);
  * vs the reference's FP32 run: 1e-3 deg per step (its FP32 state rounding).
"""
import numpy as np
import pytest

from conftest import golden, max_angle_deg, rel_l2

pytestmark = pytest.mark.gpu

MU0_F32 = float(np.float32(4e-7 * np.pi))


def dims_of(z):
    return tuple(int(v) for v in z["dims"]), tuple(float(v) for v in z["d"])


def test_rk4_vs_oracle_and_reference(cuda, lib, oracle_mod):
    import mmsb200
    z = golden("rk4_16x16x3.npz")
    dims, d = dims_of(z)
    g = mmsb200.Grid(*dims, *d)
    dt = float(z["dt"])
    og = oracle_mod.Grid(*dims, *d)
    op = oracle_mod.Params(mu0=MU0_F32, external=True, ref_stage_time=True)
    ref10 = oracle_mod.rk4_run(og, op, z["material"], z["M0"], dt, 10)
    for graph in (False, True):
        with mmsb200.Context(g, mmsb200.make_params(mu0=MU0_F32, external=True, ref_stage_time=True)) as ctx:
            ctx.state_set(z["material"], z["M0"].astype(np.float64))
            ctx.run_fixed(dt, 1, use_graph=graph)
            M1, t1 = ctx.state_get()
            ctx.run_fixed(dt, 9, use_graph=graph)
            M10, t10 = ctx.state_get()
        assert abs(t1 - dt) < 1e-25 and abs(t10 - 10 * dt) < 1e-24
        assert max_angle_deg(M10, ref10, z["material"]) < 1e-4
        assert max_angle_deg(M1, z["M_1"], z["material"]) < 1e-3
        assert max_angle_deg(M10, z["M_10"], z["material"]) < 1e-2
        # |M| = Ms on material, 0 elsewhere
        mag = np.linalg.norm(M10, axis=-1)
        assert np.allclose(mag[z["material"] != 0], 8.6e5, rtol=1e-12)
        assert np.all(mag[z["material"] == 0] == 0)


def test_graph_replay_is_bitwise_identical(cuda, lib):
    import mmsb200
    z = golden("rk4_16x16x3.npz")
    dims, d = dims_of(z)
    g = mmsb200.Grid(*dims, *d)
    out = []
    for graph in (False, True):
        with mmsb200.Context(g, mmsb200.make_params(external=True)) as ctx:
            ctx.state_set(z["material"], z["M0"].astype(np.float64))
            ctx.run_fixed(1e-13, 5, use_graph=graph)
            out.append(ctx.state_get()[0])
    assert np.array_equal(out[0], out[1])


def test_proper_stage_times_with_table_field(cuda, lib, oracle_mod):
    """stage times t + c dt and a piecewise-linear B(t) table (the external
    field forms the benchmark configurations use)"""
    import mmsb200
    z = golden("rk4_16x16x3.npz")
    dims, d = dims_of(z)
    tt = [0.0, 1e-12, 3e-12]
    bb = [[-0.05, 0.0, 0.0], [0.02, 0.01, 0.0], [0.05, -0.01, 0.002]]
    og = oracle_mod.Grid(*dims, *d)
    op = oracle_mod.Params(external=True, hext_t=tt, hext_b=bb)
    ref = oracle_mod.rk4_run(og, op, z["material"], z["M0"], 2e-13, 12)
    g = mmsb200.Grid(*dims, *d)
    with mmsb200.Context(g, mmsb200.make_params(external=True, hext_t=tt, hext_b=bb)) as ctx:
        ctx.state_set(z["material"], z["M0"].astype(np.float64))
        ctx.run_fixed(2e-13, 12)
        M, _ = ctx.state_get()
    assert max_angle_deg(M, ref, z["material"]) < 1e-4


def test_stats_match_oracle(cuda, lib, oracle_mod):
    import mmsb200
    z = golden("hfield_16x16x3.npz")
    dims, d = dims_of(z)
    og = oracle_mod.Grid(*dims, *d)
    op = oracle_mod.Params()
    M = z["M"].astype(np.float64)
    H, _, _ = oracle_mod.hfield(og, op, M)
    E, T = oracle_mod.energy_torque(og, op, z["material"], M, H)
    g = mmsb200.Grid(*dims, *d)
    with mmsb200.Context(g, mmsb200.make_params()) as ctx:
        ctx.state_set(z["material"], M)
        s = ctx.stats()
    assert abs(s["E_eV"] - E) / abs(E) < 1e-5
    assert abs(s["torque"] - T) / T < 1e-5
    mat = z["material"] != 0
    assert np.allclose(s["Mavg"], M[mat].mean(0) / 8.6e5, atol=1e-9)


def test_reference_controller_matches_reference_log(cuda, lib):
    """mms_march mode 0 restates the reference's energy/torque controller: its
    accepted-step records track dynamics.dat of the reference run"""
    import mmsb200
    z = golden("march_8x8x3.npz")
    dims, d = dims_of(z)
    rows_ref = z["dynamics"]
    g = mmsb200.Grid(*dims, *d)
    with mmsb200.Context(g, mmsb200.make_params(mu0=MU0_F32, ref_stage_time=True)) as ctx:
        ctx.state_set(z["material"], z["M0"].astype(np.float64))
        rows, st = ctx.march(float(z["finaltime"]), float(z["timestep"]), mode=0)
        Mf, _ = ctx.state_get()
    assert st == mmsb200.MMS_OK
    n = min(len(rows), len(rows_ref))
    assert abs(len(rows) - len(rows_ref)) <= 2
    assert np.array_equal(rows[:n, 0], rows_ref[:n, 0])
    for col, tol in [(1, 1e-3), (2, 1e-3), (3, 1e-4), (4, 1e-4), (5, 1e-3), (6, 1e-3), (8, 1e-3)]:
        a, b = rows[:n, col], rows_ref[:n, col]
        assert np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-3)) < tol, col
    # 159 accepted steps of an FP32-state run vs an FP64-state run
    assert max_angle_deg(Mf, z["M_final"], z["material"]) < 0.1


def test_step_doubling_controller(cuda, lib, oracle_mod):
    """mode 1: RK4 step doubling with an FP64 error estimate reaches the final
    time with steps that respect rtol; the result agrees with a fine fixed-step
    oracle run"""
    import mmsb200
    z = golden("rk4_16x16x3.npz")
    dims, d = dims_of(z)
    g = mmsb200.Grid(*dims, *d)
    T = 2e-12
    with mmsb200.Context(g, mmsb200.make_params()) as ctx:
        ctx.state_set(z["material"], z["M0"].astype(np.float64))
        rows, st = ctx.march(T, 1e-13, mode=1, rtol=1e-6, torque_stop=0.0)
        M, t = ctx.state_get()
    assert st == mmsb200.MMS_OK
    assert abs(t - T) < 1e-20
    og = oracle_mod.Grid(*dims, *d)
    fine = oracle_mod.rk4_run(og, oracle_mod.Params(), z["material"], z["M0"], T / 80, 80)
    assert max_angle_deg(M, fine, z["material"]) < 1e-3


def test_numeric_error_is_reported(cuda, lib):
    """a non-finite state is reported as MMS_ERR_NUMERIC (the NaN is injected
    on the host into the input, never on the device)"""
    import mmsb200
    z = golden("rk4_16x16x3.npz")
    dims, d = dims_of(z)
    M = z["M0"].astype(np.float64).copy()
    idx = np.argwhere(z["material"] != 0)[5]
    M[tuple(idx)] = np.nan
    g = mmsb200.Grid(*dims, *d)
    with mmsb200.Context(g, mmsb200.make_params()) as ctx:
        ctx.state_set(z["material"], M)
        ctx.run_fixed(1e-13, 1)
        with pytest.raises(mmsb200.MmsError) as e:
            ctx.state_get()
        assert e.value.status == mmsb200.MMS_ERR_NUMERIC


def test_fp32_vector3_state_io(cuda, lib):
    """the state in the reference's FP32 Vector3 layout (mms_state_*_f32,
    host and device): set widens exactly, so the steps give the bits of the
    FP64 calls; get rounds each component to nearest; empty cells read 0"""
    import torch
    import mmsb200
    z = golden("rk4_16x16x3.npz")
    dims, d = dims_of(z)
    g = mmsb200.Grid(*dims, *d)
    mat = z["material"]
    M0 = np.asarray(z["M0"], np.float32).copy()
    M0[mat == 0] = 1.0  # values at empty cells are dropped
    dt = 1e-13
    with mmsb200.Context(g, mmsb200.make_params(external=True)) as a, \
            mmsb200.Context(g, mmsb200.make_params(external=True)) as b, \
            mmsb200.Context(g, mmsb200.make_params(external=True)) as c:
        a.state_set(mat, M0.astype(np.float64))
        b.state_set_f32(mat, M0)
        c.state_set_f32_dev(torch.from_numpy(mat.astype(np.uint8)).cuda(), torch.from_numpy(M0).cuda())
        for ctx in (a, b, c):
            ctx.run_fixed(dt, 3)
        Ma, ta = a.state_get()
        Mb, tb = b.state_get()
        Mb32, tb32 = b.state_get_f32()
        out = torch.empty(M0.shape, dtype=torch.float32, device="cuda")
        c.state_get_f32_dev(out)
        c.sync()
        Mc32 = out.cpu().numpy()
    assert np.array_equal(Ma, Mb) and ta == tb == tb32 and abs(ta - 3 * dt) < 1e-25
    assert np.array_equal(Mb32, Ma.astype(np.float32))
    assert np.array_equal(Mc32, Mb32)
    assert np.all(Mb32[mat == 0] == 0) and np.all(Ma[mat == 0] == 0)


def test_time_and_dt_across_calls(cuda, lib):
    """the last stage advances the time; mms_run_fixed sets dt on the device
    only when it changes, and a state set (which clears dt) makes the next
    call set it again: t follows every call's dt, and the same steps taken
    with a change of dt between them match a context stepping them in one
    go where the dt is the same"""
    import mmsb200
    z = golden("rk4_16x16x3.npz")
    dims, d = dims_of(z)
    g = mmsb200.Grid(*dims, *d)
    mat, M0 = z["material"], z["M0"].astype(np.float64)
    d1, d2 = 1e-13, 2.5e-14
    with mmsb200.Context(g, mmsb200.make_params(external=True)) as a, \
            mmsb200.Context(g, mmsb200.make_params(external=True)) as b:
        a.state_set(mat, M0)
        a.run_fixed(d1, 2)
        a.run_fixed(d2, 1)
        a.run_fixed(d1, 1)
        Ma, ta = a.state_get()
        assert abs(ta - (3 * d1 + d2)) < 1e-26
        a.state_set(mat, M0, 1e-12)
        a.run_fixed(d1, 1)  # same dt as the last call: set again after the state set
        assert abs(a.state_get()[1] - (1e-12 + d1)) < 1e-26
        b.state_set(mat, M0)
        b.run_fixed(d1, 2, use_graph=False)
        b.run_fixed(d2, 1, use_graph=False)
        b.run_fixed(d1, 1, use_graph=False)
        Mb, tb = b.state_get()
    assert ta == tb and np.array_equal(Ma, Mb)
