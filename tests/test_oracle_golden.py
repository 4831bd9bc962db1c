"""The CPU oracle pinned against the reference's own outputs (tests/golden/).

The golden fixtures were produced by running the reference's CPU code
(tests/golden/make_golden.py).  The oracle's FP32 replicas must reproduce the
reference bit for bit; its FP64 restatement must agree within FP32 rounding.
"""
import numpy as np
import pytest

from conftest import golden, max_angle_deg, rel_l2


def grid_of(oracle, z):
    X, Y, Z = (int(v) for v in z["dims"])
    dx, dy, dz = (float(v) for v in z["d"])
    return oracle.Grid(X, Y, Z, dx, dy, dz)


def test_divergence_f32_bit_exact(oracle_mod):
    z = golden("stencils_16x16x3.npz")
    g = grid_of(oracle_mod, z)
    rho = oracle_mod.divergence_f32(g, z["M"])
    assert np.array_equal(rho, z["div"])


def test_stencils_f64(oracle_mod):
    z = golden("stencils_16x16x3.npz")
    g = grid_of(oracle_mod, z)
    assert rel_l2(oracle_mod.divergence(g, z["M"]), z["div"]) < 1e-6
    grad = oracle_mod.gradient(g, z["S"])
    assert rel_l2(grad, z["grad"]) < 1e-6
    p = oracle_mod.Params(mu0=oracle_mod.MU0_F32)
    ex = oracle_mod.exchange(g, z["M"], p)
    assert rel_l2(ex, z["exch"]) < 1e-5


@pytest.mark.parametrize("name", ["potential_16x16x3.npz", "potential_24x10x3.npz", "potential_32x32x3.npz"])
def test_direct_potential(oracle_mod, name):
    z = golden(name)
    g = grid_of(oracle_mod, z)
    # FP32 replica in the reference's accumulation order: identical bits
    assert np.array_equal(oracle_mod.potential_direct_f32(g, z["rho"]), z["phi_direct"])
    # FP64 truth vs the reference's FP32 sum
    assert rel_l2(oracle_mod.potential_direct(g, z["rho"]), z["phi_direct"]) < 5e-6


def test_reference_fmm_error_level(oracle_mod):
    """the reference tree code at P=1..3 sits at the error level its paper
    reports (~1e-3 at P=3); the oracle FP64 direct sum is the yardstick"""
    z = golden("potential_32x32x3.npz")
    g = grid_of(oracle_mod, z)
    exact = oracle_mod.potential_direct(g, z["rho"])
    errs = [rel_l2(z[f"phi_fmm_P{P}"], exact) for P in (1, 2, 3)]
    assert errs[2] < 3e-3
    assert errs[0] > errs[1] > errs[2]


def test_hfield(oracle_mod):
    z = golden("hfield_16x16x3.npz")
    g = grid_of(oracle_mod, z)
    for ext in (0, 1):
        p = oracle_mod.Params(mu0=oracle_mod.MU0_F32, external=bool(ext))
        H, rho, phi = oracle_mod.hfield(g, p, z["M"], float(z[f"t_ext{ext}"]))
        assert rel_l2(H, z[f"H_ext{ext}"]) < 1e-6
        assert rel_l2(phi, z[f"phi_ext{ext}"]) < 5e-6


def test_rk4_trajectory(oracle_mod):
    """FP64 restatement of rk4_step + time_marching order vs the FP32 reference"""
    z = golden("rk4_16x16x3.npz")
    g = grid_of(oracle_mod, z)
    p = oracle_mod.Params(mu0=oracle_mod.MU0_F32, external=True, ref_stage_time=True)
    for n in (1, 10):
        M = oracle_mod.rk4_run(g, p, z["material"], z["M0"], float(z["dt"]), n)
        assert max_angle_deg(M, z[f"M_{n}"], z["material"]) < 1e-3 * n


def test_energy_torque_matches_reference_log(oracle_mod):
    """the first accepted step of the reference driver: the oracle's energy and
    torque of the logged state agree with dynamics.dat"""
    z = golden("march_8x8x3.npz")
    g = grid_of(oracle_mod, z)
    rows = z["dynamics"]
    assert rows.shape[1] == 9 and len(rows) > 10
    # columns: tindex, t, dt, E, <Mx>, <My>, <Mz>, <|M|>, torque; dt = 1e-14/torque/2
    assert np.allclose(rows[:, 2], 1e-14 / rows[:, 8] / 2, rtol=1e-4)
    p = oracle_mod.Params(mu0=oracle_mod.MU0_F32)
    H, _, _ = oracle_mod.hfield(g, p, z["M0"])
    E0, T0 = oracle_mod.energy_torque(g, p, z["material"], z["M0"], H)
    # the first step changes the state only slightly (dt = 1e-14)
    assert abs(E0 - rows[0, 3]) / abs(rows[0, 3]) < 1e-3
    assert abs(T0 - rows[0, 8]) / rows[0, 8] < 2e-2
