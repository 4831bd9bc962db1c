"""Long trajectories: the accuracy an LLG run keeps over thousands of steps.

* 32x32x3, 5 nm cells, permalloy (Ms 8.6e5 A/m, A 1.3e-11 J/m, alpha 0.5,
  gamma 2.21e5), no external field, M uniform on the sphere from seed 2010,
  FP64 state, fixed dt = 1e-13 s: 2000 RK4 steps with the FMM (P = 4) against
  the same 2000 steps with the exact direct sum, on the full rectangle (every
  cell of the middle layer magnetic) and on the reference's default geometry
  (a 1-cell empty border, main.cpp:119-130).  Tolerance: max angle <= 1 deg
  over the magnetic cells.
* The reference's own rk4_step loop (oracle/_ref: its unmodified CPU sources,
  FP32 state, CPU direct sum), 200 steps in time_marching's accepted-step
  order (ode_functions.cpp:230-308), against this library's direct solver on
  the reference's default geometry with its stage-time convention.  The two
  differ only by the reference's FP32 state and field rounding.
* The 256x256x3 disc lattice (8 x 8 discs of radius 12 at pitch 32, one
  random in-plane direction per disc, B_x ramped -50 -> +50 mT over 10 ns):
  10^4 steps of the FMM (P = 4, leaf 8) against 10^4 steps of the exact direct
  sum: final max angle <= 1 deg.
"""
import numpy as np
import pytest

from conftest import max_angle_deg

pytestmark = pytest.mark.gpu

D = (5e-9, 5e-9, 5e-9)
MU0_F32 = float(np.float32(4e-7 * np.pi))


def _run(mmsb200, dims, solver, params, mask, M, dt, nsteps, chunk=None):
    """final FP64 state after nsteps graph-replayed RK4 steps (and the states
    after every `chunk` steps)"""
    out = []
    with mmsb200.Context(mmsb200.Grid(*dims, *D), params, solver) as ctx:
        ctx.state_set(mask, M)
        done = 0
        chunk = chunk or nsteps
        while done < nsteps:
            n = min(chunk, nsteps - done)
            ctx.run_fixed(dt, n, use_graph=True)
            done += n
            out.append(ctx.state_get()[0])
    return out


@pytest.mark.parametrize("geom", ["full", "reference_default"])
def test_c1_fmm_p4_vs_direct_2000_steps(cuda, lib, geom):
    import mmsb200
    from mmsb200 import geometry
    X = Y = 32
    Z = 3
    mask = geometry.rectangle(X, Y, Z) if geom == "full" else geometry.reference_default(X, Y, Z)
    M = geometry.random_sphere(mask, 2010)
    params = mmsb200.make_params()
    fmm = _run(mmsb200, (X, Y, Z), mmsb200.make_solver(mmsb200.SOLVER_FMM, 4), params, mask, M, 1e-13, 2000, 500)
    exact = _run(mmsb200, (X, Y, Z), mmsb200.make_solver(mmsb200.SOLVER_DIRECT), params, mask, M, 1e-13, 2000,
                 500)
    angles = [max_angle_deg(a, b, mask) for a, b in zip(fmm, exact)]
    print(f"C1 {geom}: FMM P=4 vs direct, max angle after 500/1000/1500/2000 steps: {angles}")
    assert all(np.isfinite(angles))
    assert angles[-1] <= 1.0, angles
    mag = np.linalg.norm(fmm[-1], axis=-1)
    assert np.allclose(mag[mask != 0], 8.6e5, rtol=1e-12)


def test_c1_direct_vs_reference_rk4_200_steps(cuda, lib, oracle_mod):
    import mmsb200
    from mmsb200 import geometry
    from oracle import ref
    if not ref.available():
        pytest.fail("oracle/_ref/mmsref_harness is not built (build it where the reference tree is present)")
    X = Y = 32
    Z = 3
    mask = geometry.reference_default(X, Y, Z)
    M = geometry.random_sphere(mask, 2010)
    # the reference's FP32 state: start both from the same FP32-rounded vectors
    M32 = M.astype(np.float32)
    Mref, _ = ref.rk4(mask, M32, (X, Y, Z), D, 1e-13, 200)
    params = mmsb200.make_params(mu0=MU0_F32, ref_stage_time=True)
    ours = _run(mmsb200, (X, Y, Z), mmsb200.make_solver(mmsb200.SOLVER_DIRECT), params, mask,
                M32.astype(np.float64), 1e-13, 200)[-1]
    ang = max_angle_deg(ours, Mref, mask)
    print(f"C1 reference rk4_step loop vs this library (direct), 200 steps: max angle {ang:.3e} deg")
    assert ang <= 5e-3, ang


def test_c5_fmm_vs_direct_1e4_steps(cuda, lib):
    import mmsb200
    from mmsb200 import geometry
    X = Y = 256
    Z = 3
    mask, M = geometry.per_dot_random_inplane(X, Y, Z, 12, 32, 2010)
    params = mmsb200.make_params(external=True, hext_t=[0.0, 1e-8], hext_b=[[-0.05, 0, 0], [0.05, 0, 0]])
    n = 10000
    fmm = _run(mmsb200, (X, Y, Z), mmsb200.make_solver(mmsb200.SOLVER_FMM, 4, 8), params, mask, M, 1e-13, n,
               2500)
    exact = _run(mmsb200, (X, Y, Z), mmsb200.make_solver(mmsb200.SOLVER_DIRECT), params, mask, M, 1e-13, n, 2500)
    angles = [max_angle_deg(a, b, mask) for a, b in zip(fmm, exact)]
    print(f"C5 FMM P=4 leaf 8 vs direct, max angle after 2500/5000/7500/10000 steps: {angles}")
    assert angles[-1] <= 1.0, angles
