"""GPU parity of the batched ensemble (mms_ens_*): every instance advances
exactly as the same grid does in its own context, and as the FP64 oracle.

Tolerances: vs independent single-grid contexts (same FP64 state, potentials
from a different FP32 kernel) 1e-5 deg after 10 steps; vs the FP64 oracle
1e-4 deg after 10 steps.
"""
import numpy as np
import pytest

from conftest import max_angle_deg

pytestmark = pytest.mark.gpu

D = (5e-9, 5e-9, 5e-9)


def test_ensemble_matches_single_contexts(cuda, lib):
    import mmsb200
    from mmsb200 import geometry
    from mmsb200.ensemble import Ensemble
    dims, masks, Ms, bext = geometry.ensemble_instances(7, seed=77, sides=(16, 24, 40, 64))
    dims[3] = (19, 13, 3)  # ragged sizes too
    masks[3] = geometry.rectangle(19, 13, 3)
    Ms[3] = geometry.random_sphere(masks[3], 5)
    with Ensemble(dims, D, mmsb200.make_params(external=True), bext=bext) as ens:
        ens.state_set(masks, Ms)
        ens.run_fixed(1e-13, 10, use_graph=True)
        out, t = ens.state_get()
        launches = ens.kernel_launches
    assert abs(t - 1e-12) < 1e-24
    assert launches > 0
    for i, (X, Y, Z) in enumerate(dims):
        p = mmsb200.make_params(external=True, hext_t=[0.0], hext_b=[bext[i]])
        with mmsb200.Context(mmsb200.Grid(X, Y, Z, *D), p) as ctx:
            ctx.state_set(masks[i], Ms[i])
            ctx.run_fixed(1e-13, 10)
            ref, _ = ctx.state_get()
        assert max_angle_deg(out[i], ref, masks[i]) < 1e-5, i


def test_ensemble_matches_fp64_oracle(cuda, lib, oracle_mod):
    import mmsb200
    from mmsb200 import geometry
    from mmsb200.ensemble import Ensemble
    dims, masks, Ms, bext = geometry.ensemble_instances(3, seed=5, sides=(16, 24))
    with Ensemble(dims, D, mmsb200.make_params(external=True), bext=bext) as ens:
        ens.state_set(masks, Ms)
        ens.run_fixed(1e-13, 10, use_graph=False)
        out, _ = ens.state_get()
    for i, (X, Y, Z) in enumerate(dims):
        og = oracle_mod.Grid(X, Y, Z, *D)
        op = oracle_mod.Params(external=True, hext_t=[0.0], hext_b=[bext[i]])
        ref = oracle_mod.rk4_run(og, op, masks[i], Ms[i], 1e-13, 10)
        assert max_angle_deg(out[i], ref, masks[i]) < 1e-4, i


def test_ensemble_rejects_bad_instances(cuda, lib):
    import mmsb200
    from mmsb200.ensemble import Ensemble
    with pytest.raises(mmsb200.MmsError):
        Ensemble([(300, 4, 3)], D)
    with pytest.raises(mmsb200.MmsError):
        Ensemble([(0, 4, 3)], D)


def _kinds(n, seed):
    """mask kind (0 rectangle, 1 disc, 2 ellipse) of each generated instance,
    drawn the way geometry.ensemble_instances draws it"""
    from mmsb200 import geometry
    sides = (16, 24, 32, 40, 48, 56, 64)
    out = []
    for i in range(n):
        g = geometry.rng(seed + i)
        g.choice(sides)
        g.choice(sides)
        out.append(int(g.integers(0, 3)))
    return out


def test_c4_512_instances_100_steps(cuda, lib, oracle_mod):
    """The batched-ensemble configuration: 512 instances (sides 16..64 in
    steps of 8, x 3 layers; rectangle, disc or ellipse masks; random M on the
    sphere; random in-plane |B| <= 50 mT), dt = 1e-13 s, 100 graph-replayed
    steps with the autotuned kernel shape.  A sample holding every mask kind
    at small, 32- and 64-cell sides is checked against the FP64 oracle
    (<= 1e-3 deg after 100 steps) and against independent single-grid
    contexts (<= 1e-4 deg); every instance keeps |M| = Ms."""
    import mmsb200
    from mmsb200 import geometry
    from mmsb200.ensemble import Ensemble
    n, seed, steps = 512, 2010, 100
    dims, masks, Ms, bext = geometry.ensemble_instances(n, seed=seed)
    kinds = _kinds(n, seed)
    with Ensemble(dims, D, mmsb200.make_params(external=True), bext=bext) as ens:
        ens.state_set(masks, Ms)
        ew, q, ms = ens.autotune(3)
        ens.run_fixed(1e-13, steps, use_graph=True)
        out, t = ens.state_get()
    assert abs(t - steps * 1e-13) < 1e-22
    for i in range(n):
        mag = np.linalg.norm(out[i], axis=-1)
        assert np.allclose(mag[masks[i] != 0], 8.6e5, rtol=1e-12), i
    sample = []
    for k in range(3):
        small = [i for i in range(n) if kinds[i] == k and max(dims[i][:2]) <= 24]
        mid = [i for i in range(n) if kinds[i] == k and 32 in dims[i][:2] and max(dims[i][:2]) <= 32]
        big = [i for i in range(n) if kinds[i] == k and dims[i][0] == 64]
        sample += [lst[0] for lst in (small, mid, big) if lst]
    assert len(sample) >= 8
    worst_oracle, worst_ctx = 0.0, 0.0
    for i in sample:
        X, Y, Z = dims[i]
        p = mmsb200.make_params(external=True, hext_t=[0.0], hext_b=[bext[i]])
        with mmsb200.Context(mmsb200.Grid(X, Y, Z, *D), p) as ctx:
            ctx.state_set(masks[i], Ms[i])
            ctx.run_fixed(1e-13, steps)
            ref_ctx, _ = ctx.state_get()
        a_ctx = max_angle_deg(out[i], ref_ctx, masks[i])
        worst_ctx = max(worst_ctx, a_ctx)
        assert a_ctx < 1e-4, (i, dims[i], a_ctx)
        if X * Y <= 64 * 32 or i == sample[-1]:
            og = oracle_mod.Grid(X, Y, Z, *D)
            op = oracle_mod.Params(external=True, hext_t=[0.0], hext_b=[bext[i]])
            ref = oracle_mod.rk4_run(og, op, masks[i], Ms[i], 1e-13, steps)
            a_or = max_angle_deg(out[i], ref, masks[i])
            worst_oracle = max(worst_oracle, a_or)
            assert a_or < 1e-3, (i, dims[i], a_or)
    print(f"C4: autotuned {ew} warps x {q} rows ({ms:.3f} ms per potential); sample {[dims[i] for i in sample]}; "
          f"max angle vs contexts {worst_ctx:.2e} deg, vs FP64 oracle {worst_oracle:.2e} deg")


def test_c4_512_instances_5000_steps(cuda, lib):
    """The batched-ensemble configuration at its full length: 512 instances,
    5000 graph-replayed steps of dt = 1e-13 s.  Every instance keeps |M| = Ms
    and stays finite, and one instance of each mask kind (the largest of its
    kind) ends within 1e-3 deg of an independent single-grid context run the
    same 5000 steps (measured: 6e-6 deg; bound 1e-3 deg)."""
    import mmsb200
    from mmsb200 import geometry
    from mmsb200.ensemble import Ensemble
    n, seed, steps = 512, 2010, 5000
    dims, masks, Ms, bext = geometry.ensemble_instances(n, seed=seed)
    kinds = _kinds(n, seed)
    with Ensemble(dims, D, mmsb200.make_params(external=True), bext=bext) as ens:
        ens.state_set(masks, Ms)
        ens.autotune(3)
        ens.run_fixed(1e-13, steps, use_graph=True)
        out, t = ens.state_get()
    assert abs(t - steps * 1e-13) < 1e-20
    for i in range(n):
        assert np.all(np.isfinite(out[i])), i
        mag = np.linalg.norm(out[i], axis=-1)
        assert np.allclose(mag[masks[i] != 0], 8.6e5, rtol=1e-12), i
    worst = 0.0
    for k in range(3):
        cand = [i for i in range(n) if kinds[i] == k]
        i = max(cand, key=lambda j: dims[j][0] * dims[j][1])
        X, Y, Z = dims[i]
        p = mmsb200.make_params(external=True, hext_t=[0.0], hext_b=[bext[i]])
        with mmsb200.Context(mmsb200.Grid(X, Y, Z, *D), p) as ctx:
            ctx.state_set(masks[i], Ms[i])
            ctx.run_fixed(1e-13, steps)
            ref_ctx, _ = ctx.state_get()
        a = max_angle_deg(out[i], ref_ctx, masks[i])
        worst = max(worst, a)
        assert a < 1e-3, (i, dims[i], a)
    print(f"C4 5000 steps: max angle vs single contexts {worst:.2e} deg")
