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
