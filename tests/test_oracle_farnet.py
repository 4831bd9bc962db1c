"""The FP64 restatement of the learned far-field network checks itself and the
network's starting weights: the gradient of its loss against central finite
differences, its weight layout against the library's parameter count, and the
nested-SVD start (mmsb200.farnet.h2_init) against the exact FP64 potential of
the oracle's direct sum: near field (exact) + network far field within 1e-4
relative on disc-lattice films of 64^2 and 128^2 x 3 cells."""
import numpy as np
import pytest

from conftest import rel_l2

D1 = (1.0, 1.0, 1.0)  # cell units: the network is scale free for cubic cells


@pytest.fixture(scope="module")
def w0():
    from mmsb200 import farnet
    return farnet.h2_init()


@pytest.fixture(scope="module")
def w_wide():
    from mmsb200 import farnet
    return farnet.h2_init(ne=farnet.WIDE[0], no=farnet.WIDE[1])


def _film(n, seed, oracle_mod, kind="lattice"):
    from mmsb200 import geometry
    if kind == "lattice":
        mask, M = geometry.per_dot_random_inplane(n, n, 3, 12, 32, seed)
    else:
        mask = geometry.random_blocks_mask(n, n, 3, 0.3, 4, seed)
        M = geometry.random_sphere(mask, seed + 1)
    g = oracle_mod.Grid(n, n, 3, *D1)
    u = oracle_mod.divergence(g, M / 8.6e5)
    return g, u


def test_layout_matches_library(lib):
    import mmsb200
    from mmsb200 import farnet
    from oracle import farnet as OF
    assert farnet.num_params() == OF._layout(5)["total"] == mmsb200.FarNet.num_params()
    L = mmsb200.load()
    ne, no = farnet.WIDE
    assert L.mms_surrogate_num_params(24) == farnet.num_params()
    assert L.mms_surrogate_num_params(40) == farnet.num_params(ne=ne, no=no) == OF._layout(5, ne, no)["total"]
    assert L.mms_surrogate_num_params(32) == 0
    assert farnet.width_of(farnet.num_params(ne=ne, no=no)) == (ne, no)


def test_shipped_weights_are_the_nested_svd_starts(w0, w_wide):
    """the two weight files hold h2_init's starts (trained = 0 in their meta)"""
    from mmsb200 import surrogate
    for path, w in ((surrogate.DEFAULT_WEIGHTS, w0), (surrogate.ACCURATE_WEIGHTS, w_wide)):
        got, meta = surrogate.load_weights(path)
        assert got is not None and int(meta["trained"]) == 0
        assert np.array_equal(got, w.astype(np.float32)), path


@pytest.mark.parametrize("n,kind", [(64, "lattice"), (128, "lattice"), (64, "film")])
def test_nested_svd_start_is_accurate(oracle_mod, w0, n, kind):
    from oracle import farnet as OF
    g, u = _film(n, 3, oracle_mod, kind)
    exact = oracle_mod.potential_direct(g, u)
    far, _ = OF.forward(w0, u)
    err = rel_l2(OF.near_field(u) + far, exact)
    assert err < (1e-4 if kind == "lattice" else 3e-4), err


@pytest.mark.parametrize("n,kind", [(128, "lattice"), (64, "film")])
def test_wide_start_is_ten_times_closer(oracle_mod, w0, w_wide, n, kind):
    """the accurate network (24 + 16 channels): below 1e-5 on the disc
    lattice, and at least 5x closer to the exact sum than the default"""
    from oracle import farnet as OF
    g, u = _film(n, 3, oracle_mod, kind)
    exact = oracle_mod.potential_direct(g, u)
    near = OF.near_field(u)
    err = [rel_l2(near + OF.forward(w, u)[0], exact) for w in (w0, w_wide)]
    if kind == "lattice":
        assert err[1] < 1e-5, err
    assert err[1] < err[0] / 5, err


def test_gradient_matches_finite_differences(oracle_mod, w0):
    from oracle import farnet as OF
    rng = np.random.default_rng(0)
    w = w0 * (1 + 0.05 * rng.standard_normal(w0.size))
    batch = []
    for seed in (1, 2):
        g, u = _film(64, seed, oracle_mod, "film")
        ex = oracle_mod.potential_direct(g, u)
        batch.append((u, ex - OF.near_field(u), float((ex ** 2).sum())))
    _, gr = OF.loss_and_gradient(w, batch)
    off = OF._layout(5)
    idx = [off["W"] + 5, off["V"] + 100, off[("M2L", 0)] + 10 * OF.OSZ + 3,
           off[("M2L", 1)] + 31 * OF.OSZ + OF.NE * OF.NE + 5, off[("M2M", 1)] + 2 * OF.OSZ + 7,
           off[("L2L", 1)] + 3 * OF.OSZ + OF.NE * OF.NE + 9, off[("M2L", 0)] + 4 * OF.OSZ + 17]
    for i in idx:
        # phi is linear in each single weight, so the loss is quadratic in it
        # and the central difference is exact for any step: take a large one
        h = 0.1 * max(1e-2, abs(w[i]))
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (OF.loss_and_gradient(wp, batch)[0] - OF.loss_and_gradient(wm, batch)[0]) / (2 * h)
        assert abs(gr[i] - fd) <= 1e-6 * abs(fd) + 1e-15, (i, gr[i], fd)
    # the nine near-field slots of every depth never enter the network
    for d in range(5):
        for s in (16, 17, 18, 23, 24, 25, 30, 31, 32):
            o = off[("M2L", d)] + s * OF.OSZ
            assert not np.any(gr[o:o + OF.OSZ])


def test_training_schedule_stays_within_lr_max():
    """the warm-up + cosine schedule of the training driver: never above
    lr_max, lr_max after the warm-up, lr_min at the last step, for long and
    very short runs"""
    from mmsb200.surrogate import lr_at
    for steps in (1, 2, 3, 10, 4000):
        lrs = [lr_at(i, steps, 1e-4, 1e-6, 0.02) for i in range(steps)]
        assert max(lrs) <= 1e-4 * (1 + 1e-12), (steps, max(lrs))
        assert min(lrs) >= 1e-6 * (1 - 1e-12)
        if steps > 1:
            assert abs(lrs[-1] - 1e-6) < 1e-12
    lrs = [lr_at(i, 4000, 1e-4, 1e-6, 0.02) for i in range(4000)]
    assert lrs[0] < 1e-6 * 2 and abs(max(lrs) - 1e-4) < 1e-9
