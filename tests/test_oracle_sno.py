"""The FP64 restatement of the surrogate network checks itself: its backward
against central finite differences of its own loss, and its layer-list
bookkeeping against the library's parameter count."""
import numpy as np

from oracle import sno


def test_param_count_matches_library(lib):
    import mmsb200
    assert sno.num_params() == mmsb200.SNO.num_params() == 232448


def test_patchify_roundtrip():
    u = np.random.default_rng(0).standard_normal((2, 3, 18, 23))
    H, W = sno.level_dims(18, 23)
    assert np.array_equal(sno.unpatchify(sno.patchify(u, H[0], W[0]), 18, 23), u)


def test_backward_matches_finite_differences():
    g = np.random.default_rng(5)
    u = g.standard_normal((2, 3, 20, 28))
    far = g.standard_normal((2, 3, 20, 28))
    w = sno.init_weights(11).astype(np.float64)
    loss, gw = sno.loss_and_grad(w, u, far)
    layers, _, _ = sno.architecture()
    # a few weights of every layer
    for layer in layers:
        n = layer["cout"] * sno.TAPS[layer["pat"]] * layer["cin"]
        for i in g.choice(n, 3, replace=False):
            k = layer["w_off"] + int(i)
            h = 1e-6 * max(1.0, abs(w[k]))
            wp, wm = w.copy(), w.copy()
            wp[k] += h
            wm[k] -= h
            fd = (sno.loss_and_grad(wp, u, far)[0] - sno.loss_and_grad(wm, u, far)[0]) / (2 * h)
            assert abs(fd - gw[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-5 * np.abs(gw).max(), (layer, k, fd, gw[k])


def test_network_is_linear():
    g = np.random.default_rng(9)
    w = sno.init_weights(3).astype(np.float64)
    a, b = g.standard_normal((2, 1, 3, 16, 16))
    fa, fb = sno.far_field(w, a), sno.far_field(w, b)
    assert np.allclose(sno.far_field(w, 2 * a - 3 * b), 2 * fa - 3 * fb, rtol=1e-10, atol=1e-10)
