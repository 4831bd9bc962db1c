"""The surrogate far-field network on the GPU: the tcgen05 forward, loss and
weight gradient against the FP64 restatement (oracle.sno), training, and the
surrogate solver's check / FMM fallback inside the time stepper."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case(seed, B=2, Z=3, Y=36, X=40):
    g = np.random.default_rng(seed)
    u = g.standard_normal((B, Z, Y, X)).astype(np.float32)
    far = g.standard_normal((B, Z, Y, X)).astype(np.float32)
    return u, far


@pytest.mark.parametrize("dims", [(3, 36, 40), (3, 64, 64), (1, 20, 28)])
def test_forward_matches_oracle(cuda, lib, dims):
    import torch
    import mmsb200
    from oracle import sno
    Z, Y, X = dims
    u, _ = _case(1, 2, Z, Y, X)
    w = sno.init_weights(7)
    with mmsb200.SNO(X, Y, Z, batch=2) as net:
        net.set_weights(w)
        wb = net.get_weights(bf16_rounded=True)
        assert np.array_equal(wb, sno.round_bf16(w))
        ud = torch.from_numpy(u).cuda()
        out = torch.zeros_like(ud)
        net.forward_dev(ud, out, 2)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
    ref = sno.far_field(wb.astype(np.float64), u.astype(np.float64))
    # BF16 weights are exact in both; activations are hi/lo pairs (~2^-16)
    assert rel_l2(got, ref) < 2e-5


def test_gradient_matches_oracle(cuda, lib):
    import torch
    import mmsb200
    from oracle import sno
    u, far = _case(2)
    w = sno.init_weights(8)
    with mmsb200.SNO(40, 36, 3, batch=2) as net:
        net.set_weights(w)
        wb = net.get_weights(bf16_rounded=True).astype(np.float64)
        loss, g = net.gradient(torch.from_numpy(u).cuda(), torch.from_numpy(far).cuda(), 2)
    lref, gref = sno.loss_and_grad(wb, u.astype(np.float64), far.astype(np.float64))
    assert abs(loss - lref) < 1e-5 * lref
    assert rel_l2(g, gref) < 1e-4
    layers, _, _ = sno.architecture()
    for layer in layers:
        n = layer["cout"] * sno.TAPS[layer["pat"]] * layer["cin"]
        sl = slice(layer["w_off"], layer["w_off"] + n)
        assert rel_l2(g[sl], gref[sl]) < 1e-3, layer


def test_training_fits_a_fixed_linear_map(cuda, lib):
    """Adam on the library's kernels drives the loss of a learnable target
    (the network's own output for other weights) down by orders of magnitude"""
    import torch
    import mmsb200
    from oracle import sno
    g = np.random.default_rng(3)
    B = 4
    u = g.standard_normal((16, 3, 32, 32)).astype(np.float32)
    wt = sno.init_weights(100).astype(np.float64) * 0.5
    tgt = sno.far_field(sno.round_bf16(wt).astype(np.float64), u.astype(np.float64)).astype(np.float32)
    ud, td = torch.from_numpy(u).cuda(), torch.from_numpy(tgt).cuda()
    with mmsb200.SNO(32, 32, 3, batch=B) as net:
        net.set_weights(sno.init_weights(1) * 0.5)
        losses = []
        for it in range(400):
            i = (it * B) % 16
            lr = 1e-3 if it < 300 else 2e-4
            losses.append(net.train_step(ud[i:i + B], td[i:i + B], B, lr))
    assert np.mean(losses[-10:]) < 0.05 * np.mean(losses[:5]), (losses[:5], losses[-10:])


def _surrogate_ctx(mmsb200, mask, M, w, every, tol, order=4, fast=True):
    Z, Y, X = mask.shape
    ctx = mmsb200.Context(mmsb200.Grid(X, Y, Z, 5e-9, 5e-9, 5e-9), mmsb200.make_params(),
                          mmsb200.make_solver(mmsb200.SOLVER_SURROGATE, order, 4))
    ctx.set_surrogate(w, every, tol, fast)
    ctx.state_set(mask, M)
    return ctx


@pytest.mark.parametrize("fast", [False, True])
def test_surrogate_potential_is_near_plus_network(cuda, lib, fast):
    """phi(surrogate) = exact near field + (Ms dx) net(rho dx / Ms); the fast
    mode rounds the activations to BF16"""
    import torch
    import mmsb200
    from mmsb200 import geometry
    from oracle import sno
    mask = geometry.random_blocks_mask(64, 48, 3, 0.3, 4, 5)
    M = geometry.random_sphere(mask, 6)
    w = sno.init_weights(4) * 0.1
    Ms, dx = 8.6e5, 5e-9
    grid = mmsb200.Grid(64, 48, 3, dx, dx, dx)
    with mmsb200.Context(grid, mmsb200.make_params(), mmsb200.make_solver(mmsb200.SOLVER_FMM, 4, 4)) as fctx:
        rho = torch.zeros(3 * 48 * 64, device="cuda")
        Mf = torch.from_numpy(M.astype(np.float32)).cuda()
        fctx.divergence_dev(Mf, rho)
        phi = torch.zeros_like(rho)
        near = torch.zeros_like(rho)
        fctx.potential_split_dev(rho, phi, near)
    with _surrogate_ctx(mmsb200, mask, M, w, 0, 1.0, fast=fast) as ctx:
        ps = torch.zeros_like(rho)
        ctx.potential_dev(rho, ps)
        torch.cuda.synchronize()
    u = (rho.cpu().numpy() * dx / Ms).reshape(1, 3, 48, 64).astype(np.float64)
    far = Ms * dx * sno.far_field(sno.round_bf16(w).astype(np.float64), u).ravel()
    ref = near.cpu().numpy() + far
    if fast:
        assert rel_l2(ps.cpu().numpy() - near.cpu().numpy(), far) < 1e-2
    else:
        assert rel_l2(ps.cpu().numpy(), ref) < 1e-5


def test_check_falls_back_to_fmm(cuda, lib):
    """an untrained network fails the first check; from then on the steps are
    the FMM's, bit for bit the trajectory of an FMM context from that state"""
    import mmsb200
    from mmsb200 import geometry
    from oracle import sno
    mask = geometry.disc(48, 48, 3, 22)
    M = geometry.random_inplane(mask, 12)
    with _surrogate_ctx(mmsb200, mask, M, sno.init_weights(2) * 0.1, 5, 1e-3) as ctx:
        ctx.run_fixed(1e-13, 4)
        st = ctx.surrogate_stats()
        assert st["checks"] == 0 and st["active"]
        ctx.run_fixed(1e-13, 1)          # 5th step: check
        st = ctx.surrogate_stats()
        assert st["checks"] == 1 and st["fallbacks"] == 1 and not st["active"] and st["last_err"] > 1e-3
        Mc, tc = ctx.state_get()
        ctx.run_fixed(1e-13, 10)
        Ms_, ts_ = ctx.state_get()
        assert ctx.surrogate_stats()["checks"] == 1
    with mmsb200.Context(mmsb200.Grid(48, 48, 3, 5e-9, 5e-9, 5e-9), mmsb200.make_params(),
                         mmsb200.make_solver(mmsb200.SOLVER_FMM, 4, 4)) as f:
        f.state_set(mask, Mc, tc)
        f.run_fixed(1e-13, 10)
        Mf, tf = f.state_get()
    assert np.array_equal(Ms_, Mf) and ts_ == tf


def test_check_keeps_a_passing_surrogate(cuda, lib):
    import mmsb200
    from mmsb200 import geometry
    from oracle import sno
    mask = geometry.disc(48, 48, 3, 22)
    M = geometry.random_inplane(mask, 13)
    with _surrogate_ctx(mmsb200, mask, M, sno.init_weights(2) * 0.1, 3, 1e9) as ctx:
        ctx.run_fixed(1e-13, 10)
        st = ctx.surrogate_stats()
        assert st["checks"] == 3 and st["fallbacks"] == 0 and st["active"]
        assert abs(ctx.surrogate_check() - st["last_err"]) < 0.5 * st["last_err"] + 1e-9


def test_trained_network_gain_over_near_field_only(cuda, lib):
    """What the trained network adds: on a held-out state of the benchmark
    workload (8 x 8 disc lattice, per-dot random in-plane M, seed outside the
    training set), the potential from the exact near field alone misses the
    far field entirely; near field + network recovers it to a few percent of
    the exact (direct-sum) potential."""
    import torch
    import mmsb200
    from mmsb200 import geometry, surrogate
    w, meta = surrogate.load_weights()
    assert w is not None, "trained weights missing"
    mask, M = geometry.per_dot_random_inplane(256, 256, 3, 12, 32, 4242)
    grid = mmsb200.Grid(256, 256, 3, 5e-9, 5e-9, 5e-9)
    rho = torch.zeros(3 * 256 * 256, device="cuda")
    exact, ps, phi, near = (torch.zeros_like(rho) for _ in range(4))
    with mmsb200.Context(grid, mmsb200.make_params(), mmsb200.make_solver(mmsb200.SOLVER_DIRECT)) as d:
        d.divergence_dev(torch.from_numpy(M.astype(np.float32)).cuda(), rho)
        d.potential_dev(rho, exact)
        d.sync()
    with mmsb200.Context(grid, mmsb200.make_params(), mmsb200.make_solver(mmsb200.SOLVER_FMM, 4, 4)) as f:
        f.potential_split_dev(rho, phi, near)
        f.sync()
    with _surrogate_ctx(mmsb200, mask, M, w, 0, 1.0) as s:
        s.potential_dev(rho, ps)
        s.sync()
    ex = exact.double()
    e_near = float((near.double() - ex).norm() / ex.norm())
    e_sur = float((ps.double() - ex).norm() / ex.norm())
    e_fmm = float((phi.double() - ex).norm() / ex.norm())
    assert e_near > 0.2            # the far field is a large part of phi here
    assert e_sur < 0.1 * e_near    # the network recovers > 90 % of it
    assert e_sur < 0.05
    assert e_fmm < 1e-3            # the check's reference is within the target


@pytest.mark.parametrize("tol,stays", [(1e9, True), (1e-9, False)])
def test_march_checks_on_rejected_steps(cuda, lib, tol, stays):
    """mms_march (step doubling) checks the surrogate on every rejected step:
    an oversized first step is rejected, the check runs, and with a tight
    tolerance the FMM takes over for the rest of the march, which still ends
    at the final time"""
    import mmsb200
    from mmsb200 import geometry, surrogate
    w, _ = surrogate.load_weights()
    assert w is not None
    mask = geometry.disc(48, 48, 3, 22)
    M = geometry.random_inplane(mask, 21)
    with _surrogate_ctx(mmsb200, mask, M, w, 100000, tol) as ctx:
        rows, st = ctx.march(2e-12, 1e-11, mode=1, rtol=1e-6, torque_stop=0.0)
        _, t = ctx.state_get()
        s = ctx.surrogate_stats()
    assert st == mmsb200.MMS_OK and abs(t - 2e-12) < 1e-24
    assert s["checks"] >= 1
    assert s["active"] == stays and s["fallbacks"] == (0 if stays else 1)
