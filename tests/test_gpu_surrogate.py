"""The learned far-field network on the GPU.

* Training kernels (mms_farnet_*) against the FP64 restatement (oracle.farnet):
  forward (<= 1e-5), loss (1e-6) and gradient (<= 1e-4 overall, 1e-3 per
  table: the weight gradients are split-BF16 tensor-core GEMMs, ~2^-16 per
  product), and Adam driving the loss down.
* The solver's inference pipeline (MMS_SOLVER_SURROGATE: encoder + upward
  pass, per-level interaction-list M2L, downward pass + decoder + near field)
  against the oracle's near field plus the same network (<= 3e-5, the
  tensor-core near field's split-BF16 rounding).
* The shipped weights on held-out states of the benchmark workload (256 x 256
  x 3 disc lattice, seeds outside the training set, states along LLG
  trajectories): demag phi within 1e-3 (mean and max) of the exact direct sum,
  and more accurate than the plain FMM at its default (P = 4, leaf 8), which
  is what the network gains over the method without it; its potential
  evaluation is also faster than the FMM's.
* The accurate network (24 + 16 channels, its own weights file): the same
  pipeline against the oracle, within 2e-5 of the exact sum on held-out
  states, 5x closer than the default, and faster than the FMM at P = 8.
* Inside the time stepper: 10^4 surrogate-assisted steps of the benchmark
  workload (FMM check every 50 steps, tolerance 1e-3) with no fallback and
  the final magnetisation within 1 deg of the plain-FMM trajectory; an
  untrained network fails its first check and the FMM takes over bit for
  bit; mms_march checks on rejected steps.
"""
import numpy as np
import pytest

from conftest import max_angle_deg, rel_l2

pytestmark = pytest.mark.gpu

DX = 5e-9
MS = 8.6e5


def _weights():
    from mmsb200 import surrogate
    w, _ = surrogate.load_weights()
    assert w is not None, "network weights missing (mms-gpu_b200/weights)"
    return w


def _wide_weights():
    from mmsb200 import surrogate
    w, _ = surrogate.load_weights(surrogate.ACCURATE_WEIGHTS)
    assert w is not None, "accurate network weights missing (mms-gpu_b200/weights)"
    return w


def _charges(n, seeds, oracle_mod, Y=None, kind="lattice"):
    """dimensionless charges u [B, 3, Y, n] of films (disc lattices or
    block-masked random-sphere films)"""
    from mmsb200 import geometry
    Y = Y or n
    out = []
    for s in seeds:
        if kind == "lattice":
            mask, M = geometry.per_dot_random_inplane(n, Y, 3, 12, 32, s)
        else:
            mask = geometry.random_blocks_mask(n, Y, 3, 0.3, 4, s)
            M = geometry.random_sphere(mask, s + 1)
        g = oracle_mod.Grid(n, Y, 3, 1.0, 1.0, 1.0)
        out.append(oracle_mod.divergence(g, M / MS))
    return np.stack(out)


@pytest.mark.parametrize("dims", [(64, 64), (70, 45), (40, 24), (128, 128)])
def test_forward_matches_oracle(cuda, lib, oracle_mod, dims):
    import torch
    import mmsb200
    from oracle import farnet as OF
    X, Y = dims
    w = _weights()
    u = _charges(X, (3, 4), oracle_mod, Y, "film").astype(np.float32)
    with mmsb200.FarNet(X, Y, batch=2) as net:
        net.set_weights(w)
        ud = torch.from_numpy(u).cuda()
        out = torch.zeros_like(ud)
        net.forward_dev(ud, out, 2)
        got = out.cpu().numpy()
    for b in range(2):
        ref, _ = OF.forward(w.astype(np.float64), u[b].astype(np.float64))
        assert rel_l2(got[b], ref) < 1e-5


def test_gradient_matches_oracle(cuda, lib, oracle_mod):
    import torch
    import mmsb200
    from oracle import farnet as OF
    w = _weights().astype(np.float64)
    rng = np.random.default_rng(7)
    w = (w * (1 + 0.05 * rng.standard_normal(w.size))).astype(np.float32)
    X = Y = 64
    u = _charges(X, (5, 6), oracle_mod, kind="film")
    batch = []
    for b in range(2):
        g = oracle_mod.Grid(X, Y, 3, 1.0, 1.0, 1.0)
        ex = oracle_mod.potential_direct(g, u[b])
        batch.append((u[b], ex - OF.near_field(u[b]), float((ex ** 2).sum())))
    lref, gref = OF.loss_and_gradient(w.astype(np.float64), batch)
    with mmsb200.FarNet(X, Y, batch=2) as net:
        net.set_weights(w)
        ud = torch.from_numpy(u.astype(np.float32)).cuda()
        fd = torch.from_numpy(np.stack([b[1] for b in batch]).astype(np.float32)).cuda()
        nd = torch.tensor([b[2] for b in batch], dtype=torch.float32, device="cuda")
        loss, g = net.gradient(ud, fd, nd, 2)
    assert abs(loss - lref) <= 1e-5 * lref, (loss, lref)
    assert rel_l2(g, gref) < 1e-4
    off = OF._layout(5)
    keys = ["W", "V"] + [("M2L", d) for d in range(2)] + [(n, 1) for n in ("M2M", "L2L")]
    ends = {"W": off["V"], "V": off[("M2L", 0)], ("M2L", 0): off[("M2L", 1)], ("M2L", 1): off[("M2L", 2)],
            ("M2M", 1): off[("L2L", 1)], ("L2L", 1): off[("M2M", 2)]}
    for k in keys:
        sl = slice(off[k], ends[k])
        assert rel_l2(g[sl], gref[sl]) < 1e-3, k


def test_training_reduces_the_loss(cuda, lib, oracle_mod):
    """Adam on the library's kernels fits a perturbed network back towards
    targets produced by the unperturbed one"""
    import torch
    import mmsb200
    from oracle import farnet as OF
    w = _weights().astype(np.float64)
    X = Y = 64
    u = _charges(X, (8, 9, 10, 11), oracle_mod, kind="film")
    tgt = np.stack([OF.forward(w, ub)[0] for ub in u]).astype(np.float32)
    nrm = np.array([(t.astype(np.float64) ** 2).sum() for t in tgt], np.float32) * 100.0
    rng = np.random.default_rng(1)
    wp = (w * (1 + 0.02 * rng.standard_normal(w.size))).astype(np.float32)
    with mmsb200.FarNet(X, Y, batch=4) as net:
        net.set_weights(wp)
        ud = torch.from_numpy(u.astype(np.float32)).cuda()
        td = torch.from_numpy(tgt).cuda()
        nd = torch.from_numpy(nrm).cuda()
        losses = [net.train_step(ud, td, nd, 4, 2e-4) for _ in range(150)]
    assert np.mean(losses[-5:]) < 0.2 * np.mean(losses[:3]), (losses[:3], losses[-5:])


def _surrogate_ctx(mmsb200, mask, M, w, every, tol, order=6, params=None):
    Z, Y, X = mask.shape
    ctx = mmsb200.Context(mmsb200.Grid(X, Y, Z, DX, DX, DX), params or mmsb200.make_params(),
                          mmsb200.make_solver(mmsb200.SOLVER_SURROGATE, order, 8))
    ctx.set_surrogate(w, every, tol)
    ctx.state_set(mask, M)
    return ctx


@pytest.mark.parametrize("dims", [(32, 32), (64, 64), (70, 45), (256, 256)])
def test_solver_potential_is_near_plus_network(cuda, lib, oracle_mod, dims):
    """phi(surrogate) = exact near field + dx^2 net(rho) for cubic cells;
    within 3e-5: the near field runs on the tensor cores at leaf 8 (split-BF16
    products, < 2e-5 from the FP32 near field)"""
    import torch
    import mmsb200
    from mmsb200 import geometry
    from oracle import farnet as OF
    X, Y = dims
    mask = geometry.random_blocks_mask(X, Y, 3, 0.3, 4, 5)
    M = geometry.random_sphere(mask, 6)
    w = _weights()
    rho = torch.zeros(3 * Y * X, device="cuda")
    with _surrogate_ctx(mmsb200, mask, M, w, 0, 1.0) as ctx:
        ctx.divergence_dev(torch.from_numpy(M.astype(np.float32)).cuda(), rho)
        ps = torch.zeros_like(rho)
        ctx.potential_dev(rho, ps)
        ctx.sync()
    r = rho.cpu().numpy().astype(np.float64).reshape(3, Y, X)
    far, _ = OF.forward(w.astype(np.float64), r)
    ref = DX * DX * (OF.near_field(r) + far)
    assert rel_l2(ps.cpu().numpy().reshape(3, Y, X), ref) < 3e-5


def held_out_states(n_states, seed=9100):
    """charges of held-out states of the benchmark workload: disc lattices
    with per-dot random in-plane M (seeds from 9100, outside the training
    generator's stream), each advanced 0..4000 steps along its trajectory
    with the external ramp"""
    import torch
    import mmsb200
    from mmsb200 import geometry
    X = Y = 256
    grid = mmsb200.Grid(X, Y, 3, DX, DX, DX)
    prm = mmsb200.make_params(external=True, hext_t=[0.0, 1e-8], hext_b=[[-0.05, 0, 0], [0.05, 0, 0]])
    N = 3 * X * Y
    out = []
    Mdev = torch.empty((N, 3), dtype=torch.float64, device="cuda")
    with mmsb200.Context(grid, prm, mmsb200.make_solver(mmsb200.SOLVER_FMM, 4, 8)) as dyn:
        for i in range(n_states):
            mask, M = geometry.per_dot_random_inplane(X, Y, 3, 12, 32, seed + i)
            dyn.state_set(mask, M)
            dyn.run_fixed(1e-13, 1000 * (i % 5))
            dyn.state_get_dev(Mdev)
            rho = torch.empty(N, dtype=torch.float32, device="cuda")
            dyn.divergence_dev(Mdev.float(), rho)
            out.append((mask, rho))
    return out


def test_trained_network_on_held_out_benchmark_states(cuda, lib):
    """demag phi of the network vs the exact direct sum on held-out states:
    within 1e-3 (mean and max), and below the plain FMM's error at its
    default (P = 4, leaf 8); the network's potential evaluation is faster
    than the FMM's (CUDA events, same stream)"""
    import torch
    import mmsb200
    w = _weights()
    states = held_out_states(10)
    grid = mmsb200.Grid(256, 256, 3, DX, DX, DX)
    e_sur, e_fmm = [], []
    with mmsb200.Context(grid, mmsb200.make_params(), mmsb200.make_solver(mmsb200.SOLVER_DIRECT)) as d, \
            mmsb200.Context(grid, mmsb200.make_params(), mmsb200.make_solver(mmsb200.SOLVER_FMM, 4, 8)) as f, \
            mmsb200.Context(grid, mmsb200.make_params(), mmsb200.make_solver(mmsb200.SOLVER_SURROGATE, 6, 8)) as s:
        s.set_surrogate(w, 0, 1.0)
        for _, rho in states:
            ex, pf, ps = (torch.zeros_like(rho) for _ in range(3))
            d.potential_dev(rho, ex)
            f.potential_dev(rho, pf)
            s.potential_dev(rho, ps)
            torch.cuda.synchronize()
            exd = ex.double()
            e_sur.append(float((ps.double() - exd).norm() / exd.norm()))
            e_fmm.append(float((pf.double() - exd).norm() / exd.norm()))
        times = {}
        rho = states[-1][1]
        out = torch.zeros_like(rho)
        for name, c in (("fmm", f), ("surrogate", s)):
            stream = torch.cuda.current_stream()
            for _ in range(5):
                c.potential_dev(rho, out)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(50):
                c.potential_dev(rho, out)
            e1.record(stream)
            torch.cuda.synchronize()
            times[name] = e0.elapsed_time(e1) / 50
    print(f"held-out states: network rel-L2 mean {np.mean(e_sur):.3e} max {np.max(e_sur):.3e}; "
          f"FMM P=4 mean {np.mean(e_fmm):.3e} max {np.max(e_fmm):.3e}; potential ms {times}")
    assert np.mean(e_sur) <= 1e-3 and np.max(e_sur) <= 1e-3
    assert np.mean(e_sur) < np.mean(e_fmm) and np.max(e_sur) < np.max(e_fmm)
    assert times["surrogate"] < times["fmm"], times


@pytest.mark.parametrize("dims", [(32, 32), (70, 45), (256, 256)])
def test_wide_network_potential_is_near_plus_network(cuda, lib, oracle_mod, dims):
    """the accurate network (24 + 16 channels, picked by the weight count)
    runs the same pipeline: phi = exact near field + dx^2 net(rho), against
    the oracle's restatement of the same weights (3e-5: the tensor-core near
    field's rounding)"""
    import torch
    import mmsb200
    from mmsb200 import geometry
    from oracle import farnet as OF
    X, Y = dims
    mask = geometry.random_blocks_mask(X, Y, 3, 0.3, 4, 5)
    M = geometry.random_sphere(mask, 6)
    w = _wide_weights()
    rho = torch.zeros(3 * Y * X, device="cuda")
    with _surrogate_ctx(mmsb200, mask, M, w, 0, 1.0) as ctx:
        ctx.divergence_dev(torch.from_numpy(M.astype(np.float32)).cuda(), rho)
        ps = torch.zeros_like(rho)
        ctx.potential_dev(rho, ps)
        ctx.sync()
    r = rho.cpu().numpy().astype(np.float64).reshape(3, Y, X)
    far, _ = OF.forward(w.astype(np.float64), r)
    ref = DX * DX * (OF.near_field(r) + far)
    assert rel_l2(ps.cpu().numpy().reshape(3, Y, X), ref) < 3e-5


def test_wide_network_on_held_out_states_and_against_fmm_p8(cuda, lib):
    """the accurate network on held-out states of the benchmark workload:
    within 2e-5 of the exact sum (mean and max), at least 5x closer than the
    default network, and its potential evaluation faster than the FMM's at
    P = 8 (CUDA events, same stream), whose error it approaches"""
    import torch
    import mmsb200
    states = held_out_states(5)
    grid = mmsb200.Grid(256, 256, 3, DX, DX, DX)
    e = {"wide": [], "default": [], "fmm8": []}
    times = {}
    with mmsb200.Context(grid, mmsb200.make_params(), mmsb200.make_solver(mmsb200.SOLVER_DIRECT)) as d, \
            mmsb200.Context(grid, mmsb200.make_params(), mmsb200.make_solver(mmsb200.SOLVER_FMM, 8, 8)) as f8, \
            mmsb200.Context(grid, mmsb200.make_params(), mmsb200.make_solver(mmsb200.SOLVER_SURROGATE, 6, 8)) as sw, \
            mmsb200.Context(grid, mmsb200.make_params(), mmsb200.make_solver(mmsb200.SOLVER_SURROGATE, 6, 8)) as sd:
        sw.set_surrogate(_wide_weights(), 0, 1.0)
        sd.set_surrogate(_weights(), 0, 1.0)
        for _, rho in states:
            ex = torch.zeros_like(rho)
            d.potential_dev(rho, ex)
            for name, c in (("wide", sw), ("default", sd), ("fmm8", f8)):
                p = torch.zeros_like(rho)
                c.potential_dev(rho, p)
                torch.cuda.synchronize()
                e[name].append(float((p.double() - ex.double()).norm() / ex.double().norm()))
        rho = states[-1][1]
        out = torch.zeros_like(rho)
        for name, c in (("wide", sw), ("fmm8", f8)):
            stream = torch.cuda.current_stream()
            for _ in range(5):
                c.potential_dev(rho, out)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(50):
                c.potential_dev(rho, out)
            e1.record(stream)
            torch.cuda.synchronize()
            times[name] = e0.elapsed_time(e1) / 50
    print(f"accurate network: rel-L2 mean {np.mean(e['wide']):.3e} max {np.max(e['wide']):.3e}; default "
          f"{np.mean(e['default']):.3e}; FMM P=8 {np.mean(e['fmm8']):.3e}; potential ms {times}")
    assert np.max(e["wide"]) <= 2e-5
    assert np.mean(e["wide"]) * 5 < np.mean(e["default"])
    assert times["wide"] < times["fmm8"], times


def test_assisted_run_1e4_steps_tracks_the_fmm(cuda, lib):
    """10^4 steps of the benchmark workload with the network (FMM P = 6 check
    every 50 steps, tolerance 1e-3): no fallback, every check within the
    tolerance, and the final M within 1 deg of the plain-FMM run"""
    import mmsb200
    from mmsb200 import geometry
    mask, M = geometry.per_dot_random_inplane(256, 256, 3, 12, 32, 2010)
    prm = mmsb200.make_params(external=True, hext_t=[0.0, 1e-8], hext_b=[[-0.05, 0, 0], [0.05, 0, 0]])
    n = 10000
    with _surrogate_ctx(mmsb200, mask, M, _weights(), 50, 1e-3, params=prm) as ctx:
        ctx.run_fixed(1e-13, n)
        Ms_, _ = ctx.state_get()
        st = ctx.surrogate_stats()
    with mmsb200.Context(mmsb200.Grid(256, 256, 3, DX, DX, DX), prm, mmsb200.make_solver(mmsb200.SOLVER_FMM, 4, 8)) as f:
        f.state_set(mask, M)
        f.run_fixed(1e-13, n)
        Mf, _ = f.state_get()
    ang = max_angle_deg(Ms_, Mf, mask)
    print(f"assisted 1e4 steps: {st}; final max angle vs plain FMM {ang:.3e} deg")
    assert st["checks"] == n // 50 and st["fallbacks"] == 0 and st["active"]
    assert st["max_err"] <= 1e-3
    assert ang <= 1.0


def test_check_falls_back_to_fmm(cuda, lib):
    """an untrained (zero) network fails the first check; from then on the
    steps are the FMM's, bit for bit the trajectory of an FMM context from
    that state"""
    import mmsb200
    from mmsb200 import geometry
    mask = geometry.disc(48, 48, 3, 22)
    M = geometry.random_inplane(mask, 12)
    wz = np.zeros(mmsb200.FarNet.num_params(), np.float32)
    with _surrogate_ctx(mmsb200, mask, M, wz, 5, 1e-3, order=4) as ctx:
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
    with mmsb200.Context(mmsb200.Grid(48, 48, 3, DX, DX, DX), mmsb200.make_params(),
                         mmsb200.make_solver(mmsb200.SOLVER_FMM, 4, 8)) as f:
        f.state_set(mask, Mc, tc)
        f.run_fixed(1e-13, 10)
        Mf, tf = f.state_get()
    assert np.array_equal(Ms_, Mf) and ts_ == tf


def test_check_keeps_a_passing_surrogate(cuda, lib):
    import mmsb200
    from mmsb200 import geometry
    mask = geometry.disc(48, 48, 3, 22)
    M = geometry.random_inplane(mask, 13)
    with _surrogate_ctx(mmsb200, mask, M, _weights(), 3, 1e-3) as ctx:
        ctx.run_fixed(1e-13, 10)
        st = ctx.surrogate_stats()
        assert st["checks"] == 3 and st["fallbacks"] == 0 and st["active"]
        assert st["max_err"] < 1e-3


@pytest.mark.parametrize("tol,stays", [(1e9, True), (1e-12, False)])
def test_march_checks_on_rejected_steps(cuda, lib, tol, stays):
    """mms_march (step doubling) checks the surrogate on every rejected step:
    an oversized first step is rejected, the check runs, and with a tolerance
    below the network's error the FMM takes over for the rest of the march,
    which still ends at the final time"""
    import mmsb200
    from mmsb200 import geometry
    mask = geometry.disc(48, 48, 3, 22)
    M = geometry.random_inplane(mask, 21)
    with _surrogate_ctx(mmsb200, mask, M, _weights(), 100000, tol) as ctx:
        rows, st = ctx.march(2e-12, 1e-11, mode=1, rtol=1e-6, torque_stop=0.0)
        _, t = ctx.state_get()
        s = ctx.surrogate_stats()
    assert st == mmsb200.MMS_OK and abs(t - 2e-12) < 1e-24
    assert s["checks"] >= 1
    assert s["active"] == stays and s["fallbacks"] == (0 if stays else 1)


def test_time_potential_cli(cuda, lib):
    """python -m mmsb200.surrogate --time: one JSON line with the network's and
    the FMM's potential time and error on the benchmark workload"""
    import json
    import os
    import subprocess
    import sys
    env = dict(os.environ)
    env["PYTHONPATH"] = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mms-gpu_b200")
    r = subprocess.run([sys.executable, "-m", "mmsb200.surrogate", "--time", "--evals", "10"], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["network"]["rel_l2_vs_direct"] < 1e-4 < d["fmm"]["rel_l2_vs_direct"] < 1e-3
    assert d["network"]["us"] > 0 and d["fmm"]["us"] > 0
