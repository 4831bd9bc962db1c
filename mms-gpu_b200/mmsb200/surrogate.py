"""Training and use of the learned far-field network (mms_farnet).

Training pairs are (u, far, nrm2): u = rho dx / Ms, far = (phi_FMM -
phi_near) / (Ms dx) and nrm2 = |phi_FMM / (Ms dx)|^2, taken along LLG
trajectories that the library itself integrates: instances of 64..256 cells a
side (disc lattices, discs, ellipses, rectangles, block-masked films;
in-plane, per-dot, vortex or random initial states; constant or ramped
in-plane fields up to 50 mT) placed in a 256 x 256 x 3 canvas, stepped with
the FMM, and evaluated every few steps by a high-order FMM (P = 8, leaf 8,
within ~4e-6 of the exact sum) whose exact near field
(mms_potential_split_dev) is subtracted.  The network starts from nested SVD
bases of the 1/r interactions (farnet.h2_init) and is fitted by the library's
own forward / adjoint / tensor-core weight-gradient / Adam kernels
(mms_farnet_train_step) on the relative error of the total potential.

Everything here runs through the C ABI; torch only holds device buffers.
"""
from __future__ import annotations

import math
import os
import time

import numpy as np

from . import (SOLVER_FMM, Context, FarNet, Grid, farnet, geometry, make_params, make_solver)

MS = geometry.MS_PERMALLOY
DX = 5e-9
LEAF = 8
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "weights")
DEFAULT_WEIGHTS = os.path.join(WEIGHTS_DIR, "farnet_w24_d5.npz")   # 16 + 8 channels: the default
ACCURATE_WEIGHTS = os.path.join(WEIGHTS_DIR, "farnet_w40_d5.npz")  # 24 + 16 channels: 5-10x closer to exact


# ---- training geometries ------------------------------------------------------

def _instance(rng, Z, kinds=None):
    """(mask, M) of one instance with sides drawn from 64..256; kinds: the
    geometry kinds to draw from (0, 1 disc lattices; 2 disc or ellipse; 3
    rectangle; 4 block-masked film; 5 vortex-quadrant square), all when None"""
    sides = (64, 96, 128, 160, 192, 224, 256)
    sx, sy = int(rng.choice(sides)), int(rng.choice(sides))
    kind = int(rng.integers(0, 6)) if kinds is None else int(rng.choice(kinds))
    seed = int(rng.integers(0, 2 ** 31))
    if kind in (0, 1):  # disc lattice (the benchmark's family)
        r = int(rng.integers(5, 17))
        pitch = 2 * r + int(rng.integers(2, 14))
        if kind == 0:
            mask, M = geometry.per_dot_random_inplane(sx, sy, Z, r, pitch, seed)
        else:
            mask = geometry.disc_lattice(sx, sy, Z, r, pitch)
            M = geometry.random_sphere(mask, seed)
    elif kind == 2:  # one disc or ellipse
        ax = rng.uniform(0.25, 0.5) * (sx - 2)
        ay = rng.uniform(0.25, 0.5) * (sy - 2)
        mask = geometry.from_plane(geometry.ellipse_plane(sx, sy, (sx - 1) / 2, (sy - 1) / 2, ax, ay), Z)
        M = geometry.vortex(mask, 2.0, 10.0, seed) if rng.uniform() < 0.5 else geometry.random_inplane(mask, seed)
    elif kind == 3:  # rectangle
        mask = geometry.reference_default(sx, sy, Z)
        M = geometry.single_domain(mask, phi=rng.uniform(0, 2 * np.pi)) if rng.uniform() < 0.3 else \
            geometry.random_inplane(mask, seed)
    elif kind == 4:  # block-masked film
        mask = geometry.random_blocks_mask(sx, sy, Z, rng.uniform(0.1, 0.5), 4, seed)
        M = geometry.random_sphere(mask, seed + 1)
    else:  # vortex-quadrant square
        mask = geometry.reference_default(sx, sy, Z)
        M = geometry.vortex_quadrants(mask)
    return mask, M


def _place(mask, M, X, Y, rng):
    Z, sy, sx = mask.shape
    ox, oy = int(rng.integers(0, X - sx + 1)), int(rng.integers(0, Y - sy + 1))
    m = np.zeros((Z, Y, X), np.uint8)
    v = np.zeros((Z, Y, X, 3))
    m[:, oy:oy + sy, ox:ox + sx] = mask
    v[:, oy:oy + sy, ox:ox + sx] = M
    return m, v


def _field(rng):
    """external field table: constant or a 10 ns ramp along a random in-plane direction"""
    ph = rng.uniform(0, 2 * np.pi)
    d = np.array([np.cos(ph), np.sin(ph), 0.0])
    if rng.uniform() < 0.5:
        b = 0.05 * math.sqrt(rng.uniform())
        return [0.0], [list(b * d)]
    return [0.0, 1e-8], [list(-0.05 * d), list(0.05 * d)]


def generate_pairs(n_pairs, X=256, Y=256, Z=3, snaps_per_run=50, steps_between=10, dt=1e-13, seed=2010,
                   target_order=8, progress=None, kinds=None):
    """n_pairs training pairs: torch tensors U, F [n, Z, Y, X] and N2 [n]
    (float32, cuda)"""
    import torch
    rng = np.random.Generator(np.random.Philox(seed))
    N = X * Y * Z
    U = torch.empty((n_pairs, Z, Y, X), dtype=torch.float32, device="cuda")
    F = torch.empty_like(U)
    N2 = torch.empty(n_pairs, dtype=torch.float32, device="cuda")
    grid = Grid(X, Y, Z, DX, DX, DX)
    # one stream for both contexts and for the torch copies: the charges the
    # dynamics context writes are read by the target context in order
    st = torch.cuda.Stream()
    dyn = Context(grid, make_params(), make_solver(SOLVER_FMM, 4, LEAF), stream=st.cuda_stream)
    tgt = Context(grid, make_params(), make_solver(SOLVER_FMM, target_order, LEAF), stream=st.cuda_stream)
    Mdev = torch.empty((N, 3), dtype=torch.float64, device="cuda")
    rho = torch.empty(N, dtype=torch.float32, device="cuda")
    phi = torch.empty_like(rho)
    near = torch.empty_like(rho)
    k = 0
    t0 = time.time()
    torch.cuda.synchronize()
    try:
        with torch.cuda.stream(st):
            while k < n_pairs:
                mask, M = _place(*_instance(rng, Z, kinds), X, Y, rng)
                ht, hb = _field(rng)
                dyn.set_params(make_params(external=True, hext_t=ht, hext_b=hb))
                dyn.state_set(mask, M)
                for s in range(snaps_per_run):
                    if k >= n_pairs:
                        break
                    if s:
                        dyn.run_fixed(dt, steps_between)
                    dyn.state_get_dev(Mdev)
                    dyn.divergence_dev(Mdev.float(), rho)
                    tgt.potential_split_dev(rho, phi, near)
                    U[k] = (rho * (DX / MS)).view(Z, Y, X)
                    F[k] = ((phi - near) / (MS * DX)).view(Z, Y, X)
                    N2[k] = ((phi / (MS * DX)).double() ** 2).sum().float()
                    k += 1
                if progress:
                    progress(k, time.time() - t0)
        torch.cuda.synchronize()
    finally:
        dyn.close()
        tgt.close()
    return U, F, N2


def benchmark_pairs(n_pairs, seed=777, X=256, Y=256, Z=3, steps_between=20, dt=1e-13):
    """held-out pairs of the benchmark workload itself (8 x 8 disc lattice,
    r = 12, pitch 32, per-dot random in-plane M, B_x ramp -50..+50 mT / 10 ns),
    seeds disjoint from training: U, F, N2 as generate_pairs, plus the total
    potential P [n, Z, Y, X] (dimensionless)"""
    import torch
    grid = Grid(X, Y, Z, DX, DX, DX)
    N = X * Y * Z
    U = torch.empty((n_pairs, Z, Y, X), dtype=torch.float32, device="cuda")
    F = torch.empty_like(U)
    P = torch.empty_like(U)
    Mdev = torch.empty((N, 3), dtype=torch.float64, device="cuda")
    rho = torch.empty(N, dtype=torch.float32, device="cuda")
    phi = torch.empty_like(rho)
    near = torch.empty_like(rho)
    prm = make_params(external=True, hext_t=[0.0, 1e-8], hext_b=[[-0.05, 0, 0], [0.05, 0, 0]])
    st = torch.cuda.Stream()  # one stream for both contexts and the torch copies
    torch.cuda.synchronize()
    with torch.cuda.stream(st), Context(grid, prm, make_solver(SOLVER_FMM, 4, LEAF), stream=st.cuda_stream) as dyn, \
            Context(grid, make_params(), make_solver(SOLVER_FMM, 8, LEAF), stream=st.cuda_stream) as tgt:
        per_run = 10
        for k in range(n_pairs):
            if k % per_run == 0:
                mask, M = geometry.per_dot_random_inplane(X, Y, Z, 12, 32, seed + k)
                dyn.state_set(mask, M)
            else:
                dyn.run_fixed(dt, steps_between)
            dyn.state_get_dev(Mdev)
            dyn.divergence_dev(Mdev.float(), rho)
            tgt.potential_split_dev(rho, phi, near)
            U[k] = (rho * (DX / MS)).view(Z, Y, X)
            F[k] = ((phi - near) / (MS * DX)).view(Z, Y, X)
            P[k] = (phi / (MS * DX)).view(Z, Y, X)
        torch.cuda.synchronize()
    N2 = (P.double() ** 2).flatten(1).sum(1).float()
    return U, F, N2, P


# ---- training -------------------------------------------------------------------

def evaluate(net, U, F, N2, P=None, batch=8):
    """mean and max rel-L2 of the total potential (far-field error over
    |phi|) over the pairs"""
    import torch
    out = torch.empty((batch,) + tuple(U.shape[1:]), dtype=torch.float32, device="cuda")
    et = []
    for i in range(0, U.shape[0], batch):
        nb = min(batch, U.shape[0] - i)
        net.forward_dev(U[i:i + nb], out, nb)
        d = (out[:nb] - F[i:i + nb]).double()
        et += (d.flatten(1).norm(dim=1) / N2[i:i + nb].double().sqrt()).tolist()
    return dict(total_mean=float(np.mean(et)), total_max=float(np.max(et)))


def lr_at(it, steps, lr_max, lr_min, warmup):
    """step size of step `it` of `steps`: a linear warm-up over the first
    `warmup` fraction (at least one step, never above lr_max), then a cosine
    decay from lr_max to lr_min"""
    w = it / max(1, steps - 1)
    if w < warmup:
        return lr_max * min(1.0, (it + 1) / max(1.0, warmup * steps))
    return lr_min + 0.5 * (lr_max - lr_min) * (1 + math.cos(math.pi * (w - warmup) / (1 - warmup)))


def train(U, F, N2, steps, batch=8, lr_max=1e-4, lr_min=1e-6, warmup=0.02, seed=1, weights=None, val=None,
          log_every=250, log=print):
    """fits the network (from `weights`, else the nested-SVD start) to the
    pairs with Adam on a warm-up + cosine schedule; steps are relative to
    each weight's magnitude (farnet.step_scale), so lr is a relative step;
    returns (weights, history, start weights); with `val`, the weights of the
    best validation mean"""
    import torch
    Z, Y, X = U.shape[1:]
    net = FarNet(X, Y, batch)
    w0 = np.asarray(farnet.h2_init() if weights is None else weights, np.float32)
    net.set_weights(w0)
    net.set_step_scale(farnet.step_scale(w0))
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    t0 = time.time()
    n = U.shape[0]
    perm = torch.randperm(n, generator=g)
    pos = 0
    ub = torch.empty((batch, Z, Y, X), dtype=torch.float32, device="cuda")
    fb = torch.empty_like(ub)
    nb2 = torch.empty(batch, dtype=torch.float32, device="cuda")
    best = (None, None)
    if val is not None:
        rec = dict(step=-1, s=0.0)
        rec.update(evaluate(net, *val))
        hist.append(rec)
        best = (rec["total_mean"], net.get_weights())
        if log:
            log(rec)
    for it in range(steps):
        if pos + batch > n:
            perm = torch.randperm(n, generator=g)
            pos = 0
        idx = perm[pos:pos + batch].cuda()
        pos += batch
        torch.index_select(U, 0, idx, out=ub)
        torch.index_select(F, 0, idx, out=fb)
        torch.index_select(N2, 0, idx, out=nb2)
        lr = lr_at(it, steps, lr_max, lr_min, warmup)
        loss = net.train_step(ub, fb, nb2, batch, lr)
        if it % log_every == 0 or it == steps - 1:
            rec = dict(step=it, loss_rel=math.sqrt(max(loss, 0.0)), lr=lr, s=time.time() - t0)
            if val is not None:
                rec.update(evaluate(net, *val))
                if rec["total_mean"] < best[0]:
                    best = (rec["total_mean"], net.get_weights())
            hist.append(rec)
            if log:
                log(rec)
    w = best[1] if best[1] is not None else net.get_weights()
    net.close()
    return w, hist, w0


def save_weights(path, w, meta):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, weights=np.asarray(w, np.float32), **{k: np.asarray(v) for k, v in meta.items()})


def load_weights(path=DEFAULT_WEIGHTS):
    """(weights, meta) or (None, None) when the file is absent"""
    if not os.path.exists(path):
        return None, None
    with np.load(path) as z:
        meta = {k: z[k] for k in z.files if k != "weights"}
        return z["weights"].astype(np.float32), meta


def time_potential(evals=50, X=256, Y=256, Z=3, seed=9100, order=4, weights=None):
    """one potential evaluation of the network (exact near field + learned far
    field) against the FMM at `order` (leaf 8) on a state of the benchmark
    workload (disc lattice, per-dot random in-plane M): mean time over
    `evals` back-to-back evaluations (CUDA events on the contexts' stream,
    after 5 untimed), and each one's rel-L2 error against the exact sum;
    the network runs first, then the FMM"""
    import torch
    from . import SOLVER_DIRECT, SOLVER_SURROGATE
    w = weights if weights is not None else load_weights()[0]
    if w is None:
        raise RuntimeError("network weights missing")
    grid = Grid(X, Y, Z, DX, DX, DX)
    mask, M = geometry.per_dot_random_inplane(X, Y, Z, 12, 32, seed)
    st = torch.cuda.Stream()
    out = {}
    with torch.cuda.stream(st):
        rho = torch.empty(X * Y * Z, dtype=torch.float32, device="cuda")
        ref = torch.empty_like(rho)
        with Context(grid, make_params(), make_solver(SOLVER_DIRECT), stream=st.cuda_stream) as d:
            d.divergence_dev(torch.from_numpy(M.astype(np.float32)).cuda(), rho)
            d.potential_dev(rho, ref)
            d.sync()
        for name, slv in (("network", make_solver(SOLVER_SURROGATE, 6, LEAF)),
                          ("fmm", make_solver(SOLVER_FMM, order, LEAF))):
            with Context(grid, make_params(), slv, stream=st.cuda_stream) as c:
                if name == "network":
                    c.set_surrogate(w, 0, 1.0)
                phi = torch.empty_like(rho)
                for _ in range(5):
                    c.potential_dev(rho, phi)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                for _ in range(evals):
                    c.potential_dev(rho, phi)
                e1.record(st)
                c.sync()
                torch.cuda.synchronize()
                out[name] = {"us": e0.elapsed_time(e1) * 1e3 / evals,
                             "rel_l2_vs_direct": float((phi.double() - ref.double()).norm() / ref.double().norm())}
    out["fmm"]["order"] = order
    return out


def main(argv=None):
    import argparse
    import json

    import torch
    ap = argparse.ArgumentParser(description="train the learned far-field network, or time it against the FMM")
    ap.add_argument("--time", action="store_true",
                    help="time one potential evaluation, network vs FMM, on the benchmark workload, and exit")
    ap.add_argument("--evals", type=int, default=50, help="evaluations timed with --time")
    ap.add_argument("--weights", default="default",
                    help="network timed with --time: default, accurate, or a weights file")
    ap.add_argument("--start", choices=["default", "accurate"], default=None,
                    help="write the nested-SVD start of that network (default: 16 + 8 channels, accurate: "
                         "24 + 16) to --out, or to its shipped file, and exit")
    ap.add_argument("--pairs", type=int, default=4000)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-4, help="peak relative step")
    ap.add_argument("--val", type=int, default=40)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--log", default=None)
    a = ap.parse_args(argv)
    if a.start:
        ne, no = (farnet.NE, farnet.NO) if a.start == "default" else farnet.WIDE
        out = a.out if a.out != DEFAULT_WEIGHTS else (DEFAULT_WEIGHTS if a.start == "default" else ACCURATE_WEIGHTS)
        save_weights(out, farnet.h2_init(ne=ne, no=no), dict(trained=0, width=ne + no, even=ne, odd=no,
                                                             depths=farnet.DEPTHS))
        print(json.dumps(dict(saved=out, weights=farnet.num_params(ne=ne, no=no))), flush=True)
        return
    if a.time:
        path = {"default": DEFAULT_WEIGHTS, "accurate": ACCURATE_WEIGHTS}.get(a.weights, a.weights)
        w, _ = load_weights(path)
        if w is None:
            raise SystemExit(f"no weights at {path}")
        out = time_potential(a.evals, weights=w)
        out["network"]["weights"] = os.path.basename(path)
        print(json.dumps(out), flush=True)
        return
    logf = open(a.log, "w") if a.log else None

    def log(rec):
        line = json.dumps(rec)
        print(line, flush=True)
        if logf:
            logf.write(line + "\n")
            logf.flush()

    t0 = time.time()
    U, F, N2 = generate_pairs(a.pairs, progress=lambda k, s: k % 1000 < 50 and log(dict(pairs=k, s=round(s, 1))))
    log(dict(generated=a.pairs, s=time.time() - t0))
    Uv, Fv, N2v, _ = benchmark_pairs(a.val)
    w, hist, w0 = train(U, F, N2, a.steps, a.batch, a.lr, val=(Uv, Fv, N2v), log=log)
    del U, F
    torch.cuda.empty_cache()
    start = hist[0]
    best = min((h for h in hist if "total_mean" in h), key=lambda h: h["total_mean"])
    save_weights(a.out, w, dict(pairs=a.pairs, steps=a.steps, batch=a.batch, lr=a.lr, width=farnet.NR,
                                even=farnet.NE, odd=farnet.NO, depths=farnet.DEPTHS,
                                val_start_mean=start["total_mean"], val_start_max=start["total_max"],
                                val_mean=best["total_mean"], val_max=best["total_max"], val_best_step=best["step"]))
    log(dict(saved=a.out, total_s=time.time() - t0))


if __name__ == "__main__":
    main()
