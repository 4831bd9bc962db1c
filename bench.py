#!/usr/bin/env python
"""Benchmark: LLG RK4 steps/s at 256x256x3 on one B200 (per GPU: replicas).

One "step" is one classical RK4 step of the resident FP64 state: four demag
field evaluations (divergence -> potential -> fused field/LLG/RK4 stage) plus
the time advance, captured as one CUDA graph.  Workload: a 256x256x3 grid of
5 nm cells holding an 8x8 lattice of permalloy discs (radius 12 cells, pitch
32) in the middle layer, a random in-plane direction per dot, and an external
field ramped along x from -50 to +50 mT over 10 ns; dt = 1e-13 s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--solver fmm|direct]
    python bench.py --impl reference ...   # the reference's own CPU path

Under torchrun each rank advances its own replica (seed 2010 + rank) with no
data-path collective; the timed region is bracketed by barriers and the max
over ranks is reported.  Prints ONE JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mms-gpu_b200"))

METRIC = "LLG RK4 steps/s, 256x256x3: FMM vs surrogate demag at ≤1e-3 rel err vs FP64"
WORKLOAD = "llg_rk4_disc_lattice_256x256x3"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--solver", choices=["fmm", "direct"], default=os.environ.get("MMS_BENCH_SOLVER", "fmm"))
    ap.add_argument("--order", type=int, default=4,
                    help="FMM expansion order P; 0 = autotuned on RK4 steps (fastest within 5e-4 of the exact sum)")
    ap.add_argument("--leaf", type=int, default=8, help="FMM leaf side in cells (0 = the library's default)")
    ap.add_argument("--m2l", type=int, default=int(os.environ.get("MMS_BENCH_M2L", "0")),
                    help="FMM M2L: 0 auto, 1 FP32 SIMT, 2 tensor cores (split BF16)")
    ap.add_argument("--near", type=int, default=0,
                    help="FMM near field: 0 auto (tensor cores at leaf 8), 1 FP32 k_p2p, 2 tensor cores")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--dt", type=float, default=1e-13)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the learned far-field measurement")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble measurement")
    ap.add_argument("--workload", choices=["single", "ensemble"], default="single",
                    help="single: the 256x256x3 metric; ensemble: the batched-ensemble configuration")
    ap.add_argument("--ensemble-size", type=int, default=512)
    return ap.parse_args()


def workload(size, seed):
    from mmsb200 import geometry
    X = Y = size
    Z = 3
    pitch = 32 * size // 256
    r = 12 * size // 256
    mask, M = geometry.per_dot_random_inplane(X, Y, Z, r, pitch, seed)
    hext_t = [0.0, 1e-8]
    hext_b = [[-0.05, 0.0, 0.0], [0.05, 0.0, 0.0]]
    return (X, Y, Z), (5e-9, 5e-9, 5e-9), mask, M, hext_t, hext_b


# ---------------------------------------------------------------------------- clocks
class ClockSampler:
    """samples SM clocks and throttle reasons during the timed region: NVML
    read-only queries polled every millisecond on a background thread (a
    timed region of a few milliseconds still gets samples), else nvidia-smi
    every 200 ms"""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm MHz, reason bits)
        self.smax = None
        self.run = False
        try:
            pynvml, h = nvml_handle(device_index)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.bits = (pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                         pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap)
            self.nvml, self.h = pynvml, h
        except Exception:
            self.nvml = None

    def start(self):
        if self.nvml is not None:
            self.run = True
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _poll(self):
        nv = self.nvml
        while self.run:
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.samples.append((sm, r))
            except Exception:
                pass
            time.sleep(0.001)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.run = False
            self.thread.join(timeout=5)
            sm = [x for x, _ in self.samples]
            reasons = {n for _, r in self.samples for n, bit in zip(self.NAMES, self.bits) if r & bit}
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.smax,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 1 ms polling"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        for l in self.lines:
            p = [v.strip() for v in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(self.NAMES, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# ---------------------------------------------------------------------------- helpers
def dist_init():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def profile_traffic(kernel_key):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/<kernel_key>.md, line 'traffic_bytes_per_launch: N')"""
    path = os.path.join(ROOT, "profiles", kernel_key + ".md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def cpu_baseline(dims, d, mask, M, dt, steps=2, warmup=1):
    """The reference's own CPU direct path (oracle/_ref, built from its
    sources) on all host threads: `steps` real RK4 steps after `warmup`
    untimed ones, each rk4_step (three Hfield calls inside) plus the post-step
    Hfield, the order time_marching runs an accepted step in
    (ode_functions.cpp:230-308).  steps/s = steps / their wall time."""
    sys.path.insert(0, ROOT)
    from oracle import ref
    threads = os.cpu_count() or 1
    if not ref.available():
        return None
    secs, th = ref.time_rk4(mask, M.astype(np.float32), dims, d, dt, steps, warmup=warmup, threads=threads)
    tot = float(np.sum(secs))
    return {"value": len(secs) / tot, "unit": "steps/s", "cores": th, "kind": "reference",
            "sample": f"{len(secs)} real reference RK4 steps (rk4_step + post-step Hfield, CPU direct sum, "
                      f"OpenMP) at {dims[0]}x{dims[1]}x{dims[2]} after {warmup} untimed: {tot:.2f} s",
            "seconds_per_step": tot / len(secs)}


# ---------------------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's own CPU path, timed as real RK4 steps: the unmodified
    reference sources (oracle/_ref, built from its tree) run rk4_step plus the
    post-step Hfield per step, the order of time_marching's accepted step
    (ode_functions.cpp:230-308), on all host threads.  `warmup` steps run
    untimed first; the timed steps stop early once ~120 s of work is done, and
    `steps` reports the steps actually timed."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, ROOT)
    from oracle import ref
    dims, d, mask, M, _, _ = workload(args.size, 2010)
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/mmsref_harness not built "
                          "(the reference tree was absent when building)"}))
        return 0
    threads = os.cpu_count() or 1
    # the first steps cost least (the initial in-plane state has charge only at
    # the disc edges; once M tilts, every magnetic cell of the outer layers
    # carries charge): two untimed steps reach the steady per-step cost
    warm = min(args.warmup, 2)
    secs, th = ref.time_rk4(mask, M.astype(np.float32), dims, d, args.dt, args.steps, warmup=warm,
                            threads=threads, budget_s=120.0)
    tot = float(np.sum(secs))
    v = len(secs) / tot
    N = dims[0] * dims[1] * dims[2]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": len(secs), "warmup": warm, "ms_per_step": tot / len(secs) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": list(dims), "cells": N, "cell_nm": 5,
                       "path": "reference rk4_step + post-step Hfield, CPU direct sum (calc_potential_exact, "
                               "use_gpu=0), time_marching's accepted-step order",
                       "external": "none (the reference's field is a fixed built-in ramp; the potential "
                                   "dominates the step either way)",
                       "threads": th},
            "cell_steps_per_s": v * N,
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": th, "kind": "reference",
                             "sample": f"{len(secs)} real reference RK4 steps at {dims[0]}x{dims[1]}x{dims[2]} "
                                       f"after {warm} untimed, {tot:.2f} s timed" +
                                       (f" (stopped after ~120 s of timed work, of {args.steps} asked)"
                                        if len(secs) < args.steps else "")},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import mmsb200
    ws, rank, local = dist_init()
    dims, d, mask, M, hext_t, hext_b = workload(args.size, 2010 + rank)
    X, Y, Z = dims
    N = X * Y * Z
    grid = mmsb200.Grid(X, Y, Z, *d)
    params = mmsb200.make_params(external=True, hext_t=hext_t, hext_b=hext_b)
    kind = mmsb200.SOLVER_FMM if args.solver == "fmm" else mmsb200.SOLVER_DIRECT
    solver = mmsb200.make_solver(kind, args.order, args.leaf, args.m2l, mmsb200.FAR_STAGES, args.near)
    tuned = None
    if kind == mmsb200.SOLVER_FMM and args.order == 0:
        # autotuned: fastest (P, leaf, M2L kernel) within half the metric's 1e-3 target
        Mf = torch.from_numpy(M.astype(np.float32)).cuda()
        rho0 = torch.empty((Z, Y, X), dtype=torch.float32, device="cuda")
        with mmsb200.Context(grid, params, mmsb200.make_solver(mmsb200.SOLVER_DIRECT)) as tctx:
            tctx.divergence_dev(Mf, rho0)
            tctx.sync()
        solver, tms, terr = mmsb200.autotune_fmm_steps(grid, params, mask, M, args.dt, rho0, 5e-4)
        tuned = {"P": solver.fmm_order, "leaf": solver.fmm_leaf, "m2l": solver.m2l_mode, "ms_per_step": tms,
                 "err": terr, "objective": "graph-captured RK4 step time, 20 steps per candidate"}
        args.order, args.leaf, args.m2l = solver.fmm_order, solver.fmm_leaf, solver.m2l_mode
        del Mf, rho0
    # a dedicated stream: the library's kernels and every timing event live on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = mmsb200.Context(grid, params, solver, stream=stream.cuda_stream)
    ctx.state_set(mask, M)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    # accuracy of the demag potential on the start state vs the exact (direct) sum
    acc = None
    if args.solver == "fmm":
        Mf = torch.from_numpy(M.astype(np.float32)).cuda()
        rho = torch.empty((Z, Y, X), dtype=torch.float32, device="cuda")
        phi_f = torch.empty_like(rho)
        phi_d = torch.empty_like(rho)
        ctx.divergence_dev(Mf, rho)
        ctx.potential_dev(rho, phi_f)
        with mmsb200.Context(grid, params, mmsb200.make_solver(mmsb200.SOLVER_DIRECT),
                             stream=stream.cuda_stream) as dctx:
            dctx.potential_dev(rho, phi_d)
            dctx.sync()
        acc = float((phi_f.double() - phi_d.double()).norm() / phi_d.double().norm())
        del Mf, rho, phi_f, phi_d

    # warm-up (also captures the step graph)
    ctx.run_fixed(args.dt, max(args.warmup, 3), use_graph=True)
    ctx.sync()

    # timed region: K steps, L2 flushed between steps, per-step device events
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    barrier(ws)
    torch.cuda.synchronize()
    clocks.start()
    launches0 = ctx.kernel_launches
    for k in range(args.steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        ctx.run_fixed(args.dt, 1, use_graph=True)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    launches = ctx.kernel_launches - launches0
    barrier(ws)
    clk = clocks.stop()
    ms_steps = [a.elapsed_time(b) for a, b in ev]
    ms_total = max_over_ranks(ws, float(np.sum(ms_steps)))
    ms_per_step = ms_total / args.steps
    value = ws * args.steps / (ms_total * 1e-3)

    # dominant kernel time inside one step, measured live with events around
    # one potential evaluation on the same stream (the stage kernels and the
    # divergence are the rest of the step)
    rho_t = torch.empty((Z, Y, X), dtype=torch.float32, device="cuda")
    phi_t = torch.empty_like(rho_t)
    Mf = torch.from_numpy(ctx.state_get()[0].astype(np.float32)).cuda()
    ctx.divergence_dev(Mf, rho_t)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 10
    pot_ms = []
    for _ in range(reps):
        flush.fill_(1.0)
        e0.record(stream)
        ctx.potential_dev(rho_t, phi_t)
        e1.record(stream)
        torch.cuda.synchronize()
        pot_ms.append(e0.elapsed_time(e1))
    pot_ms = float(np.median(pot_ms))
    fma_peak = mmsb200.fma_tflops()
    if args.solver == "direct":
        # sources = cells with non-zero charge (the kernel skips source-row
        # groups without charge), targets = all cells, self pairs excluded
        n_src = int(torch.count_nonzero(rho_t))
        pairs = float(N) * float(n_src) - n_src
        roof = {"kernel": "k_direct (potential, exact direct sum)", "bound": "fp32",
                "achieved": 2 * pairs / (pot_ms * 1e-3) / 1e12, "peak": fma_peak, "unit": "TFLOP/s",
                "peak_source": "measured FP32 FMA microbenchmark (mms_diag_fma_tflops), of measured",
                "algorithmic": f"2 flops (one FMA) per target-source pair: N = {N} targets x {n_src} sources "
                               "with non-zero charge (timed state), self pairs excluded"}
        roof["frac"] = roof["achieved"] / roof["peak"]
        roof["traffic"] = profile_traffic("k_direct_256x256x3")
    else:
        roof = fmm_roofline(ctx, pot_ms, fma_peak, rho_t, phi_t)
    roof["potential_ms_cold_l2"] = pot_ms

    # e2e through the public API with host buffers: H2D of the state, one step,
    # D2H of the state, every step.  The headline uses the reference's own
    # state layout (N Vector3 of FP32, as rk4_step takes and returns it); the
    # same loop with the FP64 state calls is reported beside it.
    e2e = None
    if not args.no_e2e:
        M64 = ctx.state_get()[0]
        host_mat = torch.from_numpy(mask.astype(np.uint8)).pin_memory()
        dev_mat = torch.empty(host_mat.shape, dtype=torch.uint8, device="cuda")

        def e2e_run(dtype, set_dev, get_dev, graph=False):
            """steps/s of host-state round trips; with graph the same public
            calls (copies, state set, one eager step, state get, copy back)
            are captured once into a CUDA graph and replayed every step"""
            host_M = torch.from_numpy(M64.astype(dtype)).pin_memory()
            dev_M = torch.empty(host_M.shape, dtype=host_M.dtype, device="cuda")
            out_M = torch.empty_like(host_M).pin_memory()
            t = 0.0
            # one untimed round trip first: a state set from the host has no
            # potential yet, so these steps run the evaluate-first step graph,
            # captured here (4 field evaluations per step either way)
            dev_M.copy_(host_M, non_blocking=True)
            dev_mat.copy_(host_mat, non_blocking=True)
            set_dev(dev_mat, dev_M, t)
            ctx.run_fixed(args.dt, 1, use_graph=True)
            ctx.sync()
            g = None
            if graph:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=stream, capture_error_mode="thread_local"):
                    dev_M.copy_(host_M, non_blocking=True)
                    dev_mat.copy_(host_mat, non_blocking=True)
                    set_dev(dev_mat, dev_M, t)
                    ctx.run_fixed(args.dt, 1, use_graph=False)
                    get_dev(dev_M)
                    out_M.copy_(dev_M, non_blocking=True)
                g.replay()
                torch.cuda.synchronize()
            ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
            for k in range(args.steps):
                flush.fill_(float(k))
                ev2[k][0].record(stream)
                if g is not None:
                    g.replay()
                else:
                    dev_M.copy_(host_M, non_blocking=True)
                    dev_mat.copy_(host_mat, non_blocking=True)
                    set_dev(dev_mat, dev_M, t)
                    ctx.run_fixed(args.dt, 1, use_graph=True)
                    get_dev(dev_M)
                    out_M.copy_(dev_M, non_blocking=True)
                ev2[k][1].record(stream)
                t += args.dt
            torch.cuda.synchronize()
            del g
            ms = max_over_ranks(ws, float(sum(a.elapsed_time(b) for a, b in ev2)))
            esz = host_M.element_size()
            return {"value": ws * args.steps / (ms * 1e-3), "unit": "steps/s",
                    "h2d_bytes_per_step": int(host_M.numel() * esz + host_mat.numel()),
                    "d2h_bytes_per_step": int(out_M.numel() * esz)}

        e2e = e2e_run(np.float32, ctx.state_set_f32_dev, ctx.state_get_f32_dev)
        e2e["path"] = ("mms_state_set_f32_dev + mms_run_fixed(1 step) + mms_state_get_f32_dev, pinned host "
                       "copies of M as N x 3 FP32 (the reference's Vector3 layout, as rk4_step takes it) and "
                       "the material bytes; the state between the calls stays FP64 on the device; 4 field "
                       "evaluations per step, as in the device-timed steps")
        e2e["fp64_state_io"] = e2e_run(np.float64, ctx.state_set_dev, ctx.state_get_dev)
        e2e["fp64_state_io"]["path"] = "the same with mms_state_set_dev / mms_state_get_dev (M as N x 3 FP64)"
        try:
            e2e["graph_replayed"] = e2e_run(np.float32, ctx.state_set_f32_dev, ctx.state_get_f32_dev, graph=True)
            e2e["graph_replayed"]["path"] = ("the FP32 calls above (copies, mms_state_set_f32_dev, "
                                             "mms_run_fixed(1 step, eager), mms_state_get_f32_dev, copy back) "
                                             "captured once into a CUDA graph by the caller and replayed per step")
        except RuntimeError as exc:  # the eager figures stand without it
            e2e["graph_replayed"] = {"error": str(exc).splitlines()[0]}
        # the bound the copies set: pinned H2D / D2H bandwidth of this box
        # (32 MiB copies, best of 5, CUDA events) and the step time
        h2d_gbs, d2h_gbs = pcie_bandwidth(stream)
        bound = 1.0 / (ms_per_step * 1e-3 + e2e["h2d_bytes_per_step"] / (h2d_gbs * 1e9)
                       + e2e["d2h_bytes_per_step"] / (d2h_gbs * 1e9))
        e2e["pcie"] = {"h2d_gbs": h2d_gbs, "d2h_gbs": d2h_gbs, "bound_steps_per_s": bound,
                       "frac_of_bound": e2e["value"] / bound,
                       "note": "bound = 1 / (device step time + H2D bytes / H2D bandwidth + D2H bytes / D2H "
                               "bandwidth): the copies and the step are serial in a round trip"}

    sur = None
    if args.solver == "fmm" and not args.no_surrogate:
        sur = surrogate_block(args, grid, params, mask, M, stream, flush, value)

    # the batched-ensemble configuration, measured in the same run (every rank
    # runs its cost partition of the instances; rank 0 reports)
    ens = None
    if not args.no_ensemble:
        em = ensemble_measure(args, stream, flush, ws, rank)
        ens = ensemble_summary(args, em, max_over_ranks(ws, em["ms_total"]), ws, fma_peak)

    base = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            base = cpu_baseline(dims, d, mask, M, args.dt)
        except Exception as e:  # the baseline is reported, never required
            base = {"value": None, "error": str(e)[:200]}

    kern = mmsb200.fmm_stats(ctx) if args.solver == "fmm" else None
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return 0
    cfg = {"workload": WORKLOAD, "grid": [X, Y, Z], "cells": N, "cell_nm": 5, "solver": args.solver,
           "dt_s": args.dt, "state": "fp64", "fields": "fp32",
           "geometry": "8x8 lattice of discs r=12 pitch 32 (middle layer), random in-plane M per dot",
           "external": "B_x ramp -50..+50 mT over 10 ns", "l2": f"flushed between timed steps "
           f"({L2_FLUSH_BYTES >> 20} MB write, outside the timed events)", "graph": "one CUDA graph per RK4 step",
           "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"}
    if args.solver == "fmm":
        cfg.update({"P": args.order, "leaf": args.leaf or "auto", "autotune": tuned,
                    "m2l": {0: "auto", 1: "fp32 simt", 2: "tensor cores (split bf16)"}[args.m2l],
                    "near": {0: "auto", 1: "fp32 simt", 2: "tensor cores (split bf16)"}[args.near],
                    "kernels": {"near": "k_p2p_tc (tcgen05, split bf16)" if kern["near_tc"] else "k_p2p (fp32)",
                                "m2l": "k_m2l_gemm (tcgen05, split bf16)" if kern["m2l_tc"] else "fp32"}})
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic", "config": cfg,
            "cell_steps_per_s": value * N, "gpu_launches": int(launches), "roofline": roof, "clocks": clk,
            "e2e": e2e, "cpu_baseline": base}
    if sur is not None:
        line["surrogate"] = sur
    if ens is not None:
        line["ensemble"] = ens
    if acc is not None:
        line["accuracy"] = {"demag_phi_rel_l2_vs_direct": acc,
                            "note": "direct = exact FP32 table + compensated sum, itself <= 2e-6 from FP64"}
    print(json.dumps(line))
    return 0


STAGE_KERNEL = {"p2m": "k_p2m_row", "m2m": "k_m2m_c (one launch per level)", "m2l": "k_m2l_res / k_m2l_split",
                "l2l": "k_l2l_c (one launch per level)", "l2p_p2p": "k_p2p + k_l2p"}


def surrogate_block(args, grid, params, mask, M, stream, flush, fmm_value):
    """The learned far field on the same workload: its demag error on the start
    state against the exact sum, LLG steps/s with the network alone (no
    check), and the surrogate-assisted run the metric names (FMM check every
    50 steps, 1e-3 rel-L2 tolerance, FMM takes over above it), and the FMM at
    P = 5 and 6 (the orders whose error brackets the network's) with their
    errors, and the accurate network (24 + 16 channels) beside the FMM at
    P = 8, each as K graph-replayed steps timed with CUDA events on the
    library's stream."""
    import torch
    import mmsb200
    from mmsb200 import farnet
    from mmsb200 import surrogate as S
    w, meta = S.load_weights()
    if w is None:
        return {"unavailable": "no trained weights (python -m mmsb200.surrogate)"}
    X, Y, Z = grid.xdim, grid.ydim, grid.zdim
    solver = mmsb200.make_solver(mmsb200.SOLVER_SURROGATE, 6, 8)
    out = {"network": "linear multilevel conv operator over 8x8x3 leaf boxes: encoder, 2x2 stride-2 down, "
                      "parity-aware 7x7 interaction-list convs per level, transposed up, decoder; width %d "
                      "(%d even + %d odd), %d FP32 weights; exact near field" % (farnet.NR, farnet.NE, farnet.NO,
                                                                               farnet.num_params()),
           "training": {k: (float(v) if np.ndim(v) == 0 else v.tolist()) for k, v in meta.items()},
           "check": "FMM P=6 leaf 8"}
    Mf = torch.from_numpy(M.astype(np.float32)).cuda()
    rho = torch.empty((Z, Y, X), dtype=torch.float32, device="cuda")
    phi_s, phi_d = torch.empty_like(rho), torch.empty_like(rho)
    with mmsb200.Context(grid, params, solver, stream=stream.cuda_stream) as c:
        c.set_surrogate(w, 0, 1.0)
        c.divergence_dev(Mf, rho)
        c.potential_dev(rho, phi_s)
        with mmsb200.Context(grid, params, mmsb200.make_solver(mmsb200.SOLVER_DIRECT),
                             stream=stream.cuda_stream) as dctx:
            dctx.potential_dev(rho, phi_d)
            dctx.sync()
        out["demag_phi_rel_l2_vs_direct"] = float((phi_s.double() - phi_d.double()).norm() / phi_d.double().norm())

    def steps_per_s(every, tol, nsteps, slv=solver, weights=None):
        with mmsb200.Context(grid, params, slv, stream=stream.cuda_stream) as c:
            if every is not None:
                c.set_surrogate(w if weights is None else weights, every, tol)
            c.state_set(mask, M)
            c.run_fixed(args.dt, 3)
            c.sync()
            st0 = c.surrogate_stats() if every is not None else None
            ms = 0.0
            for k in range(nsteps):
                flush.fill_(float(k))
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                c.run_fixed(args.dt, 1)
                e1.record(stream)
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1)
            if every is None:
                return nsteps / (ms * 1e-3), None
            st = c.surrogate_stats()
            st["checks"] -= st0["checks"]
            return nsteps / (ms * 1e-3), st

    n = max(args.steps, 200)
    v, _ = steps_per_s(0, 1.0, n)
    out["steps_per_s_surrogate_only"] = v
    out["speedup_surrogate_only_vs_fmm"] = v / fmm_value
    v, st = steps_per_s(50, 1e-3, n)
    out["assisted_check50_tol1e-3"] = {"steps_per_s": v, "steps": n, "checks": st["checks"],
                                       "fallbacks": st["fallbacks"], "max_check_rel_l2_vs_fmm": st["max_err"],
                                       "surrogate_active_at_end": st["active"],
                                       "speedup_vs_fmm": v / fmm_value}
    # the accurate network (24 + 16 channels, its nested-SVD start): error and
    # steps/s on the same state and steps
    wa, _ = S.load_weights(S.ACCURATE_WEIGHTS)
    if wa is not None:
        with mmsb200.Context(grid, params, solver, stream=stream.cuda_stream) as c:
            c.set_surrogate(wa, 0, 1.0)
            phi_a = torch.empty_like(rho)
            c.potential_dev(rho, phi_a)
            c.sync()
            ea = float((phi_a.double() - phi_d.double()).norm() / phi_d.double().norm())
        va, _ = steps_per_s(0, 1.0, n, weights=wa)
        out["accurate_network"] = {"weights": os.path.basename(S.ACCURATE_WEIGHTS),
                                   "channels": "24 even + 16 odd", "demag_phi_rel_l2_vs_direct": ea,
                                   "steps_per_s": va}
    # the FMM at the orders that bracket the networks' accuracy, on the same
    # state and steps: what the networks are worth at equal error
    matched = []
    for P in (5, 6, 8):
        slv = mmsb200.make_solver(mmsb200.SOLVER_FMM, P, 8)
        with mmsb200.Context(grid, params, slv, stream=stream.cuda_stream) as c:
            phi_f = torch.empty_like(rho)
            c.potential_dev(rho, phi_f)
            c.sync()
            err = float((phi_f.double() - phi_d.double()).norm() / phi_d.double().norm())
        v, _ = steps_per_s(None, None, n, slv)
        row = {"P": P, "leaf": 8, "demag_phi_rel_l2_vs_direct": err, "steps_per_s": v,
               "network_speedup": out["steps_per_s_surrogate_only"] / v}
        if "accurate_network" in out:
            row["accurate_network_speedup"] = out["accurate_network"]["steps_per_s"] / v
        matched.append(row)
    out["fmm_at_matched_accuracy"] = matched
    return out


def nvml_handle(device_index):
    """(pynvml, handle) of the torch device, found by PCI bus id; raises
    when NVML is not there"""
    import pynvml
    pynvml.nvmlInit()
    h = None
    try:
        import torch
        props = torch.cuda.get_device_properties(device_index)
        bus = getattr(props, "pci_bus_id", None)
        if bus is not None:
            dom, dev = getattr(props, "pci_domain_id", 0), getattr(props, "pci_device_id", 0)
            h = pynvml.nvmlDeviceGetHandleByPciBusId(f"{dom:08x}:{bus:02x}:{dev:02x}.0")
    except Exception:
        h = None
    if h is None:
        h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
    return pynvml, h


def pcie_bandwidth(stream, nbytes=32 << 20, reps=5):
    """best pinned host <-> device copy bandwidth (GB/s) on this box, each way"""
    import torch
    h = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    out = []
    for src, dst in ((h, d), (d, h)):
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            dst.copy_(src, non_blocking=True)
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        out.append(nbytes / (best * 1e-3) / 1e9)
    return out[0], out[1]


def bf16_peak():
    """dense BF16 tensor peak (TFLOP/s): the measured burst figure of this
    pool's B200s, else the earlier pool measurement"""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["bf16_tflops"]), "measured cuBLAS BF16 GEMM burst (MEASURED_PEAKS.json), of measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "earlier cuBLAS BF16 measurement on this pool, of fallback"


def near_pairs_occupied(rho, X, Y, Z, s):
    """near-field (target, source) pairs of the FMM with leaf side s, counting
    only sources with non-zero charge: per leaf box, its cells times the
    charged cells of its 3x3 box neighbourhood (all layers)"""
    nbx, nby = -(-X // s), -(-Y // s)
    charged = np.zeros((Z, nby * s, nbx * s), bool)
    charged[:, :Y, :X] = np.asarray(rho).reshape(Z, Y, X) != 0
    cells = np.zeros((Z, nby * s, nbx * s), bool)
    cells[:, :Y, :X] = True
    occ = charged.reshape(Z, nby, s, nbx, s).sum(axis=(0, 2, 4)).astype(np.int64)
    tgt = cells.reshape(Z, nby, s, nbx, s).sum(axis=(0, 2, 4)).astype(np.int64)
    pad = np.pad(occ, 1)
    src = sum(pad[1 + dy:1 + dy + nby, 1 + dx:1 + dx + nbx] for dy in (-1, 0, 1) for dx in (-1, 0, 1))
    return int((tgt * src).sum())


def fmm_roofline(ctx, pot_ms, fma_peak, rho, phi):
    """FMM roofline for its dominant stage: every stage is timed live with CUDA
    events over back-to-back re-launches on the library's stream, and the
    stage with the largest time is reported (at P = 4, leaf 8: the near field
    k_p2p plus k_l2p; at leaf 4: the M2L).  achieved = that stage's
    algorithmic flops (near field: 2 per target-source pair plus 2 NR per
    target; M2L: 2 (NE^2 + NO^2) per interaction-list box pair) over its time,
    against the measured FP32 FMA peak.  All stage times and flops are
    reported beside it; traffic is the committed ncu capture of that stage."""
    import mmsb200
    st = mmsb200.fmm_stats(ctx)
    times = mmsb200.fmm_stage_times(ctx, rho, phi, reps=20)
    dom = max(times, key=lambda k: times[k])
    # the near field counted from the occupancy map: sources are the cells
    # with non-zero charge (the kernel skips chargeless source rows), targets
    # every cell of the grid
    g = ctx.grid
    occ_pairs = near_pairs_occupied(rho.detach().cpu().numpy(), g.xdim, g.ydim, g.zdim, st["leaf"])
    st["stage_flops"]["l2p_p2p"] += 2.0 * (occ_pairs - st["p2p_pairs"])
    st["flops"] += 2.0 * (occ_pairs - st["p2p_pairs"])
    roof = {"kernel": f"{STAGE_KERNEL[dom]} (FMM stage {dom})", "bound": "fp32", "peak": fma_peak,
            "unit": "TFLOP/s",
            "peak_source": "measured FP32 FMA microbenchmark (mms_diag_fma_tflops), of measured"}
    roof["achieved"] = st["stage_flops"][dom] / (times[dom] * 1e-3) / 1e12 if times[dom] > 0 else 0.0
    if dom == "l2p_p2p" and st["near_tc"]:
        # near field on the tensor cores: its algorithmic flops (2 per charged
        # pair) over the stage time, which also holds the FP32 L2P
        peak, src = bf16_peak()
        roof.update({"kernel": "k_rho_split + k_p2p_tc + k_l2p (FMM stage l2p_p2p: tcgen05 near field, then L2P)",
                     "bound": "tensor", "peak": peak, "peak_source": src,
                     "achieved": 2.0 * occ_pairs / (times[dom] * 1e-3) / 1e12,
                     "issued_tensor_tflops": 3 * 2.0 * st["p2p_pairs"] / (times[dom] * 1e-3) / 1e12,
                     "issued_note": "split-BF16: 3 products per pair, every pair of the 3x3 box neighbourhood "
                                    "(charged or not), over the same stage time"})
        roof["frac"] = roof["achieved"] / peak
    else:
        roof["frac"] = roof["achieved"] / fma_peak
    roof["stage_ms"] = times
    roof["stage_flops"] = st["stage_flops"]
    roof["whole_potential_tflops"] = st["flops"] / (sum(times.values()) * 1e-3) / 1e12
    roof["plan"] = {k: st[k] for k in ("levels", "leaf", "order", "m2l_pairs")}
    roof["plan"]["p2p_pairs_all_cells"] = st["p2p_pairs"]
    roof["plan"]["p2p_pairs_charged_sources"] = occ_pairs
    roof["algorithmic"] = ("near field: 2 flops per (target, source) pair over each leaf box's 3x3 neighbourhood, "
                           "sources = cells with non-zero charge in the timed state, targets = all cells; "
                           "plus 2 NR per cell (L2P) and the leaf kernels' L2L")
    key = f"fmm_{dom}_256x256x3_P{st['order']}_leaf{st['leaf']}" + ("_tc" if dom == "l2p_p2p" and st["near_tc"] else "")
    roof["traffic"] = profile_traffic(key)
    return roof


def ensemble_measure(args, stream, flush, ws=1, rank=0):
    """The batched-ensemble configuration: `--ensemble-size` independent
    simulations (sides 16..64 in steps of 8, x3 layers, rectangle/disc/ellipse
    masks, random M, random in-plane |B| <= 50 mT; dt = 1e-13 s), one CUDA
    graph per ensemble step, the direct kernel's shape autotuned first.  Under
    torchrun the instances are partitioned over ranks by cost with no
    collective on the data path.  Returns the measurement (this rank's device
    time; the caller takes the max over ranks)."""
    import torch
    import mmsb200
    from mmsb200 import geometry
    from mmsb200.ensemble import Ensemble, cost, partition
    dims, masks, Ms, bext = geometry.ensemble_instances(args.ensemble_size, seed=2010)
    mine = partition([cost(d) for d in dims], ws, rank)
    ens = Ensemble([dims[i] for i in mine], (5e-9, 5e-9, 5e-9), mmsb200.make_params(external=True),
                   bext=[bext[i] for i in mine], stream=stream.cuda_stream)
    ens.state_set([masks[i] for i in mine], [Ms[i] for i in mine])
    ew, q, direct_ms = ens.autotune(5)
    steps = max(args.steps, 20)
    ens.run_fixed(args.dt, max(args.warmup, 3), use_graph=True)
    ens.sync()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    l0 = ens.kernel_launches
    for k in range(steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        ens.run_fixed(args.dt, 1, use_graph=True)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    launches = ens.kernel_launches - l0
    ms_total = float(sum(a.elapsed_time(b) for a, b in ev))
    cells = sum(int(np.prod(dims[i])) for i in mine)
    ens.close()

    def charge_support(mask):
        m = np.pad(mask != 0, 1)
        sup = np.zeros_like(m)
        for ax in range(3):
            sup |= np.roll(m, 1, axis=ax) | np.roll(m, -1, axis=ax)
        return int(sup[1:-1, 1:-1, 1:-1].sum())
    # one FMA per (target, source) pair, sources = cells whose charge can be
    # non-zero (a material neighbour), targets = all cells of the instance
    pairs = float(sum(charge_support(masks[i]) * float(np.prod(dims[i])) for i in mine))
    return {"steps": steps, "ms_total": ms_total, "cells": cells, "launches": int(launches), "pairs": pairs,
            "direct_ms": direct_ms, "shape": {"warps": ew, "rows": q}, "instances": len(mine)}


def ensemble_summary(args, m, ms_total, ws, fma_peak):
    value = m["steps"] / (ms_total * 1e-3)
    achieved = 2 * m["pairs"] / (m["direct_ms"] * 1e-3) / 1e12
    roof = {"kernel": "k_ens_direct (batched exact potential, persistent)", "bound": "fp32", "unit": "TFLOP/s",
            "achieved": achieved, "peak": fma_peak, "frac": achieved / fma_peak,
            "peak_source": "measured FP32 FMA microbenchmark (mms_diag_fma_tflops), of measured",
            "algorithmic": "2 flops per target-source pair (sources: cells with a material neighbour; targets: "
                           "all cells) of every instance, over the kernel's own mean time (CUDA events, "
                           "back-to-back launches after autotuning)",
            "kernel_ms": m["direct_ms"], "traffic": profile_traffic("k_ens_direct_512_instances")}
    return {"metric": f"ensemble LLG RK4 steps/s ({args.ensemble_size} instances, 16..64 x 16..64 x 3)",
            "value": value, "unit": "ensemble steps/s", "steps": m["steps"], "ms_per_step": ms_total / m["steps"],
            "cells": m["cells"], "cell_steps_per_s": value * m["cells"], "gpu_launches": m["launches"],
            "config": {"workload": "ensemble_rk4", "instances": args.ensemble_size, "solver": "direct (batched)",
                       "dt_s": args.dt, "graph": "one CUDA graph per ensemble step",
                       "autotuned_shape": m["shape"], "l2": "flushed between timed steps",
                       "parallelism": f"instance partition x{ws}" if ws > 1 else "single GPU"},
            "roofline": roof}


def run_ensemble(args):
    """`--workload ensemble`: the batched ensemble alone, as the one JSON line"""
    import torch
    import mmsb200
    ws, rank, local = dist_init()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    clocks = ClockSampler(local)
    barrier(ws)
    clocks.start()
    m = ensemble_measure(args, stream, flush, ws, rank)
    barrier(ws)
    clk = clocks.stop()
    ms_total = max_over_ranks(ws, m["ms_total"])
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = ensemble_summary(args, m, ms_total, ws, mmsb200.fma_tflops())
    line.update({"n_gpus": ws, "warmup": max(args.warmup, 3), "higher_is_better": True, "scaling": "strong",
                 "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic", "clocks": clk})
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ensemble":
        return run_ensemble(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
