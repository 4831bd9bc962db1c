"""Sharding an ensemble over ranks (CPU, gloo, world_size 2): the greedy
partition is disjoint, complete and balanced, and ranks that each advance
their own instances (FP64 oracle standing in for the device) and gather the
results reproduce a single-process run bit for bit."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT


def test_partition_is_disjoint_complete_balanced():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "mms-gpu_b200"))
    from mmsb200.ensemble import cost, partition
    from mmsb200 import geometry
    dims, _, _, _ = geometry.ensemble_instances(64, seed=3)
    costs = [cost(d) for d in dims]
    for world in (1, 2, 3, 8):
        parts = partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-9


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "mms-gpu_b200"))
    import datetime
    import torch
    import torch.distributed as dist
    import oracle
    from mmsb200 import geometry
    from mmsb200.ensemble import cost, partition
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    dims, masks, Ms, bext = geometry.ensemble_instances(6, seed=11, sides=(4, 6, 8))
    mine = partition([cost(d) for d in dims], world, rank)
    results = {}
    for i in mine:
        X, Y, Z = dims[i]
        g = oracle.Grid(X, Y, Z, 5e-9, 5e-9, 5e-9)
        p = oracle.Params(external=True, hext_t=[0.0], hext_b=[bext[i]])
        results[i] = oracle.rk4_run(g, p, masks[i], Ms[i], 1e-13, 3)
    gathered = [None] * world
    dist.all_gather_object(gathered, results)
    if rank == 0:
        merged = {}
        for r in gathered:
            merged.update(r)
        np.savez(out_path, **{str(k): v for k, v in merged.items()})
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_ensemble_matches_single_process(tmp_path, oracle_mod):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "mms-gpu_b200"))
    from mmsb200 import geometry
    out = str(tmp_path / "ens.npz")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    z = np.load(out)
    dims, masks, Ms, bext = geometry.ensemble_instances(6, seed=11, sides=(4, 6, 8))
    assert sorted(int(k) for k in z.files) == list(range(6))
    for i, (X, Y, Z) in enumerate(dims):
        g = oracle_mod.Grid(X, Y, Z, 5e-9, 5e-9, 5e-9)
        p = oracle_mod.Params(external=True, hext_t=[0.0], hext_b=[bext[i]])
        ref = oracle_mod.rk4_run(g, p, masks[i], Ms[i], 1e-13, 3)
        assert np.array_equal(z[str(i)], ref)
