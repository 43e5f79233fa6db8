"""Multi-rank batch sharding on CPU: the LPT split and the gather of results over a
world-size-2 gloo process group (the GPU solve is replaced by a stand-in solver, so
the test exercises the partition and collective plumbing without a GPU)."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

shard = importlib.import_module("g-slam_on_gpu_and_fpga_b200.shard")
synth = importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")


def test_lpt_partition_balanced_and_complete():
    rng = np.random.default_rng(0)
    costs = list(np.exp(rng.uniform(np.log(500), np.log(20000), 64)))
    for world in (1, 2, 3, 8):
        share = shard.lpt_partition(costs, world)
        flat = sorted(i for s in share for i in s)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in s) for s in share]
        # LPT bound: max load <= 4/3 optimum; the optimum is at least the mean
        assert max(loads) <= (4.0 / 3.0) * max(np.mean(loads), max(costs)) + 1e-9
    assert shard.lpt_partition(costs, 2) == shard.lpt_partition(costs, 2)  # deterministic


def fake_solver(graphs, lams, rounds, **opts):
    poses = [g.init + lam * rounds for g, lam in zip(graphs, lams)]
    return poses, [{"n": g.init.shape[0], "lam": float(lam)} for g, lam in zip(graphs, lams)]


def _worker(rank, world, port, sizes, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    graphs = [synth.city_grid(n, seed=i) for i, n in enumerate(sizes)]
    lams = np.linspace(0.1, 1.0, len(sizes))
    res = shard.solve_sharded(graphs, lams, 3, dist=dist, solver=fake_solver)
    if rank == 0:
        poses, stats = res
        ok = all(np.array_equal(poses[i], graphs[i].init + lams[i] * 3) and stats[i]["n"] == sizes[i]
                 for i in range(len(sizes)))
        out.put(ok)
    else:
        out.put(res is None)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.timeout(120)
def test_sharded_gather_world_size_2():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    sizes = [40, 200, 75, 310, 64, 90, 500]
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = [out.get(timeout=100) for _ in procs]
    for p in procs:
        p.join(timeout=30)
    assert all(results)
    assert all(p.exitcode == 0 for p in procs)
