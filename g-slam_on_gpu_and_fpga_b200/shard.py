"""Spreading a batch of independent pose graphs over GPUs (one process per GPU).

Graphs are independent, so the only exchange is the final gather of results: each
rank takes a share chosen by a greedy longest-processing-time split on estimated
cost (poses + edges, a proxy for non-zero blocks, times the iteration budget),
solves it as one batch on its GPU, and rank 0 gathers every graph's poses and
statistics back into the caller's order (torch.distributed gather_object: NCCL
on GPUs, gloo on CPU).

Not in the reference, which runs one graph per process.
"""
from __future__ import annotations

import heapq

import numpy as np


def graph_cost(g) -> float:
    """Estimated work of one graph: block rows + edges (each edge adds 2 off-diagonal
    blocks and touches 2 diagonal ones)."""
    return float(g.init.shape[0] + 2 * len(g.edge_i))


def lpt_partition(costs, n_ranks: int):
    """Greedy longest-processing-time split: indices per rank, each list ascending.
    Deterministic (ties go to the lower rank, then the lower index)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(n_ranks)]
    share = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        share[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in share]


def solve_sharded(graphs, lams, rounds: int, dist=None, solver=None, **opts):
    """Runs `rounds` Gauss-Newton rounds of every graph, spread over the ranks of
    `dist` (torch.distributed, already initialised; None = this process alone).

    solver(graphs, lams, rounds, **opts) -> (list of poses [N_q, 3], list of stats)
    defaults to a PoseGraphBatch on this rank's GPU. Returns, on rank 0, the poses and
    stats of every graph in the caller's order (None on the other ranks)."""
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    lams = np.broadcast_to(np.asarray(lams, np.float64), (len(graphs),))
    share = lpt_partition([graph_cost(g) for g in graphs], world)[rank]
    solver = solver or _batch_solver
    mine = solver([graphs[i] for i in share], lams[share], rounds, **opts) if share else ([], [])
    local = list(zip(share, mine[0], mine[1]))
    if dist is None:
        gathered = [local]
    else:
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(local, gathered, dst=0)
    if rank != 0:
        return None
    poses, stats = [None] * len(graphs), [None] * len(graphs)
    for part in gathered:
        for i, p, s in part:
            poses[i], stats[i] = p, s
    return poses, stats


def _batch_solver(graphs, lams, rounds, **opts):
    from .graph import PoseGraphBatch
    b = PoseGraphBatch.from_se2_list(graphs, lams, **opts)
    try:
        stats = None
        for _ in range(rounds):
            stats = b.round_all()
        p = b.poses
        return [b.graph_poses(q, p).copy() for q in range(len(graphs))], stats
    finally:
        b.close()
