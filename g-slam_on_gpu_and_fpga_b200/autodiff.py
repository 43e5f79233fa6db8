"""torch.autograd.Function over the Gauss-Newton solve of an SE(2) pose graph.

Forward: set lambda and the per-edge log information weights on a resident
PoseGraph, reset the poses to the initial guess, run Gauss-Newton rounds on the GPU
until the update norm falls below `diff_tol` (or `max_rounds`), return the converged
poses as a float64 tensor [N, 3].

Backward: the implicit-function adjoint (libgslam's gslam_adjoint): one FP64 PCG
solve with the exact Hessian at the converged poses plus one thread per edge, giving
dL/dlambda and dL/dlog_w [E, 3] for the incoming dL/dposes.

Not in the reference, whose programs only run the forward solve.
"""
from __future__ import annotations

import numpy as np
import torch

from .graph import PoseGraph


class GNSolve(torch.autograd.Function):
    """poses = GNSolve.apply(lam, log_w, graph, init_poses, max_rounds, diff_tol)"""

    @staticmethod
    def forward(ctx, lam, log_w, graph: PoseGraph, init_poses, max_rounds: int = 50, diff_tol: float = 1e-12):
        graph.set_weights(float(lam), log_w.detach().cpu().numpy())
        graph.poses = np.asarray(init_poses, np.float64)
        rounds = 0
        for _ in range(max_rounds):
            st = graph.round()
            rounds += 1
            if st.diff < diff_tol:
                break
        ctx.graph = graph
        ctx.rounds = rounds
        ctx.logw_shape = log_w.shape
        return torch.from_numpy(graph.poses).to(dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_poses):
        g = grad_poses.detach().to(torch.float64).cpu().numpy()
        dlam, dlogw, _, _ = ctx.graph.adjoint(g)
        return (torch.tensor(dlam, dtype=torch.float64),
                torch.from_numpy(dlogw).reshape(ctx.logw_shape).to(torch.float64),
                None, None, None, None)


def gn_solve(lam, log_w, graph: PoseGraph, init_poses, max_rounds: int = 50, diff_tol: float = 1e-12):
    """Functional form of GNSolve.apply."""
    return GNSolve.apply(lam, log_w, graph, init_poses, max_rounds, diff_tol)
