"""CPU check of the dense adjoint reference (tests/adjoint_ref.py) against central
finite differences of the dense Gauss-Newton solve, so the reference that the GPU
adjoint is compared with is itself pinned. A 150-pose city-grid walk with 5 m blocks
(51 loop closures, so the information weights matter)."""
import importlib

import numpy as np

import adjoint_ref as R


def _graph():
    synth = importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")
    return synth.city_grid(150, seed=2, block=5)


def test_dense_adjoint_matches_finite_differences():
    g = _graph()
    lam, h = 0.1, 1e-6
    p = R.gn_solve(g.init, g.edge_i, g.edge_j, g.meas, g.log_w, lam)
    _, dL = R.position_loss(p, g.gt)
    dlam, dlw, _ = R.adjoint(p, g.edge_i, g.edge_j, g.meas, g.log_w, lam, dL)
    rng = np.random.default_rng(0)
    picks = [(int(rng.integers(len(g.edge_i))), int(rng.integers(3))) for _ in range(6)]
    fd, adj = [], []
    for e, k in picks:
        lw1, lw2 = g.log_w.copy(), g.log_w.copy()
        lw1[e, k] += h
        lw2[e, k] -= h
        # restarted from the converged poses: same fixpoint, solve noise ~ the perturbation
        lp = R.position_loss(R.gn_solve(p, g.edge_i, g.edge_j, g.meas, lw1, lam), g.gt)[0]
        lm = R.position_loss(R.gn_solve(p, g.edge_i, g.edge_j, g.meas, lw2, lam), g.gt)[0]
        fd.append((lp - lm) / (2 * h))
        adj.append(dlw[e, k])
    fd, adj = np.array(fd), np.array(adj)
    assert np.linalg.norm(fd - adj) <= 1e-5 * np.linalg.norm(adj), (fd, adj)
    # lambda scales every edge weight alike: the optimum does not move
    assert abs(dlam) <= 1e-8 * np.abs(dlw).sum() + 1e-9


def test_exact_hessian_is_the_jacobian_of_the_gradient():
    """H (with the second-order terms) against central differences of xi = -g."""
    g = _graph()
    lam = 0.1
    p = R.gn_solve(g.init, g.edge_i, g.edge_j, g.meas, g.log_w, lam, rounds=3)
    H, _ = R.system(p, g.edge_i, g.edge_j, g.meas, g.log_w, lam, 0.0, exact=True)
    rng = np.random.default_rng(1)
    for col in rng.integers(0, 3 * len(p), 6):
        h = 1e-6
        p1, p2 = p.copy(), p.copy()
        p1.reshape(-1)[col] += h
        p2.reshape(-1)[col] -= h
        x1 = R.system(p1, g.edge_i, g.edge_j, g.meas, g.log_w, lam, 0.0)[1]
        x2 = R.system(p2, g.edge_i, g.edge_j, g.meas, g.log_w, lam, 0.0)[1]
        num = -(x1 - x2) / (2 * h)
        assert np.allclose(num, H[:, col], rtol=1e-5, atol=1e-5 * np.abs(H[:, col]).max())
