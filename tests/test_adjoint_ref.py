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


def test_sparse_reference_matches_dense():
    """The sparse (SuperLU) forms of the reference equal the dense ones on a small graph:
    Omega, the exact Hessian, the converged poses, the adjoint gradient, and the chord
    iteration's fixed point."""
    import scipy.sparse.linalg as spl
    G = importlib.import_module("g-slam_on_gpu_and_fpga_b200")
    cg = G.synth.city_grid(120, seed=2, block=5, k_closures=4, radius=3.0)
    for exact in (False, True):
        Hd, xd = R.system(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 0.1, 1e12, exact=exact)
        Hs, xs = R.system_sparse(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 0.1, 1e12, exact=exact)
        assert np.allclose(Hs.toarray(), Hd, rtol=0, atol=1e-9 * np.abs(Hd).max())
        assert np.array_equal(xs, xd)
        assert np.array_equal(R.rhs(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 0.1), xd)
    pd = R.gn_solve(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 0.1, anchor=1e12)
    ps = R.gn_solve_sparse(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 0.1, anchor=1e12)
    assert np.abs(ps - pd).max() <= 1e-9
    _, dL = R.position_loss(pd, cg.gt)
    _, gd, _ = R.adjoint(pd, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 0.1, dL, anchor=1e12)
    _, gs, _ = R.adjoint_sparse(pd, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 0.1, dL, anchor=1e12)
    assert np.linalg.norm(gs - gd) <= 1e-9 * np.linalg.norm(gd)
    H, _ = R.system_sparse(pd, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 0.1, 1e12)
    lw = cg.log_w.copy()
    lw[5, 1] += 1e-3
    pc = R.chord_solve_sparse(pd, cg.edge_i, cg.edge_j, cg.meas, lw, 0.1, spl.splu(H.tocsc()), anchor=1e12)
    pg = R.gn_solve_sparse(pd, cg.edge_i, cg.edge_j, cg.meas, lw, 0.1, anchor=1e12)
    assert np.abs(pc - pg).max() <= 1e-9
