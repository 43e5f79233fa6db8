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


def test_double_double_gradient_against_mpmath(oracle):
    """oracle/se2_dd.c against 200-bit mpmath on a 60-pose walk at poses with a low part:
    sin/cos of double-double angles, xi = -sum J^T Lambda e, and the position loss."""
    import mpmath as mp
    mp.mp.prec = 200
    synth = importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")
    cg = synth.city_grid(60, seed=4, block=5, k_closures=4, radius=3.0)
    rng = np.random.default_rng(3)
    hi = cg.init + rng.normal(0.0, 0.05, cg.init.shape)
    lo = rng.uniform(-1, 1, hi.shape) * np.abs(hi) * 1e-17
    for x in list(rng.uniform(-12, 12, 200)) + [0.0, np.pi / 2, -np.pi, 1e-9]:
        xl = float(rng.uniform(-1, 1)) * abs(x) * 1e-17
        (sh, sl), (ch, cl) = oracle.sincos_dd(x, xl)
        X = mp.mpf(x) + mp.mpf(xl)
        assert abs(mp.mpf(sh) + mp.mpf(sl) - mp.sin(X)) < 1e-30
        assert abs(mp.mpf(ch) + mp.mpf(cl) - mp.cos(X)) < 1e-30
    info = 0.1 * np.exp(cg.log_w)
    xh, xl = oracle.se2_rhs_dd(hi, lo, cg.edge_i, cg.edge_j, cg.meas, info)
    n = hi.shape[0]
    P = [[mp.mpf(hi[i, k]) + mp.mpf(lo[i, k]) for k in range(3)] for i in range(n)]
    xi = [mp.mpf(0)] * (3 * n)
    for e in range(len(cg.edge_i)):
        i, j = int(cg.edge_i[e]), int(cg.edge_j[e])
        c, s = mp.cos(P[i][2]), mp.sin(P[i][2])
        dx, dy = P[j][0] - P[i][0], P[j][1] - P[i][1]
        e0 = c * dx + s * dy - mp.mpf(cg.meas[e, 0])
        e1 = c * dy - s * dx - mp.mpf(cg.meas[e, 1])
        e2 = P[j][2] - P[i][2] - mp.mpf(cg.meas[e, 2])
        e2 = e2 - 2 * mp.pi * mp.nint(e2 / (2 * mp.pi))
        a0, a1, a2 = e0 * mp.mpf(info[e, 0]), e1 * mp.mpf(info[e, 1]), e2 * mp.mpf(info[e, 2])
        gi = [-c * a0 + s * a1, -s * a0 - c * a1, (c * dy - s * dx) * a0 - (c * dx + s * dy) * a1 - a2]
        gj = [c * a0 - s * a1, s * a0 + c * a1, a2]
        for k in range(3):
            xi[3 * i + k] -= gi[k]
            xi[3 * j + k] -= gj[k]
    scale = max(abs(v) for v in xi)
    err = max(abs(mp.mpf(xh[q]) + mp.mpf(xl[q]) - xi[q]) for q in range(3 * n))
    assert err <= 1e-28 * scale, (float(err), float(scale))
    lh, ll = oracle.position_loss_dd(hi, lo, cg.gt)
    ref = sum((P[i][k] - mp.mpf(cg.gt[i, k])) ** 2 for i in range(n) for k in range(2))
    assert abs(mp.mpf(lh) + mp.mpf(ll) - ref) <= 1e-29 * ref


def test_n10k_finite_differences_at_h_1e6(oracle):
    """The adjoint's configured check at N = 10,000 (lambda 0.1): central differences with
    h = 1e-6 on 32 seeded (edge, component) log weights against the exact-Hessian sparse
    reference, which the GPU adjoint matches to 1e-6 (tests/test_gpu_adjoint.py).
    With the fixed points and the loss in FP64 the differences sit on a noise floor of
    ~1e-3 at this step (noise / 2h); with double-double fixed points (chord iterations on
    the FP64 LU, xi in double-double) they agree with the reference to ~3e-7, flat in h
    from 1e-4 to 1e-8, the reference's own FP64 accuracy."""
    import scipy.sparse.linalg as spl
    synth = importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")
    lam, anchor, h = 0.1, 1e12, 1e-6
    cg = synth.city_grid(10000, seed=2)
    p = R.gn_solve_sparse(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam, anchor=anchor, rounds=60,
                          tol=1e-13)
    _, dL = R.position_loss(p, cg.gt)
    _, rdlw, _ = R.adjoint_sparse(p, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam, dL, anchor=anchor)
    H, _ = R.system_sparse(p, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam, anchor)
    lu = spl.splu(H.tocsc(), permc_spec="COLAMD")
    rng = np.random.default_rng(7)
    pairs = [(int(rng.integers(len(cg.edge_i))), int(rng.integers(3))) for _ in range(32)]
    ref = np.array([rdlw[e, k] for e, k in pairs])
    fd = R.fd_log_weights_dd(oracle, p, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam, lu, cg.gt, pairs, h)
    err_dd = np.linalg.norm(fd - ref) / np.linalg.norm(ref)
    fd64 = []
    for e, k in pairs[:8]:
        lp, lm = cg.log_w.copy(), cg.log_w.copy()
        lp[e, k] += h
        lm[e, k] -= h
        Lp = R.position_loss(R.chord_solve_sparse(p, cg.edge_i, cg.edge_j, cg.meas, lp, lam, lu, anchor=anchor,
                                                  min_rounds=4), cg.gt)[0]
        Lm = R.position_loss(R.chord_solve_sparse(p, cg.edge_i, cg.edge_j, cg.meas, lm, lam, lu, anchor=anchor,
                                                  min_rounds=4), cg.gt)[0]
        fd64.append((Lp - Lm) / (2 * h))
    err_64 = np.linalg.norm(np.array(fd64) - ref[:8]) / np.linalg.norm(ref[:8])
    print(f"N=10000, h=1e-6: double-double differences {err_dd:.2e} from the reference, FP64 ones {err_64:.2e}")
    assert err_dd <= 1e-5
    assert err_64 > 10 * err_dd   # the FP64 floor the double-double fixed points remove
