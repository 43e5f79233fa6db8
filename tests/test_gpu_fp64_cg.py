"""GPU tests of the FP64 one-reduction solver (GSLAM_PREC_FP64_CG: k_pcg_mixed with FP64
inner arithmetic, Chronopoulos-Gear recurrence, one grid reduction per iteration, no
refinement) through the C ABI, against the library's FP64 solver (the reference's
recurrence) and the oracle."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PREC_FP64, PREC_FP64_CG = 0, 2


def _se2(pkg, cg, lam=0.1, **opts):
    return pkg.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=lam, angle_wrap=1, **opts)


@pytest.fixture(scope="module")
def synth():
    return importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")


def _solve(pkg, cg, prec, **opts):
    with _se2(pkg, cg, precision=prec, **opts) as g:
        g.linearise()
        g.assemble()
        st = g.solve()
        return st, g.dx(), g.csr()


def test_iterates_follow_the_reference_recurrence(pkg, synth):
    """60 iterations, no early stop: the one-reduction recurrence produces the reference
    recurrence's iterate (equal in exact arithmetic; only rounding differs)."""
    cg = synth.city_grid(5000, seed=4)
    st64, dx64, _ = _solve(pkg, cg, PREC_FP64, tol=0.0, max_iter=60)
    stcg, dxcg, _ = _solve(pkg, cg, PREC_FP64_CG, tol=0.0, max_iter=60)
    assert st64.iterations == stcg.iterations == 60
    assert np.linalg.norm(dxcg - dx64) <= 1e-9 * np.linalg.norm(dx64)


def test_converged_solve_matches_the_oracle(pkg, oracle, synth):
    """tol 1e-10: stops on the recurrence residual (reason TOL) with the true residual
    below the tolerance and the step within 1e-6 of the exact solution (A-norm, relative).
    At tolerances this tight the one-reduction recurrence is the weaker one in finite
    precision (z carried by its own recurrence drifts from D^-1 r): on this graph it takes
    13,058 iterations against the reference recurrence's 5,201 and ends 5.6e-8 from the
    exact step where the oracle's PCG ends 9.3e-10 from it; bounded here at 4x and 1e-6."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    cg = synth.city_grid(2000, seed=3, block=5)
    tol = 1e-10
    st64, _, _ = _solve(pkg, cg, PREC_FP64, tol=tol, max_iter=200000)
    st, dx, (rp, ci, va, xi) = _solve(pkg, cg, PREC_FP64_CG, tol=tol, max_iter=200000)
    assert st.reason == pkg.abi.STOP_TOL and st.rel_residual < tol
    assert st.iterations <= 4 * st64.iterations, (st.iterations, st64.iterations)
    A = sp.csr_matrix((va, ci, rp), shape=(len(xi), len(xi)))
    x_ref, _, _ = oracle.pcg(rp, ci, va, xi, tol=tol, max_iter=400000)
    xs = spl.spsolve(A.tocsc(), xi)
    ea = lambda x: np.sqrt(max((x - xs) @ (A @ (x - xs)), 0.0))  # noqa: E731
    scale = np.sqrt(xs @ (A @ xs))
    assert ea(dx) <= 1e-6 * scale, (ea(dx) / scale, ea(x_ref) / scale)


def test_reference_settings_truncated_solve(pkg, synth):
    """tol 1e-6 / 500 iterations on a graph that does not converge in 500: both solvers
    take 500 steps and end at the same step up to rounding."""
    cg = synth.city_grid(20000, seed=5)
    st64, dx64, _ = _solve(pkg, cg, PREC_FP64)
    st, dx, _ = _solve(pkg, cg, PREC_FP64_CG)
    assert st64.iterations == st.iterations == 500
    assert st.reason == pkg.abi.STOP_MAXIT
    assert np.linalg.norm(dx - dx64) <= 1e-7 * np.linalg.norm(dx64)
    assert st.rel_residual <= 1.01 * st64.rel_residual + 1e-12


def test_rounds_follow_the_oracle(pkg, oracle, synth):
    """Ten Gauss-Newton rounds at the reference's settings: poses within 1e-8 of the
    oracle's (the reference's PCG restated in C)."""
    cg = synth.city_grid(3000, seed=6)
    poses = cg.init.copy()
    for _ in range(10):
        blocks, _ = oracle.se2_linearise(poses, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, 0.1)
        rp, ci, va, xi = oracle.csr_build_anchor(3 * cg.n_poses, cg.edge_i, cg.edge_j, blocks, 1e6)
        dx, _, _ = oracle.pcg(rp, ci, va, xi, tol=1e-6, max_iter=500)
        poses = poses + dx.reshape(-1, 3)
        poses[:, 2] = (poses[:, 2] + np.pi) % (2 * np.pi) - np.pi
    with _se2(pkg, cg, precision=PREC_FP64_CG) as g:
        for _ in range(10):
            g.round()
        got = g.poses
    d = got - poses
    d[:, 2] = (d[:, 2] + np.pi) % (2 * np.pi) - np.pi
    assert np.linalg.norm(d) <= 1e-8 * np.linalg.norm(poses)


def test_deterministic(pkg, synth):
    cg = synth.city_grid(5000, seed=9)
    out = [_solve(pkg, cg, PREC_FP64_CG)[1] for _ in range(2)]
    assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))


def test_barrier_timeout_returns_status(pkg, synth):
    """A CTA that never arrives: the bounded waits run out, the call returns
    DEVICE_TIMEOUT and the context stays usable."""
    cg = synth.city_grid(5000, seed=2)
    with _se2(pkg, cg, precision=PREC_FP64_CG, barrier_timeout_ms=20.0, test_absent_cta=1) as g:
        g.linearise()
        g.assemble()
        with pytest.raises(pkg.abi.GslamError) as e:
            g.solve()
        assert e.value.code == pkg.abi.ERR_DEVICE_TIMEOUT
        g.set_opts(test_absent_cta=-1)
        st = g.solve()
        assert st.reason in (pkg.abi.STOP_TOL, pkg.abi.STOP_MAXIT)
