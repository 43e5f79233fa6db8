"""GPU tests of the mixed-precision solver (k_pcg_mixed: FP32 inner Chronopoulos-Gear
PCG, FP64 residual / dots / D^-1 / pose accumulation, iterative refinement) through
the C ABI, against the FP64 oracle and the library's FP64 solver."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PREC_FP64, PREC_MIXED = 0, 1


def _se2(pkg, cg, lam=0.1, **opts):
    return pkg.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=lam, angle_wrap=1, **opts)


@pytest.fixture(scope="module")
def synth():
    return importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")


@pytest.mark.parametrize("n,block", [(600, 5), (2000, 20)])
def test_mixed_converges_to_the_oracle_solution(pkg, oracle, synth, n, block):
    """Refinement reaches the FP64 tolerance (on the 2000-pose walk the FP32 inner solves
    stagnate and the FP64 solver finishes): the true FP64 residual is below it and the
    solution is as close to the exact one (A-norm) as the oracle's converged FP64 PCG."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    cg = synth.city_grid(n, seed=3, block=block)
    tol = 1e-8
    with _se2(pkg, cg, precision=PREC_MIXED, tol=tol, max_iter=200000, max_refine=500) as g:
        g.linearise()
        g.assemble()
        st = g.solve()
        dx = g.dx()
        rp, ci, va, xi = g.csr()
    # refinements < 0: the FP32 inner solves stagnated and the FP64 solver finished
    assert st.reason == pkg.abi.STOP_TOL and st.refinements != 0
    A = sp.csr_matrix((va, ci, rp), shape=(len(xi), len(xi)))
    assert np.linalg.norm(A @ dx - xi) <= 1.01 * tol * np.linalg.norm(xi)
    x_ref, _, _ = oracle.pcg(rp, ci, va, xi, tol=tol, max_iter=400000)
    xs = spl.spsolve(A.tocsc(), xi)
    ea = lambda x: np.sqrt(max((x - xs) @ (A @ (x - xs)), 0.0))  # noqa: E731
    scale = np.sqrt(xs @ (A @ xs))
    assert ea(dx) <= max(1e-6 * scale, 3.0 * ea(x_ref)), (ea(dx) / scale, ea(x_ref) / scale)


def test_mixed_truncated_solve_reaches_the_fp64_residual(pkg, synth):
    """At the reference's settings (tol 1e-6, 500 iterations, no convergence on this
    graph) the mixed solve ends at the same true residual as the FP64 solve."""
    cg = synth.city_grid(20000, seed=5)
    res = {}
    for prec in (PREC_FP64, PREC_MIXED):
        with _se2(pkg, cg, precision=prec) as g:
            g.linearise()
            g.assemble()
            st = g.solve()
            assert st.iterations == 500
            res[prec] = st.rel_residual
    assert res[PREC_MIXED] <= 1.5 * res[PREC_FP64], res


def test_mixed_rounds_follow_fp64(pkg, synth):
    """Gauss-Newton rounds with converged solves: mixed and FP64 poses agree."""
    cg = synth.city_grid(1500, seed=8, block=5)
    poses = {}
    for prec in (PREC_FP64, PREC_MIXED):
        with _se2(pkg, cg, precision=prec, tol=1e-9, max_iter=100000, max_refine=500) as g:
            for _ in range(4):
                g.round()
            poses[prec] = g.poses
    d = poses[PREC_MIXED] - poses[PREC_FP64]
    d[:, 2] = (d[:, 2] + np.pi) % (2 * np.pi) - np.pi
    assert np.linalg.norm(d) <= 1e-6 * np.linalg.norm(poses[PREC_FP64])


def test_mixed_is_deterministic(pkg, synth):
    cg = synth.city_grid(5000, seed=9)
    out = []
    for _ in range(2):
        with _se2(pkg, cg, precision=PREC_MIXED) as g:
            g.linearise()
            g.assemble()
            g.solve()
            out.append(g.dx())
    assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))


def test_stagnation_falls_back_to_fp64(pkg, synth):
    """A system the FP32 inner solve cannot resolve to 1e-8: the solve still reaches the
    tolerance (FP64 after the stagnation), and reports the mixed steps as negative."""
    cg = synth.city_grid(2000, seed=3)
    with _se2(pkg, cg, precision=PREC_MIXED, tol=1e-8, max_iter=200000, max_refine=500) as g:
        g.linearise()
        g.assemble()
        st = g.solve()
    assert st.reason == pkg.abi.STOP_TOL and st.refinements < 0 and st.rel_residual < 1e-8
