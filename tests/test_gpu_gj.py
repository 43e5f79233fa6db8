"""GPU tests of the blocked Gauss-Jordan dense inverse (FP64 tensor-core trailing
updates) against numpy and against the oracle's restatement of the reference's
unblocked Gauss-Jordan (MatrixOps.c:29-91) on an assembled Omega."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [64, 300, 517])
def test_inverse_of_spd_matrix(pkg, n):
    rng = np.random.default_rng(n)
    m = rng.normal(size=(n, n))
    a = m @ m.T + n * np.eye(n)
    inv, _ = pkg.dense.gj_inverse(a)
    ref = np.linalg.inv(a)
    assert np.linalg.norm(inv - ref) <= 1e-12 * np.linalg.norm(ref)
    assert np.linalg.norm(inv @ a - np.eye(n)) <= 1e-11 * np.sqrt(n)


def test_dense_solve_of_a_pose_graph_matches_oracle_gj(pkg, oracle):
    synth = importlib.import_module("g-slam_on_gpu_and_fpga_b200.synth")
    cg = synth.city_grid(300, seed=4, block=5)
    g = pkg.PoseGraph.from_se2(cg.init, cg.edge_i, cg.edge_j, cg.meas, cg.log_w, lam=0.1)
    g.linearise()
    g.assemble()
    rp, ci, va, xi = g.csr()
    g.close()
    A = oracle.dense_from_csr(rp, ci, va)
    x, _ = pkg.dense.gj_solve(A, xi)
    inv_ref, rc = oracle.gj_inverse(A)
    assert rc == 0
    x_ref = inv_ref @ xi
    assert np.linalg.norm(x - x_ref) <= 1e-9 * np.linalg.norm(x_ref)
    assert np.linalg.norm(A @ x - xi) <= 1e-9 * np.linalg.norm(xi)
